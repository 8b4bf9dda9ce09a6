// traverse.cuh -- device-side grid traversal shared by the per-scene kernels (trace.cu) and
// the batched persistent kernel (batch.cu).
//
// Reference path (javorkk/happyray):
//   uniform DDA            src/RT/Algorithm/UGridTraverser.h:44-177
//   two-level DDA          src/RT/Algorithm/TLGridTraverser.h:45-354
//   intersector            src/RT/Algorithm/RayTriangleIntersector.h:38-92
//   camera                 src/RT/Primitive/Camera.h:35-72
//
// Execution model: the traversal is warp-synchronous.  Every lane advances its own DDA
// to its next cell or leaf, then the warp tests the triangle lists of all its lanes
// together, packed 32 (lane, triangle) pairs per round (test_lists), so that no lane idles
// while another walks a longer list.  Hits are applied in list order with the strict
// t < best rule, which is exactly the first-tested-wins result of the sequential
// intersector.  Traversal functions must therefore be called by all lanes of a warp;
// lanes without a ray pass active = false.
#pragma once

#include "hr_internal.h"
#include "hr_block.cuh"

namespace hr {
namespace {

struct Scene {
    const float4* __restrict__ tris;   // 3 float4 per triangle (current frame)
    const uint2* __restrict__ cells;
    const uint2* __restrict__ leaves;
    const uint32_t* __restrict__ prims;
    const GridDesc* desc;
    uint32_t ntri;
    int32_t kind;
    const float4* __restrict__ nrm3 = nullptr;   // path tracer: 3 vertex normals per triangle, or none
    const float* __restrict__ alb = nullptr;     // path tracer: diffuse albedo per triangle, or none
    // two-level: one bit per top cell, set for a cell with references (bit occ_bit0 + c for
    // cell c), or none; 64 times smaller than the cell records, so an empty cell costs a
    // cached bit instead of a cell-record load
    const uint32_t* __restrict__ occ = nullptr;
    uint32_t occ_bit0 = 0;
};

struct G {
    float bmin[3], bmax[3], cs[3], rcp[3];
    int32_t res[3];
};
// A grid whose build overflowed or failed holds stale or partial arrays (the host redoes
// the frame): kernels trace no triangle of it.
__device__ __forceinline__ void gate_scene(Scene& s) {
    if (__ldg(&s.desc->overflow) | __ldg(&s.desc->error)) s.ntri = 0u;
}

__device__ __forceinline__ G load_g(const GridDesc* d) {
    G g;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        g.bmin[k] = __ldg(&d->bmin[k]); g.bmax[k] = __ldg(&d->bmax[k]);
        g.cs[k] = __ldg(&d->cs[k]); g.rcp[k] = __ldg(&d->rcp[k]); g.res[k] = __ldg(&d->res[k]);
    }
    return g;
}

struct Hit {
    float t, u, v;
    uint32_t tri;
    uint32_t cells, tests;
    bool hit;
};

// a16: Moller-Trumbore of one triangle (RayTriangleIntersector.h:52-90); returns the hit
// test with strict t < tbest
__device__ __forceinline__ bool mt_test(const Scene& s, uint32_t tri, f3 o, f3 d, float tbest, float* ot, float* ou,
                                        float* ov) {
    f3 p[3];
    tri_fetch(s.tris, tri, p);
    const f3 e1 = sub(p[1], p[0]), e2 = sub(p[2], p[0]);
    const f3 pv = cross(d, e2);
    const float det = dot(e1, pv);
    const float inv = 1.0f / det;
    const f3 sv = sub(o, p[0]);
    const float u = dot(sv, pv) * inv;
    const f3 q = cross(sv, e1);
    const float v = dot(q, d) * inv;
    const float t = dot(e2, q) * inv;
    *ot = t; *ou = u; *ov = v;
    return u >= 0.0f && v >= 0.0f && u + v <= 1.0f && t > kIsectEps && t < tbest;
}

// Barycentric weights (u, v) of the hit of ray (o, d) on triangle tri, reported by the ray
// queries: Moller-Trumbore evaluated in binary64 from the binary32 inputs, once per ray.
// The traversal's binary32 weights carry up to ~6e-5 absolute error when the origin is far
// from a small triangle (the differences of nearly equal products); in binary64 the
// result is within a rounding of the exact weights of the same inputs.
__device__ __forceinline__ void refine_uv(const Scene& s, uint32_t tri, f3 o, f3 d, float* ou, float* ov) {
    f3 p[3];
    tri_fetch(s.tris, tri, p);
    const double ax = p[0].x, ay = p[0].y, az = p[0].z;
    const double e1x = (double)p[1].x - ax, e1y = (double)p[1].y - ay, e1z = (double)p[1].z - az;
    const double e2x = (double)p[2].x - ax, e2y = (double)p[2].y - ay, e2z = (double)p[2].z - az;
    const double dx = d.x, dy = d.y, dz = d.z;
    const double px = dy * e2z - dz * e2y, py = dz * e2x - dx * e2z, pz = dx * e2y - dy * e2x;
    const double det = e1x * px + e1y * py + e1z * pz;
    const double sx = (double)o.x - ax, sy = (double)o.y - ay, sz = (double)o.z - az;
    const double u = (sx * px + sy * py + sz * pz) / det;
    const double qx = sy * e1z - sz * e1y, qy = sz * e1x - sx * e1z, qz = sx * e1y - sy * e1x;
    const double v = (qx * dx + qy * dy + qz * dz) / det;
    *ou = (float)u;
    *ov = (float)v;
}

// hit modes of a traversal: closest hit, any hit, or per lane (the lane's `any` argument)
constexpr int kHitClosest = 0, kHitAny = 1, kHitMixed = 2;

__device__ __forceinline__ float shfl(float x, int src) { return __shfl_sync(kFullMask, x, src); }
__device__ __forceinline__ uint32_t shfl(uint32_t x, int src) { return __shfl_sync(kFullMask, x, src); }

// Warp-wide test of every lane's list prims[b, e); must be called by all 32 lanes, and
// returns true on the lanes whose any-hit query it answers.  The (lane, triangle) pairs of
// all lanes are numbered in lane order and tested 32 per round, one pair per lane, so no
// lane idles while another walks a longer list.  Pair j belongs to the lane whose
// [exclusive, inclusive) prefix of list lengths holds j and is tested with that lane's
// ray and current bound.  Closest hit: the hits of a round are applied one by one in pair
// order, each only if its t is strictly below the lane's best so far -- the
// first-tested-wins rule of a one-lane loop over the list.  Any hit: a lane is answered
// when one of its pairs hits; its later pairs are skipped.  STATS counts the pairs
// tested: all of a list for closest hit (as the sequential loop), whole rounds for any hit.
template <int HM, bool STATS>
__device__ __forceinline__ bool test_lists(const Scene& s, f3 o, f3 d, uint32_t b, uint32_t e, bool any, Hit& h) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t n = e - b;
    if (__ballot_sync(kFullMask, n != 0u) == 0u) return false;   // most leaves a ray crosses are empty
    // lanes whose query is an any-hit query
    const uint32_t anym = HM == kHitAny ? kFullMask : (HM == kHitClosest ? 0u : __ballot_sync(kFullMask, any));
    uint32_t incl = n;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const uint32_t x = __shfl_up_sync(kFullMask, incl, off);
        if (lane >= (uint32_t)off) incl += x;
    }
    const uint32_t total = __shfl_sync(kFullMask, incl, 31);
    // prims index of pair j of this lane: rel + j, summed in 32 bits (rel wraps when b is
    // below the lane's exclusive prefix; the sum does not)
    const uint32_t rel = b - (incl - n);
    uint32_t best = 0xffffffffu;           // pair number of this lane's best hit of this call
    uint32_t answered = 0u;                // any-hit lanes with a hit
    for (uint32_t base = 0; base < total; base += 32u) {
        const uint32_t j = base + lane;
        uint32_t own = 0;                  // number of lanes whose inclusive prefix is <= j
#pragma unroll
        for (uint32_t step = 16; step > 0; step >>= 1) {
            if (__shfl_sync(kFullMask, incl, own + step - 1u) <= j) own += step;
        }
        const f3 so = mk(shfl(o.x, own), shfl(o.y, own), shfl(o.z, own));
        const f3 sd = mk(shfl(d.x, own), shfl(d.y, own), shfl(d.z, own));
        const float bt = shfl(h.t, own);
        const uint32_t srel = shfl(rel, own);
        const bool own_any = (anym >> own) & 1u;
        const bool live = j < total && !(own_any && ((answered >> own) & 1u));
        float t = 0.0f, u = 0.0f, v = 0.0f;
        bool hit = false;
        if (live) hit = mt_test(s, __ldg(s.prims + (srel + j)), so, sd, bt, &t, &u, &v);
        if (STATS && !((anym & answered) >> lane & 1u)) {   // this lane's pairs tested in the round
            const uint32_t lo = max(incl - n, base), hi = min(incl, base + 32u);
            if (hi > lo) h.tests += hi - lo;
        }
        if (HM != kHitClosest) answered |= __reduce_or_sync(kFullMask, (hit && own_any) ? 1u << own : 0u);
        if (HM != kHitAny) {
            uint32_t hm = __ballot_sync(kFullMask, hit && !own_any);
            while (hm) {
                const int src = __ffs(hm) - 1;
                hm &= hm - 1u;
                const uint32_t ow = shfl(own, src), hj = shfl(j, src);
                const float ht = shfl(t, src), hu = shfl(u, src), hv = shfl(v, src);
                if (lane == ow && ht < h.t) {
                    h.t = ht; h.u = hu; h.v = hv; h.hit = true;
                    best = hj;
                }
            }
        }
    }
    bool done = false;
    if (HM != kHitClosest) {
        done = (answered >> lane) & 1u;
        if (done) h.hit = true;
    }
    if (HM != kHitAny && best != 0xffffffffu) h.tri = __ldg(s.prims + (rel + best));
    return done;
}

__device__ __forceinline__ int min_dim(float a, float b, float c) { return a < b ? (a < c ? 0 : 2) : (b < c ? 1 : 2); }

// One DDA step along the axis of the smallest tmax.  The state arrays are only indexed
// with constants (one branch per axis, as TLGridTraverser.h:226-290 writes it out), so
// they stay in registers.  Returns tmax of the axis before the step in *t_before and
// whether the new cell index is inside [0, res).
__device__ __forceinline__ bool dda_step(float* tmax, int32_t* cell, const float* rcp, const float* cs,
                                         const int32_t* res, float* t_before) {
    const int k = min_dim(tmax[0], tmax[1], tmax[2]);
    if (k == 0) {
        *t_before = tmax[0];
        cell[0] += rcp[0] > 0.0f ? 1 : -1;
        tmax[0] += cs[0] * fabsf(rcp[0]);
        return cell[0] < res[0] && cell[0] > -1;
    } else if (k == 1) {
        *t_before = tmax[1];
        cell[1] += rcp[1] > 0.0f ? 1 : -1;
        tmax[1] += cs[1] * fabsf(rcp[1]);
        return cell[1] < res[1] && cell[1] > -1;
    } else {
        *t_before = tmax[2];
        cell[2] += rcp[2] > 0.0f ? 1 : -1;
        tmax[2] += cs[2] * fabsf(rcp[2]);
        return cell[2] < res[2] && cell[2] > -1;
    }
}

__device__ __forceinline__ bool clip(const G& g, f3 o, const float* rcp, float* t0, float* t1) {
    float tn[3], tf[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float a = (g.bmin[k] - comp(o, k)) * rcp[k];
        float b = (g.bmax[k] - comp(o, k)) * rcp[k];
        tn[k] = hmin(a, b); tf[k] = hmax(a, b);
    }
    *t0 = hmax(hmax(tn[0], tn[1]), tn[2]);
    *t1 = hmin(hmin(tf[0], tf[1]), tf[2]);
    return *t1 > *t0 && *t1 >= 0.0f;
}

// a14: uniform grid DDA (UGridTraverser.h:76-172), warp-synchronous.  After a lane's list
// test it steps on over up to HR_UG_CELL_STEPS - 1 empty cells within the same warp step
// (an empty cell has no list to test) and keeps the range of the non-empty cell it stops
// at for the next step; each lane visits the same cells in the same order as one cell per
// step would.
#ifndef HR_UG_CELL_STEPS
#define HR_UG_CELL_STEPS 4
#endif
template <int HM, bool STATS>
__device__ void trace_ug(const Scene& s, const G& g, f3 o, f3 d, bool any, Hit& h, bool active) {
    float rcp[3] = {0.0f, 0.0f, 0.0f}, tmax[3] = {0.0f, 0.0f, 0.0f};
    int32_t cell[3] = {0, 0, 0};
    if (active) {
        rcp[0] = 1.0f / d.x; rcp[1] = 1.0f / d.y; rcp[2] = 1.0f / d.z;
        float t0, t1;
        active = clip(g, o, rcp, &t0, &t1);
        if (active) {
            f3 ep = o;
            if (t0 >= 0.0f) {
                const float te = t0 + kEps;
                ep = mk(o.x + te * d.x, o.y + te * d.y, o.z + te * d.z);
            }
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                float cf = floorf((comp(ep, k) - g.bmin[k]) * g.rcp[k]);
                cf = hmin((float)g.res[k] - 1.0f, hmax(cf, 0.0f));
                const float stp = rcp[k] > 0.0f ? 1.0f : 0.0f;
                tmax[k] = ((cf + stp) * g.cs[k] + g.bmin[k] - comp(o, k)) * rcp[k];
                cell[k] = f2i(cf);
            }
            active = cell[0] < g.res[0] && cell[0] > -1 && cell[1] < g.res[1] && cell[1] > -1 &&
                     cell[2] < g.res[2] && cell[2] > -1;
        }
    }
    const uint32_t rx = (uint32_t)g.res[0], rxy = (uint32_t)g.res[0] * (uint32_t)g.res[1];
    uint2 cr_next = make_uint2(0u, 0u);
    bool have_next = false;
    while (__any_sync(kFullMask, active)) {
        uint32_t b = 0, e = 0;
        if (active) {
            const uint2 cr = have_next ? cr_next
                                       : __ldg(s.cells + ((uint32_t)cell[0] + (uint32_t)cell[1] * rx +
                                                          (uint32_t)cell[2] * rxy));
            b = cr.x; e = cr.y;
            if (STATS) h.cells++;
        }
        const bool done = test_lists<HM, STATS>(s, o, d, b, e, any, h);
        have_next = false;
        if (active) {
            if (done) {
                active = false;
            } else {
                for (int j = 1;; ++j) {
                    float tk;
                    const bool inside = dda_step(tmax, cell, rcp, g.cs, g.res, &tk);
                    active = h.t > tk && inside;
                    if (!active || j >= HR_UG_CELL_STEPS) break;
                    const uint2 nx =
                        __ldg(s.cells + ((uint32_t)cell[0] + (uint32_t)cell[1] * rx + (uint32_t)cell[2] * rxy));
                    if (nx.y > nx.x) {
                        cr_next = nx;
                        have_next = true;
                        break;
                    }
                    if (STATS) h.cells++;
                }
            }
        }
    }
}

// Two-level DDA state of one lane (TLGridTraverser.h:79-349).
struct TL {
    float rcp[3], tmax[3], tentry;
    int32_t cell[3];
    uint32_t lbase, lres[3];   // current top cell: first leaf, sub-grid resolution
    float scs[3], tm2[3];
    int32_t c2[3];
};

// Enter the sub-grid of the current top cell at tentry (TLGridTraverser.h:145-197).
__device__ __forceinline__ void tl_enter(TL& q, const G& g, f3 o, f3 d, uint2 tc) {
    q.lbase = tc.x;
    q.lres[0] = tc.y & 0xFFu; q.lres[1] = (tc.y >> 8) & 0xFFu; q.lres[2] = (tc.y >> 16) & 0xFFu;
    const f3 e2 = mk(o.x + q.tentry * d.x, o.y + q.tentry * d.y, o.z + q.tentry * d.z);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float cres = (float)q.lres[k];
        const float srcp = g.rcp[k] * cres;
        const float mb = (float)q.cell[k] * g.cs[k] + g.bmin[k];
        float cf = floorf((comp(e2, k) - mb) * srcp);
        const float scs = 1.0f / srcp;
        q.scs[k] = scs;
        cf = hmin(cres - 1.0f, hmax(cf, 0.0f));
        const float stp = q.rcp[k] > 0.0f ? 1.0f : 0.0f;
        q.tm2[k] = ((cf + stp) * scs + mb - comp(o, k)) * q.rcp[k];
        q.c2[k] = f2i(cf);
    }
}

// Outer step (TLGridTraverser.h:296-348): returns false when the ray is done.
__device__ __forceinline__ bool tl_outer_step(TL& q, const G& g, const Hit& h) {
    float tk;
    const bool inside = dda_step(q.tmax, q.cell, q.rcp, g.cs, g.res, &tk);
    q.tentry = tk;
    return h.t > tk && inside;
}

// From the current top cell, walk to the first non-empty one and enter it; false if the
// ray leaves the grid (or is done) first.  OCC: test each cell's occupancy bit first and
// load the cell record only for a cell with references (long incoherent rays, which cross
// mostly empty cells whose records would miss in L1: the path tracer).
template <bool STATS, bool OCC = false>
__device__ __forceinline__ bool tl_seek(TL& q, const Scene& s, const G& g, f3 o, f3 d, Hit& h) {
    const uint32_t rx = (uint32_t)g.res[0], rxy = (uint32_t)g.res[0] * (uint32_t)g.res[1];
    while (true) {
        const uint32_t c = (uint32_t)q.cell[0] + (uint32_t)q.cell[1] * rx + (uint32_t)q.cell[2] * rxy;
        if (STATS) h.cells++;
        bool full = true;
        if (OCC && s.occ) {
            const uint32_t bit = s.occ_bit0 + c;
            full = ((__ldg(s.occ + (bit >> 5)) >> (bit & 31u)) & 1u) != 0u;
        }
        if (full) {
            const uint2 tc = __ldg(s.cells + c);
            if (tc.y & kNotEmptyMask) {
                tl_enter(q, g, o, d, tc);
                return true;
            }
        }
        if (!tl_outer_step(q, g, h)) return false;
    }
}

// index of the current leaf: first leaf of the top cell + x + rx * (y + ry * z)
__device__ __forceinline__ uint32_t tl_leaf(const TL& q) {
    return q.lbase + (uint32_t)q.c2[0] + q.lres[0] * (uint32_t)q.c2[1] + q.lres[0] * q.lres[1] * (uint32_t)q.c2[2];
}

// Inner step (TLGridTraverser.h:225-290): stop when the hit lies before the leaf's exit,
// else step; leaving the sub-grid continues in the top grid.  False when the ray is done.
// KL > 1: an empty next leaf (no list to test) is stepped over at once, up to KL leaves.
template <bool STATS, bool OCC = false, int KL = 1>
__device__ __forceinline__ bool tl_advance(TL& q, const Scene& s, const G& g, f3 o, f3 d, Hit& h) {
    const int32_t lres[3] = {(int32_t)q.lres[0], (int32_t)q.lres[1], (int32_t)q.lres[2]};
    for (int j = 1;; ++j) {
        float tk;
        const bool inside = dda_step(q.tm2, q.c2, q.rcp, q.scs, lres, &tk);
        if (h.t < tk) return false;
        if (!inside) return tl_outer_step(q, g, h) && tl_seek<STATS, OCC>(q, s, g, o, d, h);
        if (j >= KL) return true;
        const uint2 lr = __ldg(s.leaves + tl_leaf(q));
        if (lr.y > lr.x) return true;
        if (STATS) h.cells++;
    }
}

// Entry of a ray into the two-level grid (TLGridTraverser.h:79-143): clip to the grid
// box, the top cell at the entry point, then the first non-empty top cell entered; false
// if the ray misses the grid or leaves it (or is done) before a non-empty cell.  Per lane.
template <bool STATS, bool OCC = false>
__device__ __forceinline__ bool tl_setup(TL& q, const Scene& s, const G& g, f3 o, f3 d, Hit& h) {
    q.rcp[0] = 1.0f / d.x; q.rcp[1] = 1.0f / d.y; q.rcp[2] = 1.0f / d.z;
    float t0, t1;
    if (!clip(g, o, q.rcp, &t0, &t1)) return false;
    q.tentry = hmax(0.0f, t0);
    const f3 ep = mk(o.x + q.tentry * d.x, o.y + q.tentry * d.y, o.z + q.tentry * d.z);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float cf = floorf((comp(ep, k) - g.bmin[k]) * g.rcp[k]);
        cf = hmin((float)g.res[k] - 1.0f, hmax(cf, 0.0f));
        const float stp = q.rcp[k] > 0.0f ? 1.0f : 0.0f;
        q.tmax[k] = ((cf + stp) * g.cs[k] + g.bmin[k] - comp(o, k)) * q.rcp[k];
        q.cell[k] = f2i(cf);
    }
    if (!(q.cell[0] < g.res[0] && q.cell[0] > -1 && q.cell[1] < g.res[1] && q.cell[1] > -1 &&
          q.cell[2] < g.res[2] && q.cell[2] > -1))
        return false;
    return tl_seek<STATS, OCC>(q, s, g, o, d, h);
}

// a15: two-level DDA, warp-synchronous
#ifndef HR_RAY_LEAF_STEPS
#define HR_RAY_LEAF_STEPS 1   // camera and query rays of trace_tl: empty leaves stepped over per warp step
#endif
template <int HM, bool STATS, bool OCC = false>
__device__ void trace_tl(const Scene& s, const G& g, f3 o, f3 d, bool any, Hit& h, bool active) {
    TL q;
    if (active) active = tl_setup<STATS, OCC>(q, s, g, o, d, h);
    while (__any_sync(kFullMask, active)) {
        uint32_t b = 0, e = 0;
        if (active) {
            const uint2 lr = __ldg(s.leaves + tl_leaf(q));
            b = lr.x; e = lr.y;
            if (STATS) h.cells++;
        }
        const bool done = test_lists<HM, STATS>(s, o, d, b, e, any, h);
        if (active) active = !done && tl_advance<STATS, OCC, HR_RAY_LEAF_STEPS>(q, s, g, o, d, h);
    }
}

// Paced two-level traversal, for path and shadow rays.  A lane walking empty top cells
// takes at most K of them per warp step (and per call below), so one long walk does not
// hold back the other lanes' leaf steps and list tests; each lane's own sequence of cells
// and tests is unchanged, so the results are those of the unbounded walk.  Lane state: 0
// done, 1 in a leaf, 2 walking empty top cells.  (Camera, AO and query rays keep the
// unbounded walk of trace_tl: paced, they measured slower.)
#ifndef HR_PT_SEEK_STEPS
#define HR_PT_SEEK_STEPS 3   // path and shadow rays: empty top cells per warp step (0: unbounded)
#endif
#ifndef HR_PT_LEAF_STEPS
#define HR_PT_LEAF_STEPS 4   // path and shadow rays: leaves stepped per warp step while they are empty
#endif

// tl_seek with at most K steps over empty top cells: 1 entered a non-empty cell, 0 done
// (left the grid, or the hit lies before the next cell), 2 stopped at a top cell not yet
// looked at (the next call starts there).
template <bool STATS, bool OCC, int K>
__device__ __forceinline__ int tl_seek_n(TL& q, const Scene& s, const G& g, f3 o, f3 d, Hit& h) {
    const uint32_t rx = (uint32_t)g.res[0], rxy = (uint32_t)g.res[0] * (uint32_t)g.res[1];
    for (int i = 0;; ++i) {
        const uint32_t c = (uint32_t)q.cell[0] + (uint32_t)q.cell[1] * rx + (uint32_t)q.cell[2] * rxy;
        if (STATS) h.cells++;
        bool full = true;
        if (OCC && s.occ) {
            const uint32_t bit = s.occ_bit0 + c;
            full = ((__ldg(s.occ + (bit >> 5)) >> (bit & 31u)) & 1u) != 0u;
        }
        if (full) {
            const uint2 tc = __ldg(s.cells + c);
            if (tc.y & kNotEmptyMask) {
                tl_enter(q, g, o, d, tc);
                return 1;
            }
        }
        if (!tl_outer_step(q, g, h)) return 0;
        if (i + 1 >= K) return 2;
    }
}

// tl_setup, paced: the lane state after entering the grid
template <bool STATS, bool OCC, int K>
__device__ __forceinline__ int tl_setup_n(TL& q, const Scene& s, const G& g, f3 o, f3 d, Hit& h) {
    q.rcp[0] = 1.0f / d.x; q.rcp[1] = 1.0f / d.y; q.rcp[2] = 1.0f / d.z;
    float t0, t1;
    if (!clip(g, o, q.rcp, &t0, &t1)) return 0;
    q.tentry = hmax(0.0f, t0);
    const f3 ep = mk(o.x + q.tentry * d.x, o.y + q.tentry * d.y, o.z + q.tentry * d.z);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float cf = floorf((comp(ep, k) - g.bmin[k]) * g.rcp[k]);
        cf = hmin((float)g.res[k] - 1.0f, hmax(cf, 0.0f));
        const float stp = q.rcp[k] > 0.0f ? 1.0f : 0.0f;
        q.tmax[k] = ((cf + stp) * g.cs[k] + g.bmin[k] - comp(o, k)) * q.rcp[k];
        q.cell[k] = f2i(cf);
    }
    if (!(q.cell[0] < g.res[0] && q.cell[0] > -1 && q.cell[1] < g.res[1] && q.cell[1] > -1 &&
          q.cell[2] < g.res[2] && q.cell[2] > -1))
        return 0;
    return tl_seek_n<STATS, OCC, K>(q, s, g, o, d, h);
}

// The lane state after a warp step: a lane in a leaf (st 1) whose list test ended the ray
// (done) stops, else steps to the next leaf (tl_advance); a walking lane (st 2) walks on.
template <bool STATS, bool OCC, int K>
__device__ __forceinline__ int tl_next(TL& q, const Scene& s, const G& g, f3 o, f3 d, Hit& h, int st, bool done) {
    if (st == 1) {
        if (done) return 0;
        const int32_t lres[3] = {(int32_t)q.lres[0], (int32_t)q.lres[1], (int32_t)q.lres[2]};
        for (int j = 1;; ++j) {
            float tk;
            const bool inside = dda_step(q.tm2, q.c2, q.rcp, q.scs, lres, &tk);
            if (h.t < tk) return 0;
            if (!inside) return tl_outer_step(q, g, h) ? tl_seek_n<STATS, OCC, K>(q, s, g, o, d, h) : 0;
            if (j >= HR_PT_LEAF_STEPS) return 1;
            // an empty leaf has no list to test: step over it within this warp step
            const uint2 lr = __ldg(s.leaves + tl_leaf(q));
            if (lr.y > lr.x) return 1;
            if (STATS) h.cells++;
        }
    }
    if (st == 2) return tl_seek_n<STATS, OCC, K>(q, s, g, o, d, h);
    return 0;
}

// a15, paced (trace_tl's results)
template <int HM, bool STATS, bool OCC, int K>
__device__ void trace_tl_paced(const Scene& s, const G& g, f3 o, f3 d, bool any, Hit& h, bool active) {
    TL q;
    int st = active ? tl_setup_n<STATS, OCC, K>(q, s, g, o, d, h) : 0;
    while (__any_sync(kFullMask, st != 0)) {
        uint32_t b = 0, e = 0;
        if (st == 1) {
            const uint2 lr = __ldg(s.leaves + tl_leaf(q));
            b = lr.x; e = lr.y;
            if (STATS) h.cells++;
        }
        const bool done = test_lists<HM, STATS>(s, o, d, b, e, any, h);
        st = tl_next<STATS, OCC, K>(q, s, g, o, d, h, st, done);
    }
}

// Closest hit (ANY = false) or any hit within (1e-4, tmax) on a grid of kind KIND
// (kUniform or kTwoLevel).  The kind is a template argument so that a kernel holds the
// registers of one traversal only.  Warp-synchronous.
template <int KIND, bool ANY, bool STATS>
__device__ __forceinline__ void trace_one(const Scene& s, const G& g, f3 o, f3 d, float tmax, Hit& h, bool active) {
    h.t = tmax; h.u = 0.0f; h.v = 0.0f; h.tri = 0; h.hit = false; h.cells = 0; h.tests = 0;
    if (s.ntri == 0) return;
    constexpr int HM = ANY ? kHitAny : kHitClosest;
    if (KIND == kUniform) trace_ug<HM, STATS>(s, g, o, d, false, h, active);
    else trace_tl<HM, STATS>(s, g, o, d, false, h, active);
}

// As trace_one, with the hit mode chosen per lane: any hit where `any` is set, closest
// hit elsewhere (one traversal for the path and the shadow rays of a warp's lanes).  SEEK:
// empty top cells a lane walks per warp step (0: unbounded).
template <int KIND, bool STATS, int SEEK = HR_PT_SEEK_STEPS>
__device__ __forceinline__ void trace_mixed(const Scene& s, const G& g, f3 o, f3 d, float tmax, bool any, Hit& h,
                                            bool active) {
    h.t = tmax; h.u = 0.0f; h.v = 0.0f; h.tri = 0; h.hit = false; h.cells = 0; h.tests = 0;
    if (s.ntri == 0) return;
    if (KIND == kUniform) trace_ug<kHitMixed, STATS>(s, g, o, d, any, h, active);
    // path rays: occupancy bits
    else if constexpr (SEEK > 0) trace_tl_paced<kHitMixed, STATS, true, SEEK>(s, g, o, d, any, h, active);
    else trace_tl<kHitMixed, STATS, true>(s, g, o, d, any, h, active);
}

struct Cam {
    float pos[3], tl[3], sx[3], sy[3];
    int32_t w, h;
};

// pixel-centre ray, normalised (Camera.h:66-69 getDirection)
__device__ __forceinline__ f3 primary_dir(const Cam& c, uint32_t pix) {
    const float px = (float)(pix % (uint32_t)c.w) + 0.5f;
    const float py = (float)(pix / (uint32_t)c.w) + 0.5f;
    f3 d;
    d.x = c.tl[0] + px * c.sx[0] + py * c.sy[0];
    d.y = c.tl[1] + px * c.sx[1] + py * c.sy[1];
    d.z = c.tl[2] + px * c.sx[2] + py * c.sy[2];
    return normalize(d);
}

// Camera ray of render mode 0 for progressive image `image_id` (RTEngine.cu:409-424):
// images 0-3 take the 2 x 2 regular in-pixel pattern (RegularPixelSampler<2,2>,
// Camera.h:75-98), later ones a Gaussian offset around the pixel's corner
// (GaussianPixelSampler, Camera.h:116-132) from two PCG32 draws keyed by (image, pixel,
// seed); normalised.
__device__ __forceinline__ f3 primary_sample_dir(const Cam& c, uint32_t pix, int32_t image_id, uint64_t seed) {
    float ox, oy;
    if (image_id < 4) {
        const float tmp = (float)(image_id % 4) / 2.0f;
        oy = (truncf(tmp) + 0.5f) / 2.0f;
        ox = tmp - truncf(tmp) + 0.5f / 2.0f;
    } else {
        Pcg32 r;
        pcg_seed(r, ((uint64_t)(uint32_t)image_id << 32) | pix, seed);
        const float u1 = pcg_float(r), u2 = pcg_float(r);
        const float rad = 0.5f * sqrtf(-log_series(1.0f - u1));
        float sn, cs;
        sincos2pi(u2, &sn, &cs);
        ox = rad * cs;
        oy = rad * sn;
    }
    const float px = (float)(pix % (uint32_t)c.w) + ox;
    const float py = (float)(pix / (uint32_t)c.w) + oy;
    f3 d;
    d.x = c.tl[0] + px * c.sx[0] + py * c.sy[0];
    d.y = c.tl[1] + px * c.sx[1] + py * c.sy[1];
    d.z = c.tl[2] + px * c.sx[2] + py * c.sy[2];
    return normalize(d);
}

// simpleShade (SimpleIntegrator.h:41-126) of a hit: weights u = |(v1 - o) x (v2 - o)| / |N|,
// v = |(v2 - o) x (v0 - o)| / |N| (N the triangle's edge cross product, o the ray origin) as
// the colour (u, v, 1 - u - v), times |cos| between the unit normal and the unit direction;
// background (0.15, 0.2, 0.3) on a miss.
__device__ __forceinline__ void simple_shade(const Scene& s, bool hit, uint32_t tri, f3 o, f3 d, float* rgb) {
    if (!hit) {
        rgb[0] = 0.15f; rgb[1] = 0.2f; rgb[2] = 0.3f;
        return;
    }
    f3 p[3];
    tri_fetch(s.tris, tri, p);
    const f3 nr = cross(sub(p[1], p[0]), sub(p[2], p[0]));
    const f3 a0 = sub(p[0], o), a1 = sub(p[1], o), a2 = sub(p[2], o);
    const f3 n0 = cross(a1, a2), n1 = cross(a2, a0);
    const float inv = 1.0f / sqrtf(dot(nr, nr));
    const float u = sqrtf(dot(n0, n0)) * inv;
    const float v = sqrtf(dot(n1, n1)) * inv;
    const f3 nrm = normalize(nr);
    const f3 dn = normalize(d);
    const float cs = fmaxf(0.0f, fabsf(dot(mk(-nrm.x, -nrm.y, -nrm.z), dn)));
    rgb[0] = u * cs;
    rgb[1] = v * cs;
    rgb[2] = (1.0f - u - v) * cs;
}

__device__ __forceinline__ f3 face_normal(const Scene& s, uint32_t tri, f3 d) {
    f3 p[3];
    tri_fetch(s.tris, tri, p);
    f3 n = normalize(cross(sub(p[1], p[0]), sub(p[2], p[0])));
    if (dot(n, d) > 0.0f) n = mk(-n.x, -n.y, -n.z);
    return n;
}

// Shading normal of a path tracer hit (PathTracer.h:111-136): the triangle's vertex normals
// blended with the weights simpleShade forms from the ray origin (u of vertex 0, v of
// vertex 1, 1 - u - v of vertex 2), normalised, and turned to face the ray as the
// geometric normal is.
__device__ __forceinline__ f3 shading_normal(const Scene& s, uint32_t tri, f3 o, f3 d) {
    f3 p[3];
    tri_fetch(s.tris, tri, p);
    const f3 nr = cross(sub(p[1], p[0]), sub(p[2], p[0]));
    const f3 a0 = sub(p[0], o), a1 = sub(p[1], o), a2 = sub(p[2], o);
    const f3 n0 = cross(a1, a2), n1 = cross(a2, a0);
    const float inv = 1.0f / sqrtf(dot(nr, nr));
    const float u = sqrtf(dot(n0, n0)) * inv;
    const float v = sqrtf(dot(n1, n1)) * inv;
    const float w = 1.0f - u - v;
    const float4* q = s.nrm3 + 3 * (size_t)tri;
    const float4 m0 = __ldg(q), m1 = __ldg(q + 1), m2 = __ldg(q + 2);
    f3 n = mk(u * m0.x + v * m1.x + w * m2.x, u * m0.y + v * m1.y + w * m2.y, u * m0.z + v * m1.z + w * m2.z);
    n = normalize(n);
    if (dot(n, d) > 0.0f) n = mk(-n.x, -n.y, -n.z);
    return n;
}

__device__ __forceinline__ float blend(float old, float val, int32_t image_id) {
    const float nw = 1.0f / (float)(image_id + 1);
    const float ow = 1.0f - nw;
    return old * ow + val * nw;   // AOIntegrator.h:168-175 progressive average
}

constexpr int kTT = 128;

// Camera rays are issued in warp-sized 8x4 pixel tiles: the 32 rays of a warp start from
// the same point into a small solid angle and walk nearly the same cells.
__device__ __forceinline__ uint32_t tile_slots(const Cam& c) {
    return (((uint32_t)c.w + 7u) / 8u) * (((uint32_t)c.h + 3u) / 4u) * 32u;
}
__device__ __forceinline__ bool tile_pixel(const Cam& c, uint32_t slot, uint32_t* pix) {
    const uint32_t tile = slot >> 5, lane = slot & 31u;
    const uint32_t tx = ((uint32_t)c.w + 7u) / 8u;
    const uint32_t x = (tile % tx) * 8u + (lane & 7u), y = (tile / tx) * 4u + (lane >> 3);
    *pix = y * (uint32_t)c.w + x;
    return x < (uint32_t)c.w && y < (uint32_t)c.h;
}

// Device counters (uint64 words): [0] rays, [2] cells, [3] triangle tests of the primary
// pass; [4] rays, [5] cells, [6] tests of the secondary pass (AO samples, shadow rays);
// word 1 holds the index check of the last upload, word 7 the AO hit-pixel queue length
// (or the path tracer's tile pool) and the AO sample pool, word 8 the AO camera-ray pool.
template <bool STATS>
__device__ __forceinline__ void add_rays(unsigned long long* counter, bool secondary, uint32_t rays, uint32_t cells = 0,
                                         uint32_t tests = 0) {
    unsigned long long r = rays, c = cells, t = tests;
    for (int o = 16; o > 0; o >>= 1) {
        r += __shfl_xor_sync(kFullMask, r, o);
        if (STATS) {
            c += __shfl_xor_sync(kFullMask, c, o);
            t += __shfl_xor_sync(kFullMask, t, o);
        }
    }
    if ((threadIdx.x & 31) == 0 && counter) {
        unsigned long long* base = counter + (secondary ? 4 : 0);
        if (r) atomicAdd(base, r);
        if (STATS) {
            atomicAdd(secondary ? counter + 5 : counter + 2, c);
            atomicAdd(secondary ? counter + 6 : counter + 3, t);
        }
    }
}

// warp-uniform bound of a 1-D grid-stride loop over n items
__device__ __forceinline__ uint32_t round32(uint32_t n) { return (n + 31u) & ~31u; }

// constants of the path tracer for one grid and light collection
struct PtConsts {
    const LightSet* ls;   // device memory
    uint32_t nlights;
    float a_pi, albedo, ray_eps;
    int32_t bounces;
};
__device__ __forceinline__ PtConsts pt_consts(const G& g, const LightSet* ls, int32_t bounces, float albedo,
                                              float eps_frac) {
    PtConsts k;
    const f3 dd = mk(g.bmax[0] - g.bmin[0], g.bmax[1] - g.bmin[1], g.bmax[2] - g.bmin[2]);
    k.ray_eps = eps_frac * sqrtf(dot(dd, dd));
    k.ls = ls;
    k.nlights = __ldg(&ls->count);
    k.a_pi = albedo * 0.318309886f;
    k.albedo = albedo;
    k.bounces = bounces;
    return k;
}

__device__ __forceinline__ f3 ldf3(const float* p) { return mk(__ldg(p), __ldg(p + 1), __ldg(p + 2)); }

// distance along (o, d) to the emitting side of light q, or -1 when the ray misses it
__device__ __forceinline__ float light_hit(const LightQ* q, f3 o, f3 d) {
    const f3 n = ldf3(q->n);
    const float den = dot(d, n);
    if (!(den < 0.0f)) return -1.0f;
    const f3 c = ldf3(q->c);
    const float tl = dot(sub(c, o), n) / den;
    const f3 r = sub(mk(o.x + tl * d.x, o.y + tl * d.y, o.z + tl * d.z), c);
    const f3 nc = ldf3(q->nc);
    const float inv_nn = __ldg(&q->inv_nn);
    const float a = dot(cross(r, ldf3(q->e2)), nc) * inv_nn;
    const float b = dot(cross(ldf3(q->e1), r), nc) * inv_nn;
    return (a >= 0.0f && a <= 1.0f && b >= 0.0f && b <= 1.0f) ? tl : -1.0f;
}

// AreaLightSourceCollection::getLight (LightSource.hpp:114-126): the first light whose
// normalised running weight exceeds u, else the last
__device__ __forceinline__ uint32_t light_pick(const LightSet* ls, uint32_t n, float u) {
    const float total = __ldg(&ls->cdf[n - 1]);
    for (uint32_t i = 0; i + 1 < n; ++i)
        if (u < __ldg(&ls->cdf[i]) / total) return i;
    return n - 1;
}

struct PtCounts {
    uint32_t rays = 0, cells = 0, tests = 0, srays = 0, scells = 0, stests = 0;
};

// State of one path of the path tracer (PathTracer.h:41-372 structure).  A bounce takes
// two traversals, the path ray (closest hit) and then, if the light sample faces both
// surfaces, its shadow ray (any hit); `shadow` says which one the lane traces next.
struct PathState {
    f3 o, d;          // the ray traced next: the path ray, or the shadow ray while `shadow`
    f3 no, nd;        // while `shadow`: the path's continuation ray
    float L, beta;
    float c;          // while `shadow`: the light sample's radiance if the shadow ray is free
    float tmax;       // FLT_MAX for the path ray, the distance to the light sample for the shadow ray
    Pcg32 rng;
    int32_t bounce;
    bool shadow, last;   // last: the path ends after the shadow ray
};

// A path from the centre of pixel pix; its PCG32 stream is keyed by (image_id, pix) and seed.
__device__ __forceinline__ void path_begin(PathState& p, const Cam& cam, uint32_t pix, int32_t image_id,
                                           uint64_t seed) {
    pcg_seed(p.rng, ((uint64_t)(uint32_t)image_id << 32) | pix, seed);
    p.o = mk(cam.pos[0], cam.pos[1], cam.pos[2]);
    p.d = primary_dir(cam, pix);
    p.L = 0.0f;
    p.beta = 1.0f;
    p.tmax = FLT_MAX;
    p.bounce = 0;
    p.shadow = false;
}

// One traversal of each lane's next ray: a warp traces path rays and shadow rays together
// (trace_mixed), so lanes whose light sample needs no shadow ray do not idle while the
// others trace theirs.  Per path the operations are those of the sequential bounce loop:
// the closest hit (at bounce 0 first the camera ray against the quad light), one
// next-event sample of the light (u1, u2) whose shadow ray runs to dist - ray_eps, and a
// cosine-weighted continuation (u3, u4) with throughput x albedo; the light sample's
// radiance, formed with the throughput before the albedo factor, is added when its shadow
// ray comes back free.  Returns true while the path goes on (it ends on a miss, on hitting
// the light, or after k.bounces bounces); p.L is then its radiance.  Warp-synchronous: all
// lanes call it, lanes without a path pass alive = false.  SEEK as in trace_mixed.
template <int KIND, bool STATS, int SEEK = HR_PT_SEEK_STEPS>
__device__ __forceinline__ bool path_step(const Scene& s, const G& g, const PtConsts& k, PathState& p, bool alive,
                                          PtCounts& n) {
    if (k.bounces <= 0) return false;   // no bounce: radiance 0 (uniform over the warp)
    Hit h;
    trace_mixed<KIND, STATS, SEEK>(s, g, p.o, p.d, p.tmax, p.shadow, h, alive);
    if (!alive) return false;
    if (p.shadow) {
        n.srays += 1;
        n.scells += h.cells;
        n.stests += h.tests;
        if (!h.hit) p.L = p.L + p.c;
        p.shadow = false;
        if (p.last) return false;
        p.o = p.no;
        p.d = p.nd;
        p.tmax = FLT_MAX;
        return true;
    }
    n.rays += 1;
    n.cells += h.cells;
    n.tests += h.tests;
    if (p.bounce == 0) {
        // camera ray against the emitters: the nearest one in front of the hit ends the path
        float best = h.t;
        int32_t lit = -1;
        for (uint32_t j = 0; j < k.nlights; ++j) {
            const float tl = light_hit(&k.ls->q[j], p.o, p.d);
            if (tl > kIsectEps && tl < best) { best = tl; lit = (int32_t)j; }
        }
        if (lit >= 0) {
            p.L = p.L + __ldg(&k.ls->q[lit].emission);
            return false;
        }
    }
    if (!h.hit) return false;
    const f3 q = mk(p.o.x + h.t * p.d.x, p.o.y + h.t * p.d.y, p.o.z + h.t * p.d.z);
    f3 nrm = face_normal(s, h.tri, p.d);
    if (s.nrm3) nrm = shading_normal(s, h.tri, p.o, p.d);
    const float alb = s.alb ? __ldg(s.alb + h.tri) : k.albedo;
    const float a_pi = s.alb ? alb * 0.318309886f : k.a_pi;
    // next-event estimation: one light of the collection (by weight when there are several;
    // its radiance divided by the probability of picking it), one point on it
    uint32_t li = 0;
    if (k.nlights > 1) li = light_pick(k.ls, k.nlights, pcg_float(p.rng));
    const LightQ* lq = &k.ls->q[li];
    const f3 lc = ldf3(lq->c), le1 = ldf3(lq->e1), le2 = ldf3(lq->e2);
    const float u1 = pcg_float(p.rng), u2 = pcg_float(p.rng);
    const f3 lp = mk(lc.x + u1 * le1.x + u2 * le2.x, lc.y + u1 * le1.y + u2 * le2.y, lc.z + u1 * le1.z + u2 * le2.z);
    f3 wi = sub(lp, q);
    const float dist2 = dot(wi, wi);
    const float dist = sqrtf(dist2);
    wi = mulf(wi, 1.0f / dist);
    const float cos_s = dot(nrm, wi);
    const float cos_l = -dot(ldf3(lq->n), wi);
    const bool shadow = cos_s > 0.0f && cos_l > 0.0f;
    if (shadow) {
        p.c = p.beta * a_pi * __ldg(&lq->emission) * cos_s * cos_l * __ldg(&lq->area) / dist2;
        if (k.nlights > 1) p.c = p.c * (__ldg(&k.ls->cdf[k.nlights - 1]) / (__ldg(&lq->area) * __ldg(&lq->emission)));
    }
    p.beta = p.beta * alb;
    const float u3 = pcg_float(p.rng), u4 = pcg_float(p.rng);
    const f3 nd = cosine_dir(nrm, u3, u4);
    const f3 no = mk(q.x + k.ray_eps * nd.x, q.y + k.ray_eps * nd.y, q.z + k.ray_eps * nd.z);
    p.bounce += 1;
    const bool more = p.bounce < k.bounces;
    if (shadow) {
        p.no = no;
        p.nd = nd;
        p.last = !more;
        p.o = mk(q.x + k.ray_eps * wi.x, q.y + k.ray_eps * wi.y, q.z + k.ray_eps * wi.z);
        p.d = wi;
        p.tmax = dist - k.ray_eps;
        p.shadow = true;
        return true;
    }
    if (!more) return false;
    p.o = no;
    p.d = nd;
    return true;
}

// Lanes of a warp take pixels from a pool of 32-pixel tiles and run `spp` paths per pixel,
// one ray per lane per step (path_step); a lane whose path ends starts the pixel's
// next path (image id + 1) or takes the next pixel, so the warp stays full until the pool
// runs dry.  The per-pixel result is the progressive blend of its paths in image-id order,
// the same values as spp one-path frames.
struct PathLane {
    PathState p;
    uint32_t pix = 0;
    int32_t sample = 0;
    float val = 0.0f;
    bool has = false;
};

// Fill the lanes without a path from tile `tile` starting at slot *next (tile pixels as
// tile_pixel); advances *next.  Returns the lanes still without a path.
__device__ __forceinline__ uint32_t path_refill(PathLane& ln, const Cam& cam, uint32_t tile, uint32_t* next,
                                               int32_t image_id, uint64_t seed, const float* __restrict__ fb) {
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t need = __ballot_sync(kFullMask, !ln.has);
    while (need && *next < 32u) {
        const uint32_t rank = __popc(need & ((1u << lane) - 1u));
        const uint32_t take = min((uint32_t)__popc(need), 32u - *next);
        if (!ln.has && rank < take) {
            uint32_t q;
            if (tile_pixel(cam, tile * 32u + *next + rank, &q)) {
                ln.pix = q;
                ln.has = true;
                ln.sample = 0;
                ln.val = fb[3 * (size_t)q];
                path_begin(ln.p, cam, q, image_id, seed);
            }
        }
        *next += take;
        need = __ballot_sync(kFullMask, !ln.has);
    }
    return need;
}

// After a step: a lane whose path ended blends it in and starts the pixel's next path, or
// writes the pixel and frees itself.
__device__ __forceinline__ void path_retire(PathLane& ln, bool cont, const Cam& cam, int32_t image_id, int32_t spp,
                                            uint64_t seed, float* __restrict__ fb) {
    if (!ln.has || cont) return;
    const int32_t im = image_id + ln.sample;
    ln.val = blend(ln.val, ln.p.L, im);
    ln.sample += 1;
    if (ln.sample < spp) {
        path_begin(ln.p, cam, ln.pix, im + 1, seed);
        return;
    }
    float* o = fb + 3 * (size_t)ln.pix;
    o[0] = ln.val; o[1] = ln.val; o[2] = ln.val;
    ln.has = false;
}

}  // namespace
}  // namespace hr
