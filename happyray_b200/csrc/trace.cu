// trace.cu -- grid traversal (uniform and two-level 3D-DDA), Moller-Trumbore
// intersection and the primary / ambient-occlusion / path-tracing integrators.
//
// Reference path (javorkk/happyray):
//   uniform DDA            src/RT/Algorithm/UGridTraverser.h:44-177
//   two-level DDA          src/RT/Algorithm/TLGridTraverser.h:45-354
//   intersector            src/RT/Algorithm/RayTriangleIntersector.h:38-92
//   trace kernel           src/RT/Algorithm/RayTracingKernels.h:47-152
//   camera                 src/RT/Primitive/Camera.h:35-72
//   primary shading        src/RT/Integrator/SimpleIntegrator.h:41-126
//   ambient occlusion      src/RT/Integrator/AOIntegrator.h:64-191, 234-351; RayGenerators.h:286-342
//   path tracing           src/RT/Integrator/PathTracer.h:41-372
//
// Differences in arithmetic (all deterministic, bit-identical to the oracle):
//   * rays keep the direction and its IEEE reciprocal; the intersector and the entry
//     points use the direction itself instead of re-deriving it with __fdividef;
//   * primary ray directions are normalised, so t is a distance;
//   * no fast-math: IEEE division / square root, no FMA contraction.
#include "hr_internal.h"
#include "hr_block.cuh"

namespace hr {

namespace {

struct Scene {
    const float4* __restrict__ v;
    const uint32_t* __restrict__ idx;
    const uint2* __restrict__ cells;
    const uint2* __restrict__ leaves;
    const uint32_t* __restrict__ prims;
    const GridDesc* desc;
    uint32_t ntri;
    int32_t kind;
};

struct G {
    float bmin[3], bmax[3], cs[3], rcp[3];
    int32_t res[3];
};
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

// a16: Moller-Trumbore over prims[b, e); first-tested wins ties (strict <)
template <bool ANY, bool STATS>
__device__ __forceinline__ bool isect_range(const Scene& s, f3 o, f3 d, uint32_t b, uint32_t e, Hit& h) {
    for (uint32_t it = b; it < e; ++it) {
        const uint32_t tri = __ldg(s.prims + it);
        f3 p[3];
        tri_load(s.v, s.idx, tri, p);
        const f3 e1 = sub(p[1], p[0]), e2 = sub(p[2], p[0]);
        const f3 pv = cross(d, e2);
        const float det = dot(e1, pv);
        const float inv = 1.0f / det;
        const f3 sv = sub(o, p[0]);
        const float u = dot(sv, pv) * inv;
        const f3 q = cross(sv, e1);
        const float v = dot(q, d) * inv;
        const float t = dot(e2, q) * inv;
        if (STATS) h.tests++;
        if (u >= 0.0f && v >= 0.0f && u + v <= 1.0f && t > kIsectEps && t < h.t) {
            h.t = t; h.u = u; h.v = v; h.tri = tri; h.hit = true;
            if (ANY) return true;
        }
    }
    return false;
}

__device__ __forceinline__ int min_dim(float a, float b, float c) { return a < b ? (a < c ? 0 : 2) : (b < c ? 1 : 2); }

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

// a14: uniform grid DDA (UGridTraverser.h:76-172)
template <bool ANY, bool STATS>
__device__ void trace_ug(const Scene& s, const G& g, f3 o, f3 d, Hit& h) {
    float rcp[3] = {1.0f / d.x, 1.0f / d.y, 1.0f / d.z};
    float t0, t1;
    if (!clip(g, o, rcp, &t0, &t1)) return;
    f3 ep = o;
    if (t0 >= 0.0f) {
        const float te = t0 + kEps;
        ep = mk(o.x + te * d.x, o.y + te * d.y, o.z + te * d.z);
    }
    float tmax[3];
    int32_t cell[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float cf = floorf((comp(ep, k) - g.bmin[k]) * g.rcp[k]);
        cf = hmin((float)g.res[k] - 1.0f, hmax(cf, 0.0f));
        const float stp = rcp[k] > 0.0f ? 1.0f : 0.0f;
        tmax[k] = ((cf + stp) * g.cs[k] + g.bmin[k] - comp(o, k)) * rcp[k];
        cell[k] = f2i(cf);
    }
    bool active = cell[0] < g.res[0] && cell[0] > -1 && cell[1] < g.res[1] && cell[1] > -1 &&
                  cell[2] < g.res[2] && cell[2] > -1;
    const uint32_t rx = (uint32_t)g.res[0], rxy = (uint32_t)g.res[0] * (uint32_t)g.res[1];
    while (active) {
        const uint32_t c = (uint32_t)cell[0] + (uint32_t)cell[1] * rx + (uint32_t)cell[2] * rxy;
        const uint2 cr = __ldg(s.cells + c);
        if (STATS) h.cells++;
        if (isect_range<ANY, STATS>(s, o, d, cr.x, cr.y, h)) return;
        const int k = min_dim(tmax[0], tmax[1], tmax[2]);
        active = h.t > tmax[k];
        cell[k] += rcp[k] > 0.0f ? 1 : -1;
        tmax[k] += g.cs[k] * fabsf(rcp[k]);
        active = active && cell[k] < g.res[k] && cell[k] > -1;
    }
}

// a15: two-level DDA (TLGridTraverser.h:79-349)
template <bool ANY, bool STATS>
__device__ void trace_tl(const Scene& s, const G& g, f3 o, f3 d, Hit& h) {
    float rcp[3] = {1.0f / d.x, 1.0f / d.y, 1.0f / d.z};
    float t0, t1;
    if (!clip(g, o, rcp, &t0, &t1)) return;
    float tentry = hmax(0.0f, t0);
    const f3 ep = mk(o.x + tentry * d.x, o.y + tentry * d.y, o.z + tentry * d.z);
    float tmax[3];
    int32_t cell[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float cf = floorf((comp(ep, k) - g.bmin[k]) * g.rcp[k]);
        cf = hmin((float)g.res[k] - 1.0f, hmax(cf, 0.0f));
        const float stp = rcp[k] > 0.0f ? 1.0f : 0.0f;
        tmax[k] = ((cf + stp) * g.cs[k] + g.bmin[k] - comp(o, k)) * rcp[k];
        cell[k] = f2i(cf);
    }
    bool active = cell[0] < g.res[0] && cell[0] > -1 && cell[1] < g.res[1] && cell[1] > -1 &&
                  cell[2] < g.res[2] && cell[2] > -1;
    const uint32_t rx = (uint32_t)g.res[0], rxy = (uint32_t)g.res[0] * (uint32_t)g.res[1];
    while (active) {
        const uint32_t c = (uint32_t)cell[0] + (uint32_t)cell[1] * rx + (uint32_t)cell[2] * rxy;
        const uint2 tc = __ldg(s.cells + c);
        if (STATS) h.cells++;
        if (tc.y & kNotEmptyMask) {
            const uint32_t lres[3] = {tc.y & 0xFFu, (tc.y >> 8) & 0xFFu, (tc.y >> 16) & 0xFFu};
            const f3 e2 = mk(o.x + tentry * d.x, o.y + tentry * d.y, o.z + tentry * d.z);
            float scs[3], tm2[3];
            int32_t c2[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const float cres = (float)lres[k];
                const float srcp = g.rcp[k] * cres;
                const float mb = (float)cell[k] * g.cs[k] + g.bmin[k];
                float cf = floorf((comp(e2, k) - mb) * srcp);
                scs[k] = 1.0f / srcp;
                cf = hmin(cres - 1.0f, hmax(cf, 0.0f));
                const float stp = rcp[k] > 0.0f ? 1.0f : 0.0f;
                tm2[k] = ((cf + stp) * scs[k] + mb - comp(o, k)) * rcp[k];
                c2[k] = f2i(cf);
            }
            bool inner = true;
            while (inner) {
                const uint32_t li = tc.x + (uint32_t)c2[0] + lres[0] * (uint32_t)c2[1] + lres[0] * lres[1] * (uint32_t)c2[2];
                const uint2 lr = __ldg(s.leaves + li);
                if (STATS) h.cells++;
                if (isect_range<ANY, STATS>(s, o, d, lr.x, lr.y, h)) return;
                const int k = min_dim(tm2[0], tm2[1], tm2[2]);
                if (h.t < tm2[k]) { inner = false; active = false; }
                c2[k] += rcp[k] > 0.0f ? 1 : -1;
                tm2[k] += scs[k] * fabsf(rcp[k]);
                inner = inner && c2[k] != (int32_t)lres[k] && c2[k] != -1;
            }
        }
        if (active) {
            const int k = min_dim(tmax[0], tmax[1], tmax[2]);
            active = h.t > tmax[k];
            tentry = tmax[k];
            cell[k] += rcp[k] > 0.0f ? 1 : -1;
            tmax[k] += g.cs[k] * fabsf(rcp[k]);
            active = active && cell[k] != g.res[k] && cell[k] != -1;
        }
    }
}

template <bool ANY, bool STATS>
__device__ __forceinline__ void trace_one(const Scene& s, const G& g, f3 o, f3 d, float tmax, Hit& h) {
    h.t = tmax; h.u = 0.0f; h.v = 0.0f; h.tri = 0; h.hit = false; h.cells = 0; h.tests = 0;
    if (s.ntri == 0) return;
    if (s.kind == kUniform) trace_ug<ANY, STATS>(s, g, o, d, h);
    else trace_tl<ANY, STATS>(s, g, o, d, h);
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

__device__ __forceinline__ f3 face_normal(const Scene& s, uint32_t tri, f3 d) {
    f3 p[3];
    tri_load(s.v, s.idx, tri, p);
    f3 n = normalize(cross(sub(p[1], p[0]), sub(p[2], p[0])));
    if (dot(n, d) > 0.0f) n = mk(-n.x, -n.y, -n.z);
    return n;
}

__device__ __forceinline__ float blend(float old, float val, int32_t image_id) {
    const float nw = 1.0f / (float)(image_id + 1);
    const float ow = 1.0f - nw;
    return old * ow + val * nw;   // AOIntegrator.h:168-175 progressive average
}

constexpr int kTT = 128;

template <bool STATS>
__global__ __launch_bounds__(kTT) void k_trace_rays(Scene s, const float* __restrict__ org, const float* __restrict__ dir,
                                                    uint32_t n, int32_t* __restrict__ oid, float* __restrict__ ot,
                                                    float* __restrict__ ou, float* __restrict__ ov,
                                                    uint32_t* __restrict__ stats) {
    const G g = load_g(s.desc);
    for (uint32_t i = blockIdx.x * kTT + threadIdx.x; i < n; i += gridDim.x * kTT) {
        const f3 o = mk(__ldg(org + 3 * (size_t)i), __ldg(org + 3 * (size_t)i + 1), __ldg(org + 3 * (size_t)i + 2));
        const f3 d = mk(__ldg(dir + 3 * (size_t)i), __ldg(dir + 3 * (size_t)i + 1), __ldg(dir + 3 * (size_t)i + 2));
        Hit h;
        trace_one<false, STATS>(s, g, o, d, FLT_MAX, h);
        oid[i] = h.hit ? (int32_t)h.tri : -1;
        ot[i] = h.hit ? h.t : FLT_MAX;
        ou[i] = h.u;
        ov[i] = h.v;
        if (STATS) { stats[2 * (size_t)i] = h.cells; stats[2 * (size_t)i + 1] = h.tests; }
    }
}

template <bool STATS>
__global__ __launch_bounds__(kTT) void k_trace_primary(Scene s, Cam cam, int32_t* __restrict__ oid,
                                                       float* __restrict__ ot, float* __restrict__ ou,
                                                       float* __restrict__ ov, uint32_t* __restrict__ stats) {
    const G g = load_g(s.desc);
    const uint32_t n = (uint32_t)cam.w * (uint32_t)cam.h;
    const f3 o = mk(cam.pos[0], cam.pos[1], cam.pos[2]);
    for (uint32_t i = blockIdx.x * kTT + threadIdx.x; i < n; i += gridDim.x * kTT) {
        Hit h;
        trace_one<false, STATS>(s, g, o, primary_dir(cam, i), FLT_MAX, h);
        oid[i] = h.hit ? (int32_t)h.tri : -1;
        ot[i] = h.hit ? h.t : FLT_MAX;
        ou[i] = h.u;
        ov[i] = h.v;
        if (STATS) { stats[2 * (size_t)i] = h.cells; stats[2 * (size_t)i + 1] = h.tests; }
    }
}

__global__ __launch_bounds__(kTT) void k_occluded(Scene s, const float* __restrict__ org, const float* __restrict__ dir,
                                                  const float* __restrict__ tmax, uint32_t n, uint8_t* __restrict__ occ) {
    const G g = load_g(s.desc);
    for (uint32_t i = blockIdx.x * kTT + threadIdx.x; i < n; i += gridDim.x * kTT) {
        const f3 o = mk(org[3 * (size_t)i], org[3 * (size_t)i + 1], org[3 * (size_t)i + 2]);
        const f3 d = mk(dir[3 * (size_t)i], dir[3 * (size_t)i + 1], dir[3 * (size_t)i + 2]);
        Hit h;
        trace_one<true, false>(s, g, o, d, tmax[i], h);
        occ[i] = h.hit ? 1 : 0;
    }
}

// warp-aggregated counters: [0] rays traced, [2] cells visited, [3] triangle tests
template <bool STATS>
__device__ __forceinline__ void add_rays(unsigned long long* counter, uint32_t rays, uint32_t cells = 0,
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
        atomicAdd(counter, r);
        if (STATS) {
            atomicAdd(counter + 2, c);
            atomicAdd(counter + 3, t);
        }
    }
}

// mode 0: primary rays with barycentric false colour (SimpleIntegrator.h:41-126)
template <bool STATS>
__global__ __launch_bounds__(kTT) void k_render_primary(Scene s, Cam cam, int32_t image_id, float* __restrict__ fb,
                                                        unsigned long long* counter) {
    const G g = load_g(s.desc);
    const uint32_t n = (uint32_t)cam.w * (uint32_t)cam.h;
    const f3 o = mk(cam.pos[0], cam.pos[1], cam.pos[2]);
    const uint32_t nn = (n + kTT - 1) / kTT * kTT;
    for (uint32_t i = blockIdx.x * kTT + threadIdx.x; i < nn; i += gridDim.x * kTT) {
        uint32_t rays = 0, ncell = 0, ntest = 0;
        if (i < n) {
            const f3 d = primary_dir(cam, i);
            Hit h;
            trace_one<false, STATS>(s, g, o, d, FLT_MAX, h);
            rays = 1;
            ncell = h.cells;
            ntest = h.tests;
            float r = 0.15f, gg = 0.2f, b = 0.3f;
            if (h.hit) {
                const f3 nrm = face_normal(s, h.tri, d);
                const float cs = fabsf(dot(nrm, d));
                r = (1.0f - h.u - h.v) * cs; gg = h.u * cs; b = h.v * cs;
            }
            fb[3 * (size_t)i] = blend(fb[3 * (size_t)i], r, image_id);
            fb[3 * (size_t)i + 1] = blend(fb[3 * (size_t)i + 1], gg, image_id);
            fb[3 * (size_t)i + 2] = blend(fb[3 * (size_t)i + 2], b, image_id);
        }
        add_rays<STATS>(counter, rays, ncell, ntest);
    }
}

// mode 3: ambient occlusion (AOIntegrator.h:234-351, RayGenerators.h:286-342), with the
// configured sample count, radius alpha and a PCG32 stream per (image, pixel, seed)
template <bool STATS>
__global__ __launch_bounds__(kTT) void k_render_ao(Scene s, Cam cam, int32_t spp, float alpha_frac, float alpha_abs,
                                                   uint64_t seed, int32_t image_id, float* __restrict__ fb,
                                                   unsigned long long* counter) {
    const G g = load_g(s.desc);
    float alpha = alpha_abs;
    if (!(alpha > 0.0f)) {
        const f3 dd = mk(g.bmax[0] - g.bmin[0], g.bmax[1] - g.bmin[1], g.bmax[2] - g.bmin[2]);
        alpha = alpha_frac * sqrtf(dot(dd, dd));
    }
    const float off = 0.01f * alpha;
    const uint32_t n = (uint32_t)cam.w * (uint32_t)cam.h;
    const f3 o = mk(cam.pos[0], cam.pos[1], cam.pos[2]);
    const uint32_t nn = (n + kTT - 1) / kTT * kTT;
    for (uint32_t pix = blockIdx.x * kTT + threadIdx.x; pix < nn; pix += gridDim.x * kTT) {
        uint32_t rays = 0, ncell = 0, ntest = 0;
        if (pix < n) {
            const f3 d = primary_dir(cam, pix);
            Hit h;
            trace_one<false, STATS>(s, g, o, d, FLT_MAX, h);
            rays = 1;
            ncell = h.cells;
            ntest = h.tests;
            float vis = 1.0f;
            if (h.hit) {
                const f3 p = mk(o.x + h.t * d.x, o.y + h.t * d.y, o.z + h.t * d.z);
                const f3 nrm = face_normal(s, h.tri, d);
                Pcg32 rng;
                pcg_seed(rng, ((uint64_t)(uint32_t)image_id << 32) | pix, seed);
                int32_t unocc = 0;
                for (int32_t k = 0; k < spp; ++k) {
                    const float u1 = pcg_float(rng), u2 = pcg_float(rng);
                    const f3 w = cosine_dir(nrm, u1, u2);
                    const f3 ao = mk(p.x + off * w.x, p.y + off * w.y, p.z + off * w.z);
                    Hit hs;
                    trace_one<true, STATS>(s, g, ao, w, alpha, hs);
                    unocc += hs.hit ? 0 : 1;
                    ncell += hs.cells;
                    ntest += hs.tests;
                }
                rays += (uint32_t)spp;
                vis = (float)unocc / (float)spp;
            }
            const float val = blend(fb[3 * (size_t)pix], vis, image_id);
            fb[3 * (size_t)pix] = val;
            fb[3 * (size_t)pix + 1] = val;
            fb[3 * (size_t)pix + 2] = val;
        }
        add_rays<STATS>(counter, rays, ncell, ntest);
    }
}

struct LightP {
    float c[3], e1[3], e2[3];
    float emission;
};

// mode 1/2: path tracing with next-event estimation (PathTracer.h:41-372 structure)
template <bool STATS>
__global__ __launch_bounds__(kTT) void k_render_pt(Scene s, Cam cam, LightP l, int32_t bounces, float albedo,
                                                   float eps_frac, uint64_t seed, int32_t image_id,
                                                   float* __restrict__ fb, unsigned long long* counter) {
    const G g = load_g(s.desc);
    const f3 dd = mk(g.bmax[0] - g.bmin[0], g.bmax[1] - g.bmin[1], g.bmax[2] - g.bmin[2]);
    const float ray_eps = eps_frac * sqrtf(dot(dd, dd));
    const f3 lc = mk(l.c[0], l.c[1], l.c[2]), le1 = mk(l.e1[0], l.e1[1], l.e1[2]), le2 = mk(l.e2[0], l.e2[1], l.e2[2]);
    const f3 lcr = cross(le1, le2);
    const float larea = sqrtf(dot(lcr, lcr));
    const float a_pi = albedo * 0.318309886f;
    const uint32_t n = (uint32_t)cam.w * (uint32_t)cam.h;
    const uint32_t nn = (n + kTT - 1) / kTT * kTT;
    for (uint32_t pix = blockIdx.x * kTT + threadIdx.x; pix < nn; pix += gridDim.x * kTT) {
        uint32_t rays = 0, ncell = 0, ntest = 0;
        if (pix < n) {
            Pcg32 rng;
            pcg_seed(rng, ((uint64_t)(uint32_t)image_id << 32) | pix, seed);
            f3 o = mk(cam.pos[0], cam.pos[1], cam.pos[2]);
            f3 d = primary_dir(cam, pix);
            float L = 0.0f, beta = 1.0f;
            for (int32_t bounce = 0; bounce < bounces; ++bounce) {
                Hit h;
                trace_one<false, STATS>(s, g, o, d, FLT_MAX, h);
                rays += 1;
                ncell += h.cells;
                ntest += h.tests;
                if (bounce == 0 && d.z > 0.0f) {
                    const float tl = (lc.z - o.z) / d.z;
                    const float px = o.x + tl * d.x, py = o.y + tl * d.y;
                    const float fx = (px - lc.x) / le1.x, fy = (py - lc.y) / le2.y;
                    if (tl > kIsectEps && tl < h.t && fx >= 0.0f && fx <= 1.0f && fy >= 0.0f && fy <= 1.0f) {
                        L = L + l.emission;
                        break;
                    }
                }
                if (!h.hit) break;
                const f3 p = mk(o.x + h.t * d.x, o.y + h.t * d.y, o.z + h.t * d.z);
                const f3 nrm = face_normal(s, h.tri, d);
                const float u1 = pcg_float(rng), u2 = pcg_float(rng);
                const f3 lp = mk(lc.x + u1 * le1.x + u2 * le2.x, lc.y + u1 * le1.y + u2 * le2.y,
                                 lc.z + u1 * le1.z + u2 * le2.z);
                f3 wi = sub(lp, p);
                const float dist2 = dot(wi, wi);
                const float dist = sqrtf(dist2);
                wi = mulf(wi, 1.0f / dist);
                const float cos_s = dot(nrm, wi), cos_l = wi.z;
                if (cos_s > 0.0f && cos_l > 0.0f) {
                    const f3 so = mk(p.x + ray_eps * wi.x, p.y + ray_eps * wi.y, p.z + ray_eps * wi.z);
                    Hit hs;
                    trace_one<true, STATS>(s, g, so, wi, dist - ray_eps, hs);
                    rays += 1;
                    ncell += hs.cells;
                    ntest += hs.tests;
                    if (!hs.hit) L = L + beta * a_pi * l.emission * cos_s * cos_l * larea / dist2;
                }
                beta = beta * albedo;
                const float u3 = pcg_float(rng), u4 = pcg_float(rng);
                d = cosine_dir(nrm, u3, u4);
                o = mk(p.x + ray_eps * d.x, p.y + ray_eps * d.y, p.z + ray_eps * d.z);
            }
            const float val = blend(fb[3 * (size_t)pix], L, image_id);
            fb[3 * (size_t)pix] = val;
            fb[3 * (size_t)pix + 1] = val;
            fb[3 * (size_t)pix + 2] = val;
        }
        add_rays<STATS>(counter, rays, ncell, ntest);
    }
}

Scene make_scene(hr_ctx* c) {
    Scene s;
    s.v = c->verts.as<float4>();
    s.idx = c->idx.as<uint32_t>();
    s.cells = c->g.cells.as<uint2>();
    s.leaves = c->g.leaves.as<uint2>();
    s.prims = c->g.prims.as<uint32_t>();
    s.desc = c->g.desc.as<GridDesc>();
    s.ntri = c->ntri;
    s.kind = c->built_kind;
    return s;
}

Cam make_cam(const hr_ctx* c) {
    Cam k;
    for (int i = 0; i < 3; ++i) {
        k.pos[i] = c->cam.pos[i]; k.tl[i] = c->cam.top_left[i];
        k.sx[i] = c->cam.step_x[i]; k.sy[i] = c->cam.step_y[i];
    }
    k.w = c->cam.w; k.h = c->cam.h;
    return k;
}

int grid_for(const hr_ctx* c, uint32_t n) {
    uint32_t b = (n + kTT - 1) / kTT;
    uint32_t cap = (uint32_t)c->num_sms * 16u;
    return (int)(b < 1 ? 1 : (b > cap ? cap : b));
}

}  // namespace

int launch_trace_rays(hr_ctx* c, const float* org, const float* dir, uint32_t n, int32_t* id, float* t, float* u,
                      float* v, uint32_t* stats) {
    if (n == 0) return 0;
    Scene s = make_scene(c);
    c->launches += 1;
    if (stats) k_trace_rays<true><<<grid_for(c, n), kTT, 0, c->stream>>>(s, org, dir, n, id, t, u, v, stats);
    else k_trace_rays<false><<<grid_for(c, n), kTT, 0, c->stream>>>(s, org, dir, n, id, t, u, v, nullptr);
    return cuda_check(c, cudaGetLastError(), "trace_rays launch");
}

int launch_trace_primary(hr_ctx* c, int32_t* id, float* t, float* u, float* v, uint32_t* stats) {
    Scene s = make_scene(c);
    Cam k = make_cam(c);
    const uint32_t n = (uint32_t)k.w * (uint32_t)k.h;
    if (n == 0) return 0;
    c->launches += 1;
    if (stats) k_trace_primary<true><<<grid_for(c, n), kTT, 0, c->stream>>>(s, k, id, t, u, v, stats);
    else k_trace_primary<false><<<grid_for(c, n), kTT, 0, c->stream>>>(s, k, id, t, u, v, nullptr);
    return cuda_check(c, cudaGetLastError(), "trace_primary launch");
}

int launch_occluded(hr_ctx* c, const float* org, const float* dir, const float* tmax, uint32_t n, uint8_t* occ) {
    if (n == 0) return 0;
    c->launches += 1;
    k_occluded<<<grid_for(c, n), kTT, 0, c->stream>>>(make_scene(c), org, dir, tmax, n, occ);
    return cuda_check(c, cudaGetLastError(), "occluded launch");
}

int launch_render(hr_ctx* c, int32_t mode, int32_t image_id, float* d_fb) {
    Scene s = make_scene(c);
    Cam k = make_cam(c);
    const uint32_t n = (uint32_t)k.w * (uint32_t)k.h;
    if (n == 0) return 0;
    unsigned long long* ctr = c->counters.as<unsigned long long>();
    const int gb = grid_for(c, n);
    c->launches += 1;
    const bool st = c->collect_stats;
    switch (mode) {
    case 0:
        if (st) k_render_primary<true><<<gb, kTT, 0, c->stream>>>(s, k, image_id, d_fb, ctr);
        else k_render_primary<false><<<gb, kTT, 0, c->stream>>>(s, k, image_id, d_fb, ctr);
        break;
    case 1:
    case 2: {
        LightP l;
        for (int i = 0; i < 3; ++i) { l.c[i] = c->light.corner[i]; l.e1[i] = c->light.e1[i]; l.e2[i] = c->light.e2[i]; }
        l.emission = c->light.emission;
        if (st)
            k_render_pt<true><<<gb, kTT, 0, c->stream>>>(s, k, l, c->ip.pt_bounces, c->ip.albedo, c->ip.ray_eps_frac,
                                                         c->ip.seed, image_id, d_fb, ctr);
        else
            k_render_pt<false><<<gb, kTT, 0, c->stream>>>(s, k, l, c->ip.pt_bounces, c->ip.albedo, c->ip.ray_eps_frac,
                                                          c->ip.seed, image_id, d_fb, ctr);
        break;
    }
    case 3:
        if (st)
            k_render_ao<true><<<gb, kTT, 0, c->stream>>>(s, k, c->ip.ao_samples, c->ip.ao_radius_frac,
                                                         c->ip.ao_radius_abs, c->ip.seed, image_id, d_fb, ctr);
        else
            k_render_ao<false><<<gb, kTT, 0, c->stream>>>(s, k, c->ip.ao_samples, c->ip.ao_radius_frac,
                                                          c->ip.ao_radius_abs, c->ip.seed, image_id, d_fb, ctr);
        break;
    default:
        return set_error(c, 1, "render: unknown mode %d", mode);
    }
    return cuda_check(c, cudaGetLastError(), "render launch");
}

}  // namespace hr
