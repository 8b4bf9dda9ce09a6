// hier.cu -- instanced two-level grid hierarchy: one uniform grid per object (built for
// all objects at once, segmented by object), a uniform grid over the instances' world
// boxes, and the nested traversal (instance grid -> instance box -> ray in object space
// -> object grid).
//
// Reference path (javorkk/happyray):
//   structure              src/RT/Structure/TwoLevelGridHierarchy.h:569-697, 750-952
//   object grids           src/RT/Algorithm/TLGridHierarchySortBuilder.cu:20-225, 522-682
//                          (bounds and resolution: src/RT/RTEngine.cu:261-330)
//   instance grid          src/RT/Algorithm/TLGridHierarchySortBuilder.cu:260-520
//   traversal              src/RT/Algorithm/TLGridHierarchyTraverser.h:45-405
//
// Arithmetic follows the oracle (oracle/hr_oracle.c, orc_hier_*) operation by operation,
// so cells, lists and hits compare bit-exact.  Deliberate differences from the reference
// (all recorded with the others of the project): the instance grid spans the union of the
// instance boxes (the reference uses the scene's vertex bounds, which must then contain
// every instance); rays carry their direction, so the object-space direction is the
// world -> object rotation applied to it, not re-derived from reciprocals.
#include "happyray.h"
#include "build_dev.cuh"
#include "traverse.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#ifndef HR_HIER_MIN_BLOCKS
#define HR_HIER_MIN_BLOCKS 8   // blocks per SM the trace kernel's register budget must allow (8: 64 registers)
#endif
#ifndef HR_HIER_WARP_POOL
#define HR_HIER_WARP_POOL 1   // trace warps take 32 consecutive rays from a pool once all lanes are done
#endif

namespace hr {
namespace {

struct HierObj {   // the layout of hr_hier_object
    float bmin[3], bmax[3], cs[3], rcp[3];
    int32_t res[3];
    uint32_t cell_off, tri_begin, tri_count;
};
static_assert(sizeof(HierObj) == 72, "object record layout");

struct HierInst {   // 80 bytes, five float4 loads
    float4 r0, r1, r2;   // rows of the world -> object map
    float4 lo;           // world box min; w = object index (bits)
    float4 hi;           // world box max
};

constexpr float kObjPad = 10.0f * kEps;   // RTEngine.cu:291-296

// ---- object grids ------------------------------------------------------------------

__global__ void k_hier_obj_init(int32_t* __restrict__ enc, uint32_t nobj) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nobj; k += gridDim.x * blockDim.x) {
        enc[6 * k + 0] = enc[6 * k + 1] = enc[6 * k + 2] = fenc(FLT_MAX);
        enc[6 * k + 3] = enc[6 * k + 4] = enc[6 * k + 5] = fenc(-FLT_MAX);
    }
}

// Per triangle: its three vertices into `tris` and its box into its object's bounds
// (objects are consecutive triangle ranges; a warp whose triangles share one object
// reduces first and adds one set of atomics).
__global__ __launch_bounds__(kBT) void k_hier_tris(const float4* __restrict__ verts, const uint32_t* __restrict__ idx,
                                                   const uint32_t* __restrict__ tri_begin, uint32_t nobj,
                                                   uint32_t ntri, float4* __restrict__ tris, int32_t* __restrict__ enc) {
    const uint32_t lane = threadIdx.x & 31u;
    for (uint32_t base = blockIdx.x * blockDim.x; base < ntri; base += gridDim.x * blockDim.x) {
        const uint32_t t = base + threadIdx.x;
        const bool valid = t < ntri;
        f3 lo = mk(FLT_MAX, FLT_MAX, FLT_MAX), hi = mk(-FLT_MAX, -FLT_MAX, -FLT_MAX);
        uint32_t obj = 0xffffffffu;
        if (valid) {
            f3 p[3];
            tri_load(verts, idx, t, p);
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                tris[3 * (size_t)t + c] = make_float4(p[c].x, p[c].y, p[c].z, 0.0f);
                lo = vmin(lo, p[c]);
                hi = vmax(hi, p[c]);
            }
            obj = find_segment(tri_begin, nobj, t);
        }
        const uint32_t o0 = __shfl_sync(kFullMask, obj, 0);
        if (__all_sync(kFullMask, !valid || obj == o0) && o0 != 0xffffffffu) {
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                lo = vmin(lo, mk(__shfl_xor_sync(kFullMask, lo.x, off), __shfl_xor_sync(kFullMask, lo.y, off),
                                 __shfl_xor_sync(kFullMask, lo.z, off)));
                hi = vmax(hi, mk(__shfl_xor_sync(kFullMask, hi.x, off), __shfl_xor_sync(kFullMask, hi.y, off),
                                 __shfl_xor_sync(kFullMask, hi.z, off)));
            }
            if (lane == 0) obj = o0;
            else obj = 0xffffffffu;
        }
        if (obj != 0xffffffffu) {
            int32_t* e = enc + 6 * (size_t)obj;
            atomicMin(e + 0, fenc(lo.x)); atomicMin(e + 1, fenc(lo.y)); atomicMin(e + 2, fenc(lo.z));
            atomicMax(e + 3, fenc(hi.x)); atomicMax(e + 4, fenc(hi.y)); atomicMax(e + 5, fenc(hi.z));
        }
    }
}

// Object grid geometry (RTEngine.cu:288-327 / countGridCellsMultiUniformGrid,
// TLGridHierarchySortBuilder.cu:20-57): bounds padded by 10 EPS, res = max(1,
// (int)(diag * (density * N / volume)^(1/3))) per axis, cell size diag / res.
__global__ void k_hier_obj_setup(const int32_t* __restrict__ enc, const uint32_t* __restrict__ tri_begin,
                                 uint32_t nobj, float density, HierObj* __restrict__ objs, uint32_t* __restrict__ cnt,
                                 uint32_t* __restrict__ err, unsigned long long* __restrict__ total) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nobj; k += gridDim.x * blockDim.x) {
        HierObj g;
        g.tri_begin = tri_begin[k];
        g.tri_count = tri_begin[k + 1] - tri_begin[k];
        const f3 lo = mk(fdec(enc[6 * k]), fdec(enc[6 * k + 1]), fdec(enc[6 * k + 2]));
        const f3 hi = mk(fdec(enc[6 * k + 3]), fdec(enc[6 * k + 4]), fdec(enc[6 * k + 5]));
        g.bmin[0] = lo.x - kObjPad; g.bmin[1] = lo.y - kObjPad; g.bmin[2] = lo.z - kObjPad;
        g.bmax[0] = hi.x + kObjPad; g.bmax[1] = hi.y + kObjPad; g.bmax[2] = hi.z + kObjPad;
        const f3 d = mk(g.bmax[0] - g.bmin[0], g.bmax[1] - g.bmin[1], g.bmax[2] - g.bmin[2]);
        const float vol = d.x * d.y * d.z;
        const float m = pow_third(density * (float)g.tri_count / vol);
        const f3 r = mulf(d, m);
        const int32_t ri[3] = {f2i(r.x), f2i(r.y), f2i(r.z)};
        uint64_t cells = 1;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            g.res[a] = ri[a] > 0 ? ri[a] : 1;
            const float dk = comp(d, a), rk = (float)g.res[a];
            g.cs[a] = dk / rk;
            g.rcp[a] = rk / dk;
            cells *= (uint64_t)g.res[a];
        }
        g.cell_off = 0;
        if (cells > (1ull << 30)) {   // more cells than the 32-bit keys can hold
            atomicOr(err, 1u);
            cells = 1;
        }
        objs[k] = g;
        cnt[k] = (uint32_t)cells;
        atomicAdd(total, (unsigned long long)cells);
    }
}

__global__ void k_hier_obj_offsets(const uint32_t* __restrict__ off, uint32_t nobj, HierObj* __restrict__ objs) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nobj; k += gridDim.x * blockDim.x)
        objs[k].cell_off = off[k];
}

// cell range of a triangle box in its object grid: countPairsMultiUniformGrid,
// TLGridHierarchySortBuilder.cu:122-145 (both ends clamped into [0, res))
__device__ __forceinline__ uint32_t obj_cell_range(f3 lo, f3 hi, const HierObj& g, int32_t* rlo, int32_t* rhi) {
    const float af[3] = {(lo.x - g.bmin[0]) * g.rcp[0], (lo.y - g.bmin[1]) * g.rcp[1], (lo.z - g.bmin[2]) * g.rcp[2]};
    const float bf[3] = {(hi.x - g.bmin[0]) * g.rcp[0] + 1.0f, (hi.y - g.bmin[1]) * g.rcp[1] + 1.0f,
                         (hi.z - g.bmin[2]) * g.rcp[2] + 1.0f};
    uint32_t n = 1;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        rlo[k] = min(g.res[k] - 1, max(0, f2i(af[k])));
        rhi[k] = max(1, min(g.res[k], f2i(bf[k])));
        const int32_t e = rhi[k] - rlo[k];
        n *= (uint32_t)(e > 0 ? e : 0);
    }
    return n;
}

__device__ __forceinline__ uint32_t tri_pairs(const float4* __restrict__ tris, const HierObj* __restrict__ objs,
                                              const uint32_t* __restrict__ tri_begin, uint32_t nobj, uint32_t t,
                                              HierObj* g, int32_t* rlo, int32_t* rhi) {
    f3 p[3], lo, hi;
    tri_fetch(tris, t, p);
    tri_bbox(p, &lo, &hi);
    *g = objs[find_segment(tri_begin, nobj, t)];
    return obj_cell_range(lo, hi, *g, rlo, rhi);
}

// pairs per block of kBT triangles (the block sums are scanned into block offsets)
__global__ __launch_bounds__(kBT) void k_hier_count(const float4* __restrict__ tris, const HierObj* __restrict__ objs,
                                                    const uint32_t* __restrict__ tri_begin, uint32_t nobj,
                                                    uint32_t ntri, uint32_t* __restrict__ bsum) {
    const uint32_t t = blockIdx.x * kBT + threadIdx.x;
    uint32_t n = 0;
    if (t < ntri) {
        HierObj g;
        int32_t rlo[3], rhi[3];
        n = tri_pairs(tris, objs, tri_begin, nobj, t, &g, rlo, rhi);
    }
    uint32_t total;
    block_excl_scan<uint32_t, kBT>(n, &total);
    if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

// pairs in triangle order (writeKeysAndValuesMultiUniformGrid, .cu:151-225): key = the
// object's first cell + x + rx (y + ry z), value = triangle id; z, y, x loops
__global__ __launch_bounds__(kBT) void k_hier_write(const float4* __restrict__ tris, const HierObj* __restrict__ objs,
                                                    const uint32_t* __restrict__ tri_begin, uint32_t nobj,
                                                    uint32_t ntri, const uint32_t* __restrict__ boff,
                                                    uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
    const uint32_t t = blockIdx.x * kBT + threadIdx.x;
    HierObj g;
    int32_t rlo[3] = {0, 0, 0}, rhi[3] = {0, 0, 0};
    uint32_t n = 0;
    if (t < ntri) n = tri_pairs(tris, objs, tri_begin, nobj, t, &g, rlo, rhi);
    uint32_t total;
    uint32_t w = block_excl_scan<uint32_t, kBT>(n, &total) + boff[blockIdx.x];
    if (n == 0) return;
    const uint32_t rx = (uint32_t)g.res[0], rxy = (uint32_t)g.res[0] * (uint32_t)g.res[1];
    for (int32_t z = rlo[2]; z < rhi[2]; ++z)
        for (int32_t y = rlo[1]; y < rhi[1]; ++y)
            for (int32_t x = rlo[0]; x < rhi[0]; ++x) {
                keys[w] = (uint32_t)x + (uint32_t)y * rx + (uint32_t)z * rxy + g.cell_off;
                vals[w] = t;
                ++w;
            }
}

// ---- instance grid -----------------------------------------------------------------

// One block: the union of the instance boxes, padded as the scene bounds
// (WFObjectUploader.h:112-114); resolution max(1, (int)(diag * (density * n /
// volume)^(1/3))) (TLGridHierarchySortBuilder.cu:275-286), cell size diag / res
// (TLGridHierarchyMemoryManager.h:111-119).
__global__ __launch_bounds__(kBT) void k_hier_top_setup(const HierInst* __restrict__ inst, uint32_t ninst,
                                                        float density, GridDesc* __restrict__ d) {
    f3 lo = mk(FLT_MAX, FLT_MAX, FLT_MAX), hi = mk(-FLT_MAX, -FLT_MAX, -FLT_MAX);
    for (uint32_t i = threadIdx.x; i < ninst; i += kBT) {
        const float4 a = inst[i].lo, b = inst[i].hi;
        lo = vmin(lo, mk(a.x, a.y, a.z));
        hi = vmax(hi, mk(b.x, b.y, b.z));
    }
    __shared__ float s[6][kBT];
    s[0][threadIdx.x] = lo.x; s[1][threadIdx.x] = lo.y; s[2][threadIdx.x] = lo.z;
    s[3][threadIdx.x] = hi.x; s[4][threadIdx.x] = hi.y; s[5][threadIdx.x] = hi.z;
    __syncthreads();
    if (threadIdx.x != 0) return;
    for (int j = 1; j < kBT; ++j) {
        lo = vmin(lo, mk(s[0][j], s[1][j], s[2][j]));
        hi = vmax(hi, mk(s[3][j], s[4][j], s[5][j]));
    }
    const f3 dd = sub(hi, lo);
    const float pad = 0.001f * sqrtf(dot(dd, dd));
    d->bmin[0] = lo.x - pad; d->bmin[1] = lo.y - pad; d->bmin[2] = lo.z - pad;
    d->bmax[0] = hi.x + pad; d->bmax[1] = hi.y + pad; d->bmax[2] = hi.z + pad;
    const f3 e = mk(d->bmax[0] - d->bmin[0], d->bmax[1] - d->bmin[1], d->bmax[2] - d->bmin[2]);
    const float vol = e.x * e.y * e.z;
    const float m = pow_third(density * (float)ninst / vol);
    const f3 r = mulf(e, m);
    d->res[0] = max(1, f2i(r.x)); d->res[1] = max(1, f2i(r.y)); d->res[2] = max(1, f2i(r.z));
    uint64_t cells = 1;
    for (int k = 0; k < 3; ++k) {
        const float dk = comp(e, k), rk = (float)d->res[k];
        d->cs[k] = dk / rk;
        d->rcp[k] = rk / dk;
        cells *= (uint64_t)d->res[k];
    }
    d->overflow = 0u;
    d->error = cells > (1ull << 30) ? 1u : 0u;
    d->ncells = d->error ? 1u : (uint32_t)cells;
    d->kind = kUniform;
    d->ntri = ninst;
}

// instance box -> cell range of the instance grid (UniformGridBuildKernels.h:56-73)
__device__ __forceinline__ uint32_t inst_cell_range(const HierInst& I, const GridDesc& d, int32_t* rlo, int32_t* rhi) {
    const float af[3] = {(I.lo.x - d.bmin[0]) * d.rcp[0], (I.lo.y - d.bmin[1]) * d.rcp[1], (I.lo.z - d.bmin[2]) * d.rcp[2]};
    const float bf[3] = {(I.hi.x - d.bmin[0]) * d.rcp[0] + 1.0f, (I.hi.y - d.bmin[1]) * d.rcp[1] + 1.0f,
                         (I.hi.z - d.bmin[2]) * d.rcp[2] + 1.0f};
    uint32_t n = 1;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        rlo[k] = max(0, f2i(af[k]));
        rhi[k] = min(d.res[k], f2i(bf[k]));
        const int32_t e = rhi[k] - rlo[k];
        n *= (uint32_t)(e > 0 ? e : 0);
    }
    return n;
}

__global__ void k_hier_inst_count(const HierInst* __restrict__ inst, uint32_t ninst, const GridDesc* __restrict__ d,
                                  uint32_t* __restrict__ cnt) {
    const GridDesc g = *d;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < ninst; i += gridDim.x * blockDim.x) {
        int32_t rlo[3], rhi[3];
        cnt[i] = g.error ? 0u : inst_cell_range(inst[i], g, rlo, rhi);
    }
}

__global__ void k_hier_inst_write(const HierInst* __restrict__ inst, uint32_t ninst, const GridDesc* __restrict__ d,
                                  const uint32_t* __restrict__ off, uint32_t* __restrict__ keys,
                                  uint32_t* __restrict__ vals) {
    const GridDesc g = *d;
    if (g.error) return;
    const uint32_t rx = (uint32_t)g.res[0], rxy = (uint32_t)g.res[0] * (uint32_t)g.res[1];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < ninst; i += gridDim.x * blockDim.x) {
        int32_t rlo[3], rhi[3];
        inst_cell_range(inst[i], g, rlo, rhi);
        uint32_t w = off[i];
        for (int32_t z = rlo[2]; z < rhi[2]; ++z)
            for (int32_t y = rlo[1]; y < rhi[1]; ++y)
                for (int32_t x = rlo[0]; x < rhi[0]; ++x) {
                    keys[w] = (uint32_t)x + (uint32_t)y * rx + (uint32_t)z * rxy;
                    vals[w] = i;
                    ++w;
                }
    }
}

// ---- traversal ---------------------------------------------------------------------

struct HierView {
    const float4* tris;
    const HierObj* objs;
    const HierInst* inst;
    const GridDesc* top;
    const uint2* top_cells;
    const uint32_t* inst_ids;
    const uint2* obj_cells;
    const uint32_t* prims;
};

// slab test against a box (BBox.hpp:64-79 fastClip)
__device__ __forceinline__ void box_clip(const float* bmin, const float* bmax, f3 o, const float* rcp, float* t0,
                                         float* t1) {
    float tn[3], tf[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float a = (bmin[k] - comp(o, k)) * rcp[k];
        const float b = (bmax[k] - comp(o, k)) * rcp[k];
        tn[k] = hmin(a, b); tf[k] = hmax(a, b);
    }
    *t0 = hmax(hmax(tn[0], tn[1]), tn[2]);
    *t1 = hmin(hmin(tf[0], tf[1]), tf[2]);
}

struct HHit {
    float t, u, v;
    int32_t inst, tri;
};

// per-ray work counters (STATS instances): instance-grid cells, instance boxes tested,
// instances entered, object-grid cells, triangle tests
struct HCount {
    uint32_t top_cells = 0, inst_tests = 0, inst_entered = 0, obj_cells = 0, tri_tests = 0;
};

// One instance (GeometryInstanceTraverser, TLGridHierarchyTraverser.h:45-205): the world
// box interval, the ray in object space, the object grid's DDA from the current best t.
// Returns true when the instance's hit is accepted (inside the box interval, closer).
template <bool STATS>
__device__ bool hier_instance(const HierView& H, uint32_t ii, f3 o, f3 d, const float* rcp, HHit& h, HCount& n) {
    const HierInst I = H.inst[ii];
    const float blo[3] = {I.lo.x, I.lo.y, I.lo.z}, bhi[3] = {I.hi.x, I.hi.y, I.hi.z};
    float te1, tx1;
    box_clip(blo, bhi, o, rcp, &te1, &tx1);
    if (STATS) n.inst_tests++;
    if (!(tx1 > te1 && tx1 >= 0.0f && te1 < h.t)) return false;
    if (STATS) n.inst_entered++;
    const f3 ot = mk(I.r0.x * o.x + I.r0.y * o.y + I.r0.z * o.z + I.r0.w,
                     I.r1.x * o.x + I.r1.y * o.y + I.r1.z * o.z + I.r1.w,
                     I.r2.x * o.x + I.r2.y * o.y + I.r2.z * o.z + I.r2.w);
    const f3 dt = mk(I.r0.x * d.x + I.r0.y * d.y + I.r0.z * d.z, I.r1.x * d.x + I.r1.y * d.y + I.r1.z * d.z,
                     I.r2.x * d.x + I.r2.y * d.y + I.r2.z * d.z);
    const float rt[3] = {1.0f / dt.x, 1.0f / dt.y, 1.0f / dt.z};
    const HierObj g = H.objs[__float_as_uint(I.lo.w)];
    Scene s;
    s.tris = H.tris;
    float rayT = h.t, bu = 0.0f, bv = 0.0f;
    int32_t best = -1;
    float te, tx;
    box_clip(g.bmin, g.bmax, ot, rt, &te, &tx);
    bool flag = tx > te && tx >= 0.0f && te < rayT;
    f3 ep = ot;
    if (te >= 0.0f) {
        const float sc = te + kEps;
        ep = mk(ot.x + sc * dt.x, ot.y + sc * dt.y, ot.z + sc * dt.z);
    }
    float tmax[3];
    int32_t cell[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float cf = floorf((comp(ep, k) - g.bmin[k]) * g.rcp[k]);
        cf = rt[k] > 0.0f ? hmin((float)g.res[k] - 1.0f, cf) : hmax(cf, 0.0f);
        const float stp = rt[k] > 0.0f ? 1.0f : 0.0f;
        tmax[k] = ((cf + stp) * g.cs[k] + g.bmin[k] - comp(ot, k)) * rt[k];
        cell[k] = f2i(cf);
        flag = flag && (rt[k] > 0.0f ? cell[k] < g.res[k] : cell[k] > -1);
    }
    const uint32_t rx = (uint32_t)g.res[0], rxy = (uint32_t)g.res[0] * (uint32_t)g.res[1];
    while (flag) {
        if (cell[0] < g.res[0] && cell[0] > -1 && cell[1] < g.res[1] && cell[1] > -1 && cell[2] < g.res[2] &&
            cell[2] > -1) {
            const uint2 cr = __ldg(H.obj_cells + (g.cell_off + (uint32_t)cell[0] + (uint32_t)cell[1] * rx +
                                                  (uint32_t)cell[2] * rxy));
            if (STATS) {
                n.obj_cells++;
                n.tri_tests += cr.y - cr.x;
            }
            for (uint32_t it = cr.x; it < cr.y; ++it) {
                const uint32_t tri = __ldg(H.prims + it);
                float t, u, v;
                if (mt_test(s, tri, ot, dt, rayT, &t, &u, &v)) {
                    rayT = t; bu = u; bv = v; best = (int32_t)tri;
                }
            }
        }
        const int k = min_dim(tmax[0], tmax[1], tmax[2]);
        float tk;
        if (k == 0) {
            tk = tmax[0];
            cell[0] += rt[0] > 0.0f ? 1 : -1;
            tmax[0] += g.cs[0] * fabsf(rt[0]);
            flag = flag && rayT > tk && (rt[0] > 0.0f ? cell[0] < g.res[0] : cell[0] > -1);
        } else if (k == 1) {
            tk = tmax[1];
            cell[1] += rt[1] > 0.0f ? 1 : -1;
            tmax[1] += g.cs[1] * fabsf(rt[1]);
            flag = flag && rayT > tk && (rt[1] > 0.0f ? cell[1] < g.res[1] : cell[1] > -1);
        } else {
            tk = tmax[2];
            cell[2] += rt[2] > 0.0f ? 1 : -1;
            tmax[2] += g.cs[2] * fabsf(rt[2]);
            flag = flag && rayT > tk && (rt[2] > 0.0f ? cell[2] < g.res[2] : cell[2] > -1);
        }
    }
    if (best >= 0 && rayT < h.t && rayT >= te1 && rayT < tx1) {
        h.t = rayT; h.u = bu; h.v = bv; h.inst = (int32_t)ii; h.tri = best;
        return true;
    }
    return false;
}

// instance-grid DDA (TLGridHierarchyTraverser.h:220-405); ANY stops at the first
// accepted hit
template <bool ANY, bool STATS>
__device__ void hier_trace(const HierView& H, const GridDesc& g, f3 o, f3 d, HHit& h, HCount& n) {
    const float rcp[3] = {1.0f / d.x, 1.0f / d.y, 1.0f / d.z};
    float t0, t1;
    box_clip(g.bmin, g.bmax, o, rcp, &t0, &t1);
    if (!(t1 > t0 && t1 >= 0.0f)) return;
    f3 ep = o;
    if (t0 >= 0.0f) {
        const float sc = t0 + kEps;
        ep = mk(o.x + sc * d.x, o.y + sc * d.y, o.z + sc * d.z);
    }
    float tmax[3];
    int32_t cell[3];
    bool active = true;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float cf = floorf((comp(ep, k) - g.bmin[k]) * g.rcp[k]);
        const float stp = rcp[k] > 0.0f ? 1.0f : 0.0f;
        tmax[k] = ((cf + stp) * g.cs[k] + g.bmin[k] - comp(o, k)) * rcp[k];
        cell[k] = f2i(cf);
        active = active && (rcp[k] > 0.0f ? cell[k] < g.res[k] : cell[k] > -1);
    }
    const uint32_t rx = (uint32_t)g.res[0], rxy = (uint32_t)g.res[0] * (uint32_t)g.res[1];
    while (active) {
        if (cell[0] < g.res[0] && cell[0] > -1 && cell[1] < g.res[1] && cell[1] > -1 && cell[2] < g.res[2] &&
            cell[2] > -1) {
            const uint2 cr = __ldg(H.top_cells + ((uint32_t)cell[0] + (uint32_t)cell[1] * rx + (uint32_t)cell[2] * rxy));
            if (STATS) n.top_cells++;
            for (uint32_t it = cr.x; it < cr.y; ++it)
                if (hier_instance<STATS>(H, __ldg(H.inst_ids + it), o, d, rcp, h, n) && ANY) return;
        }
        const int k = min_dim(tmax[0], tmax[1], tmax[2]);
        float tk;
        if (k == 0) {
            tk = tmax[0];
            cell[0] += rcp[0] > 0.0f ? 1 : -1;
            tmax[0] += g.cs[0] * fabsf(rcp[0]);
            active = h.t > tk && (rcp[0] > 0.0f ? cell[0] < g.res[0] : cell[0] > -1);
        } else if (k == 1) {
            tk = tmax[1];
            cell[1] += rcp[1] > 0.0f ? 1 : -1;
            tmax[1] += g.cs[1] * fabsf(rcp[1]);
            active = h.t > tk && (rcp[1] > 0.0f ? cell[1] < g.res[1] : cell[1] > -1);
        } else {
            tk = tmax[2];
            cell[2] += rcp[2] > 0.0f ? 1 : -1;
            tmax[2] += g.cs[2] * fabsf(rcp[2]);
            active = h.t > tk && (rcp[2] > 0.0f ? cell[2] < g.res[2] : cell[2] > -1);
        }
    }
}

template <bool ANY, bool STATS>
__global__ __launch_bounds__(kTT, HR_HIER_MIN_BLOCKS) void k_hier_trace(HierView H, const float* __restrict__ org,
                                                       const float* __restrict__ dir, const float* __restrict__ tmax,
                                                       uint32_t n, int32_t* __restrict__ oinst,
                                                       int32_t* __restrict__ otri, float* __restrict__ ot,
                                                       float* __restrict__ ou, float* __restrict__ ov,
                                                       uint8_t* __restrict__ occ, uint32_t* __restrict__ stats,
                                                       uint32_t* pool) {
    const GridDesc g = *H.top;
#if HR_HIER_WARP_POOL
    // a warp takes 32 consecutive rays from the pool once all its lanes are done, so its
    // lanes trace neighbouring rays together (rays listed in pixel tiles stay coherent)
    const uint32_t lane = threadIdx.x & 31u;
    while (true) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(pool, 32u);
        base = __shfl_sync(kFullMask, base, 0);
        if (base >= n) break;
        const uint32_t i = base + lane;
        if (i >= n) continue;
#else
    for (uint32_t i = blockIdx.x * kTT + threadIdx.x; i < n; i += gridDim.x * kTT) {
#endif
        const f3 o = mk(__ldg(org + 3 * (size_t)i), __ldg(org + 3 * (size_t)i + 1), __ldg(org + 3 * (size_t)i + 2));
        const f3 d = mk(__ldg(dir + 3 * (size_t)i), __ldg(dir + 3 * (size_t)i + 1), __ldg(dir + 3 * (size_t)i + 2));
        HHit h;
        h.t = ANY ? __ldg(tmax + i) : FLT_MAX;
        h.u = 0.0f; h.v = 0.0f; h.inst = -1; h.tri = -1;
        HCount c;
        if (!g.error) hier_trace<ANY, STATS>(H, g, o, d, h, c);
        if (STATS) {
            uint32_t* st = stats + 5 * (size_t)i;
            st[0] = c.top_cells; st[1] = c.inst_tests; st[2] = c.inst_entered; st[3] = c.obj_cells; st[4] = c.tri_tests;
        }
        if (ANY) {
            occ[i] = h.inst >= 0 ? 1 : 0;
        } else {
            oinst[i] = h.inst;
            otri[i] = h.tri;
            ot[i] = h.inst >= 0 ? h.t : FLT_MAX;
            ou[i] = h.u;
            ov[i] = h.v;
        }
    }
}

int key_bits(uint64_t n) {
    int b = 1;
    while (b < 32 && ((uint64_t)1 << b) <= n) ++b;
    return b;
}

}  // namespace
}  // namespace hr

using namespace hr;

struct hr_hier {
    hr_ctx* c = nullptr;   // stream, device, error text, sort scratch
    uint32_t nv = 0, ntri = 0, nobj = 0, ninst = 0;
    float top_density = 1.2f, obj_density = 1.2f;
    bool objects_dirty = true, have_objects = false, have_instances = false, built = false;
    DevBuf tri_begin, enc, objs, cnt, obj_cells, prims;
    DevBuf inst, top_desc, icnt, top_cells, inst_ids, words;   // words: [0] cells [1] pairs [2] top pairs [3] err [4] nobj [5] ninst [7] ray pool
    uint32_t num_obj_cells = 0, num_pairs = 0, num_top_pairs = 0;
    GridDesc top{};
    DevBuf rays;   // host-call staging: org, dir, tmax, outputs
};

namespace hr {
namespace {

void free_dev(DevBuf& b, cudaStream_t s) {
    if (b.p) cudaFreeAsync(b.p, s);
    b.p = nullptr;
    b.bytes = 0;
}

int grid_of(const hr_ctx* c, uint64_t n, int bt) {
    const uint64_t b = (n + (uint64_t)bt - 1) / (uint64_t)bt;
    const uint64_t cap = (uint64_t)c->num_sms * 16u;
    return (int)std::max<uint64_t>(1, std::min(b, cap));
}

// blocks of the trace launch: resident blocks on every SM with the warp ray pool,
// enough blocks for one ray per thread otherwise
template <bool ANY, bool STATS>
int hier_grid(hr_ctx* c, uint32_t n) {
    const int want = grid_of(c, n, kTT);
    if (!HR_HIER_WARP_POOL) return want;
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_hier_trace<ANY, STATS>, kTT, 0) != cudaSuccess || nb < 1) {
        cudaGetLastError();
        nb = 1;
    }
    return std::max(1, std::min(want, nb * c->num_sms));
}


// level two: object grids
int build_objects(hr_hier* h) {
    hr_ctx* c = h->c;
    cudaStream_t s = c->stream;
    GridBuffers& B = c->g;
    uint32_t* words = h->words.as<uint32_t>();
    const uint32_t nb = (h->ntri + kBT - 1) / kBT;
    int rc;
    if ((rc = cuda_check(c, cudaMemsetAsync(words + 8, 0, 8, s), "hier counts")) ||
        (rc = ensure(c, h->enc, sizeof(int32_t) * 6 * h->nobj)) || (rc = ensure(c, h->objs, sizeof(HierObj) * h->nobj)) ||
        (rc = ensure(c, h->cnt, sizeof(uint32_t) * (h->nobj + 1))) ||
        (rc = ensure(c, c->tris, sizeof(float4) * 3 * (size_t)h->ntri)) ||
        (rc = ensure(c, B.block_sums, sizeof(uint32_t) * (nb + 1))) ||
        (rc = ensure(c, B.scan_partials, sizeof(uint32_t) * (scan_partials_words(h->nobj) + 2))))
        return rc;
    c->launches += 6;   // five kernels and the block-sum scan; the other scan counts its own
    k_hier_obj_init<<<grid_of(c, h->nobj, 256), 256, 0, s>>>(h->enc.as<int32_t>(), h->nobj);
    k_hier_tris<<<grid_of(c, h->ntri, kBT), kBT, 0, s>>>(c->verts.as<float4>(), c->idx.as<uint32_t>(),
                                                         h->tri_begin.as<uint32_t>(), h->nobj, h->ntri,
                                                         c->tris.as<float4>(), h->enc.as<int32_t>());
    k_hier_obj_setup<<<grid_of(c, h->nobj, 256), 256, 0, s>>>(h->enc.as<int32_t>(), h->tri_begin.as<uint32_t>(),
                                                              h->nobj, h->obj_density, h->objs.as<HierObj>(),
                                                              h->cnt.as<uint32_t>(), words + 3,
                                                              reinterpret_cast<unsigned long long*>(words + 8));
    if ((rc = exclusive_scan_u32(c, h->cnt.as<uint32_t>(), words + 4, h->nobj, words + 0,
                                 B.scan_partials.as<uint32_t>(), s)))
        return rc;
    k_hier_obj_offsets<<<grid_of(c, h->nobj, 256), 256, 0, s>>>(h->cnt.as<uint32_t>(), h->nobj, h->objs.as<HierObj>());
    k_hier_count<<<nb, kBT, 0, s>>>(c->tris.as<float4>(), h->objs.as<HierObj>(), h->tri_begin.as<uint32_t>(), h->nobj,
                                    h->ntri, B.block_sums.as<uint32_t>());
    if ((rc = scan_block_sums(c, B.block_sums.as<uint32_t>(), nb, words + 1, words + 3, 0xffffffffu, 2u, words + 6, s)))
        return rc;
    uint32_t hw[10];
    if ((rc = cuda_check(c, cudaMemcpyAsync(hw, words, sizeof(hw), cudaMemcpyDeviceToHost, s), "hier counts")) ||
        (rc = cuda_check(c, cudaStreamSynchronize(s), "hier counts")))
        return rc;
    uint64_t cells64;
    std::memcpy(&cells64, hw + 8, 8);
    if (hw[3] || cells64 >= (1ull << 31))
        return set_error(c, HR_ERR_INVALID_ARG, "hier: the object grids need more than 2^31 cells or 2^32 pairs");
    h->num_obj_cells = hw[0];
    h->num_pairs = hw[1];
    const size_t np = std::max<size_t>(h->num_pairs, 1);
    const int kb = key_bits(h->num_obj_cells);
    if ((rc = ensure(c, B.keys_a, 4 * np)) || (rc = ensure(c, B.vals_a, 4 * np)) || (rc = ensure(c, B.keys_b, 4 * np)) ||
        (rc = ensure(c, B.vals_b, 4 * np)) || (rc = ensure(c, h->prims, 4 * np)) ||
        (rc = ensure(c, h->obj_cells, sizeof(uint2) * std::max<uint32_t>(h->num_obj_cells, 1))) ||
        (rc = ensure(c, B.tile_hist, sizeof(uint32_t) * radix_tile_hist_words(np, kb))) ||
        (rc = ensure(c, B.row_total, sizeof(uint32_t) * kRadixRowWords)))
        return rc;
    c->launches += 1;
    k_hier_write<<<nb, kBT, 0, s>>>(c->tris.as<float4>(), h->objs.as<HierObj>(), h->tri_begin.as<uint32_t>(), h->nobj,
                                    h->ntri, B.block_sums.as<uint32_t>(), B.keys_a.as<uint32_t>(),
                                    B.vals_a.as<uint32_t>());
    const int passes = radix_sort_passes(kb);
    uint32_t* sorted = (passes % 2 == 1) ? B.keys_b.as<uint32_t>() : B.keys_a.as<uint32_t>();
    if ((rc = radix_sort_pairs(c, B.keys_a.as<uint32_t>(), B.vals_a.as<uint32_t>(), B.keys_b.as<uint32_t>(),
                               B.vals_b.as<uint32_t>(), sorted, h->prims.as<uint32_t>(), words + 1, np, kb,
                               B.tile_hist.as<uint32_t>(), B.tile_hist.bytes, B.row_total.as<uint32_t>(), s)))
        return rc;
    // k_fill_u2 / k_cell_ranges read the overflow bits of a descriptor: the instance
    // grid's, cleared here
    GridDesc* td = h->top_desc.as<GridDesc>();
    if ((rc = cuda_check(c, cudaMemsetAsync(td, 0, sizeof(GridDesc), s), "hier desc"))) return rc;
    const int gc = grid_of(c, h->num_obj_cells, 256);
    c->launches += 2;
    k_fill_u2<<<gc, 256, 0, s>>>(h->obj_cells.as<uint2>(), words + 0, td, make_uint2(0u, 0u));
    k_cell_ranges<<<grid_of(c, np, 256), 256, 0, s>>>(sorted, words + 1, words + 0, td, h->obj_cells.as<uint2>());
    return cuda_check(c, cudaGetLastError(), "hier object grids");
}

// level one: instance grid
int build_instances(hr_hier* h) {
    hr_ctx* c = h->c;
    cudaStream_t s = c->stream;
    GridBuffers& B = c->g;
    uint32_t* words = h->words.as<uint32_t>();
    GridDesc* td = h->top_desc.as<GridDesc>();
    int rc;
    if ((rc = ensure(c, h->icnt, sizeof(uint32_t) * (h->ninst + 1))) ||
        (rc = ensure(c, B.scan_partials, sizeof(uint32_t) * (scan_partials_words(std::max(h->ninst, h->nobj)) + 2))))
        return rc;
    c->launches += 2;
    k_hier_top_setup<<<1, kBT, 0, s>>>(h->inst.as<HierInst>(), h->ninst, h->top_density, td);
    k_hier_inst_count<<<grid_of(c, h->ninst, 256), 256, 0, s>>>(h->inst.as<HierInst>(), h->ninst, td,
                                                                h->icnt.as<uint32_t>());
    if ((rc = exclusive_scan_u32(c, h->icnt.as<uint32_t>(), words + 5, h->ninst, words + 2,
                                 B.scan_partials.as<uint32_t>(), s)))
        return rc;
    uint32_t ntp = 0;
    if ((rc = cuda_check(c, cudaMemcpyAsync(&h->top, td, sizeof(GridDesc), cudaMemcpyDeviceToHost, s), "hier top")) ||
        (rc = cuda_check(c, cudaMemcpyAsync(&ntp, words + 2, 4, cudaMemcpyDeviceToHost, s), "hier top")) ||
        (rc = cuda_check(c, cudaStreamSynchronize(s), "hier top")))
        return rc;
    if (h->top.error) return set_error(c, HR_ERR_INVALID_ARG, "hier: the instance grid has more than 2^30 cells");
    h->num_top_pairs = ntp;
    const size_t np = std::max<size_t>(ntp, 1);
    const int kb = key_bits(h->top.ncells);
    if ((rc = ensure(c, B.keys_a, 4 * np)) || (rc = ensure(c, B.vals_a, 4 * np)) || (rc = ensure(c, B.keys_b, 4 * np)) ||
        (rc = ensure(c, B.vals_b, 4 * np)) || (rc = ensure(c, h->inst_ids, 4 * np)) ||
        (rc = ensure(c, h->top_cells, sizeof(uint2) * h->top.ncells)) ||
        (rc = ensure(c, B.tile_hist, sizeof(uint32_t) * radix_tile_hist_words(np, kb))) ||
        (rc = ensure(c, B.row_total, sizeof(uint32_t) * kRadixRowWords)))
        return rc;
    c->launches += 1;
    k_hier_inst_write<<<grid_of(c, h->ninst, 256), 256, 0, s>>>(h->inst.as<HierInst>(), h->ninst, td,
                                                                h->icnt.as<uint32_t>(), B.keys_a.as<uint32_t>(),
                                                                B.vals_a.as<uint32_t>());
    const int passes = radix_sort_passes(kb);
    uint32_t* sorted = (passes % 2 == 1) ? B.keys_b.as<uint32_t>() : B.keys_a.as<uint32_t>();
    if ((rc = radix_sort_pairs(c, B.keys_a.as<uint32_t>(), B.vals_a.as<uint32_t>(), B.keys_b.as<uint32_t>(),
                               B.vals_b.as<uint32_t>(), sorted, h->inst_ids.as<uint32_t>(), words + 2, np, kb,
                               B.tile_hist.as<uint32_t>(), B.tile_hist.bytes, B.row_total.as<uint32_t>(), s)))
        return rc;
    c->launches += 2;
    k_fill_u2<<<grid_of(c, h->top.ncells, 256), 256, 0, s>>>(h->top_cells.as<uint2>(), &td->ncells, td,
                                                             make_uint2(0u, 0u));
    k_cell_ranges<<<grid_of(c, np, 256), 256, 0, s>>>(sorted, words + 2, &td->ncells, td, h->top_cells.as<uint2>());
    return cuda_check(c, cudaGetLastError(), "hier instance grid");
}

HierView view(hr_hier* h) {
    HierView v;
    v.tris = h->c->tris.as<float4>();
    v.objs = h->objs.as<HierObj>();
    v.inst = h->inst.as<HierInst>();
    v.top = h->top_desc.as<GridDesc>();
    v.top_cells = h->top_cells.as<uint2>();
    v.inst_ids = h->inst_ids.as<uint32_t>();
    v.obj_cells = h->obj_cells.as<uint2>();
    v.prims = h->prims.as<uint32_t>();
    return v;
}

bool bad_hier(const hr_hier* h) { return !h || !h->c; }

}  // namespace
}  // namespace hr

extern "C" {

hr_status hr_hier_create(hr_hier** out, int32_t device, void* stream) {
    if (!out) return HR_ERR_INVALID_ARG;
    *out = nullptr;
    hr_hier* h = new (std::nothrow) hr_hier();
    if (!h) return HR_ERR_OUT_OF_MEMORY;
    hr_status st = hr_create(&h->c, device, stream);
    if (st != HR_OK) {
        delete h;
        return st;
    }
    DeviceGuard dg(h->c->device);
    int rc;
    if ((rc = ensure(h->c, h->words, 64)) || (rc = ensure(h->c, h->top_desc, sizeof(GridDesc))) ||
        (rc = cuda_check(h->c, cudaMemsetAsync(h->words.p, 0, 64, h->c->stream), "hier init"))) {
        hr_hier_destroy(h);
        return (hr_status)rc;
    }
    *out = h;
    return HR_OK;
}

void hr_hier_destroy(hr_hier* h) {
    if (!h) return;
    if (h->c) {
        DeviceGuard dg(h->c->device);
        cudaStream_t s = h->c->stream;
        DevBuf* bufs[] = {&h->tri_begin, &h->enc, &h->objs, &h->cnt, &h->obj_cells, &h->prims, &h->inst,
                          &h->top_desc, &h->icnt, &h->top_cells, &h->inst_ids, &h->words, &h->rays};
        for (DevBuf* b : bufs) free_dev(*b, s);
        cudaStreamSynchronize(s);
        hr_destroy(h->c);
    }
    delete h;
}

const char* hr_hier_last_error(const hr_hier* h) { return h && h->c ? h->c->err.c_str() : "no hierarchy"; }

hr_status hr_hier_set_objects(hr_hier* h, const float* verts_xyz, uint32_t nv, const uint32_t* idx, uint32_t ntri,
                              const uint32_t* counts, uint32_t nobj) {
    if (bad_hier(h) || !verts_xyz || !idx || !counts || nv == 0 || ntri == 0 || nobj == 0) return HR_ERR_INVALID_ARG;
    hr_ctx* c = h->c;
    std::vector<uint32_t> begin(nobj + 1, 0u);
    for (uint32_t k = 0; k < nobj; ++k) {
        if (counts[k] == 0) return (hr_status)set_error(c, HR_ERR_INVALID_ARG, "hier: object %u has no triangle", k);
        begin[k + 1] = begin[k] + counts[k];
        if (begin[k + 1] < begin[k] || begin[k + 1] > ntri) break;
    }
    if (begin[nobj] != ntri)
        return (hr_status)set_error(c, HR_ERR_INVALID_ARG, "hier: object triangle counts do not sum to %u", ntri);
    for (size_t i = 0; i < 3 * (size_t)ntri; ++i)
        if (idx[i] >= nv) return (hr_status)set_error(c, HR_ERR_INVALID_ARG, "hier: triangle index out of range");
    for (size_t i = 0; i < 3 * (size_t)nv; ++i)
        if (!std::isfinite(verts_xyz[i])) return (hr_status)set_error(c, HR_ERR_INVALID_ARG, "hier: non-finite vertex");
    DeviceGuard dg(c->device);
    cudaStream_t s = c->stream;
    int rc;
    if ((rc = ensure(c, c->staging, 12 * (size_t)nv)) || (rc = ensure(c, c->verts, sizeof(float4) * (size_t)nv)) ||
        (rc = ensure(c, c->idx, 12 * (size_t)ntri)) || (rc = ensure(c, h->tri_begin, 4 * ((size_t)nobj + 1))) ||
        (rc = cuda_check(c, cudaMemcpyAsync(c->staging.p, verts_xyz, 12 * (size_t)nv, cudaMemcpyHostToDevice, s), "verts")) ||
        (rc = cuda_check(c, cudaMemcpyAsync(c->idx.p, idx, 12 * (size_t)ntri, cudaMemcpyHostToDevice, s), "indices")) ||
        (rc = cuda_check(c, cudaMemcpyAsync(h->tri_begin.p, begin.data(), 4 * ((size_t)nobj + 1), cudaMemcpyHostToDevice, s),
                         "objects")))
        return (hr_status)rc;
    expand_xyz(c->staging.as<float>(), c->verts.as<float4>(), nv, grid_of(c, nv, 256), s);
    if ((rc = cuda_check(c, cudaStreamSynchronize(s), "hier objects"))) return (hr_status)rc;
    h->nv = nv;
    h->ntri = ntri;
    h->nobj = nobj;
    h->have_objects = true;
    h->objects_dirty = true;
    h->built = false;
    if ((rc = cuda_check(c, cudaMemcpyAsync(h->words.as<uint32_t>() + 4, &nobj, 4, cudaMemcpyHostToDevice, s), "hier")))
        return (hr_status)rc;
    return (hr_status)cuda_check(c, cudaStreamSynchronize(s), "hier objects");
}

hr_status hr_hier_set_instances(hr_hier* h, const hr_instance* inst, uint32_t n) {
    if (bad_hier(h) || !inst || n == 0) return HR_ERR_INVALID_ARG;
    hr_ctx* c = h->c;
    if (!h->have_objects) return (hr_status)set_error(c, HR_ERR_NOT_READY, "hier: set the objects first");
    std::vector<HierInst> hi(n);
    for (uint32_t i = 0; i < n; ++i) {
        const hr_instance& r = inst[i];
        if (r.object >= h->nobj) return (hr_status)set_error(c, HR_ERR_INVALID_ARG, "hier: instance %u: no object %u", i, r.object);
        for (int k = 0; k < 12; ++k)
            if (!std::isfinite(r.m[k])) return (hr_status)set_error(c, HR_ERR_INVALID_ARG, "hier: instance %u: bad matrix", i);
        for (int k = 0; k < 3; ++k)
            if (!std::isfinite(r.bmin[k]) || !std::isfinite(r.bmax[k]) || !(r.bmin[k] <= r.bmax[k]))
                return (hr_status)set_error(c, HR_ERR_INVALID_ARG, "hier: instance %u: bad box", i);
        uint32_t ob = r.object;
        float fob;
        std::memcpy(&fob, &ob, 4);
        hi[i].r0 = make_float4(r.m[0], r.m[1], r.m[2], r.m[3]);
        hi[i].r1 = make_float4(r.m[4], r.m[5], r.m[6], r.m[7]);
        hi[i].r2 = make_float4(r.m[8], r.m[9], r.m[10], r.m[11]);
        hi[i].lo = make_float4(r.bmin[0], r.bmin[1], r.bmin[2], fob);
        hi[i].hi = make_float4(r.bmax[0], r.bmax[1], r.bmax[2], 0.0f);
    }
    DeviceGuard dg(c->device);
    int rc;
    if ((rc = ensure(c, h->inst, sizeof(HierInst) * n)) ||
        (rc = cuda_check(c, cudaMemcpyAsync(h->inst.p, hi.data(), sizeof(HierInst) * n, cudaMemcpyHostToDevice, c->stream),
                         "instances")) ||
        (rc = cuda_check(c, cudaMemcpyAsync(h->words.as<uint32_t>() + 5, &n, 4, cudaMemcpyHostToDevice, c->stream),
                         "instances")) ||
        (rc = cuda_check(c, cudaStreamSynchronize(c->stream), "instances")))
        return (hr_status)rc;
    h->ninst = n;
    h->have_instances = true;
    h->built = false;
    return HR_OK;
}

hr_status hr_hier_set_densities(hr_hier* h, float top, float obj) {
    if (bad_hier(h) || !(top > 0.0f) || !(obj > 0.0f) || !std::isfinite(top) || !std::isfinite(obj)) return HR_ERR_INVALID_ARG;
    if (obj != h->obj_density) h->objects_dirty = true;
    h->top_density = top;
    h->obj_density = obj;
    h->built = false;
    return HR_OK;
}

hr_status hr_hier_build(hr_hier* h) {
    if (bad_hier(h)) return HR_ERR_INVALID_ARG;
    hr_ctx* c = h->c;
    if (!h->have_objects || !h->have_instances)
        return (hr_status)set_error(c, HR_ERR_NOT_READY, "hier: set objects and instances first");
    DeviceGuard dg(c->device);
    int rc;
    if (h->objects_dirty) {
        if ((rc = build_objects(h))) return (hr_status)rc;
        h->objects_dirty = false;
    }
    if ((rc = build_instances(h))) return (hr_status)rc;
    if ((rc = cuda_check(c, cudaStreamSynchronize(c->stream), "hier build"))) return (hr_status)rc;
    h->built = true;
    return HR_OK;
}

hr_status hr_hier_get_info(hr_hier* h, hr_hier_info* info) {
    if (bad_hier(h) || !info) return HR_ERR_INVALID_ARG;
    if (!h->built) return (hr_status)set_error(h->c, HR_ERR_NOT_READY, "hier: not built");
    std::memset(info, 0, sizeof(*info));
    info->num_objects = h->nobj;
    info->num_instances = h->ninst;
    info->num_triangles = h->ntri;
    info->num_object_cells = h->num_obj_cells;
    info->num_pairs = h->num_pairs;
    for (int k = 0; k < 3; ++k) {
        info->top_res[k] = h->top.res[k];
        info->top_bmin[k] = h->top.bmin[k];
        info->top_bmax[k] = h->top.bmax[k];
    }
    info->num_top_cells = h->top.ncells;
    info->num_top_pairs = h->num_top_pairs;
    info->launches = h->c->launches;
    return HR_OK;
}

hr_status hr_hier_download(hr_hier* h, hr_hier_object* objects, uint32_t* object_cells, uint32_t* triangles,
                           uint32_t* top_cells, uint32_t* instances) {
    if (bad_hier(h)) return HR_ERR_INVALID_ARG;
    hr_ctx* c = h->c;
    if (!h->built) return (hr_status)set_error(c, HR_ERR_NOT_READY, "hier: not built");
    DeviceGuard dg(c->device);
    struct { void* dst; const DevBuf* src; size_t bytes; } cp[] = {
        {objects, &h->objs, sizeof(HierObj) * h->nobj},
        {object_cells, &h->obj_cells, sizeof(uint2) * h->num_obj_cells},
        {triangles, &h->prims, 4 * (size_t)h->num_pairs},
        {top_cells, &h->top_cells, sizeof(uint2) * h->top.ncells},
        {instances, &h->inst_ids, 4 * (size_t)h->num_top_pairs},
    };
    for (auto& x : cp) {
        if (!x.dst || x.bytes == 0) continue;
        int rc = cuda_check(c, cudaMemcpyAsync(x.dst, x.src->p, x.bytes, cudaMemcpyDeviceToHost, c->stream), "hier download");
        if (rc) return (hr_status)rc;
    }
    return (hr_status)cuda_check(c, cudaStreamSynchronize(c->stream), "hier download");
}

hr_status hr_hier_trace_rays_device(hr_hier* h, const float* org, const float* dir, uint32_t n, int32_t* inst_id,
                                    int32_t* tri_id, float* t, float* u, float* v) {
    if (bad_hier(h) || (n && (!org || !dir || !inst_id || !tri_id || !t || !u || !v))) return HR_ERR_INVALID_ARG;
    hr_ctx* c = h->c;
    if (!h->built) return (hr_status)set_error(c, HR_ERR_NOT_READY, "hier: build first");
    if (n == 0) return HR_OK;
    DeviceGuard dg(c->device);
    c->launches += 1;
    uint32_t* pool = h->words.as<uint32_t>() + 7;
    if (cudaMemsetAsync(pool, 0, 4, c->stream) != cudaSuccess)
        return (hr_status)cuda_check(c, cudaGetLastError(), "hier ray pool");
    k_hier_trace<false, false><<<hier_grid<false, false>(c, n), kTT, 0, c->stream>>>(view(h), org, dir, nullptr, n,
                                                                                    inst_id, tri_id, t, u, v, nullptr,
                                                                                    nullptr, pool);
    return (hr_status)cuda_check(c, cudaGetLastError(), "hier trace launch");
}

hr_status hr_hier_trace_stats_device(hr_hier* h, const float* org, const float* dir, uint32_t n, int32_t* inst_id,
                                     int32_t* tri_id, float* t, float* u, float* v, uint32_t* stats) {
    if (bad_hier(h) || (n && (!org || !dir || !inst_id || !tri_id || !t || !u || !v || !stats))) return HR_ERR_INVALID_ARG;
    hr_ctx* c = h->c;
    if (!h->built) return (hr_status)set_error(c, HR_ERR_NOT_READY, "hier: build first");
    if (n == 0) return HR_OK;
    DeviceGuard dg(c->device);
    c->launches += 1;
    uint32_t* pool = h->words.as<uint32_t>() + 7;
    if (cudaMemsetAsync(pool, 0, 4, c->stream) != cudaSuccess)
        return (hr_status)cuda_check(c, cudaGetLastError(), "hier ray pool");
    k_hier_trace<false, true><<<hier_grid<false, true>(c, n), kTT, 0, c->stream>>>(view(h), org, dir, nullptr, n,
                                                                                  inst_id, tri_id, t, u, v, nullptr,
                                                                                  stats, pool);
    return (hr_status)cuda_check(c, cudaGetLastError(), "hier trace launch");
}

hr_status hr_hier_trace_rays(hr_hier* h, const float* org, const float* dir, uint32_t n, int32_t* inst_id,
                             int32_t* tri_id, float* t, float* u, float* v) {
    if (bad_hier(h) || (n && (!org || !dir || !inst_id || !tri_id || !t || !u || !v))) return HR_ERR_INVALID_ARG;
    hr_ctx* c = h->c;
    if (!h->built) return (hr_status)set_error(c, HR_ERR_NOT_READY, "hier: build first");
    if (n == 0) return HR_OK;
    DeviceGuard dg(c->device);
    cudaStream_t s = c->stream;
    int rc;
    if ((rc = ensure(c, h->rays, 44 * (size_t)n))) return (hr_status)rc;
    float* dorg = h->rays.as<float>();
    float* ddir = dorg + 3 * (size_t)n;
    int32_t* di = reinterpret_cast<int32_t*>(ddir + 3 * (size_t)n);
    int32_t* dt = di + n;
    float* dtt = reinterpret_cast<float*>(dt + n);
    float* du = dtt + n;
    float* dv = du + n;
    if ((rc = cuda_check(c, cudaMemcpyAsync(dorg, org, 12 * (size_t)n, cudaMemcpyHostToDevice, s), "rays")) ||
        (rc = cuda_check(c, cudaMemcpyAsync(ddir, dir, 12 * (size_t)n, cudaMemcpyHostToDevice, s), "rays")))
        return (hr_status)rc;
    if ((rc = hr_hier_trace_rays_device(h, dorg, ddir, n, di, dt, dtt, du, dv))) return (hr_status)rc;
    void* outs[] = {inst_id, tri_id, t, u, v};
    const void* srcs[] = {di, dt, dtt, du, dv};
    for (int k = 0; k < 5; ++k)
        if ((rc = cuda_check(c, cudaMemcpyAsync(outs[k], srcs[k], 4 * (size_t)n, cudaMemcpyDeviceToHost, s), "hits")))
            return (hr_status)rc;
    return (hr_status)cuda_check(c, cudaStreamSynchronize(s), "hier trace");
}

hr_status hr_hier_occluded(hr_hier* h, const float* org, const float* dir, const float* tmax, uint32_t n,
                           uint8_t* occluded) {
    if (bad_hier(h) || (n && (!org || !dir || !tmax || !occluded))) return HR_ERR_INVALID_ARG;
    hr_ctx* c = h->c;
    if (!h->built) return (hr_status)set_error(c, HR_ERR_NOT_READY, "hier: build first");
    if (n == 0) return HR_OK;
    DeviceGuard dg(c->device);
    cudaStream_t s = c->stream;
    int rc;
    if ((rc = ensure(c, h->rays, 29 * (size_t)n + 16))) return (hr_status)rc;
    float* dorg = h->rays.as<float>();
    float* ddir = dorg + 3 * (size_t)n;
    float* dtm = ddir + 3 * (size_t)n;
    uint8_t* docc = reinterpret_cast<uint8_t*>(dtm + n);
    if ((rc = cuda_check(c, cudaMemcpyAsync(dorg, org, 12 * (size_t)n, cudaMemcpyHostToDevice, s), "rays")) ||
        (rc = cuda_check(c, cudaMemcpyAsync(ddir, dir, 12 * (size_t)n, cudaMemcpyHostToDevice, s), "rays")) ||
        (rc = cuda_check(c, cudaMemcpyAsync(dtm, tmax, 4 * (size_t)n, cudaMemcpyHostToDevice, s), "rays")))
        return (hr_status)rc;
    c->launches += 1;
    uint32_t* pool = h->words.as<uint32_t>() + 7;
    if ((rc = cuda_check(c, cudaMemsetAsync(pool, 0, 4, s), "hier ray pool"))) return (hr_status)rc;
    k_hier_trace<true, false><<<hier_grid<true, false>(c, n), kTT, 0, s>>>(view(h), dorg, ddir, dtm, n, nullptr, nullptr,
                                                                          nullptr, nullptr, nullptr, docc, nullptr, pool);
    if ((rc = cuda_check(c, cudaGetLastError(), "hier occluded launch")) ||
        (rc = cuda_check(c, cudaMemcpyAsync(occluded, docc, n, cudaMemcpyDeviceToHost, s), "occluded")))
        return (hr_status)rc;
    return (hr_status)cuda_check(c, cudaStreamSynchronize(s), "hier occluded");
}

}  // extern "C"
