// build_dev.cuh -- device-side pieces of the grid build shared by the per-scene pipeline
// (build.cu) and the batched pipeline (batch.cu).
//
// Reference path (javorkk/happyray):
//   resolution                 src/RT/Algorithm/UGridSortBuilder.h:78-92, TLGridSortBuilder.h:80-92
//   exact triangle/box test    src/RT/Algorithm/UniformGridBuildKernels.cu:8-48, 299-366
//   cell ranges                src/RT/Algorithm/UniformGridBuildKernels.h:384-487
//   leaf resolution            src/RT/Algorithm/TLGridBuildKernels.h:55-87, 338-377
#pragma once

#include "hr_internal.h"
#include "hr_block.cuh"

namespace hr {
namespace {

constexpr int kBT = 256;   // build block size

__device__ __forceinline__ float pow_third(float x) { return (float)pow((double)x, (double)0.3333333f); }

__device__ __forceinline__ void desc_init(GridDesc* d, int32_t kind, uint32_t ntri, uint32_t error) {
    d->bmin_enc[0] = d->bmin_enc[1] = d->bmin_enc[2] = fenc(FLT_MAX);
    d->bmax_enc[0] = d->bmax_enc[1] = d->bmax_enc[2] = fenc(-FLT_MAX);
    d->ncells = d->npairs = d->ntop_pairs = d->nleaves = 0u;
    d->overflow = 0u;
    d->error = error;
    d->kind = kind;
    d->ntri = ntri;
}

// a2: padded bounds (WFObjectUploader.h:112-114) and resolution (UGridSortBuilder.h:78-92,
// UGridMemoryManager.cu:338-345, UGridMemoryManager.h:93-101) from the reduced bounds of
// d; returns the cell count (64-bit, the caller checks it against its capacity).
__device__ __forceinline__ uint64_t grid_setup(GridDesc* d, float density) {
    f3 lo = mk(fdec(d->bmin_enc[0]), fdec(d->bmin_enc[1]), fdec(d->bmin_enc[2]));
    f3 hi = mk(fdec(d->bmax_enc[0]), fdec(d->bmax_enc[1]), fdec(d->bmax_enc[2]));
    f3 dd = sub(hi, lo);
    float diag = sqrtf(dot(dd, dd));
    float pad = 0.001f * diag;
    d->bmin[0] = lo.x - pad; d->bmin[1] = lo.y - pad; d->bmin[2] = lo.z - pad;
    d->bmax[0] = hi.x + pad; d->bmax[1] = hi.y + pad; d->bmax[2] = hi.z + pad;
    f3 e = mk(d->bmax[0] - d->bmin[0], d->bmax[1] - d->bmin[1], d->bmax[2] - d->bmin[2]);
    float vol = e.x * e.y * e.z;
    float m = pow_third(density * (float)d->ntri / vol);
    e = mulf(e, m);
    int32_t r[3] = {f2i(e.x), f2i(e.y), f2i(e.z)};
    if (r[0] <= 0 || r[1] <= 0 || r[2] <= 0) r[0] = r[1] = r[2] = 32;
    for (int k = 0; k < 3; ++k) {
        d->res[k] = r[k];
        float dk = d->bmax[k] - d->bmin[k];
        d->cs[k] = dk / (float)r[k];
        d->rcp[k] = (float)r[k] / dk;
    }
    return (uint64_t)r[0] * (uint64_t)r[1] * (uint64_t)r[2];
}

__device__ __forceinline__ void reduce_bounds(f3 lo, f3 hi, GridDesc* d) {
    __shared__ float s[6][kBT / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lo.x = hmin(lo.x, __shfl_xor_sync(kFullMask, lo.x, o));
        lo.y = hmin(lo.y, __shfl_xor_sync(kFullMask, lo.y, o));
        lo.z = hmin(lo.z, __shfl_xor_sync(kFullMask, lo.z, o));
        hi.x = hmax(hi.x, __shfl_xor_sync(kFullMask, hi.x, o));
        hi.y = hmax(hi.y, __shfl_xor_sync(kFullMask, hi.y, o));
        hi.z = hmax(hi.z, __shfl_xor_sync(kFullMask, hi.z, o));
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) { s[0][w] = lo.x; s[1][w] = lo.y; s[2][w] = lo.z; s[3][w] = hi.x; s[4][w] = hi.y; s[5][w] = hi.z; }
    __syncthreads();
    if (threadIdx.x < 6) {
        float v = s[threadIdx.x][0];
        for (int i = 1; i < kBT / 32; ++i) v = threadIdx.x < 3 ? hmin(v, s[threadIdx.x][i]) : hmax(v, s[threadIdx.x][i]);
        if (threadIdx.x < 3) atomicMin(&d->bmin_enc[threadIdx.x], fenc(v));
        else atomicMax(&d->bmax_enc[threadIdx.x - 3], fenc(v));
    }
}

struct DescRegs {
    f3 bmin, cs;
    float rcp[3];
    int32_t res[3];
    uint32_t ncells;
};
__device__ __forceinline__ DescRegs load_desc(const GridDesc* d) {
    DescRegs r;
    r.bmin = mk(d->bmin[0], d->bmin[1], d->bmin[2]);
    r.cs = mk(d->cs[0], d->cs[1], d->cs[2]);
    for (int k = 0; k < 3; ++k) { r.rcp[k] = d->rcp[k]; r.res[k] = d->res[k]; }
    r.ncells = d->ncells;
    return r;
}

// exact triangle/box test, UniformGridBuildKernels.cu:8-48, 299-366
__device__ __forceinline__ bool axis_test(float a, float b, float fa, float fb, float v0a, float v0b,
                                          float v1a, float v1b, float ha, float hb) {
    float p0 = a * v0a + b * v0b;
    float p1 = a * v1a + b * v1b;
    float mn = hmin(p0, p1), mx = hmax(p0, p1);
    float rad = fa * ha + fb * hb;
    return !(mn > rad + kEps || mx + kEps < -rad);
}
__device__ __forceinline__ bool sat_overlap(f3 nrm, f3 c, const f3* tv, f3 h) {
    f3 v0 = sub(tv[0], c), v1 = sub(tv[1], c), v2 = sub(tv[2], c);
    f3 e0 = sub(v1, v0), e1 = sub(v2, v1), e2 = sub(v0, v2);
    bool pass = true;
    f3 mn, mx;
    mn.x = (nrm.x > 0.0f) ? -h.x : h.x;
    mn.y = (nrm.y > 0.0f) ? -h.y : h.y;
    mn.z = (nrm.z > 0.0f) ? -h.z : h.z;
    mx = mk(-mn.x, -mn.y, -mn.z);
    mx = sub(mx, v0);
    mn = sub(mn, v0);
    pass = pass && dot(nrm, mn) <= 0.0f && dot(nrm, mx) > 0.0f;
    f3 fe = mk(fabsf(e0.x), fabsf(e0.y), fabsf(e0.z));
    pass = pass && axis_test(e0.z, -e0.y, fe.z, fe.y, v0.y, v0.z, v2.y, v2.z, h.y, h.z);
    pass = pass && axis_test(-e0.z, e0.x, fe.z, fe.x, v0.x, v0.z, v2.x, v2.z, h.x, h.z);
    pass = pass && axis_test(e0.y, -e0.x, fe.y, fe.x, v1.x, v1.y, v2.x, v2.y, h.x, h.y);
    fe = mk(fabsf(e1.x), fabsf(e1.y), fabsf(e1.z));
    pass = pass && axis_test(e1.z, -e1.y, fe.z, fe.y, v0.y, v0.z, v2.y, v2.z, h.y, h.z);
    pass = pass && axis_test(-e1.z, e1.x, fe.z, fe.x, v0.x, v0.z, v2.x, v2.z, h.x, h.z);
    pass = pass && axis_test(e1.y, -e1.x, fe.y, fe.x, v0.x, v0.y, v1.x, v1.y, h.x, h.y);
    fe = mk(fabsf(e2.x), fabsf(e2.y), fabsf(e2.z));
    pass = pass && axis_test(e2.z, -e2.y, fe.z, fe.y, v0.y, v0.z, v1.y, v1.z, h.y, h.z);
    pass = pass && axis_test(-e2.z, e2.x, fe.z, fe.x, v0.x, v0.z, v1.x, v1.z, h.x, h.z);
    pass = pass && axis_test(e2.y, -e2.x, fe.y, fe.x, v1.x, v1.y, v2.x, v2.y, h.x, h.y);
    return pass;
}

__global__ void k_fill_u2(uint2* a, const uint32_t* d_count, const GridDesc* d, uint2 val) {
    if (d->overflow | d->error) return;   // counts may exceed the buffers after an overflow
    const uint32_t n = *d_count;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a[i] = val;
}

// a7 / a13: cell (or leaf) ranges from sorted keys (UniformGridBuildKernels.h:384-487,
// TLGridBuildKernels.h:750-834); keys >= *d_ncells (rejected exact-insertion pairs) are skipped
__global__ void k_cell_ranges(const uint32_t* __restrict__ keys, const uint32_t* d_count, const uint32_t* d_ncells,
                              const GridDesc* d, uint2* cells) {
    if (d->overflow | d->error) return;
    const uint32_t n = *d_count, C = *d_ncells;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t k = keys[i];
        if (k >= C) continue;
        if (i == 0 || keys[i - 1] != k) cells[k].x = i;
        if (i + 1 == n || keys[i + 1] != k) cells[k].y = i + 1;
    }
}

// a8: leaf resolution of a top cell (TLGridBuildKernels.h:55-87)
struct LeafGeom { uint32_t res[3]; bool leaf; };
__device__ __forceinline__ LeafGeom leaf_geom(const DescRegs& g, uint32_t refs, float leaf_density) {
    LeafGeom lg;
    float vol = g.cs.x * g.cs.y * g.cs.z;
    float m = pow_third(leaf_density * (float)refs / vol);
    lg.leaf = refs <= kLeafRefsMax;
    float r0 = hmin(255.0f, hmax(1.0f, g.cs.x * m));
    float r1 = hmin(255.0f, hmax(1.0f, g.cs.y * m));
    float r2 = hmin(255.0f, hmax(1.0f, g.cs.z * m));
    lg.res[0] = lg.leaf ? 1u : (uint32_t)r0;
    lg.res[1] = lg.leaf ? 1u : (uint32_t)r1;
    lg.res[2] = lg.leaf ? 1u : (uint32_t)r2;
    return lg;
}

// sub-cell range of a triangle inside top cell c (TLGridBuildKernels.h:338-377)
__device__ __forceinline__ uint32_t leaf_range(const DescRegs& g, const uint32_t* lres, uint32_t c, f3 lo, f3 hi,
                                               CRange* r) {
    const uint32_t rx = (uint32_t)g.res[0], rxy = (uint32_t)g.res[0] * (uint32_t)g.res[1];
    const uint32_t cc[3] = {c % rx, (c % rxy) / rx, c / rxy};
    f3 org;
    org.x = (float)cc[0] * g.cs.x + g.bmin.x;
    org.y = (float)cc[1] * g.cs.y + g.bmin.y;
    org.z = (float)cc[2] * g.cs.z + g.bmin.z;
    float srcp[3] = {(float)lres[0] / g.cs.x, (float)lres[1] / g.cs.y, (float)lres[2] / g.cs.z};
    int32_t ires[3] = {(int32_t)lres[0], (int32_t)lres[1], (int32_t)lres[2]};
    return cell_range(lo, hi, org, srcp, ires, r);
}

// The count passes keep each triangle's cell range, 16-bit coordinates (lo | hi << 16 per
// axis in .x .y .z, pair count in .w), so that the scatter pass reads 16 bytes per
// triangle instead of its 48-byte vertex record; a grid with an axis of more than 65,535
// cells keeps recomputing them from the vertices.
__device__ __forceinline__ bool ranges_fit(const int32_t* res) {
    return res[0] <= 65535 && res[1] <= 65535 && res[2] <= 65535;
}
__device__ __forceinline__ uint4 pack_range(const CRange& r, uint32_t n) {
    uint32_t w[3];
#pragma unroll
    for (int k = 0; k < 3; ++k)
        w[k] = (uint32_t)min(max(r.lo[k], 0), 65535) | ((uint32_t)min(max(r.hi[k], 0), 65535) << 16);
    return make_uint4(w[0], w[1], w[2], n);
}
__device__ __forceinline__ uint32_t unpack_range(uint4 q, CRange* r) {
    r->lo[0] = (int32_t)(q.x & 0xFFFFu); r->hi[0] = (int32_t)(q.x >> 16);
    r->lo[1] = (int32_t)(q.y & 0xFFFFu); r->hi[1] = (int32_t)(q.y >> 16);
    r->lo[2] = (int32_t)(q.z & 0xFFFFu); r->hi[2] = (int32_t)(q.z >> 16);
    return q.w;
}

// Per top-level reference the leaf count pass keeps what the leaf scatter pass needs, 16 bytes:
// .x = lo.x | lo.y << 8 | lo.z << 16 | lres.x << 24, .y = hi.x | hi.y << 8 | hi.z << 16 |
// lres.y << 24 (sub-grid coordinates and resolutions are below 256), .z = the top cell's
// first leaf, .w = the triangle.
__device__ __forceinline__ uint4 pack_ref(const CRange& r, const uint32_t* lres, uint32_t base, uint32_t tri) {
    uint32_t a = 0, b = 0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        a |= (uint32_t)min(max(r.lo[k], 0), 255) << (8 * k);
        b |= (uint32_t)min(max(r.hi[k], 0), 255) << (8 * k);
    }
    return make_uint4(a | (lres[0] << 24), b | (lres[1] << 24), base, tri);
}

__global__ void k_check_leaves(GridDesc* d, uint32_t cap_leaves) {
    if (d->overflow | d->error) return;   // the leaf total is meaningless after an earlier overflow
    if (d->nleaves > cap_leaves) d->overflow |= kOvfLeaves;
}

// a9: first leaf of every top cell (prepareTopLevelCellRanges, TLGridBuildKernels.h:130-147)
__global__ void k_tl_cell_begin(const uint32_t* __restrict__ leaf_begin, const GridDesc* d, uint2* top_cells) {
    if (d->overflow | d->error) return;
    const uint32_t C = d->ncells;
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < C; c += gridDim.x * blockDim.x)
        top_cells[c].x = leaf_begin[c];
}

}  // namespace
}  // namespace hr
