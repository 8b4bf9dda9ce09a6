// build.cu -- per-frame construction of uniform and two-level grids on the device.
//
// Reference path (javorkk/happyray):
//   keyframe lerp + bounds     src/Application/WFObjectUploader.h:82-114 (host loop there;
//                              fused into the first device pass here)
//   resolution                 src/RT/Algorithm/UGridSortBuilder.h:78-92, TLGridSortBuilder.h:80-92
//   pair count                 src/RT/Algorithm/UniformGridBuildKernels.h:40-105
//   pair scatter               UniformGridBuildKernels.h:180-252, exact SAT .cu:224-383
//   radix sort                 src/Utils/Sort.cu:31-53
//   cell ranges                UniformGridBuildKernels.h:384-487
//   leaf cells / leaf pairs    src/RT/Algorithm/TLGridBuildKernels.h:45-147, 304-409, 536-663, 750-834
//
// The reference sorts every (cell, triangle) pair globally by cell key with a radix sort,
// once for the top level and once for the leaves.  Here no global sort is made: cells are
// counted and scanned, each pair takes a slot in its cell's range through an atomic cursor,
// and each cell's short list is ordered afterwards, where it already sits.  Pipeline:
//
//   1 k_frame_bounds    key-frame interpolation + bounds (a1); the last block to finish pads
//                       the bounds and sets the resolution (a2); per-cell counters zeroed
//   2 k_count_cells     per triangle: the per-triangle vertex record and one count per
//                       overlapped cell (a3; with exact insertion only the cells the SAT
//                       test accepts, and one count per rejected pair in an extra bucket)
//   3 k_cell_scan       per cell: (two-level) leaf resolution and flags of the top cell (a8);
//                       tile-local scans of the reference and leaf counts; the last block
//                       scans the tile totals (a4, a9)
//   4 k_place           per (triangle, cell) pair: a slot in the cell's range; two-level: the
//                       pair's leaf sub-range and leaf pair count (a5, a10)
//   two-level:
//   5 k_lp_scan         per top cell: scan of the leaf pair counts (a11 offsets)
//   6 k_leaf_cells      per top cell: its references ordered by triangle, then a stable
//                       counting sort of its leaf pairs into its leaves (a11-a13); cells too
//                       large for one warp are listed for
//   7 k_leaf_cells_big  one CTA per listed cell: CTA-wide radix sorts in global scratch
//   uniform:
//   5 k_ug_cells        per cell: its list sorted by triangle, the cell range written (a6, a7)
//   6 k_ug_cells_big    one CTA per listed cell
//
// Results are identical to the reference's with every cell's list in ascending triangle
// order (the reference's in-cell order comes from atomics and is nondeterministic): a
// leaf's list is its cell's references in ascending triangle order filtered by overlap,
// which is what the reference's stable sort of pairs written in that order gives.  The
// uniform grid with exact insertion keeps the reference's array layout: rejected pairs
// follow all cell lists in the primitive array, in triangle order.
#include "build_dev.cuh"

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>

namespace hr {

namespace {

constexpr int kTileT = 256;                         // threads of the per-cell tile kernels
constexpr int kTileI = 8;                           // cells per thread there
constexpr uint32_t kCellTile = kTileT * kTileI;     // cells per tile
constexpr uint32_t kNone = 0xffffffffu;
constexpr int kWarpRefs = 128;                      // cells a warp orders: references ...
constexpr int kWarpLeaves = 1024;                   // ... and leaves (two-level)
constexpr int kWarpList = 256;                      // uniform cells a warp sorts
constexpr int kBigT = 512;                          // threads of the one-CTA-per-cell kernels
constexpr int kBigW = kBigT / 32;
constexpr int kBigIpt = 8;
constexpr uint32_t kBigChunk = kBigT * kBigIpt;

// control words
enum : int { kTicketBounds = 0, kTicketCells = 1, kTicketLeafPairs = 2, kBigCount = 4, kBigNext = 5, kCtlWords = 16 };

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

// The key-frame pair and weight of the next interpolating build, written in stream order
// ahead of it so that a captured build graph replays for any frame time:
// sel = (frame a, frame b, bits of coeff, 0).
__global__ void k_frame_select(int4* sel, int32_t a, int32_t b, float coeff) {
    *sel = make_int4(a, b, __float_as_int(coeff), 0);
}

// min (k < 3) / max (k >= 3) of six ordered-int encoded bounds over the block; every
// thread gets the result.  Encoded integers order -0 below +0, so the result does not
// depend on the order of the reduction.
__device__ __forceinline__ void block_minmax6(int32_t v[6]) {
    __shared__ int32_t s[6][kBT / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            const int32_t y = __shfl_xor_sync(kFullMask, v[k], o);
            v[k] = k < 3 ? min(v[k], y) : max(v[k], y);
        }
    }
    const int w = threadIdx.x >> 5;
    if (lane_id() == 0)
        for (int k = 0; k < 6; ++k) s[k][w] = v[k];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        int32_t r = s[k][0];
        for (int i = 1; i < kBT / 32; ++i) r = k < 3 ? min(r, s[k][i]) : max(r, s[k][i]);
        v[k] = r;
    }
    __syncthreads();
}

// 1: key-frame interpolation + bounds (WFObjectUploader.h:82-114).  The frames and weight
// come from sel; coeff applies to frame b: v = a * (1 - c) + b * c.  With kf == nullptr
// the vertices are only reduced.  The block that finishes last pads the bounds and sets
// the resolution (UGridSortBuilder.h:78-92), checking the cell count against cap_cells.
// The per-cell counters of the later stages are zeroed here (nzero words each).
__global__ __launch_bounds__(kBT) void k_frame_bounds(const float4* __restrict__ kf, const int4* __restrict__ sel,
                                                      float4* __restrict__ out, uint32_t nv, GridDesc* d,
                                                      int4* part, uint32_t* ctl, uint32_t* z0, uint32_t* z1,
                                                      uint32_t* z2, uint32_t nzero, int32_t kind, uint32_t ntri,
                                                      const uint32_t* bad_index_count, float density,
                                                      uint32_t cap_cells) {
    f3 lo = mk(FLT_MAX, FLT_MAX, FLT_MAX), hi = mk(-FLT_MAX, -FLT_MAX, -FLT_MAX);
    const float4* a = nullptr;
    const float4* b = nullptr;
    float coeff = 0.0f;
    if (kf) {
        const int4 q = *sel;
        a = kf + (size_t)q.x * nv;
        b = kf + (size_t)q.y * nv;
        coeff = __int_as_float(q.z);
    }
    const float w1 = 1.0f - coeff;
    for (uint32_t i = blockIdx.x * kBT + threadIdx.x; i < nv; i += gridDim.x * kBT) {
        f3 p;
        if (a) {
            float4 qa = __ldg(a + i), qb = __ldg(b + i);
            p.x = qa.x * w1 + qb.x * coeff;
            p.y = qa.y * w1 + qb.y * coeff;
            p.z = qa.z * w1 + qb.z * coeff;
            out[i] = make_float4(p.x, p.y, p.z, 0.0f);
        } else {
            float4 q = __ldg(out + i);
            p = mk(q.x, q.y, q.z);
        }
        lo = vmin(p, lo);
        hi = vmax(p, hi);
    }
    for (uint32_t i = blockIdx.x * kBT + threadIdx.x; i < nzero; i += gridDim.x * kBT) {
        z0[i] = 0u;
        z1[i] = 0u;
        if (z2) z2[i] = 0u;
    }
    int32_t e[6] = {fenc(lo.x), fenc(lo.y), fenc(lo.z), fenc(hi.x), fenc(hi.y), fenc(hi.z)};
    block_minmax6(e);
    __shared__ bool s_last;
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = make_int4(e[0], e[1], e[2], 0);
        part[2 * blockIdx.x + 1] = make_int4(e[3], e[4], e[5], 0);
        __threadfence();
        s_last = atomicAdd(ctl + kTicketBounds, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    int32_t m[6] = {INT_MAX, INT_MAX, INT_MAX, INT_MIN, INT_MIN, INT_MIN};
    for (uint32_t i = threadIdx.x; i < gridDim.x; i += kBT) {
        const int4 p = __ldcg(part + 2 * i), q = __ldcg(part + 2 * i + 1);
        m[0] = min(m[0], p.x); m[1] = min(m[1], p.y); m[2] = min(m[2], p.z);
        m[3] = max(m[3], q.x); m[4] = max(m[4], q.y); m[5] = max(m[5], q.z);
    }
    block_minmax6(m);
    if (threadIdx.x == 0) {
        desc_init(d, kind, ntri, *bad_index_count != 0u ? 1u : 0u);
        for (int k = 0; k < 3; ++k) { d->bmin_enc[k] = m[k]; d->bmax_enc[k] = m[3 + k]; }
        const uint64_t nc = grid_setup(d, density);
        if (nc >= (uint64_t)cap_cells) {
            // publish zero cells so later stages do nothing; the host regrows from req_cells
            d->overflow |= kOvfCells;
            d->req_cells = nc > 0xfffffff0ull ? 0xfffffff0u : (uint32_t)nc;
            d->ncells = 0u;
        } else {
            d->ncells = (uint32_t)nc;
        }
        ctl[kTicketBounds] = 0u;
        ctl[kBigCount] = 0u;
        ctl[kBigNext] = 0u;
    }
}

// A block's triangles and their cell boxes, for the block-wide enumeration of pairs: pair
// j of the block belongs to the triangle whose run [off[k], off[k + 1]) holds j, and is the
// (j - off[k])-th cell of its box, x fastest, then y, then z (UniformGridBuildKernels.h:237-249).
struct BlockTris {
    uint32_t off[kBT + 1];
    int32_t lo[kBT][3];
    uint32_t ex[kBT][2];
};

__device__ __forceinline__ void pair_cell(const BlockTris& s, int k, uint32_t l, int32_t* x, int32_t* y, int32_t* z,
                                          uint32_t* dx, uint32_t* dy, uint32_t* dz) {
    const uint32_t ex = s.ex[k][0], ey = s.ex[k][1];
    const uint32_t a = l / ex, c = a / ey;
    *dx = l - a * ex;
    *dy = a - c * ey;
    *dz = c;
    *x = s.lo[k][0] + (int32_t)*dx;
    *y = s.lo[k][1] + (int32_t)*dy;
    *z = s.lo[k][2] + (int32_t)*dz;
}

// centre coordinate of the n-th cell of a run (n = 0, 1, ...) as the reference's loop forms it:
// start - step, then step added n + 1 times (UniformGridBuildKernels.cu:285-300)
__device__ __forceinline__ float run_centre(float start, float step, uint32_t n) {
    float c = start - step;
    for (uint32_t i = 0; i <= n; ++i) c += step;
    return c;
}

// exact triangle/box test of a pair (UniformGridBuildKernels.cu:275-366): the test box has
// its centre at cell min + 0.505 cell and half size 0.505 cell
__device__ __forceinline__ bool pair_sat(const DescRegs& g, const f3* tv, f3 nrm, const int32_t* lo, uint32_t dx,
                                         uint32_t dy, uint32_t dz) {
    const f3 h = mulf(g.cs, 0.505f);
    f3 mc = mk((float)lo[0], (float)lo[1], (float)lo[2]);
    mc = mk(mc.x * g.cs.x, mc.y * g.cs.y, mc.z * g.cs.z);
    mc = add(add(mc, g.bmin), h);
    const f3 c = mk(run_centre(mc.x, g.cs.x, dx), run_centre(mc.y, g.cs.y, dy), run_centre(mc.z, g.cs.z, dz));
    return sat_overlap(nrm, c, tv, h);
}

// 2: per triangle its cell box; one count per overlapped cell (UniformGridBuildKernels.h:40-105),
// aggregated over the lanes of a warp that count the same cell.  With EXACT, cells the SAT
// test rejects are counted in the extra bucket ncells.  The pass also writes the
// per-triangle vertex record (3 float4) that the later passes and the traversal read.
template <bool EXACT>
__global__ __launch_bounds__(kBT) void k_count_cells(const float4* __restrict__ v, const uint32_t* __restrict__ idx,
                                                     uint32_t ntri, const GridDesc* d, float4* __restrict__ tris,
                                                     uint32_t* __restrict__ cell_cnt) {
    if (d->overflow | d->error) return;
    const DescRegs g = load_desc(d);
    __shared__ BlockTris s;
    __shared__ float s_tv[EXACT ? kBT : 1][12];   // vertices and unit normal
    const uint32_t t = blockIdx.x * kBT + threadIdx.x;
    uint32_t n = 0;
    if (t < ntri) {
        f3 p[3], lo, hi;
        CRange r;
        tri_load(v, idx, t, p);
        float4* q = tris + 3 * (size_t)t;
        q[0] = make_float4(p[0].x, p[0].y, p[0].z, 0.0f);
        q[1] = make_float4(p[1].x, p[1].y, p[1].z, 0.0f);
        q[2] = make_float4(p[2].x, p[2].y, p[2].z, 0.0f);
        tri_bbox(p, &lo, &hi);
        n = cell_range(lo, hi, g.bmin, g.rcp, g.res, &r);
        for (int k = 0; k < 3; ++k) s.lo[threadIdx.x][k] = r.lo[k];
        s.ex[threadIdx.x][0] = (uint32_t)max(r.hi[0] - r.lo[0], 1);
        s.ex[threadIdx.x][1] = (uint32_t)max(r.hi[1] - r.lo[1], 1);
        if (EXACT) {
            const f3 nrm = normalize(cross(sub(p[1], p[0]), sub(p[2], p[0])));
            float* w = s_tv[threadIdx.x];
            w[0] = p[0].x; w[1] = p[0].y; w[2] = p[0].z; w[3] = p[1].x; w[4] = p[1].y; w[5] = p[1].z;
            w[6] = p[2].x; w[7] = p[2].y; w[8] = p[2].z; w[9] = nrm.x; w[10] = nrm.y; w[11] = nrm.z;
        }
    }
    uint32_t tot;
    s.off[threadIdx.x] = block_excl_scan<uint32_t, kBT>(n, &tot);
    __syncthreads();
    const uint32_t rx = (uint32_t)g.res[0], rxy = (uint32_t)g.res[0] * (uint32_t)g.res[1];
    const uint32_t lane = lane_id();
    for (uint32_t base = 0; base < tot; base += kBT) {
        const uint32_t j = base + threadIdx.x;
        uint32_t key = kNone;
        if (j < tot) {
            const int k = block_owner<kBT>(s.off, j);
            int32_t x, y, z;
            uint32_t dx, dy, dz;
            pair_cell(s, k, j - s.off[k], &x, &y, &z, &dx, &dy, &dz);
            key = (uint32_t)x + (uint32_t)y * rx + (uint32_t)z * rxy;
            if (EXACT) {
                const float* w = s_tv[k];
                const f3 tv[3] = {mk(w[0], w[1], w[2]), mk(w[3], w[4], w[5]), mk(w[6], w[7], w[8])};
                if (!pair_sat(g, tv, mk(w[9], w[10], w[11]), s.lo[k], dx, dy, dz)) key = g.ncells;
            }
        }
        const uint32_t peers = __match_any_sync(kFullMask, key);
        if (key != kNone && lane == (uint32_t)(__ffs(peers) - 1)) atomicAdd(cell_cnt + key, (uint32_t)__popc(peers));
    }
}

// 3: per cell (and, uniform, the bucket of rejected pairs after the last cell): the
// two-level top cell's leaf resolution and flags (countLeafLevelCells,
// TLGridBuildKernels.h:45-122; packed as TwoLevelGridCell, TwoLevelGrid.h:38-161), then
// the tile-local exclusive scan of (references, leaves).  The block that finishes last
// turns the tile totals into tile offsets and publishes the totals, or an overflow.
template <bool TL>
__global__ __launch_bounds__(kTileT) void k_cell_scan(GridDesc* d, const uint32_t* __restrict__ cell_cnt,
                                                      float leaf_density, uint2* __restrict__ cells,
                                                      uint2* __restrict__ cell_scan, uint2* tile_sums, uint32_t* ctl,
                                                      uint32_t cap_refs, uint32_t cap_leaves) {
    if (d->overflow | d->error) return;
    const DescRegs g = load_desc(d);
    const uint32_t C = TL ? g.ncells : g.ncells + 1u;
    const uint32_t ntiles = (C + kCellTile - 1) / kCellTile;
    if (blockIdx.x >= ntiles) return;
    const uint32_t c0 = blockIdx.x * kCellTile + threadIdx.x * kTileI;
    uint2 val[kTileI];
    uint2 sum = make_uint2(0u, 0u);
#pragma unroll
    for (int k = 0; k < kTileI; ++k) {
        const uint32_t c = c0 + k;
        val[k] = make_uint2(0u, 0u);
        if (c < C) {
            const uint32_t refs = cell_cnt[c];
            uint32_t nl = 0;
            if (TL) {
                const LeafGeom lg = leaf_geom(g, refs, leaf_density);
                uint32_t y = (lg.res[0] & 0xFFu) | ((lg.res[1] & 0xFFu) << 8) | ((lg.res[2] & 0xFFu) << 16);
                if (lg.leaf) y |= kLeafMask;
                if (refs != 0) y |= kNotEmptyMask;
                cells[c].y = y;
                nl = lg.res[0] * lg.res[1] * lg.res[2];
            }
            val[k] = make_uint2(refs, nl);
            sum = sum + val[k];
        }
    }
    uint2 tot;
    uint2 run = block_excl_scan<uint2, kTileT>(sum, &tot);
#pragma unroll
    for (int k = 0; k < kTileI; ++k) {
        if (c0 + k < C) cell_scan[c0 + k] = run;
        run = run + val[k];
    }
    __shared__ bool s_last;
    if (threadIdx.x == 0) {
        tile_sums[blockIdx.x] = tot;
        __threadfence();
        s_last = atomicAdd(ctl + kTicketCells, 1u) == ntiles - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    uint2 carry = make_uint2(0u, 0u);
    for (uint32_t b = 0; b < ntiles; b += kTileT) {
        const uint32_t i = b + threadIdx.x;
        const uint2 x = i < ntiles ? __ldcg(tile_sums + i) : make_uint2(0u, 0u);
        uint2 t;
        const uint2 ex = block_excl_scan<uint2, kTileT>(x, &t);
        if (i < ntiles) tile_sums[i] = carry + ex;
        carry = carry + t;
    }
    if (threadIdx.x == 0) {
        ctl[kTicketCells] = 0u;
        if (TL) {
            if (carry.x > cap_refs) {
                d->overflow |= kOvfTopPairs;
                d->req_pairs = carry.x;
                d->ntop_pairs = 0u;
            } else {
                d->ntop_pairs = carry.x;
            }
            d->nleaves = carry.y;
            if (carry.y > cap_leaves) d->overflow |= kOvfLeaves;
        } else {
            if (carry.x > cap_refs) {
                d->overflow |= kOvfPairs;
                d->req_pairs = carry.x;
                d->npairs = 0u;
            } else {
                d->npairs = carry.x;
            }
        }
    }
}

__device__ __forceinline__ uint32_t cell_first(const uint2* __restrict__ cell_scan, const uint2* __restrict__ tile_sums,
                                               uint32_t c) {
    return __ldg(&cell_scan[c].x) + __ldg(&tile_sums[c / kCellTile].x);
}

// 4: per (triangle, cell) pair a slot in the cell's range [first, first + count), taken by
// the warp's lanes of one cell together from the cell's cursor.  Two-level: the slot gets
// the triangle, its box in the top cell's leaf grid (TLGridBuildKernels.h:338-377) and its
// leaf pair count, which is also summed per top cell (countLeafLevelPairs,
// TLGridBuildKernels.h:304-409).  Uniform: the slot gets the triangle.
template <bool TL, bool EXACT>
__global__ __launch_bounds__(kBT) void k_place(const float4* __restrict__ tris, uint32_t ntri, const GridDesc* d,
                                               uint32_t* __restrict__ cell_cur, const uint2* __restrict__ cell_scan,
                                               const uint2* __restrict__ tile_sums, const uint2* __restrict__ cells,
                                               uint4* __restrict__ refs4, uint32_t* __restrict__ refs1,
                                               uint32_t* __restrict__ cell_lp) {
    if (d->overflow | d->error) return;
    const DescRegs g = load_desc(d);
    __shared__ BlockTris s;
    __shared__ float s_tv[(EXACT || TL) ? kBT : 1][12];   // EXACT: vertices + normal; TL: box lo, hi
    const uint32_t t = blockIdx.x * kBT + threadIdx.x;
    uint32_t n = 0;
    if (t < ntri) {
        f3 p[3], lo, hi;
        CRange r;
        tri_fetch(tris, t, p);
        tri_bbox(p, &lo, &hi);
        n = cell_range(lo, hi, g.bmin, g.rcp, g.res, &r);
        for (int k = 0; k < 3; ++k) s.lo[threadIdx.x][k] = r.lo[k];
        s.ex[threadIdx.x][0] = (uint32_t)max(r.hi[0] - r.lo[0], 1);
        s.ex[threadIdx.x][1] = (uint32_t)max(r.hi[1] - r.lo[1], 1);
        float* w = s_tv[(EXACT || TL) ? threadIdx.x : 0];
        if (EXACT) {
            const f3 nrm = normalize(cross(sub(p[1], p[0]), sub(p[2], p[0])));
            w[0] = p[0].x; w[1] = p[0].y; w[2] = p[0].z; w[3] = p[1].x; w[4] = p[1].y; w[5] = p[1].z;
            w[6] = p[2].x; w[7] = p[2].y; w[8] = p[2].z; w[9] = nrm.x; w[10] = nrm.y; w[11] = nrm.z;
        } else if (TL) {
            w[0] = lo.x; w[1] = lo.y; w[2] = lo.z; w[3] = hi.x; w[4] = hi.y; w[5] = hi.z;
        }
    }
    uint32_t tot;
    s.off[threadIdx.x] = block_excl_scan<uint32_t, kBT>(n, &tot);
    __syncthreads();
    const uint32_t rx = (uint32_t)g.res[0], rxy = (uint32_t)g.res[0] * (uint32_t)g.res[1];
    const uint32_t lane = lane_id();
    for (uint32_t base = 0; base < tot; base += kBT) {
        const uint32_t j = base + threadIdx.x;
        uint32_t key = kNone;
        int k = 0;
        if (j < tot) {
            k = block_owner<kBT>(s.off, j);
            int32_t x, y, z;
            uint32_t dx, dy, dz;
            pair_cell(s, k, j - s.off[k], &x, &y, &z, &dx, &dy, &dz);
            key = (uint32_t)x + (uint32_t)y * rx + (uint32_t)z * rxy;
            if (EXACT) {
                const float* w = s_tv[k];
                const f3 tv[3] = {mk(w[0], w[1], w[2]), mk(w[3], w[4], w[5]), mk(w[6], w[7], w[8])};
                if (!pair_sat(g, tv, mk(w[9], w[10], w[11]), s.lo[k], dx, dy, dz)) key = g.ncells;
            }
        }
        const uint32_t peers = __match_any_sync(kFullMask, key);
        const uint32_t leader = (uint32_t)(__ffs(peers) - 1);
        uint32_t old = 0;
        if (key != kNone && lane == leader) old = atomicAdd(cell_cur + key, (uint32_t)__popc(peers));
        old = __shfl_sync(kFullMask, old, (int)leader);
        uint32_t npl = 0;
        if (key != kNone) {
            const uint32_t slot = cell_first(cell_scan, tile_sums, key) + old + (uint32_t)__popc(peers & ((1u << lane) - 1u));
            const uint32_t tri = blockIdx.x * kBT + (uint32_t)k;
            if (TL) {
                const uint32_t yv = __ldg(&cells[key].y);
                const uint32_t lres[3] = {yv & 0xFFu, (yv >> 8) & 0xFFu, (yv >> 16) & 0xFFu};
                const float* w = s_tv[k];
                CRange r;
                npl = leaf_range(g, lres, key, mk(w[0], w[1], w[2]), mk(w[3], w[4], w[5]), &r);
                uint32_t a = 0, b = 0;
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    a |= (uint32_t)min(max(r.lo[q], 0), 255) << (8 * q);
                    b |= (uint32_t)min(max(r.hi[q], 0), 255) << (8 * q);
                }
                refs4[slot] = make_uint4(a, b, tri, npl);
            } else {
                refs1[slot] = tri;
            }
        }
        if (TL) {
            const uint32_t sum = __reduce_add_sync(peers, npl);
            if (key != kNone && lane == leader && sum) atomicAdd(cell_lp + key, sum);
        }
    }
}

// 5 (two-level): tile-local exclusive scan of the leaf pair counts of the top cells; the
// last block turns the tile totals into offsets and publishes the total or an overflow.
__global__ __launch_bounds__(kTileT) void k_lp_scan(GridDesc* d, const uint32_t* __restrict__ cell_lp,
                                                    uint32_t* __restrict__ lp_scan, uint32_t* lp_tiles, uint32_t* ctl,
                                                    uint32_t cap_leaf_pairs) {
    if (d->overflow | d->error) return;
    const uint32_t C = d->ncells;
    const uint32_t ntiles = (C + kCellTile - 1) / kCellTile;
    if (blockIdx.x >= ntiles) return;
    const uint32_t c0 = blockIdx.x * kCellTile + threadIdx.x * kTileI;
    uint32_t val[kTileI], sum = 0;
#pragma unroll
    for (int k = 0; k < kTileI; ++k) {
        val[k] = c0 + k < C ? cell_lp[c0 + k] : 0u;
        sum += val[k];
    }
    uint32_t tot;
    uint32_t run = block_excl_scan<uint32_t, kTileT>(sum, &tot);
#pragma unroll
    for (int k = 0; k < kTileI; ++k) {
        if (c0 + k < C) lp_scan[c0 + k] = run;
        run += val[k];
    }
    __shared__ bool s_last;
    if (threadIdx.x == 0) {
        lp_tiles[blockIdx.x] = tot;
        __threadfence();
        s_last = atomicAdd(ctl + kTicketLeafPairs, 1u) == ntiles - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    uint64_t carry = 0;
    for (uint32_t b = 0; b < ntiles; b += kTileT) {
        const uint32_t i = b + threadIdx.x;
        const uint32_t x = i < ntiles ? __ldcg(lp_tiles + i) : 0u;
        uint32_t t;
        const uint32_t ex = block_excl_scan<uint32_t, kTileT>(x, &t);
        if (i < ntiles) lp_tiles[i] = (uint32_t)carry + ex;
        carry += t;
    }
    if (threadIdx.x == 0) {
        ctl[kTicketLeafPairs] = 0u;
        if (carry > cap_leaf_pairs) {
            d->overflow |= kOvfLeafPairs;
            d->req_leaf_pairs = carry > 0xffffffffull ? 0xffffffffu : (uint32_t)carry;
            d->npairs = 0u;
        } else {
            d->npairs = (uint32_t)carry;
        }
    }
}

// Where a top cell's data lives: its references [rb, rb + R) in refs4, its leaves
// [lb, lb + nl), its leaf pairs [pb, pb + P) in prims, its packed cell word y.
struct TopCell {
    uint32_t rb, R, lb, nl, pb, P, y;
    uint32_t lres[3];
};
__device__ __forceinline__ TopCell top_cell(uint32_t c, const uint32_t* __restrict__ cell_cnt,
                                            const uint2* __restrict__ cell_scan, const uint2* __restrict__ tile_sums,
                                            const uint2* __restrict__ cells, const uint32_t* __restrict__ cell_lp,
                                            const uint32_t* __restrict__ lp_scan, const uint32_t* __restrict__ lp_tiles) {
    TopCell tc;
    const uint2 sc = __ldg(cell_scan + c), ts = __ldg(tile_sums + c / kCellTile);
    tc.rb = sc.x + ts.x;
    tc.lb = sc.y + ts.y;
    tc.R = __ldg(cell_cnt + c);
    tc.y = __ldg(&cells[c].y);
    tc.lres[0] = tc.y & 0xFFu; tc.lres[1] = (tc.y >> 8) & 0xFFu; tc.lres[2] = (tc.y >> 16) & 0xFFu;
    tc.nl = tc.lres[0] * tc.lres[1] * tc.lres[2];
    tc.pb = __ldg(lp_scan + c) + __ldg(lp_tiles + c / kCellTile);
    tc.P = __ldg(cell_lp + c);
    return tc;
}

// leaf index of the j-th leaf of a reference's box (x fastest, then y, then z)
__device__ __forceinline__ uint32_t ref_leaf(uint4 q, uint32_t j, const uint32_t* lres) {
    const uint32_t lx = q.x & 0xFFu, ly = (q.x >> 8) & 0xFFu, lz = (q.x >> 16) & 0xFFu;
    const uint32_t ex = (q.y & 0xFFu) - lx, ey = ((q.y >> 8) & 0xFFu) - ly;
    const uint32_t a = j / ex, dz = a / ey;
    const uint32_t dx = j - a * ex, dy = a - dz * ey;
    return (lx + dx) + (ly + dy) * lres[0] + (lz + dz) * lres[0] * lres[1];
}

// bitonic sort of n (a power of two, >= 32) keys in shared memory by one warp
template <class K>
__device__ __forceinline__ void warp_bitonic(K* s, uint32_t n) {
    const uint32_t lane = lane_id();
    for (uint32_t k = 2; k <= n; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t i = lane; i < n; i += 32) {
                const uint32_t ixj = i ^ j;
                if (ixj > i) {
                    const K a = s[i], b = s[ixj];
                    if ((a > b) == ((i & k) == 0)) { s[i] = b; s[ixj] = a; }
                }
            }
            __syncwarp();
        }
    }
}

__device__ __forceinline__ uint32_t pow2_at_least(uint32_t n) {
    uint32_t p = 32;
    while (p < n) p <<= 1;
    return p;
}

// One warp orders a top cell with at most kWarpRefs references and kWarpLeaves leaves:
// references sorted by triangle (bitonic, 64-bit keys triangle << 32 | index); leaf pair
// counts in shared memory, their scan gives the leaf ranges; then the references are
// placed one at a time in ascending triangle order, the leaves of each spread over the lanes.
__device__ void warp_leaf_cell(const TopCell& tc, const uint4* __restrict__ refs4, uint2* __restrict__ leaves,
                               uint32_t* __restrict__ prims, unsigned long long* s_key, uint32_t* s_cur) {
    const uint32_t lane = lane_id();
    const uint32_t n2 = pow2_at_least(tc.R);
    for (uint32_t i = lane; i < n2; i += 32)
        s_key[i] = i < tc.R ? ((unsigned long long)__ldg(&refs4[tc.rb + i].z) << 32) | i : ~0ull;
    for (uint32_t l = lane; l < tc.nl; l += 32) s_cur[l] = 0u;
    __syncwarp();
    warp_bitonic(s_key, n2);
    for (uint32_t i = lane; i < tc.R; i += 32) {
        const uint4 q = __ldg(refs4 + tc.rb + i);
        for (uint32_t j = 0; j < q.w; ++j) atomicAdd(s_cur + ref_leaf(q, j, tc.lres), 1u);
    }
    __syncwarp();
    // exclusive scan over the leaves, one contiguous run per lane; leaf ranges written
    const uint32_t per = (tc.nl + 31) / 32;
    const uint32_t l0 = min(tc.nl, lane * per), l1 = min(tc.nl, l0 + per);
    uint32_t sum = 0;
    for (uint32_t l = l0; l < l1; ++l) sum += s_cur[l];
    uint32_t inc = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(kFullMask, inc, o);
        if ((int)lane >= o) inc += y;
    }
    uint32_t run = inc - sum;
    for (uint32_t l = l0; l < l1; ++l) {
        const uint32_t cnt = s_cur[l];
        leaves[tc.lb + l] = cnt ? make_uint2(tc.pb + run, tc.pb + run + cnt) : make_uint2(0u, 0u);
        s_cur[l] = run;
        run += cnt;
    }
    __syncwarp();
    for (uint32_t k = 0; k < tc.R; ++k) {
        const uint32_t i = (uint32_t)s_key[k];
        const uint4 q = __ldg(refs4 + tc.rb + i);
        for (uint32_t j = lane; j < q.w; j += 32) {
            const uint32_t l = ref_leaf(q, j, tc.lres);
            const uint32_t slot = s_cur[l];
            s_cur[l] = slot + 1u;
            prims[tc.pb + slot] = q.z;
        }
        __syncwarp();
    }
}

// 6 (two-level): per top cell, one thread each: the first leaf goes to the cell word; an
// empty cell gets its one empty leaf; a cell of at most kLeafRefsMax references has one
// leaf (TLGridBuildKernels.h:77) holding the references that overlap it, in ascending
// triangle order.  Larger cells are ordered by a warp of the block, or listed for
// k_leaf_cells_big.
__global__ __launch_bounds__(256) void k_leaf_cells(const GridDesc* d, const uint32_t* __restrict__ cell_cnt,
                                                    const uint2* __restrict__ cell_scan,
                                                    const uint2* __restrict__ tile_sums, uint2* __restrict__ cells,
                                                    const uint32_t* __restrict__ cell_lp,
                                                    const uint32_t* __restrict__ lp_scan,
                                                    const uint32_t* __restrict__ lp_tiles,
                                                    const uint4* __restrict__ refs4, uint2* __restrict__ leaves,
                                                    uint32_t* __restrict__ prims, uint32_t* ctl,
                                                    uint32_t* __restrict__ big_list) {
    if (d->overflow | d->error) return;
    const uint32_t C = d->ncells;
    __shared__ uint32_t s_q[256];
    __shared__ uint32_t s_nq;
    __shared__ unsigned long long s_key[8][kWarpRefs];
    __shared__ uint32_t s_cur[8][kWarpLeaves];
    if (threadIdx.x == 0) s_nq = 0;
    __syncthreads();
    const uint32_t c = blockIdx.x * 256 + threadIdx.x;
    if (c < C) {
        const TopCell tc = top_cell(c, cell_cnt, cell_scan, tile_sums, cells, cell_lp, lp_scan, lp_tiles);
        cells[c].x = tc.lb;
        if (tc.R <= kLeafRefsMax) {
            uint32_t tl[kLeafRefsMax];
            uint32_t m = 0;
            for (uint32_t i = 0; i < tc.R; ++i) {
                const uint4 q = __ldg(refs4 + tc.rb + i);
                if (q.w == 0) continue;
                uint32_t p = m++;
                while (p > 0 && tl[p - 1] > q.z) { tl[p] = tl[p - 1]; --p; }
                tl[p] = q.z;
            }
            for (uint32_t i = 0; i < m; ++i) prims[tc.pb + i] = tl[i];
            leaves[tc.lb] = m ? make_uint2(tc.pb, tc.pb + m) : make_uint2(0u, 0u);
        } else if (tc.R <= kWarpRefs && tc.nl <= kWarpLeaves) {
            s_q[atomicAdd(&s_nq, 1u)] = c;
        } else {
            big_list[atomicAdd(ctl + kBigCount, 1u)] = c;
        }
    }
    __syncthreads();
    const uint32_t w = threadIdx.x >> 5;
    for (uint32_t i = w; i < s_nq; i += 8) {
        const TopCell tc = top_cell(s_q[i], cell_cnt, cell_scan, tile_sums, cells, cell_lp, lp_scan, lp_tiles);
        warp_leaf_cell(tc, refs4, leaves, prims, s_key[w], s_cur[w]);
    }
}

struct BigSmem {
    uint32_t cur[256];                 // digit counts, then running digit cursors
    uint32_t whist[kBigW][256];        // per warp and digit: count, then output base
    uint32_t red[kBigW];
    uint32_t item;
};

// Stable LSD radix sort of n (key, value) pairs in global memory by one CTA, over the low
// `bits` bits of the keys in 8-bit digits.  Each pass: digit histogram, then chunks of
// kBigChunk pairs in order, ranked within a warp by match_any and across warps by per-warp
// digit counts.  vals may be null.  Returns 0 when the result is in (ka, va), 1 in (kb, vb).
__device__ int cta_radix_sort(uint32_t* ka, uint32_t* va, uint32_t* kb, uint32_t* vb, uint32_t n, int bits,
                              BigSmem& sm) {
    const int passes = (bits + 7) / 8;
    const uint32_t lane = lane_id(), w = threadIdx.x >> 5;
    const uint32_t lt = (1u << lane) - 1u;
    for (int p = 0; p < passes; ++p) {
        const uint32_t* sk = (p & 1) ? kb : ka;
        const uint32_t* sv = (p & 1) ? vb : va;
        uint32_t* dk = (p & 1) ? ka : kb;
        uint32_t* dv = (p & 1) ? va : vb;
        const int shift = 8 * p;
        for (uint32_t i = threadIdx.x; i < 256; i += kBigT) sm.cur[i] = 0u;
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < n; i += kBigT) atomicAdd(&sm.cur[(sk[i] >> shift) & 255u], 1u);
        __syncthreads();
        if (w == 0) {   // exclusive scan of the 256 digit counts, 8 per lane
            uint32_t x[8], s = 0;
#pragma unroll
            for (int k = 0; k < 8; ++k) { x[k] = sm.cur[lane * 8 + k]; s += x[k]; }
            uint32_t inc = s;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(kFullMask, inc, o);
                if ((int)lane >= o) inc += y;
            }
            uint32_t run = inc - s;
#pragma unroll
            for (int k = 0; k < 8; ++k) { sm.cur[lane * 8 + k] = run; run += x[k]; }
        }
        __syncthreads();
        for (uint32_t base = 0; base < n; base += kBigChunk) {
            for (uint32_t i = threadIdx.x; i < kBigW * 256; i += kBigT) (&sm.whist[0][0])[i] = 0u;
            __syncthreads();
            uint32_t key[kBigIpt], val[kBigIpt], dig[kBigIpt], rank[kBigIpt];
#pragma unroll
            for (int r = 0; r < kBigIpt; ++r) {
                const uint32_t i = base + (w * kBigIpt + r) * 32 + lane;
                const bool valid = i < n;
                key[r] = valid ? sk[i] : 0u;
                val[r] = valid && sv ? sv[i] : 0u;
                dig[r] = valid ? (key[r] >> shift) & 255u : 256u;
                const uint32_t peers = __match_any_sync(kFullMask, dig[r]);
                const uint32_t leader = (uint32_t)(__ffs(peers) - 1);
                uint32_t b = 0;
                if (valid && lane == leader) {
                    b = sm.whist[w][dig[r]];
                    sm.whist[w][dig[r]] = b + (uint32_t)__popc(peers);
                }
                b = __shfl_sync(kFullMask, b, (int)leader);
                rank[r] = b + (uint32_t)__popc(peers & lt);
                __syncwarp();
            }
            __syncthreads();
            for (uint32_t dd = threadIdx.x; dd < 256; dd += kBigT) {
                uint32_t run = sm.cur[dd];
                for (uint32_t ww = 0; ww < kBigW; ++ww) {
                    const uint32_t t = sm.whist[ww][dd];
                    sm.whist[ww][dd] = run;
                    run += t;
                }
                sm.cur[dd] = run;
            }
            __syncthreads();
#pragma unroll
            for (int r = 0; r < kBigIpt; ++r) {
                if (dig[r] < 256u) {
                    const uint32_t pos = sm.whist[w][dig[r]] + rank[r];
                    dk[pos] = key[r];
                    if (dv) dv[pos] = val[r];
                }
            }
            __syncthreads();
        }
    }
    return passes & 1;
}

__device__ __forceinline__ int bit_width(uint32_t x) { return x ? 32 - __clz(x) : 0; }

// min (first) and max (second) of x over the CTA; every thread gets the result
__device__ __forceinline__ uint2 cta_minmax(uint32_t lo, uint32_t hi, BigSmem& sm) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lo = min(lo, __shfl_xor_sync(kFullMask, lo, o));
        hi = max(hi, __shfl_xor_sync(kFullMask, hi, o));
    }
    const uint32_t w = threadIdx.x >> 5;
    if (lane_id() == 0) sm.red[w] = lo;
    __syncthreads();
    uint32_t a = sm.red[0];
    for (uint32_t i = 1; i < kBigW; ++i) a = min(a, sm.red[i]);
    __syncthreads();
    if (lane_id() == 0) sm.red[w] = hi;
    __syncthreads();
    uint32_t b = sm.red[0];
    for (uint32_t i = 1; i < kBigW; ++i) b = max(b, sm.red[i]);
    __syncthreads();
    return make_uint2(a, b);
}

// exclusive scan of one value per thread over the CTA (kBigT threads); total to *tot
__device__ __forceinline__ uint32_t cta_excl_scan(uint32_t x, uint32_t* tot, BigSmem& sm) {
    const uint32_t lane = lane_id(), w = threadIdx.x >> 5;
    uint32_t inc = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(kFullMask, inc, o);
        if ((int)lane >= o) inc += y;
    }
    if (lane == 31) sm.red[w] = inc;
    __syncthreads();
    uint32_t before = 0, all = 0;
    for (uint32_t i = 0; i < kBigW; ++i) {
        const uint32_t v = sm.red[i];
        if (i < w) before += v;
        all += v;
    }
    __syncthreads();
    *tot = all;
    return before + inc - x;
}

// 7 (two-level): one CTA per listed top cell, taken from a work counter.  The cell's
// references are sorted by triangle (keys triangle - smallest triangle, values reference
// index), its leaf pairs are written in that order (keys leaf, values triangle) and sorted
// stably by leaf; leaf ranges and the primitive list follow from the sorted keys.
// Scratch: rk/rv pairs per top-level reference, lk/lv pairs per leaf pair.
__global__ __launch_bounds__(kBigT) void k_leaf_cells_big(const GridDesc* d, const uint32_t* __restrict__ cell_cnt,
                                                          const uint2* __restrict__ cell_scan,
                                                          const uint2* __restrict__ tile_sums,
                                                          const uint2* __restrict__ cells,
                                                          const uint32_t* __restrict__ cell_lp,
                                                          const uint32_t* __restrict__ lp_scan,
                                                          const uint32_t* __restrict__ lp_tiles,
                                                          const uint4* __restrict__ refs4, uint2* __restrict__ leaves,
                                                          uint32_t* __restrict__ prims, uint32_t* ctl,
                                                          const uint32_t* __restrict__ big_list, uint32_t* rka,
                                                          uint32_t* rva, uint32_t* rkb, uint32_t* rvb, uint32_t* lka,
                                                          uint32_t* lva, uint32_t* lkb, uint32_t* lvb) {
    if (d->overflow | d->error) return;
    __shared__ BigSmem sm;
    const uint32_t nbig = ctl[kBigCount];
    for (;;) {
        if (threadIdx.x == 0) sm.item = atomicAdd(ctl + kBigNext, 1u);
        __syncthreads();
        const uint32_t item = sm.item;
        __syncthreads();
        if (item >= nbig) return;
        const TopCell tc = top_cell(big_list[item], cell_cnt, cell_scan, tile_sums, cells, cell_lp, lp_scan, lp_tiles);
        // references sorted by triangle
        uint32_t lo = kNone, hi = 0;
        for (uint32_t i = threadIdx.x; i < tc.R; i += kBigT) {
            const uint32_t tri = __ldg(&refs4[tc.rb + i].z);
            lo = min(lo, tri);
            hi = max(hi, tri);
        }
        const uint2 mm = cta_minmax(lo, hi, sm);
        for (uint32_t i = threadIdx.x; i < tc.R; i += kBigT) {
            rka[tc.rb + i] = __ldg(&refs4[tc.rb + i].z) - mm.x;
            rva[tc.rb + i] = i;
        }
        __syncthreads();
        const int rs = cta_radix_sort(rka + tc.rb, rva + tc.rb, rkb + tc.rb, rvb + tc.rb, tc.R, bit_width(mm.y - mm.x), sm);
        const uint32_t* sidx = (rs ? rvb : rva) + tc.rb;   // reference index by rank
        uint32_t* off = (rs ? rka : rkb) + tc.rb;           // free half: leaf pair offset by rank
        // leaf pairs in ascending triangle order
        uint32_t carry = 0;
        for (uint32_t b = 0; b < tc.R; b += kBigT) {
            const uint32_t k = b + threadIdx.x;
            const uint32_t np = k < tc.R ? __ldg(&refs4[tc.rb + sidx[k]].w) : 0u;
            uint32_t t;
            const uint32_t ex = cta_excl_scan(np, &t, sm);
            if (k < tc.R) off[k] = carry + ex;
            carry += t;
        }
        __syncthreads();
        for (uint32_t k = threadIdx.x; k < tc.R; k += kBigT) {
            const uint4 q = __ldg(refs4 + tc.rb + sidx[k]);
            const uint32_t o = tc.pb + off[k];
            for (uint32_t j = 0; j < q.w; ++j) {
                lka[o + j] = ref_leaf(q, j, tc.lres);
                lva[o + j] = q.z;
            }
        }
        for (uint32_t l = threadIdx.x; l < tc.nl; l += kBigT) leaves[tc.lb + l] = make_uint2(0u, 0u);
        __syncthreads();
        const int ls = cta_radix_sort(lka + tc.pb, lva + tc.pb, lkb + tc.pb, lvb + tc.pb, tc.P, bit_width(tc.nl - 1u), sm);
        const uint32_t* sk = (ls ? lkb : lka) + tc.pb;
        const uint32_t* sv = (ls ? lvb : lva) + tc.pb;
        for (uint32_t i = threadIdx.x; i < tc.P; i += kBigT) {
            const uint32_t key = sk[i];
            if (i == 0 || sk[i - 1] != key) leaves[tc.lb + key].x = tc.pb + i;
            if (i + 1 == tc.P || sk[i + 1] != key) leaves[tc.lb + key].y = tc.pb + i + 1;
            prims[tc.pb + i] = sv[i];
        }
        __syncthreads();
    }
}

// 5 (uniform): per cell its range, and its list -- placed in any order -- sorted by
// triangle into prims (a6, a7); the bucket after the last cell holds the pairs exact
// insertion rejected (their triangles, in order).  Short lists by one thread, longer by a
// warp of the block, the longest listed for k_ug_cells_big.
__global__ __launch_bounds__(256) void k_ug_cells(const GridDesc* d, const uint32_t* __restrict__ cell_cnt,
                                                  const uint2* __restrict__ cell_scan,
                                                  const uint2* __restrict__ tile_sums, uint2* __restrict__ cells,
                                                  const uint32_t* __restrict__ refs1, uint32_t* __restrict__ prims,
                                                  uint32_t* ctl, uint32_t* __restrict__ big_list) {
    if (d->overflow | d->error) return;
    const uint32_t C = d->ncells;
    __shared__ uint32_t s_q[256];
    __shared__ uint32_t s_nq;
    __shared__ uint32_t s_key[8][kWarpList];
    if (threadIdx.x == 0) s_nq = 0;
    __syncthreads();
    const uint32_t c = blockIdx.x * 256 + threadIdx.x;
    if (c <= C) {
        const uint32_t b = cell_first(cell_scan, tile_sums, c), R = __ldg(cell_cnt + c);
        if (c < C) cells[c] = R ? make_uint2(b, b + R) : make_uint2(0u, 0u);
        if (R <= 16) {
            uint32_t tl[16];
            for (uint32_t i = 0; i < R; ++i) {
                const uint32_t x = __ldg(refs1 + b + i);
                uint32_t p = i;
                while (p > 0 && tl[p - 1] > x) { tl[p] = tl[p - 1]; --p; }
                tl[p] = x;
            }
            for (uint32_t i = 0; i < R; ++i) prims[b + i] = tl[i];
        } else if (R <= kWarpList) {
            s_q[atomicAdd(&s_nq, 1u)] = c;
        } else {
            big_list[atomicAdd(ctl + kBigCount, 1u)] = c;
        }
    }
    __syncthreads();
    const uint32_t w = threadIdx.x >> 5, lane = lane_id();
    for (uint32_t i = w; i < s_nq; i += 8) {
        const uint32_t cc = s_q[i];
        const uint32_t b = cell_first(cell_scan, tile_sums, cc), R = __ldg(cell_cnt + cc);
        const uint32_t n2 = pow2_at_least(R);
        for (uint32_t k = lane; k < n2; k += 32) s_key[w][k] = k < R ? __ldg(refs1 + b + k) : kNone;
        __syncwarp();
        warp_bitonic(s_key[w], n2);
        for (uint32_t k = lane; k < R; k += 32) prims[b + k] = s_key[w][k];
        __syncwarp();
    }
}

// 6 (uniform): one CTA per listed cell: its list sorted by triangle with a CTA-wide radix
// sort in global scratch (keys triangle - smallest triangle).
__global__ __launch_bounds__(kBigT) void k_ug_cells_big(const GridDesc* d, const uint32_t* __restrict__ cell_cnt,
                                                        const uint2* __restrict__ cell_scan,
                                                        const uint2* __restrict__ tile_sums,
                                                        const uint32_t* __restrict__ refs1, uint32_t* __restrict__ prims,
                                                        uint32_t* ctl, const uint32_t* __restrict__ big_list,
                                                        uint32_t* ka, uint32_t* kb) {
    if (d->overflow | d->error) return;
    __shared__ BigSmem sm;
    const uint32_t nbig = ctl[kBigCount];
    for (;;) {
        if (threadIdx.x == 0) sm.item = atomicAdd(ctl + kBigNext, 1u);
        __syncthreads();
        const uint32_t item = sm.item;
        __syncthreads();
        if (item >= nbig) return;
        const uint32_t c = big_list[item];
        const uint32_t b = cell_first(cell_scan, tile_sums, c), R = __ldg(cell_cnt + c);
        uint32_t lo = kNone, hi = 0;
        for (uint32_t i = threadIdx.x; i < R; i += kBigT) {
            const uint32_t x = __ldg(refs1 + b + i);
            lo = min(lo, x);
            hi = max(hi, x);
        }
        const uint2 mm = cta_minmax(lo, hi, sm);
        for (uint32_t i = threadIdx.x; i < R; i += kBigT) ka[b + i] = __ldg(refs1 + b + i) - mm.x;
        __syncthreads();
        const int rs = cta_radix_sort(ka + b, nullptr, kb + b, nullptr, R, bit_width(mm.y - mm.x), sm);
        const uint32_t* sk = (rs ? kb : ka) + b;
        for (uint32_t i = threadIdx.x; i < R; i += kBigT) prims[b + i] = sk[i] + mm.x;
        __syncthreads();
    }
}

}  // namespace

// Everything a captured build depends on: grid kind and settings, sizes and capacities,
// and the addresses of every buffer the build reads or writes.
static std::vector<uint8_t> build_graph_key(const hr_ctx* c, int32_t kind, int32_t exact, float dens) {
    const GridBuffers& B = c->g;
    const DevBuf* bufs[] = {&B.desc, &c->tris, &B.cells, &B.leaves, &B.prims, &B.keys_a, &B.vals_a, &B.keys_b,
                            &B.vals_b, &B.lkeys_a, &B.lvals_a, &B.lkeys_b, &B.lvals_b, &B.cell_cnt, &B.cell_cur,
                            &B.cell_lp, &B.cell_scan, &B.lp_scan, &B.tile_sums, &B.lp_tiles, &B.refs, &B.ctl,
                            &B.bounds_part, &B.big_list, &c->verts, &c->idx, &c->counters, &c->keyframes,
                            &c->frame_sel};
    std::vector<uint8_t> k;
    auto put = [&](const void* p, size_t n) {
        const uint8_t* b = static_cast<const uint8_t*>(p);
        k.insert(k.end(), b, b + n);
    };
    // the frame pair and weight are not part of it: the graph reads them from frame_sel
    const int32_t ints[5] = {kind, exact, c->timing ? 1 : 0, c->num_sms, c->lerp_pending ? 1 : 0};
    const uint32_t sizes[3] = {c->ntri, c->nverts, c->nkeyframes};
    const float dens_all[3] = {dens, c->leaf_density, c->ug_density};
    const size_t caps[4] = {B.cap_cells, B.cap_pairs, B.cap_leaf_pairs, B.cap_leaves};
    put(ints, sizeof(ints));
    put(sizes, sizeof(sizes));
    put(dens_all, sizeof(dens_all));
    put(caps, sizeof(caps));
    for (const DevBuf* b : bufs) {
        put(&b->p, sizeof(b->p));
        put(&b->bytes, sizeof(b->bytes));
    }
    return k;
}

void drop_build_graph(hr_ctx* c) {
    if (c->build_exec) cudaGraphExecDestroy(c->build_exec);
    c->build_exec = nullptr;
    c->build_key.clear();
}

// Host orchestration of one build.  With wait, syncs and reports the overflow bits in
// *ovf_out; without, only enqueues (the descriptor lands in c->desc_pinned when the stream
// has passed the build).  Returns HR status code (0 = ok).
static int build_once_impl(hr_ctx* c, int32_t kind, int32_t exact, uint32_t* ovf_out, bool wait) {
    cudaStream_t s = c->stream;
    GridBuffers& B = c->g;
    const uint32_t ntri = c->ntri;
    const bool tl = kind == kTwoLevel;
    const bool ex = !tl && exact;
    const float dens = tl ? c->top_density : c->ug_density;
    // capacity of the cell array is a bound (prod res <= density * N), not a guess
    const size_t cells_bound = (size_t)(std::floor((double)dens * (double)ntri * 1.01)) + 32768u + 64u;
    if (B.cap_cells < cells_bound) B.cap_cells = cells_bound;
    if (B.cap_pairs == 0) B.cap_pairs = (size_t)ntri * (tl ? 3u : 6u) + 4096u;
    if (tl) {
        if (B.cap_leaf_pairs == 0) B.cap_leaf_pairs = (size_t)ntri * 4u + 4096u;
        if (B.cap_leaves == 0) B.cap_leaves = (size_t)(c->leaf_density * 2.0f * (float)B.cap_pairs) + B.cap_cells;
    }
    const size_t cap_pairs = B.cap_pairs;   // uniform pairs, or top-level references
    const size_t ncell_words = B.cap_cells + 1;   // + the bucket of rejected pairs
    const size_t ntiles = (ncell_words + kCellTile - 1) / kCellTile;
    const uint32_t nblocks = (ntri + kBT - 1) / kBT;
    const int gridv = std::max(1, std::min((int)((c->nverts + kBT - 1) / kBT), c->num_sms * 8));
    int rc;
    if ((rc = ensure(c, B.desc, sizeof(GridDesc)))) return rc;
    if ((rc = ensure(c, c->frame_sel, sizeof(int4)))) return rc;
    if ((rc = ensure(c, c->tris, sizeof(float4) * 3 * (size_t)ntri))) return rc;
    if ((rc = ensure(c, B.cells, sizeof(uint2) * B.cap_cells))) return rc;
    if ((rc = ensure(c, B.cell_cnt, sizeof(uint32_t) * ncell_words))) return rc;
    if ((rc = ensure(c, B.cell_cur, sizeof(uint32_t) * ncell_words))) return rc;
    if ((rc = ensure(c, B.cell_scan, sizeof(uint2) * ncell_words))) return rc;
    if ((rc = ensure(c, B.tile_sums, sizeof(uint2) * (ntiles + 1)))) return rc;
    if ((rc = ensure(c, B.big_list, sizeof(uint32_t) * ncell_words))) return rc;
    if ((rc = ensure(c, B.bounds_part, sizeof(int4) * 2 * (size_t)gridv))) return rc;
    if ((rc = ensure(c, B.keys_a, sizeof(uint32_t) * cap_pairs))) return rc;
    if ((rc = ensure(c, B.keys_b, sizeof(uint32_t) * cap_pairs))) return rc;
    if (!B.ctl.p) {
        if ((rc = ensure(c, B.ctl, sizeof(uint32_t) * kCtlWords))) return rc;
        if ((rc = cuda_check(c, cudaMemsetAsync(B.ctl.p, 0, sizeof(uint32_t) * kCtlWords, s), "build control"))) return rc;
    }
    if (tl) {
        if ((rc = ensure(c, B.cell_lp, sizeof(uint32_t) * ncell_words))) return rc;
        if ((rc = ensure(c, B.lp_scan, sizeof(uint32_t) * ncell_words))) return rc;
        if ((rc = ensure(c, B.lp_tiles, sizeof(uint32_t) * (ntiles + 1)))) return rc;
        if ((rc = ensure(c, B.refs, sizeof(uint4) * cap_pairs))) return rc;
        if ((rc = ensure(c, B.vals_a, sizeof(uint32_t) * cap_pairs))) return rc;
        if ((rc = ensure(c, B.vals_b, sizeof(uint32_t) * cap_pairs))) return rc;
        if ((rc = ensure(c, B.leaves, sizeof(uint2) * B.cap_leaves))) return rc;
        if ((rc = ensure(c, B.prims, sizeof(uint32_t) * B.cap_leaf_pairs))) return rc;
        if ((rc = ensure(c, B.lkeys_a, sizeof(uint32_t) * B.cap_leaf_pairs))) return rc;
        if ((rc = ensure(c, B.lvals_a, sizeof(uint32_t) * B.cap_leaf_pairs))) return rc;
        if ((rc = ensure(c, B.lkeys_b, sizeof(uint32_t) * B.cap_leaf_pairs))) return rc;
        if ((rc = ensure(c, B.lvals_b, sizeof(uint32_t) * B.cap_leaf_pairs))) return rc;
    } else {
        if ((rc = ensure(c, B.refs, sizeof(uint32_t) * cap_pairs))) return rc;
        if ((rc = ensure(c, B.prims, sizeof(uint32_t) * cap_pairs))) return rc;
    }
    GridDesc* d = B.desc.as<GridDesc>();
    uint32_t* ctl = B.ctl.as<uint32_t>();
    const uint32_t cap32 = (uint32_t)std::min(cap_pairs, (size_t)0xffffffffu);
    const uint32_t ncb = (uint32_t)((ncell_words + 255) / 256);   // blocks of one cell per thread
    const uint32_t ntb = (uint32_t)ntiles;                         // blocks of one cell tile each
    const int nbig = c->num_sms * 2;
    // the whole build as one enqueue (returns an HR status)
    auto enqueue = [&]() -> int {
        int ev = 0;
        auto mark = [&]() {
            if (c->timing && ev < 16) {
                if (c->build_capturing) cudaEventRecordWithFlags(c->ev[ev++], s, cudaEventRecordExternal);
                else cudaEventRecord(c->ev[ev++], s);
            }
        };
        mark();
        c->launches += 1 + (nblocks > 0 ? 2 : 0) + 1 + 2 + (tl ? 1 : 0);
        k_frame_bounds<<<gridv, kBT, 0, s>>>(c->lerp_pending ? c->keyframes.as<float4>() : nullptr,
                                             c->frame_sel.as<int4>(), c->verts.as<float4>(), c->nverts, d,
                                             B.bounds_part.as<int4>(), ctl, B.cell_cnt.as<uint32_t>(),
                                             B.cell_cur.as<uint32_t>(), tl ? B.cell_lp.as<uint32_t>() : nullptr,
                                             (uint32_t)ncell_words, kind, ntri, c->counters.as<uint32_t>() + 2, dens,
                                             (uint32_t)std::min(B.cap_cells, (size_t)0xffffffffu));
        mark();
        if (nblocks > 0) {
            if (ex)
                k_count_cells<true><<<nblocks, kBT, 0, s>>>(c->verts.as<float4>(), c->idx.as<uint32_t>(), ntri, d,
                                                            c->tris.as<float4>(), B.cell_cnt.as<uint32_t>());
            else
                k_count_cells<false><<<nblocks, kBT, 0, s>>>(c->verts.as<float4>(), c->idx.as<uint32_t>(), ntri, d,
                                                             c->tris.as<float4>(), B.cell_cnt.as<uint32_t>());
        }
        mark();
        if (tl)
            k_cell_scan<true><<<ntb, kTileT, 0, s>>>(d, B.cell_cnt.as<uint32_t>(), c->leaf_density, B.cells.as<uint2>(),
                                                     B.cell_scan.as<uint2>(), B.tile_sums.as<uint2>(), ctl, cap32,
                                                     (uint32_t)std::min(B.cap_leaves, (size_t)0xffffffffu));
        else
            k_cell_scan<false><<<ntb, kTileT, 0, s>>>(d, B.cell_cnt.as<uint32_t>(), 0.0f, B.cells.as<uint2>(),
                                                      B.cell_scan.as<uint2>(), B.tile_sums.as<uint2>(), ctl, cap32, 0u);
        mark();
        if (nblocks > 0) {
            const float4* tr = c->tris.as<float4>();
            uint32_t* cur = B.cell_cur.as<uint32_t>();
            const uint2* cs = B.cell_scan.as<uint2>();
            const uint2* ts = B.tile_sums.as<uint2>();
            if (tl)
                k_place<true, false><<<nblocks, kBT, 0, s>>>(tr, ntri, d, cur, cs, ts, B.cells.as<uint2>(),
                                                             B.refs.as<uint4>(), nullptr, B.cell_lp.as<uint32_t>());
            else if (ex)
                k_place<false, true><<<nblocks, kBT, 0, s>>>(tr, ntri, d, cur, cs, ts, nullptr, nullptr,
                                                             B.refs.as<uint32_t>(), nullptr);
            else
                k_place<false, false><<<nblocks, kBT, 0, s>>>(tr, ntri, d, cur, cs, ts, nullptr, nullptr,
                                                              B.refs.as<uint32_t>(), nullptr);
        }
        mark();
        if (tl) {
            k_lp_scan<<<ntb, kTileT, 0, s>>>(d, B.cell_lp.as<uint32_t>(), B.lp_scan.as<uint32_t>(),
                                             B.lp_tiles.as<uint32_t>(), ctl,
                                             (uint32_t)std::min(B.cap_leaf_pairs, (size_t)0xffffffffu));
            k_leaf_cells<<<ncb, 256, 0, s>>>(d, B.cell_cnt.as<uint32_t>(), B.cell_scan.as<uint2>(), B.tile_sums.as<uint2>(),
                                             B.cells.as<uint2>(), B.cell_lp.as<uint32_t>(), B.lp_scan.as<uint32_t>(),
                                             B.lp_tiles.as<uint32_t>(), B.refs.as<uint4>(), B.leaves.as<uint2>(),
                                             B.prims.as<uint32_t>(), ctl, B.big_list.as<uint32_t>());
            mark();
            k_leaf_cells_big<<<nbig, kBigT, 0, s>>>(d, B.cell_cnt.as<uint32_t>(), B.cell_scan.as<uint2>(),
                                                    B.tile_sums.as<uint2>(), B.cells.as<uint2>(), B.cell_lp.as<uint32_t>(),
                                                    B.lp_scan.as<uint32_t>(), B.lp_tiles.as<uint32_t>(),
                                                    B.refs.as<uint4>(), B.leaves.as<uint2>(), B.prims.as<uint32_t>(),
                                                    ctl, B.big_list.as<uint32_t>(), B.keys_a.as<uint32_t>(),
                                                    B.vals_a.as<uint32_t>(), B.keys_b.as<uint32_t>(),
                                                    B.vals_b.as<uint32_t>(), B.lkeys_a.as<uint32_t>(),
                                                    B.lvals_a.as<uint32_t>(), B.lkeys_b.as<uint32_t>(),
                                                    B.lvals_b.as<uint32_t>());
        } else {
            k_ug_cells<<<ncb, 256, 0, s>>>(d, B.cell_cnt.as<uint32_t>(), B.cell_scan.as<uint2>(), B.tile_sums.as<uint2>(),
                                           B.cells.as<uint2>(), B.refs.as<uint32_t>(), B.prims.as<uint32_t>(), ctl,
                                           B.big_list.as<uint32_t>());
            mark();
            k_ug_cells_big<<<nbig, kBigT, 0, s>>>(d, B.cell_cnt.as<uint32_t>(), B.cell_scan.as<uint2>(),
                                                  B.tile_sums.as<uint2>(), B.refs.as<uint32_t>(), B.prims.as<uint32_t>(),
                                                  ctl, B.big_list.as<uint32_t>(), B.keys_a.as<uint32_t>(),
                                                  B.keys_b.as<uint32_t>());
        }
        mark();
        c->nstages = ev;
        return 0;
    };
    // A rebuild identical to the previous one (the same frame, sizes, buffers and
    // settings: a mesh rebuilt every frame) is captured once as a CUDA graph and then
    // replayed: one launch instead of one per kernel, so small builds are not paced by the
    // host's launch rate.  An animated mesh replays the same graph for every frame time:
    // the frame pair and weight go to frame_sel first, outside the graph (only when the
    // word does not hold this selection already).
    if (c->lerp_pending) {
        uint32_t cb;
        std::memcpy(&cb, &c->frame_coeff, sizeof(cb));
        const int32_t want[3] = {c->frame_a, c->frame_b, (int32_t)cb};
        if (!c->frame_sel_valid || std::memcmp(want, c->frame_sel_host, sizeof(want)) != 0) {
            c->frame_sel_valid = false;
            k_frame_select<<<1, 1, 0, s>>>(c->frame_sel.as<int4>(), c->frame_a, c->frame_b, c->frame_coeff);
            c->launches += 1;
            if ((rc = cuda_check(c, cudaGetLastError(), "frame selection"))) return rc;
            std::memcpy(c->frame_sel_host, want, sizeof(want));
            c->frame_sel_valid = true;
        }
    }
    bool enqueued = false;
    std::vector<uint8_t> key;
    if (HR_BUILD_GRAPH && wait && c->build_graph_ok) key = build_graph_key(c, kind, exact, dens);
    if (!key.empty() && (key == c->build_key || key == c->last_build_key)) {
        if (c->build_exec && key == c->build_key) {
            if (cudaGraphLaunch(c->build_exec, s) == cudaSuccess) {
                c->launches += c->build_graph_launches;
                c->nstages = c->build_graph_stages;
                enqueued = true;
            } else {
                cudaGetLastError();
                drop_build_graph(c);
                c->build_graph_ok = false;
            }
        } else {
            drop_build_graph(c);
            cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
            if (cudaStreamIsCapturing(s, &cs) == cudaSuccess && cs == cudaStreamCaptureStatusNone &&
                cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
                const uint64_t l0 = c->launches;
                c->build_capturing = true;
                const int erc = enqueue();
                c->build_capturing = false;
                cudaGraph_t g = nullptr;
                const cudaError_t e = cudaStreamEndCapture(s, &g);
                if (erc) {
                    if (g) cudaGraphDestroy(g);
                    cudaGetLastError();
                    return erc;
                }
                if (e == cudaSuccess && g && cudaGraphInstantiate(&c->build_exec, g, 0) == cudaSuccess &&
                    cudaGraphLaunch(c->build_exec, s) == cudaSuccess) {
                    c->build_key = std::move(key);
                    c->build_graph_launches = c->launches - l0;
                    c->build_graph_stages = c->nstages;
                    enqueued = true;
                } else {   // not capturable here: build directly from now on
                    cudaGetLastError();
                    drop_build_graph(c);
                    c->build_graph_ok = false;
                    c->launches = l0;
                }
                if (g) cudaGraphDestroy(g);
            } else {
                cudaGetLastError();
            }
        }
    }
    if (!enqueued && (rc = enqueue())) return rc;
    c->last_build_key = std::move(key);
    if ((rc = cuda_check(c, cudaGetLastError(), "build launch"))) return rc;
    if (!wait) {
        if (!c->desc_pinned && cudaMallocHost((void**)&c->desc_pinned, sizeof(GridDesc)) != cudaSuccess) {
            cudaGetLastError();
            return set_error(c, 2, "pinned descriptor allocation failed");
        }
        return cuda_check(c, cudaMemcpyAsync(c->desc_pinned, d, sizeof(GridDesc), cudaMemcpyDeviceToHost, s),
                          "descriptor download");
    }
    if ((rc = cuda_check(c, cudaMemcpyAsync(&c->host_desc, d, sizeof(GridDesc), cudaMemcpyDeviceToHost, s),
                         "descriptor download")))
        return rc;
    if ((rc = cuda_check(c, cudaStreamSynchronize(s), "build"))) return rc;
    if (c->timing)
        for (int i = 0; i + 1 < c->nstages; ++i) cudaEventElapsedTime(&c->stage_ms[i], c->ev[i], c->ev[i + 1]);
    if (c->host_desc.error) return set_error(c, 1, "triangle index out of range of the uploaded vertices");
    *ovf_out = c->host_desc.overflow;
    return 0;
}

// A failed build may have stopped anywhere after the frame word's launch, so the word is
// rewritten by the next build that interpolates.
static int build_once(hr_ctx* c, int32_t kind, int32_t exact, uint32_t* ovf_out, bool wait) {
    const int rc = build_once_impl(c, kind, exact, ovf_out, wait);
    if (rc) c->frame_sel_valid = false;
    return rc;
}

// grow what overflowed from the exact sizes the device computed
static void grow_caps(hr_ctx* c, const GridDesc& hd, uint32_t ovf) {
    GridBuffers& B = c->g;
    if (ovf & kOvfCells) B.cap_cells = (size_t)hd.req_cells + 64u;
    if (ovf & (kOvfPairs | kOvfTopPairs)) B.cap_pairs = (size_t)(hd.req_pairs * 1.25) + 4096u;
    if (ovf & kOvfLeaves) B.cap_leaves = (size_t)(hd.nleaves * 1.25) + 4096u;
    if (ovf & kOvfLeafPairs) B.cap_leaf_pairs = (size_t)(hd.req_leaf_pairs * 1.25) + 4096u;
}

// After a build that fit: capacities follow the largest sizes seen so far plus 15%
// (an overflow later grows them again and rebuilds).
static void fit_caps(hr_ctx* c, const GridDesc& hd, int32_t kind) {
    GridBuffers& B = c->g;
    const size_t top = kind == kUniform ? hd.npairs : hd.ntop_pairs;
    B.seen_pairs = std::max(B.seen_pairs, top);
    auto fit = [](size_t& cap, size_t seen) {
        const size_t want = seen + seen / 7 + 4096;
        if (cap > want + want / 2) cap = want;   // only when the estimate is far above
    };
    fit(B.cap_pairs, B.seen_pairs);
    if (kind == kTwoLevel) {
        B.seen_leaves = std::max(B.seen_leaves, (size_t)hd.nleaves);
        B.seen_leaf_pairs = std::max(B.seen_leaf_pairs, (size_t)hd.npairs);
        fit(B.cap_leaves, B.seen_leaves);
        fit(B.cap_leaf_pairs, B.seen_leaf_pairs);
    }
}

int build_grid(hr_ctx* c, int32_t kind, int32_t exact) {
    GridBuffers& B = c->g;
    if (c->built_kind != kind) {
        B.cap_pairs = 0; B.cap_leaf_pairs = 0; B.cap_leaves = 0;
        B.seen_pairs = B.seen_leaves = B.seen_leaf_pairs = 0;
    }
    c->async_pending = false;
    for (int attempt = 0; attempt < 6; ++attempt) {
        uint32_t ovf = 0;
        int rc = build_once(c, kind, exact, &ovf, true);
        if (rc) return rc;
        if (ovf == 0) {
            c->built_kind = kind;
            c->built = true;
            c->lerp_pending = false;
            fit_caps(c, c->host_desc, kind);
            return 0;
        }
        grow_caps(c, c->host_desc, ovf);
    }
    return set_error(c, 3, "grid build: capacity did not converge");
}

int build_grid_async(hr_ctx* c, int32_t kind, int32_t exact) {
    if (c->built_kind != kind) return build_grid(c, kind, exact);   // a new kind is sized synchronously
    uint32_t ovf = 0;
    int rc = build_once(c, kind, exact, &ovf, false);
    if (rc) return rc;
    c->built = true;
    c->lerp_pending = false;
    c->async_pending = true;
    return 0;
}

int build_async_result(hr_ctx* c, bool* fit) {
    *fit = true;
    if (!c->async_pending) return 0;
    c->async_pending = false;
    c->host_desc = *c->desc_pinned;
    if (c->host_desc.error) return set_error(c, 1, "triangle index out of range of the uploaded vertices");
    const uint32_t ovf = c->host_desc.overflow;
    if (ovf) {
        *fit = false;
        c->built = false;
        grow_caps(c, c->host_desc, ovf);
    }
    return 0;
}

}  // namespace hr
