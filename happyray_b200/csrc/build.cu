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
// Differences in structure (results are identical to the reference's, canonicalised to
// ascending triangle id inside every cell):
//   * each triangle's pairs are written at its own exclusive-scan offset (block sums +
//     in-block scan) instead of a shared-memory atomicAdd slot, so the stable sort
//     yields ascending triangle ids per cell without any extra pass;
//   * all sizes (bounds, resolution, pair counts, leaf counts) stay in a device-side
//     descriptor; the whole build is enqueued without a host round trip and capacity
//     overflow is reported by flag;
//   * leaf-level pairs are likewise written at per-reference scan offsets in top-level
//     reference order, so the stable leaf sort gives ascending triangle ids per leaf;
//   * the pair-count pass also writes a per-triangle vertex array (3 float4) that the
//     later passes and the traversal read with one contiguous load per triangle.
#include "build_dev.cuh"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>

namespace hr {

namespace {

// ctl: the build's control words, whose work-list length and counter restart at zero
__global__ void k_desc_init(GridDesc* d, int32_t kind, uint32_t ntri, const uint32_t* bad_index_count, uint32_t* ctl) {
    // the error flag is set by the index check of the last upload
    desc_init(d, kind, ntri, *bad_index_count != 0u ? 1u : 0u);
    ctl[0] = 0u;   // kBigCount
    ctl[1] = 0u;   // kBigNext
}

// The key-frame pair and weight of the next interpolating build, written in stream order
// ahead of it so that a captured build graph replays for any frame time:
// sel = (frame a, frame b, bits of coeff, 0).
__global__ void k_frame_select(int4* sel, int32_t a, int32_t b, float coeff) {
    *sel = make_int4(a, b, __float_as_int(coeff), 0);
}

// a1: fused keyframe interpolation + bounds (WFObjectUploader.h:82-110).  The frames and
// coeff come from sel; coeff applies to frame b: v = a * (1 - c) + b * c.  With
// kf == nullptr the vertices are only reduced.
__global__ __launch_bounds__(kBT) void k_lerp_bounds(const float4* __restrict__ kf, const int4* __restrict__ sel,
                                                     float4* __restrict__ out, uint32_t nv, GridDesc* d) {
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
    reduce_bounds(lo, hi, d);
}

// a2: padded bounds and resolution, single thread
__global__ void k_grid_setup(GridDesc* d, float density, uint32_t cap_cells) {
    const uint64_t nc = grid_setup(d, density);
    if (nc >= (uint64_t)cap_cells) {
        // publish zero cells so later stages do nothing; the host regrows from req_cells
        d->overflow |= kOvfCells;
        d->req_cells = nc > 0xfffffff0ull ? 0xfffffff0u : (uint32_t)nc;
        d->ncells = 0u;
    } else {
        d->ncells = (uint32_t)nc;
    }
}

// a3: pair count, one triangle per thread; block sums for the scan (UniformGridBuildKernels.h:40-105).
// Also writes the per-triangle vertex array (3 float4) that the later build passes and the
// traversal read instead of gathering through the index buffer.
__global__ __launch_bounds__(kBT) void k_count_pairs(const float4* __restrict__ v, const uint32_t* __restrict__ idx,
                                                     uint32_t ntri, const GridDesc* d, uint32_t* block_sums,
                                                     float4* __restrict__ tris, uint4* __restrict__ rng) {
    if (d->overflow | d->error) {
        if (threadIdx.x == 0) block_sums[blockIdx.x] = 0u;
        return;
    }
    const DescRegs g = load_desc(d);
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
        if (rng && ranges_fit(g.res)) rng[t] = pack_range(r, n);
    }
    uint32_t tot;
    block_excl_scan<uint32_t, kBT>(n, &tot);
    if (threadIdx.x == 0) block_sums[blockIdx.x] = tot;
}

// a5: pair scatter at the triangle's exclusive-scan offset.  Keys are x + y*rx + z*rx*ry;
// with EXACT a cell rejected by the SAT test gets key = ncells (sorted last, skipped).
template <bool EXACT>
__global__ __launch_bounds__(kBT) void k_write_pairs(const float4* __restrict__ tris, uint32_t ntri, const GridDesc* d,
                                                     const uint32_t* block_sums, const uint4* __restrict__ rng,
                                                     uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
    if (d->overflow | d->error) return;
    const DescRegs g = load_desc(d);
    const uint32_t t = blockIdx.x * kBT + threadIdx.x;
    uint32_t n = 0;
    f3 p[3], lo, hi;
    CRange r;
    if (t < ntri) {
        if (!EXACT && rng && ranges_fit(g.res)) {
            n = unpack_range(__ldg(rng + t), &r);   // the range k_count_pairs found
        } else {
            tri_fetch(tris, t, p);
            tri_bbox(p, &lo, &hi);
            n = cell_range(lo, hi, g.bmin, g.rcp, g.res, &r);
        }
    }
    const uint32_t rx = (uint32_t)g.res[0], rxy = (uint32_t)g.res[0] * (uint32_t)g.res[1];
    if (!EXACT) {
        PairRun run;
        if (n) run = {(uint32_t)r.lo[0] + (uint32_t)r.lo[1] * rx + (uint32_t)r.lo[2] * rxy,
                      (uint32_t)(r.hi[0] - r.lo[0]), (uint32_t)(r.hi[1] - r.lo[1]), rx, rxy, t};
        block_write_runs<kBT>(n, run, block_sums[blockIdx.x], keys, vals);
        return;
    }
    uint32_t tot;
    uint32_t slot = block_excl_scan<uint32_t, kBT>(n, &tot) + block_sums[blockIdx.x];
    if (n == 0) return;
    const f3 nrm = normalize(cross(sub(p[1], p[0]), sub(p[2], p[0])));
    const f3 h = mulf(g.cs, 0.505f);
    f3 mc = mk((float)r.lo[0], (float)r.lo[1], (float)r.lo[2]);
    mc = mk(mc.x * g.cs.x, mc.y * g.cs.y, mc.z * g.cs.z);
    mc = add(add(mc, g.bmin), h);
    f3 c;
    c.z = mc.z - g.cs.z;
    for (int32_t z = r.lo[2]; z < r.hi[2]; ++z) {
        c.z += g.cs.z;
        c.y = mc.y - g.cs.y;
        for (int32_t y = r.lo[1]; y < r.hi[1]; ++y) {
            c.y += g.cs.y;
            c.x = mc.x - g.cs.x;
            for (int32_t x = r.lo[0]; x < r.hi[0]; ++x, ++slot) {
                c.x += g.cs.x;
                keys[slot] = sat_overlap(nrm, c, p, h) ? (uint32_t)x + (uint32_t)y * rx + (uint32_t)z * rxy
                                                       : g.ncells;
                vals[slot] = t;
            }
        }
    }
}

// a8: per top cell: leaf resolution, flags, leaf-cell count (countLeafLevelCells,
// TLGridBuildKernels.h:45-122); packed y of TwoLevelGridCell (TwoLevelGrid.h:38-161)
__global__ void k_tl_cells(const uint2* __restrict__ top_ranges, const GridDesc* d, float leaf_density,
                           uint32_t* __restrict__ leaf_cnt, uint2* __restrict__ top_cells) {
    if (d->overflow | d->error) return;
    const DescRegs g = load_desc(d);
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < g.ncells; c += gridDim.x * blockDim.x) {
        const uint2 rg = top_ranges[c];
        const uint32_t refs = rg.y - rg.x;
        const LeafGeom lg = leaf_geom(g, refs, leaf_density);
        uint32_t y = (lg.res[0] & 0xFFu) | ((lg.res[1] & 0xFFu) << 8) | ((lg.res[2] & 0xFFu) << 16);
        if (lg.leaf) y |= kLeafMask;
        if (refs != 0) y |= kNotEmptyMask;
        top_cells[c].y = y;
        leaf_cnt[c] = lg.res[0] * lg.res[1] * lg.res[2];
    }
}

// sub-cell range of top-level reference i: its top cell (sorted key), triangle, cell sub-grid
__device__ __forceinline__ uint32_t ref_leaf_range(const DescRegs& g, const uint32_t* __restrict__ top_keys,
                                                   const uint32_t* __restrict__ top_refs,
                                                   const float4* __restrict__ tris,
                                                   const uint2* __restrict__ top_cells, uint32_t i, uint32_t* cell,
                                                   uint32_t* tri, uint32_t* lres, CRange* r) {
    *cell = __ldg(top_keys + i);
    *tri = __ldg(top_refs + i);
    const uint32_t y = top_cells[*cell].y;
    lres[0] = y & 0xFFu; lres[1] = (y >> 8) & 0xFFu; lres[2] = (y >> 16) & 0xFFu;
    f3 p[3], lo, hi;
    tri_fetch(tris, *tri, p);
    tri_bbox(p, &lo, &hi);
    return leaf_range(g, lres, *cell, lo, hi, r);
}

// a10: leaf pair count per top-level reference, block sums (countLeafLevelPairs,
// TLGridBuildKernels.h:304-409)
__global__ __launch_bounds__(kBT) void k_leaf_count_pairs(const uint32_t* __restrict__ top_keys,
                                                          const uint32_t* __restrict__ top_refs,
                                                          const float4* __restrict__ tris,
                                                          const GridDesc* d, const uint2* __restrict__ top_cells,
                                                          uint32_t* block_sums, uint4* __restrict__ refrng) {
    if (d->overflow | d->error) {
        if (threadIdx.x == 0) block_sums[blockIdx.x] = 0u;
        return;
    }
    const DescRegs g = load_desc(d);
    const uint32_t i = blockIdx.x * kBT + threadIdx.x;
    uint32_t n = 0;
    if (i < d->ntop_pairs) {
        uint32_t cell, tri, lres[3];
        CRange r;
        n = ref_leaf_range(g, top_keys, top_refs, tris, top_cells, i, &cell, &tri, lres, &r);
        if (refrng) refrng[i] = pack_ref(r, lres, top_cells[cell].x, tri);
    }
    uint32_t tot;
    block_excl_scan<uint32_t, kBT>(n, &tot);
    if (threadIdx.x == 0) block_sums[blockIdx.x] = tot;
}

// a11: leaf pairs in reference order at each reference's scan offset; key = first leaf of
// the top cell + local sub-cell index (writeLeafLevelKeysAndValues, TLGridBuildKernels.h:536-663).
// The references are sorted by (top cell, triangle), so each top cell's leaf pairs form one
// segment [cell_pb, cell_pe) in ascending triangle order; the first and last reference of a
// cell record the segment's ends.
__global__ __launch_bounds__(kBT) void k_leaf_write_pairs(const uint4* __restrict__ refrng, const GridDesc* d,
                                                          const uint32_t* block_sums, uint32_t* __restrict__ keys,
                                                          uint32_t* __restrict__ vals,
                                                          const uint32_t* __restrict__ top_keys,
                                                          uint32_t* __restrict__ cell_pb, uint32_t* __restrict__ cell_pe) {
    if (d->overflow | d->error) return;
    const uint32_t i = blockIdx.x * kBT + threadIdx.x;
    uint32_t n = 0, tri = 0, base = 0, lres[2] = {1u, 1u};
    CRange r;
    if (i < d->ntop_pairs) {   // the sub-cell range k_leaf_count_pairs found
        const uint4 q = __ldg(refrng + i);
        n = 1;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            r.lo[k] = (int32_t)((q.x >> (8 * k)) & 0xFFu);
            r.hi[k] = (int32_t)((q.y >> (8 * k)) & 0xFFu);
            const int32_t e = r.hi[k] - r.lo[k];
            n *= (uint32_t)(e > 0 ? e : 0);
        }
        lres[0] = q.x >> 24;
        lres[1] = q.y >> 24;
        base = q.z;
        tri = q.w;
    }
    PairRun run;
    if (n) run = {base + (uint32_t)r.lo[0] + (uint32_t)r.lo[1] * lres[0] + (uint32_t)r.lo[2] * lres[0] * lres[1],
                  (uint32_t)(r.hi[0] - r.lo[0]), (uint32_t)(r.hi[1] - r.lo[1]), lres[0], lres[0] * lres[1], tri};
    const uint32_t at = block_write_runs<kBT>(n, run, block_sums[blockIdx.x], keys, vals);
    const uint32_t nref = d->ntop_pairs;
    if (i < nref) {
        const uint32_t cell = __ldg(top_keys + i);
        if (i == 0 || __ldg(top_keys + i - 1) != cell) cell_pb[cell] = at;
        if (i + 1 == nref || __ldg(top_keys + i + 1) != cell) cell_pe[cell] = at + n;
    }
}

// Build control words in device memory: the big-cell list length and its work counter,
// reset by k_desc_init at the start of every build.
enum : int { kBigCount = 0, kBigNext = 1, kCtlWords = 16 };

constexpr int kSegT = 512;                       // threads of the per-segment CTA kernel
constexpr int kSegW = kSegT / 32;
constexpr int kSegIpt = 8;
constexpr uint32_t kSegChunk = kSegT * kSegIpt;  // items ranked per chunk
constexpr uint32_t kSegCap = 24576;              // items a segment sorts in shared memory
constexpr int kSegPosBits = 17;                  // position of an item in its segment
constexpr size_t kSegDynSmem = sizeof(uint32_t) * 2 * kSegCap;

// a13 for the common cases, one thread per top cell (prepareLeafCellRanges,
// TLGridBuildKernels.h:750-834): an empty cell's single leaf is empty; a cell with one
// leaf holds its whole segment, already in ascending triangle order.  Cells with more
// leaves are listed for k_leaf_cells_big.
__global__ void k_leaf_cells(const GridDesc* d, const uint2* __restrict__ top_ranges, const uint2* __restrict__ cells,
                             const uint32_t* __restrict__ cell_pb, const uint32_t* __restrict__ cell_pe,
                             const uint32_t* __restrict__ vals, uint2* __restrict__ leaves,
                             uint32_t* __restrict__ prims, uint32_t* ctl, uint32_t* __restrict__ big_list) {
    if (d->overflow | d->error) return;
    const uint32_t C = d->ncells;
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < C; c += gridDim.x * blockDim.x) {
        const uint2 tr = top_ranges[c];
        const uint2 cw = cells[c];
        const uint32_t y = cw.y;
        const uint32_t nl = (y & 0xFFu) * ((y >> 8) & 0xFFu) * ((y >> 16) & 0xFFu);
        if (tr.y == tr.x) {
            leaves[cw.x] = make_uint2(0u, 0u);
        } else if (nl == 1u) {
            const uint32_t pb = cell_pb[c], pe = cell_pe[c];
            leaves[cw.x] = pe > pb ? make_uint2(pb, pe) : make_uint2(0u, 0u);
            for (uint32_t i = pb; i < pe; ++i) prims[i] = __ldg(vals + i);
        } else {
            big_list[atomicAdd(ctl + kBigCount, 1u)] = c;
        }
    }
}

struct SegSmem {
    uint32_t cur[256];            // digit counts, then running digit cursors
    uint32_t whist[kSegW][256];   // per warp and digit: count, then output base
    uint32_t item;
};

// Stable LSD radix sort by one CTA of the n words at a (b: the other half of the
// ping-pong; shared memory, or global scratch for large segments) on the bits [shift, shift + 8 * passes) in 8-bit digits.  Each pass counts
// the digits, then ranks chunks of kSegChunk words in order: within a warp by match_any,
// across warps by per-warp digit counts.  Returns the buffer holding the result.
template <class Wd>
__device__ Wd* cta_smem_radix(Wd* a, Wd* b, uint32_t n, int shift, int passes, SegSmem& sm) {
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    const uint32_t lt = (1u << lane) - 1u;
    for (int p = 0; p < passes; ++p) {
        const Wd* src = (p & 1) ? b : a;
        Wd* dst = (p & 1) ? a : b;
        const int sh = shift + 8 * p;
        for (uint32_t i = threadIdx.x; i < 256; i += kSegT) sm.cur[i] = 0u;
        __syncthreads();
        for (uint32_t base = 0; base < n; base += kSegT) {
            const uint32_t i = base + threadIdx.x;
            const uint32_t dg = i < n ? (uint32_t)(src[i] >> sh) & 255u : 256u;
            const uint32_t peers = __match_any_sync(kFullMask, dg);
            if (dg < 256u && lane == (uint32_t)(__ffs(peers) - 1)) atomicAdd(&sm.cur[dg], (uint32_t)__popc(peers));
        }
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
        for (uint32_t base = 0; base < n; base += kSegChunk) {
            for (uint32_t i = threadIdx.x; i < kSegW * 256; i += kSegT) (&sm.whist[0][0])[i] = 0u;
            __syncthreads();
            Wd key[kSegIpt];
            uint32_t dig[kSegIpt], rank[kSegIpt];
#pragma unroll
            for (int r = 0; r < kSegIpt; ++r) {
                const uint32_t i = base + (w * kSegIpt + r) * 32 + lane;
                key[r] = i < n ? src[i] : (Wd)0;
                dig[r] = i < n ? (uint32_t)(key[r] >> sh) & 255u : 256u;
            }
#pragma unroll
            for (int r = 0; r < kSegIpt; ++r) {
                const uint32_t peers = __match_any_sync(kFullMask, dig[r]);
                const uint32_t leader = (uint32_t)(__ffs(peers) - 1);
                uint32_t bb = 0;
                if (dig[r] < 256u && lane == leader) {
                    bb = sm.whist[w][dig[r]];
                    sm.whist[w][dig[r]] = bb + (uint32_t)__popc(peers);
                }
                bb = __shfl_sync(kFullMask, bb, (int)leader);
                rank[r] = bb + (uint32_t)__popc(peers & lt);
                __syncwarp();
            }
            __syncthreads();
            for (uint32_t dd = threadIdx.x; dd < 256; dd += kSegT) {
                uint32_t run = sm.cur[dd];
                for (uint32_t ww = 0; ww < kSegW; ++ww) {
                    const uint32_t t = sm.whist[ww][dd];
                    sm.whist[ww][dd] = run;
                    run += t;
                }
                sm.cur[dd] = run;
            }
            __syncthreads();
#pragma unroll
            for (int r = 0; r < kSegIpt; ++r)
                if (dig[r] < 256u) dst[sm.whist[w][dig[r]] + rank[r]] = key[r];
            __syncthreads();
        }
    }
    return (passes & 1) ? b : a;
}

__device__ __forceinline__ int bit_width(uint32_t x) { return x ? 32 - __clz(x) : 0; }

// a11-a13 for top cells with more than one leaf: one CTA per listed cell, taken from a work
// counter.  The cell's segment of leaf pairs is in ascending triangle order; it is sorted
// stably by local leaf index: the words (leaf << 17 | position in the segment) are
// radix-sorted on their leaf bits in shared memory, the leaf ranges follow from the sorted
// words and each list takes its triangles from the positions.  A segment of more than
// kSegCap pairs or a cell of more than 2^15 leaves sorts 64-bit words (leaf << 32 |
// position) the same way in global scratch (g64: 2 words per leaf pair).
__global__ __launch_bounds__(kSegT, 1) void k_leaf_cells_big(const GridDesc* d, const uint2* __restrict__ cells,
                                                             const uint32_t* __restrict__ cell_pb,
                                                             const uint32_t* __restrict__ cell_pe,
                                                             const uint32_t* __restrict__ keys,
                                                             const uint32_t* __restrict__ vals,
                                                             uint2* __restrict__ leaves, uint32_t* __restrict__ prims,
                                                             uint32_t* ctl, const uint32_t* __restrict__ big_list,
                                                             unsigned long long* g64) {
    if (d->overflow | d->error) return;
    __shared__ SegSmem sm;
    extern __shared__ uint32_t s_buf[];
    const uint32_t nbig = ctl[kBigCount];
    const uint32_t npairs = d->npairs;
    for (;;) {
        if (threadIdx.x == 0) sm.item = atomicAdd(ctl + kBigNext, 1u);
        __syncthreads();
        const uint32_t item = sm.item;
        __syncthreads();
        if (item >= nbig) return;
        const uint32_t c = big_list[item];
        const uint2 cw = cells[c];
        const uint32_t lb = cw.x, y = cw.y;
        const uint32_t nl = (y & 0xFFu) * ((y >> 8) & 0xFFu) * ((y >> 16) & 0xFFu);
        const uint32_t pb = cell_pb[c], P = cell_pe[c] - pb;
        const int lbits = bit_width(nl - 1u);
        for (uint32_t l = threadIdx.x; l < nl; l += kSegT) leaves[lb + l] = make_uint2(0u, 0u);
        if (P <= kSegCap && lbits <= 32 - kSegPosBits) {
            for (uint32_t i = threadIdx.x; i < P; i += kSegT)
                s_buf[i] = ((__ldg(keys + pb + i) - lb) << kSegPosBits) | i;
            __syncthreads();
            const uint32_t* sw = cta_smem_radix(s_buf, s_buf + kSegCap, P, kSegPosBits, (lbits + 7) / 8, sm);
            for (uint32_t s = threadIdx.x; s < P; s += kSegT) {
                const uint32_t wv = sw[s], l = wv >> kSegPosBits;
                prims[pb + s] = __ldg(vals + pb + (wv & ((1u << kSegPosBits) - 1u)));
                if (s == 0 || (sw[s - 1] >> kSegPosBits) != l) leaves[lb + l].x = pb + s;
                if (s + 1 == P || (sw[s + 1] >> kSegPosBits) != l) leaves[lb + l].y = pb + s + 1;
            }
        } else {
            unsigned long long* a = g64 + pb;
            unsigned long long* b = g64 + npairs + pb;
            for (uint32_t i = threadIdx.x; i < P; i += kSegT)
                a[i] = ((unsigned long long)(__ldg(keys + pb + i) - lb) << 32) | i;
            __syncthreads();
            const unsigned long long* sw = cta_smem_radix(a, b, P, 32, (lbits + 7) / 8, sm);
            for (uint32_t s = threadIdx.x; s < P; s += kSegT) {
                const unsigned long long wv = sw[s];
                const uint32_t l = (uint32_t)(wv >> 32);
                prims[pb + s] = __ldg(vals + pb + (uint32_t)wv);
                if (s == 0 || (uint32_t)(sw[s - 1] >> 32) != l) leaves[lb + l].x = pb + s;
                if (s + 1 == P || (uint32_t)(sw[s + 1] >> 32) != l) leaves[lb + l].y = pb + s + 1;
            }
        }
        __syncthreads();
    }
}

int key_bits_for(size_t max_key) {
    int b = 1;
    while (b < 32 && ((size_t)1 << b) <= max_key) ++b;
    return b;
}


}  // namespace

// Everything a captured build depends on: grid kind and settings, sizes and capacities,
// and the addresses of every buffer the build reads or writes.
static std::vector<uint8_t> build_graph_key(const hr_ctx* c, int32_t kind, int32_t exact, float dens) {
    const GridBuffers& B = c->g;
    const DevBuf* bufs[] = {&B.desc, &c->tris, &B.cells, &B.keys_a, &B.tri_ranges, &B.vals_a, &B.keys_b, &B.vals_b,
                            &B.block_sums, &B.tile_hist, &B.row_total, &B.prims, &B.top_ranges, &B.top_refs,
                            &B.ref_ranges, &B.leaf_cnt, &B.scan_partials, &B.leaves, &B.lkeys_a, &B.lvals_a,
                            &B.cell_pb, &B.cell_pe, &B.ctl, &B.big_list, &B.seg_words, &c->verts, &c->idx,
                            &c->counters, &c->keyframes, &c->frame_sel};
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
    const float dens = kind == kUniform ? c->ug_density : c->top_density;
    // capacity of the cell array is a bound (prod res <= density * N), not a guess
    const size_t cells_bound = (size_t)(std::floor((double)dens * (double)ntri * 1.01)) + 32768u + 64u;
    if (B.cap_cells < cells_bound) B.cap_cells = cells_bound;
    if (B.cap_pairs == 0) B.cap_pairs = (size_t)ntri * (kind == kUniform ? 6u : 3u) + 4096u;
    if (kind == kTwoLevel) {
        if (B.cap_leaf_pairs == 0) B.cap_leaf_pairs = (size_t)ntri * 4u + 4096u;
        if (B.cap_leaves == 0) B.cap_leaves = (size_t)(c->leaf_density * 2.0f * (float)B.cap_pairs) + B.cap_cells;
    }
    const size_t cap_pairs = B.cap_pairs;   // uniform pairs, or top-level pairs for two-level
    const uint32_t nblocks = (ntri + kBT - 1) / kBT;
    const int key_bits = key_bits_for(B.cap_cells);
    const int passes = radix_sort_passes(key_bits);
    const uint32_t nref_blocks = (uint32_t)((cap_pairs + kBT - 1) / kBT);   // per top-level reference
    size_t hist_words = radix_tile_hist_words(cap_pairs, key_bits);
    int rc;
    if ((rc = ensure(c, B.desc, sizeof(GridDesc)))) return rc;
    if ((rc = ensure(c, c->frame_sel, sizeof(int4)))) return rc;
    if ((rc = ensure(c, c->tris, sizeof(float4) * 3 * (size_t)ntri))) return rc;
    if ((rc = ensure(c, B.cells, sizeof(uint2) * B.cap_cells))) return rc;
    if ((rc = ensure(c, B.keys_a, sizeof(uint32_t) * cap_pairs))) return rc;
    if ((rc = ensure(c, B.tri_ranges, sizeof(uint4) * (size_t)ntri))) return rc;
    if ((rc = ensure(c, B.vals_a, sizeof(uint32_t) * cap_pairs))) return rc;
    if ((rc = ensure(c, B.keys_b, sizeof(uint32_t) * cap_pairs))) return rc;
    if ((rc = ensure(c, B.vals_b, sizeof(uint32_t) * cap_pairs))) return rc;
    if ((rc = ensure(c, B.block_sums, sizeof(uint32_t) * (std::max(nblocks, nref_blocks) + 1)))) return rc;
    if ((rc = ensure(c, B.tile_hist, sizeof(uint32_t) * hist_words))) return rc;
    if ((rc = ensure(c, B.row_total, sizeof(uint32_t) * kRadixRowWords))) return rc;
    if (!B.ctl.p && (rc = ensure(c, B.ctl, sizeof(uint32_t) * kCtlWords))) return rc;
    if (kind == kUniform) {
        if ((rc = ensure(c, B.prims, sizeof(uint32_t) * cap_pairs))) return rc;
    } else {
        if ((rc = ensure(c, B.top_ranges, sizeof(uint2) * B.cap_cells))) return rc;
        if ((rc = ensure(c, B.top_refs, sizeof(uint32_t) * cap_pairs))) return rc;
        if ((rc = ensure(c, B.ref_ranges, sizeof(uint4) * cap_pairs))) return rc;
        if ((rc = ensure(c, B.leaf_cnt, sizeof(uint32_t) * B.cap_cells))) return rc;
        if ((rc = ensure(c, B.scan_partials, sizeof(uint32_t) * (scan_partials_words(B.cap_cells) + 2)))) return rc;
        if ((rc = ensure(c, B.leaves, sizeof(uint2) * B.cap_leaves))) return rc;
        if ((rc = ensure(c, B.lkeys_a, sizeof(uint32_t) * B.cap_leaf_pairs))) return rc;
        if ((rc = ensure(c, B.lvals_a, sizeof(uint32_t) * B.cap_leaf_pairs))) return rc;
        if ((rc = ensure(c, B.prims, sizeof(uint32_t) * B.cap_leaf_pairs))) return rc;
        if ((rc = ensure(c, B.cell_pb, sizeof(uint32_t) * B.cap_cells))) return rc;
        if ((rc = ensure(c, B.cell_pe, sizeof(uint32_t) * B.cap_cells))) return rc;
        if ((rc = ensure(c, B.big_list, sizeof(uint32_t) * B.cap_cells))) return rc;
        if ((rc = ensure(c, B.seg_words, sizeof(unsigned long long) * 2 * B.cap_leaf_pairs))) return rc;
        static bool attr_set[64] = {};   // per device, once per process
        const int dv = c->device & 63;
        if (!attr_set[dv]) {
            if ((rc = cuda_check(c, cudaFuncSetAttribute(k_leaf_cells_big, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                         (int)kSegDynSmem), "leaf kernel shared memory")))
                return rc;
            attr_set[dv] = true;
        }
    }
    GridDesc* d = B.desc.as<GridDesc>();
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
        // launches of this function (radix sort and scans count their own)
        c->launches += 3 + (nblocks > 0 ? 3 : 0) + 2 + (kind == kTwoLevel ? 6 : 0);
        k_desc_init<<<1, 1, 0, s>>>(d, kind, ntri, c->counters.as<uint32_t>() + 2, B.ctl.as<uint32_t>());
        const int gridv = std::max(1, std::min((int)((c->nverts + kBT - 1) / kBT), c->num_sms * 8));
        k_lerp_bounds<<<gridv, kBT, 0, s>>>(c->lerp_pending ? c->keyframes.as<float4>() : nullptr,
                                            c->frame_sel.as<int4>(), c->verts.as<float4>(), c->nverts, d);
        k_grid_setup<<<1, 1, 0, s>>>(d, dens, (uint32_t)std::min(B.cap_cells, (size_t)0xffffffffu));
        mark();
        const float4* v = c->verts.as<float4>();
        const uint32_t* ix = c->idx.as<uint32_t>();
        uint32_t* bsum = B.block_sums.as<uint32_t>();
        uint32_t* d_np = kind == kUniform ? &d->npairs : &d->ntop_pairs;
        if (nblocks > 0) {
            k_count_pairs<<<nblocks, kBT, 0, s>>>(v, ix, ntri, d, bsum, c->tris.as<float4>(), B.tri_ranges.as<uint4>());
            if ((rc = scan_block_sums(c, bsum, nblocks, d_np, &d->overflow, (uint32_t)std::min(cap_pairs, (size_t)0xffffffffu),
                                      kind == kUniform ? kOvfPairs : kOvfTopPairs, &d->req_pairs, s)))
                return rc;
            if (kind == kUniform && exact)
                k_write_pairs<true><<<nblocks, kBT, 0, s>>>(c->tris.as<float4>(), ntri, d, bsum, nullptr,
                                                            B.keys_a.as<uint32_t>(), B.vals_a.as<uint32_t>());
            else
                k_write_pairs<false><<<nblocks, kBT, 0, s>>>(c->tris.as<float4>(), ntri, d, bsum, B.tri_ranges.as<uint4>(),
                                                             B.keys_a.as<uint32_t>(), B.vals_a.as<uint32_t>());
        }
        mark();
        uint32_t* sorted_keys = (passes % 2 == 1) ? B.keys_b.as<uint32_t>() : B.keys_a.as<uint32_t>();
        uint32_t* sorted_vals = kind == kUniform ? B.prims.as<uint32_t>() : B.top_refs.as<uint32_t>();
        if ((rc = radix_sort_pairs(c, B.keys_a.as<uint32_t>(), B.vals_a.as<uint32_t>(), B.keys_b.as<uint32_t>(),
                                   B.vals_b.as<uint32_t>(), sorted_keys, sorted_vals, d_np, cap_pairs, key_bits,
                                   B.tile_hist.as<uint32_t>(), B.tile_hist.bytes, B.row_total.as<uint32_t>(), s)))
            return rc;
        mark();
        uint2* ranges = kind == kUniform ? B.cells.as<uint2>() : B.top_ranges.as<uint2>();
        const int gcells = std::max(1, std::min((int)((B.cap_cells + 255) / 256), c->num_sms * 16));
        k_fill_u2<<<gcells, 256, 0, s>>>(ranges, &d->ncells, d, make_uint2(0u, 0u));
        const int gpairs = std::max(1, std::min((int)((cap_pairs + 255) / 256), c->num_sms * 16));
        k_cell_ranges<<<gpairs, 256, 0, s>>>(sorted_keys, d_np, &d->ncells, d, ranges);
        mark();
        if (kind == kTwoLevel) {
            // leaf level, TLGridSortBuilder.h:256-410: leaf cells per top cell, scan, leaf pairs
            // per reference in reference order, stable sort by leaf, leaf ranges
            k_tl_cells<<<gcells, 256, 0, s>>>(ranges, d, c->leaf_density, B.leaf_cnt.as<uint32_t>(), B.cells.as<uint2>());
            uint32_t* sp = B.scan_partials.as<uint32_t>();
            if ((rc = exclusive_scan_u32(c, B.leaf_cnt.as<uint32_t>(), &d->ncells, B.cap_cells, &d->nleaves, sp, s)))
                return rc;
            k_check_leaves<<<1, 1, 0, s>>>(d, (uint32_t)std::min(B.cap_leaves, (size_t)0xffffffffu));
            k_tl_cell_begin<<<gcells, 256, 0, s>>>(B.leaf_cnt.as<uint32_t>(), d, B.cells.as<uint2>());
            mark();
            uint32_t* lsum = B.block_sums.as<uint32_t>();
            k_leaf_count_pairs<<<nref_blocks, kBT, 0, s>>>(sorted_keys, B.top_refs.as<uint32_t>(), c->tris.as<float4>(), d,
                                                           B.cells.as<uint2>(), lsum, B.ref_ranges.as<uint4>());
            if ((rc = scan_block_sums(c, lsum, nref_blocks, &d->npairs, &d->overflow,
                                      (uint32_t)std::min(B.cap_leaf_pairs, (size_t)0xffffffffu), kOvfLeafPairs,
                                      &d->req_leaf_pairs, s)))
                return rc;
            k_leaf_write_pairs<<<nref_blocks, kBT, 0, s>>>(B.ref_ranges.as<uint4>(), d, lsum, B.lkeys_a.as<uint32_t>(),
                                                           B.lvals_a.as<uint32_t>(), sorted_keys, B.cell_pb.as<uint32_t>(),
                                                           B.cell_pe.as<uint32_t>());
            mark();
            // a12-a13: each top cell's segment sorted stably by leaf where it lies
            c->launches += 2;
            k_leaf_cells<<<gcells, 256, 0, s>>>(d, ranges, B.cells.as<uint2>(), B.cell_pb.as<uint32_t>(),
                                                B.cell_pe.as<uint32_t>(), B.lvals_a.as<uint32_t>(), B.leaves.as<uint2>(),
                                                B.prims.as<uint32_t>(), B.ctl.as<uint32_t>(), B.big_list.as<uint32_t>());
            k_leaf_cells_big<<<c->num_sms, kSegT, kSegDynSmem, s>>>(
                d, B.cells.as<uint2>(), B.cell_pb.as<uint32_t>(), B.cell_pe.as<uint32_t>(), B.lkeys_a.as<uint32_t>(),
                B.lvals_a.as<uint32_t>(), B.leaves.as<uint2>(), B.prims.as<uint32_t>(), B.ctl.as<uint32_t>(),
                B.big_list.as<uint32_t>(), B.seg_words.as<unsigned long long>());
            mark();
        }
        c->nstages = ev;
        return 0;
    };
    // A rebuild identical to the previous one (the same frame, sizes, buffers and
    // settings: a mesh rebuilt every frame) is captured once as a CUDA graph and then
    // replayed: one launch instead of about 35, so small builds are not paced by the host's
    // launch rate.  An animated mesh replays the same graph for every frame time: the frame
    // pair and weight go to frame_sel first, outside the graph.
    // (only when the word does not hold this selection already: a static mesh whose frame
    // time is set every frame launches nothing extra)
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
// (an overflow later grows them again and rebuilds).  Smaller capacities mean fewer
// blocks in the per-reference passes, fewer radix tiles and shorter histogram scans.
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
