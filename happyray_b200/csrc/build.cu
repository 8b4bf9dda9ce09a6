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

__global__ void k_desc_init(GridDesc* d, int32_t kind, uint32_t ntri, const uint32_t* bad_index_count) {
    // the error flag is set by the index check of the last upload
    desc_init(d, kind, ntri, *bad_index_count != 0u ? 1u : 0u);
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
// With cell_count (two-level), the kernel's threads also clear the per-top-cell reference
// counts that k_write_pairs accumulates.
__global__ __launch_bounds__(kBT) void k_count_pairs(const float4* __restrict__ v, const uint32_t* __restrict__ idx,
                                                     uint32_t ntri, const GridDesc* d, uint32_t* block_sums,
                                                     float4* __restrict__ tris, uint4* __restrict__ rng,
                                                     uint32_t* __restrict__ cell_count) {
    if (d->overflow | d->error) {
        if (threadIdx.x == 0) block_sums[blockIdx.x] = 0u;
        return;
    }
    const DescRegs g = load_desc(d);
    if (cell_count)
        for (uint32_t c = blockIdx.x * kBT + threadIdx.x; c < g.ncells; c += gridDim.x * kBT) cell_count[c] = 0u;
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
// With cell_count, every pair's cell is also counted there (the two-level build needs the
// number of references per top cell, not their sorted order).
template <bool EXACT>
__global__ __launch_bounds__(kBT) void k_write_pairs(const float4* __restrict__ tris, uint32_t ntri, const GridDesc* d,
                                                     const uint32_t* block_sums, const uint4* __restrict__ rng,
                                                     uint32_t* __restrict__ keys, uint32_t* __restrict__ vals,
                                                     uint32_t* __restrict__ cell_count) {
    if (d->overflow | d->error) return;
    const DescRegs g = load_desc(d);
    const uint32_t bx = gridDim.x - 1u - blockIdx.x;   // last block first (see k_leaf_write_pairs)
    const uint32_t t = bx * kBT + threadIdx.x;
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
        block_write_runs<kBT>(n, run, block_sums[bx], keys, vals, cell_count);
        return;
    }
    uint32_t tot;
    uint32_t slot = block_excl_scan<uint32_t, kBT>(n, &tot) + block_sums[bx];
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
// leaf_cnt holds each top cell's reference count on entry (k_write_pairs) and its leaf
// count on return.
// occ gets one bit per top cell (set: the cell has references), a word per warp pass.
// Launched with a block size that is a multiple of 32.
__global__ void k_tl_cells(const GridDesc* d, float leaf_density, uint32_t* __restrict__ leaf_cnt,
                           uint2* __restrict__ top_cells, uint32_t* __restrict__ occ) {
    if (d->overflow | d->error) return;
    const DescRegs g = load_desc(d);
    const uint32_t lane = threadIdx.x & 31u;
    // warp-uniform trip count: the 32 cells of a pass share one occupancy word
    for (uint32_t c0 = blockIdx.x * blockDim.x + threadIdx.x - lane; c0 < g.ncells; c0 += gridDim.x * blockDim.x) {
        const uint32_t c = c0 + lane;
        bool full = false;
        if (c < g.ncells) {
            const uint32_t refs = leaf_cnt[c];
            const LeafGeom lg = leaf_geom(g, refs, leaf_density);
            uint32_t y = (lg.res[0] & 0xFFu) | ((lg.res[1] & 0xFFu) << 8) | ((lg.res[2] & 0xFFu) << 16);
            if (lg.leaf) y |= kLeafMask;
            if (refs != 0) y |= kNotEmptyMask;
            top_cells[c].y = y;
            leaf_cnt[c] = lg.res[0] * lg.res[1] * lg.res[2];
            full = refs != 0;
        }
        const uint32_t word = __ballot_sync(0xffffffffu, full);
        if (lane == 0) occ[c0 >> 5] = word;
    }
}

// sub-cell range of top-level reference i (pairs in triangle order): its top cell, triangle,
// cell sub-grid
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
// TLGridBuildKernels.h:304-409); the references are the top-level pairs as written, in
// triangle order
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
// Blocks take the references from the end first: a block's work is its pair count, and a
// mesh's large triangles (a ground plane over thousands of cells) tend to sit at one end of
// it; launched last, their long blocks would run alone at the end of the kernel.
__global__ __launch_bounds__(kBT) void k_leaf_write_pairs(const uint4* __restrict__ refrng, const GridDesc* d,
                                                          const uint32_t* block_sums, uint32_t* __restrict__ keys,
                                                          uint32_t* __restrict__ vals) {
    if (d->overflow | d->error) return;
    const uint32_t bx = gridDim.x - 1u - blockIdx.x;
    const uint32_t i = bx * kBT + threadIdx.x;
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
    block_write_runs<kBT>(n, run, block_sums[bx], keys, vals);
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
                            &B.block_sums, &B.tile_hist, &B.row_total, &B.prims,
                            &B.ref_ranges, &B.leaf_cnt, &B.occ, &B.scan_partials, &B.leaves, &B.lkeys_a, &B.lvals_a,
                            &B.lkeys_b, &B.lvals_b, &c->verts, &c->idx, &c->counters, &c->keyframes, &c->frame_sel};
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

// status of a built descriptor whose error word is set
static int desc_error(hr_ctx* c) {
    if (c->host_desc.error & kDescErrBarrier) {
        c->small_build_max_tris = 0;   // the pipeline from now on
        return set_error(c, 1, "grid build: a barrier of the single-launch build gave up waiting");
    }
    return set_error(c, 1, "triangle index out of range of the uploaded vertices");
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
    const int leaf_bits = key_bits_for(B.cap_leaves);
    const int leaf_passes = radix_sort_passes(leaf_bits);
    const uint32_t nref_blocks = (uint32_t)((cap_pairs + kBT - 1) / kBT);   // per top-level reference
    const size_t hist_words = kind == kUniform ? radix_tile_hist_words(cap_pairs, key_bits)
                                               : radix_tile_hist_words(B.cap_leaf_pairs, leaf_bits);
    int rc;
    if ((rc = ensure(c, B.desc, sizeof(GridDesc)))) return rc;
    if ((rc = ensure(c, c->frame_sel, sizeof(int4)))) return rc;
    if ((rc = ensure(c, c->tris, sizeof(float4) * 3 * (size_t)ntri))) return rc;
    if ((rc = ensure(c, B.cells, sizeof(uint2) * B.cap_cells))) return rc;
    if ((rc = ensure(c, B.keys_a, sizeof(uint32_t) * cap_pairs))) return rc;
    if ((rc = ensure(c, B.tri_ranges, sizeof(uint4) * (size_t)ntri))) return rc;
    if ((rc = ensure(c, B.vals_a, sizeof(uint32_t) * cap_pairs))) return rc;
    if ((rc = ensure(c, B.block_sums, sizeof(uint32_t) * (std::max(nblocks, nref_blocks) + 1)))) return rc;
    if ((rc = ensure(c, B.tile_hist, sizeof(uint32_t) * hist_words))) return rc;
    if ((rc = ensure(c, B.row_total, sizeof(uint32_t) * kRadixRowWords))) return rc;
    if (kind == kUniform) {   // the sort's second buffers (the two-level top level is not sorted)
        if ((rc = ensure(c, B.keys_b, sizeof(uint32_t) * cap_pairs))) return rc;
        if ((rc = ensure(c, B.vals_b, sizeof(uint32_t) * cap_pairs))) return rc;
        if ((rc = ensure(c, B.prims, sizeof(uint32_t) * cap_pairs))) return rc;
    } else {
        if ((rc = ensure(c, B.ref_ranges, sizeof(uint4) * cap_pairs))) return rc;
        if ((rc = ensure(c, B.leaf_cnt, sizeof(uint32_t) * B.cap_cells))) return rc;
        if ((rc = ensure(c, B.occ, sizeof(uint32_t) * (B.cap_cells / 32 + 1)))) return rc;
        if ((rc = ensure(c, B.scan_partials, sizeof(uint32_t) * (scan_partials_words(B.cap_cells) + 2)))) return rc;
        if ((rc = ensure(c, B.leaves, sizeof(uint2) * B.cap_leaves))) return rc;
        if ((rc = ensure(c, B.lkeys_a, sizeof(uint32_t) * B.cap_leaf_pairs))) return rc;
        if ((rc = ensure(c, B.lvals_a, sizeof(uint32_t) * B.cap_leaf_pairs))) return rc;
        if ((rc = ensure(c, B.lkeys_b, sizeof(uint32_t) * B.cap_leaf_pairs))) return rc;
        if ((rc = ensure(c, B.lvals_b, sizeof(uint32_t) * B.cap_leaf_pairs))) return rc;
        if ((rc = ensure(c, B.prims, sizeof(uint32_t) * B.cap_leaf_pairs))) return rc;
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
        c->launches += 3 + (nblocks > 0 ? 3 : 0) + (kind == kTwoLevel ? 9 : 2);
        k_desc_init<<<1, 1, 0, s>>>(d, kind, ntri, c->counters.as<uint32_t>() + 2);
        const int gridv = std::max(1, std::min((int)((c->nverts + kBT - 1) / kBT), c->num_sms * 8));
        k_lerp_bounds<<<gridv, kBT, 0, s>>>(c->lerp_pending ? c->keyframes.as<float4>() : nullptr,
                                            c->frame_sel.as<int4>(), c->verts.as<float4>(), c->nverts, d);
        k_grid_setup<<<1, 1, 0, s>>>(d, dens, (uint32_t)std::min(B.cap_cells, (size_t)0xffffffffu));
        mark();
        const float4* v = c->verts.as<float4>();
        const uint32_t* ix = c->idx.as<uint32_t>();
        uint32_t* bsum = B.block_sums.as<uint32_t>();
        uint32_t* d_np = kind == kUniform ? &d->npairs : &d->ntop_pairs;
        // two-level: the references per top cell are counted as the pairs are written
        uint32_t* cell_count = kind == kTwoLevel ? B.leaf_cnt.as<uint32_t>() : nullptr;
        if (nblocks > 0) {
            k_count_pairs<<<nblocks, kBT, 0, s>>>(v, ix, ntri, d, bsum, c->tris.as<float4>(), B.tri_ranges.as<uint4>(),
                                                  cell_count);
            if ((rc = scan_block_sums(c, bsum, nblocks, d_np, &d->overflow, (uint32_t)std::min(cap_pairs, (size_t)0xffffffffu),
                                      kind == kUniform ? kOvfPairs : kOvfTopPairs, &d->req_pairs, s)))
                return rc;
            if (kind == kUniform && exact)
                k_write_pairs<true><<<nblocks, kBT, 0, s>>>(c->tris.as<float4>(), ntri, d, bsum, nullptr,
                                                            B.keys_a.as<uint32_t>(), B.vals_a.as<uint32_t>(), nullptr);
            else
                k_write_pairs<false><<<nblocks, kBT, 0, s>>>(c->tris.as<float4>(), ntri, d, bsum, B.tri_ranges.as<uint4>(),
                                                             B.keys_a.as<uint32_t>(), B.vals_a.as<uint32_t>(), cell_count);
        }
        mark();
        const int gcells = std::max(1, std::min((int)((B.cap_cells + 255) / 256), c->num_sms * 16));
        if (kind == kUniform) {
            // a6-a7: pairs sorted by cell, cell ranges
            uint32_t* sorted_keys = (passes % 2 == 1) ? B.keys_b.as<uint32_t>() : B.keys_a.as<uint32_t>();
            if ((rc = radix_sort_pairs(c, B.keys_a.as<uint32_t>(), B.vals_a.as<uint32_t>(), B.keys_b.as<uint32_t>(),
                                       B.vals_b.as<uint32_t>(), sorted_keys, B.prims.as<uint32_t>(), d_np, cap_pairs,
                                       key_bits, B.tile_hist.as<uint32_t>(), B.tile_hist.bytes,
                                       B.row_total.as<uint32_t>(), s)))
                return rc;
            mark();
            k_fill_u2<<<gcells, 256, 0, s>>>(B.cells.as<uint2>(), &d->ncells, d, make_uint2(0u, 0u));
            const int gpairs = std::max(1, std::min((int)((cap_pairs + 255) / 256), c->num_sms * 16));
            k_cell_ranges<<<gpairs, 256, 0, s>>>(sorted_keys, d_np, &d->ncells, d, B.cells.as<uint2>());
            mark();
        } else {
            // Leaf level, TLGridSortBuilder.h:256-410: leaf cells per top cell, scan, leaf pairs
            // per top-level reference, stable sort by leaf, leaf ranges.  The reference sorts
            // the top-level pairs by cell first; here they stay in triangle order: the leaf
            // level needs only each top cell's reference count (counted as they were written),
            // and the one stable sort by global leaf index then orders every leaf's list by
            // triangle exactly as the two sorts would.
            k_tl_cells<<<gcells, 256, 0, s>>>(d, c->leaf_density, B.leaf_cnt.as<uint32_t>(), B.cells.as<uint2>(),
                                              B.occ.as<uint32_t>());
            uint32_t* sp = B.scan_partials.as<uint32_t>();
            if ((rc = exclusive_scan_u32(c, B.leaf_cnt.as<uint32_t>(), &d->ncells, B.cap_cells, &d->nleaves, sp, s)))
                return rc;
            k_check_leaves<<<1, 1, 0, s>>>(d, (uint32_t)std::min(B.cap_leaves, (size_t)0xffffffffu));
            k_tl_cell_begin<<<gcells, 256, 0, s>>>(B.leaf_cnt.as<uint32_t>(), d, B.cells.as<uint2>());
            mark();
            uint32_t* lsum = B.block_sums.as<uint32_t>();
            k_leaf_count_pairs<<<nref_blocks, kBT, 0, s>>>(B.keys_a.as<uint32_t>(), B.vals_a.as<uint32_t>(),
                                                           c->tris.as<float4>(), d, B.cells.as<uint2>(), lsum,
                                                           B.ref_ranges.as<uint4>());
            if ((rc = scan_block_sums(c, lsum, nref_blocks, &d->npairs, &d->overflow,
                                      (uint32_t)std::min(B.cap_leaf_pairs, (size_t)0xffffffffu), kOvfLeafPairs,
                                      &d->req_leaf_pairs, s)))
                return rc;
            k_leaf_write_pairs<<<nref_blocks, kBT, 0, s>>>(B.ref_ranges.as<uint4>(), d, lsum, B.lkeys_a.as<uint32_t>(),
                                                           B.lvals_a.as<uint32_t>());
            mark();
            uint32_t* leaf_keys = (leaf_passes % 2 == 1) ? B.lkeys_b.as<uint32_t>() : B.lkeys_a.as<uint32_t>();
            if ((rc = radix_sort_pairs(c, B.lkeys_a.as<uint32_t>(), B.lvals_a.as<uint32_t>(), B.lkeys_b.as<uint32_t>(),
                                       B.lvals_b.as<uint32_t>(), leaf_keys, B.prims.as<uint32_t>(), &d->npairs,
                                       B.cap_leaf_pairs, leaf_bits, B.tile_hist.as<uint32_t>(), B.tile_hist.bytes,
                                       B.row_total.as<uint32_t>(), s)))
                return rc;
            mark();
            const int gleaves = std::max(1, std::min((int)((B.cap_leaves + 255) / 256), c->num_sms * 16));
            k_fill_u2<<<gleaves, 256, 0, s>>>(B.leaves.as<uint2>(), &d->nleaves, d, make_uint2(0u, 0u));
            const int glp = std::max(1, std::min((int)((B.cap_leaf_pairs + 255) / 256), c->num_sms * 16));
            k_cell_ranges<<<glp, 256, 0, s>>>(leaf_keys, &d->npairs, &d->nleaves, d, B.leaves.as<uint2>());
            mark();
        }
        c->nstages = ev;
        return 0;
    };
    // A rebuild identical to the previous one (the same frame, sizes, buffers and
    // settings: a mesh rebuilt every frame) is captured once as a CUDA graph and then
    // replayed: one launch instead of about 35, so small builds are not paced by the host's
    // launch rate.  An animated mesh replays the same graph for every frame time: the frame
    // pair and weight go to frame_sel first, outside the graph.  Asynchronous builds (the
    // server's rebuilds) replay it too; a stream wait enqueued before the capture stays
    // outside the graph and orders its launch.
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
    bool enqueued = false, single = false;
    // a small uniform build: one cooperative launch instead of the pipeline (build_small.cu)
    if (kind == kUniform && wait && (rc = build_small_uniform(c, exact, key_bits, &single))) return rc;
    if (single) {
        enqueued = true;
        c->nstages = 0;
    }
    std::vector<uint8_t> key;
    if (!enqueued && HR_BUILD_GRAPH && c->build_graph_ok) key = build_graph_key(c, kind, exact, dens);
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
    if (single && (c->host_desc.error & kDescErrBarrier)) {
        // the single launch gave up at a barrier: the pipeline builds it, from now on too
        c->small_build_max_tris = 0;
        return build_once_impl(c, kind, exact, ovf_out, wait);
    }
    if (c->timing)
        for (int i = 0; i + 1 < c->nstages; ++i) cudaEventElapsedTime(&c->stage_ms[i], c->ev[i], c->ev[i + 1]);
    if (c->host_desc.error) return desc_error(c);
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
    if (c->host_desc.error) return desc_error(c);
    const uint32_t ovf = c->host_desc.overflow;
    if (ovf) {
        *fit = false;
        c->built = false;
        grow_caps(c, c->host_desc, ovf);
    }
    return 0;
}

}  // namespace hr
