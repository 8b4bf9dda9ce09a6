// batch.cu -- many independent scenes built and rendered together.
//
// The reference renders one scene held in static globals (src/RT/RTEngine.cu:91-181); a
// batch of scenes there means one full build + render per scene, each ~40 launches and a
// host round trip.  Here a batch of scenes of uneven size is
//   * built by ONE segmented two-level-grid pipeline: every kernel covers all scenes, so
//     the launch count is fixed whatever the number of scenes.  Scene s owns top cells
//     [cell_off[s], cell_off[s+1]) of one global cell array and its triangles are
//     [tri_off[s], tri_off[s] + ntri[s]) of one global triangle array; top-level pair keys
//     are cell_off[s] + the scene-local cell key, leaf keys are global leaf indices, so
//     one stable radix sort per level orders the references of all scenes at once.
//     Within a cell the order is by global triangle id = scene-local id + tri_off[s], so
//     every scene's grid equals the one the per-scene pipeline (build.cu) builds, shifted
//     by the scene's offsets;
//   * rendered by ONE persistent launch (k_trace_jobs): warps take 32-pixel tiles of any
//     scene from a global work counter, trace the camera rays and, for AO, the samples of
//     the tile's hit pixels from a ray queue kept in registers (no global queue, no
//     second launch); the per-pixel random streams are those of the per-scene kernels,
//     so images are bit-identical too;
//   * captured, build and render, in one CUDA graph that a step replays.
//
// Per-scene pipeline it segments: TLGridSortBuilder.h:66-452 with the kernels of
// TLGridBuildKernels.h:45-834 and UniformGridBuildKernels.h:40-252 (top level).
#include "build_dev.cuh"
#include "traverse.cuh"
#include "../../include/happyray.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

namespace hr {

// per-scene record of a batch (device copy written by the host)
struct BScene {
    uint32_t tri_off, ntri, vert_off, nverts;
    float top, leaf;
    uint32_t pad[2];
};

namespace {

// ---------------------------------------------------------------------------------
// segmented build.  Blocks of the per-triangle (per-vertex) passes never straddle two
// scenes: chunk b covers kBT triangles (vertices) of scene chunk[b].x from chunk[b].y.

// scene-local vertex indices -> global, with each scene's range check (the per-scene
// upload's index check); bad indices count into *bad and fail the build
__global__ __launch_bounds__(kBT) void kb_global_indices(uint32_t* __restrict__ idx, const uint2* __restrict__ tchunk,
                                                         const BScene* __restrict__ sc, uint32_t* bad) {
    const uint2 ch = tchunk[blockIdx.x];
    const BScene S = sc[ch.x];
    const uint32_t t = ch.y + threadIdx.x;
    uint32_t nbad = 0;
    if (t < S.tri_off + S.ntri) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            uint32_t v = idx[3 * (size_t)t + k];
            if (v >= S.nverts) { ++nbad; v = 0; }
            idx[3 * (size_t)t + k] = v + S.vert_off;
        }
    }
    if (nbad) atomicAdd(bad, nbad);
}

__global__ void kb_init(const BScene* __restrict__ sc, uint32_t nsc, GridDesc* descs, GridDesc* bd, uint32_t ntri,
                        const uint32_t* bad) {
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < nsc; s += gridDim.x * blockDim.x)
        desc_init(descs + s, kTwoLevel, sc[s].ntri, 0u);
    if (blockIdx.x == 0 && threadIdx.x == 0) desc_init(bd, kTwoLevel, ntri, *bad != 0u ? 1u : 0u);
}

// a1: scene bounds (no keyframe interpolation: batch scenes are static)
__global__ __launch_bounds__(kBT) void kb_bounds(const float4* __restrict__ v, const uint2* __restrict__ vchunk,
                                                 const BScene* __restrict__ sc, GridDesc* descs) {
    const uint2 ch = vchunk[blockIdx.x];
    const uint32_t end = sc[ch.x].vert_off + sc[ch.x].nverts;
    const uint32_t i = ch.y + threadIdx.x;
    f3 lo = mk(FLT_MAX, FLT_MAX, FLT_MAX), hi = mk(-FLT_MAX, -FLT_MAX, -FLT_MAX);
    if (i < end) {
        const float4 q = __ldg(v + i);
        const f3 p = mk(q.x, q.y, q.z);
        lo = vmin(p, lo);
        hi = vmax(p, hi);
    }
    reduce_bounds(lo, hi, descs + ch.x);
}

// a2 for every scene + exclusive scan of the scenes' cell counts -> cell_off.  A scene
// above kMaxSceneCells top cells sets error 2 (the sums stay in 32 bits).
constexpr uint32_t kMaxSceneCells = 1u << 22;
__global__ __launch_bounds__(1024) void kb_setup(const BScene* __restrict__ sc, uint32_t nsc, GridDesc* descs,
                                                 uint32_t* cell_off, GridDesc* bd, uint32_t cap_cells) {
    uint64_t carry = 0;
    bool big = false;
    for (uint32_t b = 0; b < nsc; b += 1024) {
        const uint32_t s = b + threadIdx.x;
        uint32_t nc = 0;
        if (s < nsc) {
            const uint64_t n64 = grid_setup(descs + s, sc[s].top);
            if (n64 > kMaxSceneCells) big = true;
            nc = n64 > kMaxSceneCells ? kMaxSceneCells : (uint32_t)n64;
            descs[s].ncells = nc;
        }
        uint32_t tot;
        const uint32_t ex = block_excl_scan<uint32_t, 1024>(nc, &tot);
        if (s < nsc) cell_off[s] = (uint32_t)(carry + ex);
        carry += tot;
    }
    if (big) atomicOr(&bd->error, 2u);
    if (threadIdx.x == 0) {
        cell_off[nsc] = (uint32_t)carry;
        if (carry >= (uint64_t)cap_cells) {
            bd->overflow |= kOvfCells;
            bd->req_cells = (uint32_t)carry;
            bd->ncells = 0u;
        } else {
            bd->ncells = (uint32_t)carry;
        }
    }
}

// a3 per scene chunk: pair count + the per-triangle vertex array; also clears the per-top-cell
// reference counts kb_write_pairs accumulates, and adds the chunk's pairs to its scene's
// top-level pair count
__global__ __launch_bounds__(kBT) void kb_count_pairs(const float4* __restrict__ v, const uint32_t* __restrict__ idx,
                                                      const uint2* __restrict__ tchunk, const BScene* __restrict__ sc,
                                                      GridDesc* __restrict__ descs, const GridDesc* bd,
                                                      uint32_t* block_sums, float4* __restrict__ tris,
                                                      uint4* __restrict__ rng, uint32_t* __restrict__ cell_count) {
    if (bd->overflow | bd->error) {
        if (threadIdx.x == 0) block_sums[blockIdx.x] = 0u;
        return;
    }
    for (uint32_t c = blockIdx.x * kBT + threadIdx.x; c < bd->ncells; c += gridDim.x * kBT) cell_count[c] = 0u;
    const uint2 ch = tchunk[blockIdx.x];
    const uint32_t end = sc[ch.x].tri_off + sc[ch.x].ntri;
    const DescRegs g = load_desc(descs + ch.x);
    const uint32_t t = ch.y + threadIdx.x;
    uint32_t n = 0;
    if (t < end) {
        f3 p[3], lo, hi;
        CRange r;
        tri_load(v, idx, t, p);
        float4* q = tris + 3 * (size_t)t;
        q[0] = make_float4(p[0].x, p[0].y, p[0].z, 0.0f);
        q[1] = make_float4(p[1].x, p[1].y, p[1].z, 0.0f);
        q[2] = make_float4(p[2].x, p[2].y, p[2].z, 0.0f);
        tri_bbox(p, &lo, &hi);
        n = cell_range(lo, hi, g.bmin, g.rcp, g.res, &r);
        if (ranges_fit(g.res)) rng[t] = pack_range(r, n);
    }
    uint32_t tot;
    block_excl_scan<uint32_t, kBT>(n, &tot);
    if (threadIdx.x == 0) {
        block_sums[blockIdx.x] = tot;
        if (tot) atomicAdd(&descs[ch.x].ntop_pairs, tot);
    }
}

// a5 per scene chunk: key = the scene's first top cell + local cell key, value = global
// triangle id
__global__ __launch_bounds__(kBT) void kb_write_pairs(const float4* __restrict__ tris, const uint2* __restrict__ tchunk,
                                                      const BScene* __restrict__ sc, const GridDesc* __restrict__ descs,
                                                      const uint32_t* __restrict__ cell_off, const GridDesc* bd,
                                                      const uint32_t* block_sums, const uint4* __restrict__ rng,
                                                      uint32_t* __restrict__ keys, uint32_t* __restrict__ vals,
                                                      uint32_t* __restrict__ cell_count) {
    if (bd->overflow | bd->error) return;
    const uint2 ch = tchunk[blockIdx.x];
    const uint32_t end = sc[ch.x].tri_off + sc[ch.x].ntri;
    const DescRegs g = load_desc(descs + ch.x);
    const uint32_t t = ch.y + threadIdx.x;
    uint32_t n = 0;
    CRange r;
    if (t < end) {
        if (ranges_fit(g.res)) {
            n = unpack_range(__ldg(rng + t), &r);   // the range kb_count_pairs found
        } else {
            f3 p[3], lo, hi;
            tri_fetch(tris, t, p);
            tri_bbox(p, &lo, &hi);
            n = cell_range(lo, hi, g.bmin, g.rcp, g.res, &r);
        }
    }
    const uint32_t base = __ldg(cell_off + ch.x);
    const uint32_t rx = (uint32_t)g.res[0], rxy = (uint32_t)g.res[0] * (uint32_t)g.res[1];
    PairRun run;
    if (n) run = {base + (uint32_t)r.lo[0] + (uint32_t)r.lo[1] * rx + (uint32_t)r.lo[2] * rxy,
                  (uint32_t)(r.hi[0] - r.lo[0]), (uint32_t)(r.hi[1] - r.lo[1]), rx, rxy, t};
    block_write_runs<kBT>(n, run, block_sums[blockIdx.x], keys, vals, cell_count);
}

// a8 per global top cell, with the cell's scene found by binary search; leaf_cnt holds the
// cell's reference count on entry and its leaf count on return
__global__ void kb_tl_cells(const BScene* __restrict__ sc,
                            const GridDesc* __restrict__ descs, const uint32_t* __restrict__ cell_off, uint32_t nsc,
                            const GridDesc* bd, uint32_t* __restrict__ leaf_cnt, uint2* __restrict__ top_cells,
                            uint32_t* __restrict__ occ) {
    if (bd->overflow | bd->error) return;
    const uint32_t C = bd->ncells;
    const uint32_t lane = threadIdx.x & 31u;
    // warp-uniform trip count: the 32 cells of a pass share one occupancy word (global cell bits)
    for (uint32_t c0 = blockIdx.x * blockDim.x + threadIdx.x - lane; c0 < C; c0 += gridDim.x * blockDim.x) {
        const uint32_t c = c0 + lane;
        bool full = false;
        if (c < C) {
            const uint32_t s = find_segment(cell_off, nsc, c);
            const DescRegs g = load_desc(descs + s);
            const uint32_t refs = leaf_cnt[c];
            const LeafGeom lg = leaf_geom(g, refs, sc[s].leaf);
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

// sub-cell range of top-level reference i inside its (scene-local) top cell
__device__ __forceinline__ uint32_t bref_leaf_range(const GridDesc* __restrict__ descs,
                                                    const uint32_t* __restrict__ cell_off, uint32_t nsc,
                                                    const uint32_t* __restrict__ top_keys,
                                                    const uint32_t* __restrict__ top_refs,
                                                    const float4* __restrict__ tris,
                                                    const uint2* __restrict__ top_cells, uint32_t i, uint32_t* cell,
                                                    uint32_t* tri, uint32_t* lres, CRange* r) {
    *cell = __ldg(top_keys + i);
    *tri = __ldg(top_refs + i);
    const uint32_t s = find_segment(cell_off, nsc, *cell);
    const DescRegs g = load_desc(descs + s);
    const uint32_t y = top_cells[*cell].y;
    lres[0] = y & 0xFFu; lres[1] = (y >> 8) & 0xFFu; lres[2] = (y >> 16) & 0xFFu;
    f3 p[3], lo, hi;
    tri_fetch(tris, *tri, p);
    tri_bbox(p, &lo, &hi);
    return leaf_range(g, lres, *cell - __ldg(cell_off + s), lo, hi, r);
}

// a10
__global__ __launch_bounds__(kBT) void kb_leaf_count_pairs(const uint32_t* __restrict__ top_keys,
                                                           const uint32_t* __restrict__ top_refs,
                                                           const float4* __restrict__ tris,
                                                           const GridDesc* __restrict__ descs,
                                                           const uint32_t* __restrict__ cell_off, uint32_t nsc,
                                                           const GridDesc* bd, const uint2* __restrict__ top_cells,
                                                           uint32_t* block_sums, uint4* __restrict__ refrng) {
    if (bd->overflow | bd->error) {
        if (threadIdx.x == 0) block_sums[blockIdx.x] = 0u;
        return;
    }
    const uint32_t i = blockIdx.x * kBT + threadIdx.x;
    uint32_t n = 0;
    if (i < bd->ntop_pairs) {
        uint32_t cell, tri, lres[3];
        CRange r;
        n = bref_leaf_range(descs, cell_off, nsc, top_keys, top_refs, tris, top_cells, i, &cell, &tri, lres, &r);
        refrng[i] = pack_ref(r, lres, top_cells[cell].x, tri);
    }
    uint32_t tot;
    block_excl_scan<uint32_t, kBT>(n, &tot);
    if (threadIdx.x == 0) block_sums[blockIdx.x] = tot;
}

// a11: key = first (global) leaf of the top cell + local sub-cell index, from the packed
// sub-cell range kb_leaf_count_pairs kept for every reference
__global__ __launch_bounds__(kBT) void kb_leaf_write_pairs(const uint4* __restrict__ refrng, const GridDesc* bd,
                                                           const uint32_t* block_sums, uint32_t* __restrict__ keys,
                                                           uint32_t* __restrict__ vals) {
    if (bd->overflow | bd->error) return;
    const uint32_t i = blockIdx.x * kBT + threadIdx.x;
    uint32_t n = 0;
    PairRun run;
    if (i < bd->ntop_pairs) {
        const uint4 q = __ldg(refrng + i);
        int32_t lo[3], e[3];
        n = 1;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            lo[k] = (int32_t)((q.x >> (8 * k)) & 0xFFu);
            e[k] = (int32_t)((q.y >> (8 * k)) & 0xFFu) - lo[k];
            n *= (uint32_t)(e[k] > 0 ? e[k] : 0);
        }
        const uint32_t l0 = q.x >> 24, l1 = q.y >> 24;
        if (n) run = {q.z + (uint32_t)lo[0] + (uint32_t)lo[1] * l0 + (uint32_t)lo[2] * l0 * l1, (uint32_t)e[0],
                      (uint32_t)e[1], l0, l0 * l1, q.w};
    }
    block_write_runs<kBT>(n, run, block_sums[blockIdx.x], keys, vals);
}

template <class T>
T* dev(const DevBuf& b) { return b.as<T>(); }

}  // namespace
}  // namespace hr

using namespace hr;

struct hr_batch {
    hr_ctx* c = nullptr;   // stream, device, error text, launch count, grid buffers
    uint32_t nsc = 0, ntri = 0, nverts = 0, ntchunk = 0, nvchunk = 0;
    uint64_t npix = 0;
    std::vector<BScene> sc;
    std::vector<Camera> cams;
    std::vector<int32_t> spp;
    std::vector<uint64_t> px_off;
    DevBuf d_sc, d_descs, d_bdesc, d_cell_off, d_tchunk, d_vchunk, d_jobs, d_tile_off, d_work, d_fb, d_bad;
    GridDesc* h_bdesc = nullptr;   // pinned: batch totals of the last step
    Job* h_jobs = nullptr;         // pinned job table
    size_t h_jobs_cap = 0;
    int32_t block_threads = 256, tile_w = 8;
    float alpha_frac = 0.1f;
    uint64_t seed = 0x853c49e6748fea9bULL;
    int32_t image_id = -1;         // image id baked into the uploaded job table
    bool use_graph = true;
    bool planned = false;          // capacities fit the current scenes / densities
    bool jobs_valid = false;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint64_t graph_launches = 0;
    cudaEvent_t ev[4] = {};
    float t_build = -1.0f, t_render = -1.0f, t_total = -1.0f;
    int persist_blocks = 0;
    uint32_t ntiles = 0;
    uint64_t secondary_rays = 0;
};

namespace hr {
namespace {

int berr(hr_batch* b, int code, const char* msg) { return set_error(b->c, code, "%s", msg); }

void drop_graph(hr_batch* b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
}

// allocations for the current capacities (never inside a capture)
int batch_alloc(hr_batch* b) {
    hr_ctx* c = b->c;
    GridBuffers& B = c->g;
    const size_t cap_pairs = B.cap_pairs;
    const int leaf_bits = std::max(1, (int)std::ceil(std::log2((double)B.cap_leaves + 1.0)));
    size_t hist = radix_tile_hist_words(B.cap_leaf_pairs, leaf_bits);
    const size_t nref_blocks = (cap_pairs + kBT - 1) / kBT;
    int rc;
    if ((rc = ensure(c, B.cells, sizeof(uint2) * B.cap_cells))) return rc;
    if ((rc = ensure(c, B.leaf_cnt, sizeof(uint32_t) * B.cap_cells))) return rc;
    if ((rc = ensure(c, B.occ, sizeof(uint32_t) * (B.cap_cells / 32 + 1)))) return rc;
    if ((rc = ensure(c, B.scan_partials, sizeof(uint32_t) * (scan_partials_words(B.cap_cells) + 2)))) return rc;
    if ((rc = ensure(c, B.keys_a, sizeof(uint32_t) * cap_pairs))) return rc;
    if ((rc = ensure(c, B.vals_a, sizeof(uint32_t) * cap_pairs))) return rc;
    if ((rc = ensure(c, B.ref_ranges, sizeof(uint4) * cap_pairs))) return rc;
    if ((rc = ensure(c, B.tri_ranges, sizeof(uint4) * std::max<size_t>(b->ntri, 1)))) return rc;
    if ((rc = ensure(c, B.block_sums, sizeof(uint32_t) * (std::max((size_t)b->ntchunk, nref_blocks) + 1)))) return rc;
    if ((rc = ensure(c, B.tile_hist, sizeof(uint32_t) * hist))) return rc;
    if ((rc = ensure(c, B.row_total, sizeof(uint32_t) * kRadixRowWords))) return rc;
    if ((rc = ensure(c, B.leaves, sizeof(uint2) * B.cap_leaves))) return rc;
    if ((rc = ensure(c, B.lkeys_a, sizeof(uint32_t) * B.cap_leaf_pairs))) return rc;
    if ((rc = ensure(c, B.lvals_a, sizeof(uint32_t) * B.cap_leaf_pairs))) return rc;
    if ((rc = ensure(c, B.lkeys_b, sizeof(uint32_t) * B.cap_leaf_pairs))) return rc;
    if ((rc = ensure(c, B.lvals_b, sizeof(uint32_t) * B.cap_leaf_pairs))) return rc;
    if ((rc = ensure(c, B.prims, sizeof(uint32_t) * B.cap_leaf_pairs))) return rc;
    return 0;
}

// Enqueue the whole segmented build on the batch stream (no allocation, no host sync).
int enqueue_build(hr_batch* b) {
    hr_ctx* c = b->c;
    cudaStream_t s = c->stream;
    GridBuffers& B = c->g;
    const size_t cap_pairs = B.cap_pairs;
    const int leaf_bits = std::max(1, (int)std::ceil(std::log2((double)B.cap_leaves + 1.0)));
    const uint32_t nref_blocks = (uint32_t)((cap_pairs + kBT - 1) / kBT);
    GridDesc* descs = dev<GridDesc>(b->d_descs);
    GridDesc* bd = dev<GridDesc>(b->d_bdesc);
    const BScene* sc = dev<BScene>(b->d_sc);
    uint32_t* cell_off = dev<uint32_t>(b->d_cell_off);
    const uint2* tch = dev<uint2>(b->d_tchunk);
    float4* tris = c->tris.as<float4>();
    uint32_t* bsum = B.block_sums.as<uint32_t>();
    int rc;
    c->launches += 14;   // this function's kernels, both block-sum scans included
    kb_init<<<(b->nsc + 255) / 256, 256, 0, s>>>(sc, b->nsc, descs, bd, b->ntri, dev<uint32_t>(b->d_bad));
    kb_bounds<<<b->nvchunk, kBT, 0, s>>>(c->verts.as<float4>(), dev<uint2>(b->d_vchunk), sc, descs);
    kb_setup<<<1, 1024, 0, s>>>(sc, b->nsc, descs, cell_off, bd, (uint32_t)std::min(B.cap_cells, (size_t)0xffffffffu));
    // the top-level pairs stay in triangle order (as the per-scene build: the leaf level needs
    // only each top cell's reference count, counted as they are written)
    kb_count_pairs<<<b->ntchunk, kBT, 0, s>>>(c->verts.as<float4>(), c->idx.as<uint32_t>(), tch, sc, descs, bd, bsum, tris,
                                              B.tri_ranges.as<uint4>(), B.leaf_cnt.as<uint32_t>());
    if ((rc = scan_block_sums(c, bsum, b->ntchunk, &bd->ntop_pairs, &bd->overflow,
                              (uint32_t)std::min(cap_pairs, (size_t)0xffffffffu), kOvfTopPairs, &bd->req_pairs, s)))
        return rc;
    kb_write_pairs<<<b->ntchunk, kBT, 0, s>>>(tris, tch, sc, descs, cell_off, bd, bsum, B.tri_ranges.as<uint4>(),
                                              B.keys_a.as<uint32_t>(), B.vals_a.as<uint32_t>(), B.leaf_cnt.as<uint32_t>());
    const int gcells = std::max(1, std::min((int)((B.cap_cells + 255) / 256), c->num_sms * 16));
    kb_tl_cells<<<gcells, 256, 0, s>>>(sc, descs, cell_off, b->nsc, bd, B.leaf_cnt.as<uint32_t>(), B.cells.as<uint2>(),
                                       B.occ.as<uint32_t>());
    if ((rc = exclusive_scan_u32(c, B.leaf_cnt.as<uint32_t>(), &bd->ncells, B.cap_cells, &bd->nleaves,
                                 B.scan_partials.as<uint32_t>(), s)))
        return rc;
    k_check_leaves<<<1, 1, 0, s>>>(bd, (uint32_t)std::min(B.cap_leaves, (size_t)0xffffffffu));
    k_tl_cell_begin<<<gcells, 256, 0, s>>>(B.leaf_cnt.as<uint32_t>(), bd, B.cells.as<uint2>());
    kb_leaf_count_pairs<<<nref_blocks, kBT, 0, s>>>(B.keys_a.as<uint32_t>(), B.vals_a.as<uint32_t>(), tris, descs, cell_off,
                                                    b->nsc, bd, B.cells.as<uint2>(), bsum, B.ref_ranges.as<uint4>());
    if ((rc = scan_block_sums(c, bsum, nref_blocks, &bd->npairs, &bd->overflow,
                              (uint32_t)std::min(B.cap_leaf_pairs, (size_t)0xffffffffu), kOvfLeafPairs,
                              &bd->req_leaf_pairs, s)))
        return rc;
    kb_leaf_write_pairs<<<nref_blocks, kBT, 0, s>>>(B.ref_ranges.as<uint4>(), bd, bsum, B.lkeys_a.as<uint32_t>(),
                                                    B.lvals_a.as<uint32_t>());
    const int lpasses = radix_sort_passes(leaf_bits);
    uint32_t* leaf_keys = (lpasses % 2 == 1) ? B.lkeys_b.as<uint32_t>() : B.lkeys_a.as<uint32_t>();
    if ((rc = radix_sort_pairs(c, B.lkeys_a.as<uint32_t>(), B.lvals_a.as<uint32_t>(), B.lkeys_b.as<uint32_t>(),
                               B.lvals_b.as<uint32_t>(), leaf_keys, B.prims.as<uint32_t>(), &bd->npairs,
                               B.cap_leaf_pairs, leaf_bits, B.tile_hist.as<uint32_t>(), B.tile_hist.bytes, B.row_total.as<uint32_t>(),
                               s)))
        return rc;
    const int gleaves = std::max(1, std::min((int)((B.cap_leaves + 255) / 256), c->num_sms * 16));
    k_fill_u2<<<gleaves, 256, 0, s>>>(B.leaves.as<uint2>(), &bd->nleaves, bd, make_uint2(0u, 0u));
    const int glp = std::max(1, std::min((int)((B.cap_leaf_pairs + 255) / 256), c->num_sms * 16));
    k_cell_ranges<<<glp, 256, 0, s>>>(leaf_keys, &bd->npairs, &bd->nleaves, bd, B.leaves.as<uint2>());
    return cuda_check(c, cudaGetLastError(), "batch build launch");
}

// job table for the current scenes and image id (pinned host copy -> device)
int upload_jobs(hr_batch* b, int32_t image_id) {
    hr_ctx* c = b->c;
    if (b->h_jobs_cap < b->nsc) {
        if (b->h_jobs) cudaFreeHost(b->h_jobs);
        b->h_jobs = nullptr;
        b->h_jobs_cap = 0;
        if (cudaMallocHost((void**)&b->h_jobs, sizeof(Job) * b->nsc) != cudaSuccess) {
            cudaGetLastError();
            return berr(b, HR_ERR_OUT_OF_MEMORY, "batch: pinned job table allocation failed");
        }
        b->h_jobs_cap = b->nsc;
    }
    int rc;
    if ((rc = cuda_check(c, cudaStreamSynchronize(c->stream), "batch job table"))) return rc;   // previous copy done
    for (uint32_t i = 0; i < b->nsc; ++i) {
        Job& J = b->h_jobs[i];
        std::memset(&J, 0, sizeof(Job));
        J.tris = c->tris.as<float4>();
        J.cells = c->g.cells.as<uint2>();
        J.leaves = c->g.leaves.as<uint2>();
        J.prims = c->g.prims.as<uint32_t>();
        J.desc = dev<GridDesc>(b->d_descs) + i;
        J.cells_offset = dev<uint32_t>(b->d_cell_off) + i;
        J.occ = c->g.occ.as<uint32_t>();
        J.status = dev<GridDesc>(b->d_bdesc);   // overflow and error bits of the whole batch build
        J.fb = dev<float>(b->d_fb) + 3 * b->px_off[i];
        const Camera& k = b->cams[i];
        for (int q = 0; q < 3; ++q) {
            J.cam_pos[q] = k.pos[q]; J.cam_tl[q] = k.top_left[q]; J.cam_sx[q] = k.step_x[q]; J.cam_sy[q] = k.step_y[q];
        }
        J.w = k.w;
        J.h = k.h;
        J.ntri = b->sc[i].ntri;
        J.kind = kTwoLevel;
        J.mode = b->spp[i] > 0 ? kJobAO : kJobPrimary;
        J.spp = b->spp[i];
        J.image_id = image_id;
        J.alpha_frac = b->alpha_frac;
        J.alpha_abs = 0.0f;
        J.seed = b->seed;
    }
    if ((rc = cuda_check(c, cudaMemcpyAsync(b->d_jobs.p, b->h_jobs, sizeof(Job) * b->nsc, cudaMemcpyHostToDevice,
                                            c->stream), "batch job upload")))
        return rc;
    b->image_id = image_id;
    return 0;
}

// tiles per job for the current tile shape
int upload_tiles(hr_batch* b) {
    hr_ctx* c = b->c;
    std::vector<uint32_t> off(b->nsc + 1, 0u);
    for (uint32_t i = 0; i < b->nsc; ++i) {
        Job j{};
        j.mode = kJobAO;
        j.w = b->cams[i].w;
        j.h = b->cams[i].h;
        off[i + 1] = off[i] + job_tiles(j, b->tile_w);
    }
    b->ntiles = off[b->nsc];
    int rc;
    if ((rc = ensure(c, b->d_tile_off, sizeof(uint32_t) * (b->nsc + 1)))) return rc;
    if ((rc = cuda_check(c, cudaMemcpyAsync(b->d_tile_off.p, off.data(), sizeof(uint32_t) * (b->nsc + 1),
                                            cudaMemcpyHostToDevice, c->stream), "batch tiles")))
        return rc;
    b->persist_blocks = job_blocks_per_sm(b->block_threads, false) * c->num_sms;
    return cuda_check(c, cudaStreamSynchronize(c->stream), "batch tiles");
}

int enqueue_render(hr_batch* b) {
    hr_ctx* c = b->c;
    cudaStream_t s = c->stream;
    int rc;
    if ((rc = cuda_check(c, cudaMemsetAsync(b->d_work.p, 0, sizeof(uint32_t), s), "batch work reset"))) return rc;
    return launch_jobs(c, dev<Job>(b->d_jobs), dev<uint32_t>(b->d_tile_off), b->nsc, dev<uint32_t>(b->d_work),
                       b->tile_w, b->block_threads, b->persist_blocks, false, s);
}

// one step's work on the stream: build, render, totals to pinned host memory
int enqueue_step(hr_batch* b, bool capturing) {
    hr_ctx* c = b->c;
    cudaStream_t s = c->stream;
    int rc;
    // inside a capture an event must be an external record node to be recorded on replay
    auto mark = [&](cudaEvent_t e) {
        if (capturing) cudaEventRecordWithFlags(e, s, cudaEventRecordExternal);
        else cudaEventRecord(e, s);
    };
    mark(b->ev[0]);
    if ((rc = enqueue_build(b))) return rc;
    mark(b->ev[1]);
    if ((rc = enqueue_render(b))) return rc;
    mark(b->ev[2]);
    return cuda_check(c, cudaMemcpyAsync(b->h_bdesc, b->d_bdesc.p, sizeof(GridDesc), cudaMemcpyDeviceToHost, s),
                      "batch totals");
}

// Size every buffer by running the build eagerly until nothing overflows, then capture.
int plan(hr_batch* b) {
    hr_ctx* c = b->c;
    GridBuffers& B = c->g;
    drop_graph(b);
    b->planned = false;
    if (B.cap_cells == 0) {
        double cells = 32768.0;
        for (const BScene& S : b->sc) cells += std::floor((double)S.top * (double)S.ntri * 1.01) + 64.0;
        B.cap_cells = (size_t)cells;
        B.cap_pairs = (size_t)b->ntri * 3u + 4096u;
        B.cap_leaf_pairs = (size_t)b->ntri * 4u + 4096u;
        double leaves = (double)B.cap_cells;
        for (const BScene& S : b->sc) leaves += 2.0 * (double)S.leaf * (3.0 * S.ntri + 16.0);
        B.cap_leaves = (size_t)leaves;
    }
    int rc;
    for (int attempt = 0; attempt < 8; ++attempt) {
        if ((rc = batch_alloc(b))) return rc;
        if ((rc = enqueue_build(b))) return rc;
        if ((rc = cuda_check(c, cudaMemcpyAsync(b->h_bdesc, b->d_bdesc.p, sizeof(GridDesc), cudaMemcpyDeviceToHost,
                                                c->stream), "batch totals")))
            return rc;
        if ((rc = cuda_check(c, cudaStreamSynchronize(c->stream), "batch plan"))) return rc;
        const GridDesc hd = *b->h_bdesc;
        if (hd.error & 1u) return berr(b, HR_ERR_INVALID_ARG, "batch: a triangle index is out of range of its scene");
        if (hd.error & 2u) return berr(b, HR_ERR_INVALID_ARG, "batch: a scene's top-level grid exceeds 4M cells");
        const uint32_t ovf = hd.overflow;
        if (ovf == 0) {
            // capacities (which size the per-reference passes, radix tiles and scans) follow
            // the planned sizes plus 15% instead of the first estimates
            auto fit = [](size_t& cap, size_t need) {
                const size_t want = need + need / 7 + 4096;
                if (cap > want + want / 2) cap = want;
            };
            fit(B.cap_pairs, hd.ntop_pairs);
            fit(B.cap_leaf_pairs, hd.npairs);
            fit(B.cap_leaves, hd.nleaves);
            b->planned = true;
            break;
        }
        if (ovf & kOvfCells) B.cap_cells = (size_t)(hd.req_cells * 1.125) + 64u;
        if (ovf & kOvfTopPairs) B.cap_pairs = (size_t)(hd.req_pairs * 1.125) + 4096u;
        if (ovf & kOvfLeaves) B.cap_leaves = (size_t)(hd.nleaves * 1.125) + 4096u;
        if (ovf & kOvfLeafPairs) B.cap_leaf_pairs = (size_t)(hd.req_leaf_pairs * 1.125) + 4096u;
    }
    if (!b->planned) return berr(b, HR_ERR_CAPACITY_RETRY, "batch: grid capacities did not converge");
    // the fitted capacities can need a LARGER radix histogram than the ones allocated
    // above: fewer key bits may mean fewer passes of wider digits (19 bits: 3 passes of
    // 7-bit digits; 18 bits: 2 passes of 9-bit digits, 4x the words per tile)
    if ((rc = batch_alloc(b))) return rc;
    b->jobs_valid = false;   // grid buffers may have moved
    if (!b->use_graph) return 0;
    const uint64_t l0 = c->launches;
    if ((rc = cuda_check(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal), "capture begin")))
        return rc;
    rc = enqueue_step(b, true);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    if (rc) { if (g) cudaGraphDestroy(g); return rc; }
    if ((rc = cuda_check(c, e, "capture end"))) return rc;
    b->graph = g;
    if ((rc = cuda_check(c, cudaGraphInstantiate(&b->exec, g, 0), "graph instantiate"))) { drop_graph(b); return rc; }
    b->graph_launches = c->launches - l0;
    c->launches = l0;
    return 0;
}

int run_step(hr_batch* b, int32_t image_id) {
    hr_ctx* c = b->c;
    int rc;
    for (int attempt = 0; attempt < 3; ++attempt) {
        if (!b->planned && (rc = plan(b))) return rc;
        if (!b->jobs_valid || b->image_id != image_id) {
            if ((rc = upload_jobs(b, image_id))) return rc;
            b->jobs_valid = true;
        }
        if (b->use_graph) {
            if ((rc = cuda_check(c, cudaGraphLaunch(b->exec, c->stream), "graph launch"))) return rc;
            c->launches += b->graph_launches;
        } else if ((rc = enqueue_step(b, false))) {
            return rc;
        }
        cudaEventRecord(b->ev[3], c->stream);
        if ((rc = cuda_check(c, cudaStreamSynchronize(c->stream), "batch step"))) return rc;
        const GridDesc hd = *b->h_bdesc;
        if (hd.error) return berr(b, HR_ERR_INVALID_ARG, "batch: invalid scene data");
        if (hd.overflow == 0) {
            float ms;
            b->t_build = cudaEventElapsedTime(&ms, b->ev[0], b->ev[1]) == cudaSuccess ? ms : -1.0f;
            b->t_render = cudaEventElapsedTime(&ms, b->ev[1], b->ev[2]) == cudaSuccess ? ms : -1.0f;
            b->t_total = cudaEventElapsedTime(&ms, b->ev[0], b->ev[3]) == cudaSuccess ? ms : -1.0f;
            cudaGetLastError();
            return 0;
        }
        b->planned = false;   // sizes changed under the plan: replan and redo the step
    }
    return berr(b, HR_ERR_CAPACITY_RETRY, "batch: step did not fit its plan");
}

bool valid_batch(const hr_batch* b) { return b && b->c; }

}  // namespace
}  // namespace hr

extern "C" {

hr_status hr_batch_create(hr_batch** out, int32_t device, void* stream) {
    if (!out) return HR_ERR_INVALID_ARG;
    *out = nullptr;
    hr_batch* b = new (std::nothrow) hr_batch();
    if (!b) return HR_ERR_OUT_OF_MEMORY;
    hr_status st = hr_create(&b->c, device, stream);
    if (st != HR_OK) { delete b; return st; }
    DeviceGuard dg(b->c->device);
    for (auto& e : b->ev) cudaEventCreate(&e);
    if (cudaMallocHost((void**)&b->h_bdesc, sizeof(GridDesc)) != cudaSuccess) {
        cudaGetLastError();
        hr_batch_destroy(b);
        return HR_ERR_OUT_OF_MEMORY;
    }
    std::memset(b->h_bdesc, 0, sizeof(GridDesc));
    int rc;
    if ((rc = ensure(b->c, b->d_work, 16)) || (rc = ensure(b->c, b->d_bad, 16)) ||
        (rc = ensure(b->c, b->d_bdesc, sizeof(GridDesc)))) {
        hr_batch_destroy(b);
        return (hr_status)rc;
    }
    *out = b;
    return HR_OK;
}

void hr_batch_destroy(hr_batch* b) {
    if (!b) return;
    if (b->c) {
        DeviceGuard dg(b->c->device);
        cudaStreamSynchronize(b->c->stream);
        drop_graph(b);
        DevBuf* bufs[] = {&b->d_sc, &b->d_descs, &b->d_bdesc, &b->d_cell_off, &b->d_tchunk, &b->d_vchunk,
                          &b->d_jobs, &b->d_tile_off, &b->d_work, &b->d_fb, &b->d_bad};
        for (DevBuf* d : bufs)
            if (d->p) cudaFreeAsync(d->p, b->c->stream);
        for (auto& e : b->ev) if (e) cudaEventDestroy(e);
        if (b->h_bdesc) cudaFreeHost(b->h_bdesc);
        if (b->h_jobs) cudaFreeHost(b->h_jobs);
        hr_destroy(b->c);
    }
    delete b;
}

const char* hr_batch_last_error(const hr_batch* b) { return b && b->c ? b->c->err.c_str() : "null batch"; }

hr_status hr_batch_set_scenes(hr_batch* b, const hr_batch_scene* scenes, uint32_t n) {
    if (!valid_batch(b) || (n && !scenes)) return HR_ERR_INVALID_ARG;
    hr_ctx* c = b->c;
    DeviceGuard dg(c->device);
    uint64_t ntri = 0, nverts = 0, npix = 0;
    for (uint32_t i = 0; i < n; ++i) {
        const hr_batch_scene& S = scenes[i];
        if (!S.vertices_xyz || !S.indices || S.num_triangles == 0 || S.num_vertices == 0)
            return (hr_status)set_error(c, HR_ERR_INVALID_ARG, "batch: scene %u has no mesh", i);
        if (S.width <= 0 || S.height <= 0 || !(S.cam_fov_deg > 0.0f && S.cam_fov_deg < 180.0f) || S.ao_samples < 0)
            return (hr_status)set_error(c, HR_ERR_INVALID_ARG, "batch: scene %u has an invalid camera or sample count", i);
        ntri += S.num_triangles;
        nverts += S.num_vertices;
        npix += (uint64_t)S.width * (uint64_t)S.height;
    }
    if (ntri > 0x7fffffffull || nverts > 0x7fffffffull)
        return (hr_status)set_error(c, HR_ERR_INVALID_ARG, "batch: more than 2^31 triangles or vertices");
    cudaStreamSynchronize(c->stream);
    drop_graph(b);
    b->planned = false;
    b->jobs_valid = false;
    b->nsc = n;
    b->ntri = (uint32_t)ntri;
    b->nverts = (uint32_t)nverts;
    b->npix = npix;
    b->sc.assign(n, BScene{});
    b->cams.assign(n, Camera{});
    b->spp.assign(n, 0);
    b->px_off.assign(n, 0);
    std::vector<uint2> tch, vch;
    uint32_t to = 0, vo = 0;
    uint64_t po = 0;
    for (uint32_t i = 0; i < n; ++i) {
        const hr_batch_scene& S = scenes[i];
        BScene& R = b->sc[i];
        R.tri_off = to; R.ntri = S.num_triangles; R.vert_off = vo; R.nverts = S.num_vertices;
        R.top = S.top_density > 0.0f ? S.top_density : 0.0625f;
        R.leaf = S.leaf_density > 0.0f ? S.leaf_density : 2.0f;
        for (uint32_t t = 0; t < S.num_triangles; t += kBT) tch.push_back(make_uint2(i, to + t));
        for (uint32_t v = 0; v < S.num_vertices; v += kBT) vch.push_back(make_uint2(i, vo + v));
        camera_init(&b->cams[i], S.cam_position, S.cam_orientation, S.cam_up, S.cam_fov_deg, S.width, S.height);
        b->spp[i] = S.ao_samples;
        b->px_off[i] = po;
        to += S.num_triangles;
        vo += S.num_vertices;
        po += (uint64_t)S.width * (uint64_t)S.height;
    }
    b->ntchunk = (uint32_t)tch.size();
    b->nvchunk = (uint32_t)vch.size();
    // the grid capacities are re-derived by the next plan
    c->g.cap_cells = c->g.cap_pairs = c->g.cap_leaf_pairs = c->g.cap_leaves = 0;
    int rc;
    if ((rc = ensure(c, b->d_sc, sizeof(BScene) * std::max(n, 1u))) ||
        (rc = ensure(c, b->d_descs, sizeof(GridDesc) * std::max(n, 1u))) ||
        (rc = ensure(c, b->d_cell_off, sizeof(uint32_t) * (n + 1))) ||
        (rc = ensure(c, b->d_tchunk, sizeof(uint2) * std::max<size_t>(tch.size(), 1))) ||
        (rc = ensure(c, b->d_vchunk, sizeof(uint2) * std::max<size_t>(vch.size(), 1))) ||
        (rc = ensure(c, c->verts, sizeof(float4) * std::max<uint64_t>(nverts, 1))) ||
        (rc = ensure(c, c->staging, sizeof(float) * 3 * std::max<uint64_t>(nverts, 1))) ||
        (rc = ensure(c, c->idx, sizeof(uint32_t) * 3 * std::max<uint64_t>(ntri, 1))) ||
        (rc = ensure(c, c->tris, sizeof(float4) * 3 * std::max<uint64_t>(ntri, 1))) ||
        (rc = ensure(c, b->d_fb, sizeof(float) * 3 * std::max<uint64_t>(npix, 1))) ||
        (rc = ensure(c, b->d_jobs, sizeof(Job) * std::max(n, 1u))))
        return (hr_status)rc;
    cudaStream_t s = c->stream;
    for (uint32_t i = 0; i < n; ++i) {
        const hr_batch_scene& S = scenes[i];
        const BScene& R = b->sc[i];
        if ((rc = cuda_check(c, cudaMemcpyAsync(c->staging.as<float>() + 3 * (size_t)R.vert_off, S.vertices_xyz,
                                                sizeof(float) * 3 * (size_t)R.nverts, cudaMemcpyHostToDevice, s),
                             "batch vertices")) ||
            (rc = cuda_check(c, cudaMemcpyAsync(c->idx.as<uint32_t>() + 3 * (size_t)R.tri_off, S.indices,
                                                sizeof(uint32_t) * 3 * (size_t)R.ntri, cudaMemcpyHostToDevice, s),
                             "batch indices")))
            return (hr_status)rc;
    }
    if ((rc = cuda_check(c, cudaMemcpyAsync(b->d_sc.p, b->sc.data(), sizeof(BScene) * n, cudaMemcpyHostToDevice, s),
                         "batch scenes")) ||
        (rc = cuda_check(c, cudaMemcpyAsync(b->d_tchunk.p, tch.data(), sizeof(uint2) * tch.size(), cudaMemcpyHostToDevice, s),
                         "batch chunks")) ||
        (rc = cuda_check(c, cudaMemcpyAsync(b->d_vchunk.p, vch.data(), sizeof(uint2) * vch.size(), cudaMemcpyHostToDevice, s),
                         "batch chunks")) ||
        (rc = cuda_check(c, cudaMemsetAsync(b->d_bad.p, 0, sizeof(uint32_t), s), "batch index check")) ||
        (rc = cuda_check(c, cudaMemsetAsync(b->d_fb.p, 0, sizeof(float) * 3 * npix, s), "batch framebuffer")))
        return (hr_status)rc;
    if (nverts) {
        const size_t nv = nverts;
        const int grid = (int)std::min<size_t>((nv + 255) / 256, (size_t)c->num_sms * 16);
        expand_xyz(c->staging.as<float>(), c->verts.as<float4>(), nv, grid, s);
    }
    if (b->ntchunk) {
        kb_global_indices<<<b->ntchunk, kBT, 0, s>>>(c->idx.as<uint32_t>(), dev<uint2>(b->d_tchunk), dev<BScene>(b->d_sc),
                                                     dev<uint32_t>(b->d_bad));
        c->launches += 2;
    }
    if ((rc = cuda_check(c, cudaGetLastError(), "batch upload"))) return (hr_status)rc;
    if ((rc = upload_tiles(b))) return (hr_status)rc;
    return HR_OK;
}

hr_status hr_batch_set_vertices(hr_batch* b, const float* xyz, uint32_t nv) {
    if (!valid_batch(b) || (nv && !xyz)) return HR_ERR_INVALID_ARG;
    hr_ctx* c = b->c;
    if (nv != b->nverts)
        return (hr_status)set_error(c, HR_ERR_INVALID_ARG, "batch: %u vertices given, the batch has %u", nv, b->nverts);
    if (nv == 0) return HR_OK;
    DeviceGuard dg(c->device);
    int rc = cuda_check(c, cudaMemcpyAsync(c->staging.p, xyz, sizeof(float) * 3 * (size_t)nv, cudaMemcpyHostToDevice,
                                           c->stream), "batch vertices");
    if (rc) return (hr_status)rc;
    const int grid = (int)std::min<size_t>(((size_t)nv + 255) / 256, (size_t)c->num_sms * 16);
    expand_xyz(c->staging.as<float>(), c->verts.as<float4>(), nv, grid, c->stream);
    c->launches += 1;
    return (hr_status)cuda_check(c, cudaGetLastError(), "batch vertices");
}

hr_status hr_batch_download_images(hr_batch* b, float* rgb, uint64_t nfloats) {
    if (!valid_batch(b) || !rgb) return HR_ERR_INVALID_ARG;
    hr_ctx* c = b->c;
    if (nfloats != 3 * b->npix)
        return (hr_status)set_error(c, HR_ERR_INVALID_ARG, "batch: %llu floats given, the images hold %llu",
                                    (unsigned long long)nfloats, (unsigned long long)(3 * b->npix));
    DeviceGuard dg(c->device);
    int rc = cuda_check(c, cudaMemcpyAsync(rgb, b->d_fb.p, sizeof(float) * nfloats, cudaMemcpyDeviceToHost, c->stream),
                        "batch images");
    if (!rc) rc = cuda_check(c, cudaStreamSynchronize(c->stream), "batch images");
    return (hr_status)rc;
}

hr_status hr_batch_set_densities(hr_batch* b, uint32_t scene, float top, float leaf) {
    if (!valid_batch(b) || !(top > 0.0f) || !(leaf > 0.0f)) return HR_ERR_INVALID_ARG;
    if (scene != 0xffffffffu && scene >= b->nsc)
        return (hr_status)set_error(b->c, HR_ERR_INVALID_ARG, "batch: scene %u out of range", scene);
    for (uint32_t i = 0; i < b->nsc; ++i)
        if (scene == 0xffffffffu || scene == i) { b->sc[i].top = top; b->sc[i].leaf = leaf; }
    DeviceGuard dg(b->c->device);
    cudaStreamSynchronize(b->c->stream);
    int rc = cuda_check(b->c, cudaMemcpyAsync(b->d_sc.p, b->sc.data(), sizeof(BScene) * b->nsc, cudaMemcpyHostToDevice,
                                              b->c->stream), "batch densities");
    if (rc) return (hr_status)rc;
    b->c->g.cap_cells = b->c->g.cap_pairs = b->c->g.cap_leaf_pairs = b->c->g.cap_leaves = 0;
    b->planned = false;
    return HR_OK;
}

hr_status hr_batch_set_launch(hr_batch* b, int32_t block_threads, int32_t tile_w) {
    if (!valid_batch(b)) return HR_ERR_INVALID_ARG;
    if (block_threads < 32 || block_threads > 256 || block_threads % 32 != 0 || tile_w < 1 || tile_w > 32 ||
        (tile_w & (tile_w - 1)) != 0)
        return (hr_status)set_error(b->c, HR_ERR_INVALID_ARG, "batch: launch shape %d threads, tile width %d",
                                    block_threads, tile_w);
    DeviceGuard dg(b->c->device);
    cudaStreamSynchronize(b->c->stream);
    b->block_threads = block_threads;
    b->tile_w = tile_w;
    drop_graph(b);
    b->planned = false;
    return b->nsc ? (hr_status)upload_tiles(b) : HR_OK;
}

hr_status hr_batch_set_integrator(hr_batch* b, float ao_radius_fraction, uint64_t seed) {
    if (!valid_batch(b) || !(ao_radius_fraction > 0.0f)) return HR_ERR_INVALID_ARG;
    b->alpha_frac = ao_radius_fraction;
    b->seed = seed;
    b->jobs_valid = false;
    return HR_OK;
}

hr_status hr_batch_set_graph(hr_batch* b, int32_t use_graph) {
    if (!valid_batch(b)) return HR_ERR_INVALID_ARG;
    DeviceGuard dg(b->c->device);
    cudaStreamSynchronize(b->c->stream);
    b->use_graph = use_graph != 0;
    drop_graph(b);
    b->planned = false;
    return HR_OK;
}

hr_status hr_batch_run(hr_batch* b, int32_t image_id) {
    if (!valid_batch(b) || image_id < 0) return HR_ERR_INVALID_ARG;
    if (b->nsc == 0) return (hr_status)set_error(b->c, HR_ERR_NOT_READY, "batch: no scenes");
    DeviceGuard dg(b->c->device);
    return (hr_status)run_step(b, image_id);
}

hr_status hr_batch_get_times(hr_batch* b, float* build_ms, float* render_ms, float* total_ms) {
    if (!valid_batch(b)) return HR_ERR_INVALID_ARG;
    if (build_ms) *build_ms = b->t_build;
    if (render_ms) *render_ms = b->t_render;
    if (total_ms) *total_ms = b->t_total;
    return HR_OK;
}

hr_status hr_batch_get_counters(hr_batch* b, uint64_t out[8], int32_t reset) {
    if (!valid_batch(b) || !out) return HR_ERR_INVALID_ARG;
    hr_ctx* c = b->c;
    DeviceGuard dg(c->device);
    uint64_t w[8];
    int rc = cuda_check(c, cudaMemcpyAsync(w, c->counters.p, sizeof(w), cudaMemcpyDeviceToHost, c->stream), "counters");
    if (!rc) rc = cuda_check(c, cudaStreamSynchronize(c->stream), "counters");
    if (rc) return (hr_status)rc;
    out[0] = w[0] + w[4];
    out[1] = c->launches;
    out[2] = b->nsc;
    out[3] = b->npix;
    out[4] = w[4];
    out[5] = out[6] = out[7] = 0;
    if (reset) {
        const uint64_t keep = w[1];
        std::memset(w, 0, sizeof(w));
        w[1] = keep;
        rc = cuda_check(c, cudaMemcpyAsync(c->counters.p, w, sizeof(w), cudaMemcpyHostToDevice, c->stream), "counters");
        if (!rc) rc = cuda_check(c, cudaStreamSynchronize(c->stream), "counters");
    }
    return (hr_status)rc;
}

hr_status hr_batch_image_device(hr_batch* b, uint32_t scene, float** d_rgb) {
    if (!valid_batch(b) || !d_rgb) return HR_ERR_INVALID_ARG;
    if (scene >= b->nsc) return (hr_status)set_error(b->c, HR_ERR_INVALID_ARG, "batch: scene %u out of range", scene);
    *d_rgb = dev<float>(b->d_fb) + 3 * b->px_off[scene];
    return HR_OK;
}

hr_status hr_batch_get_image(hr_batch* b, uint32_t scene, float* rgb) {
    if (!valid_batch(b) || !rgb) return HR_ERR_INVALID_ARG;
    if (scene >= b->nsc) return (hr_status)set_error(b->c, HR_ERR_INVALID_ARG, "batch: scene %u out of range", scene);
    hr_ctx* c = b->c;
    DeviceGuard dg(c->device);
    const size_t n = (size_t)b->cams[scene].w * (size_t)b->cams[scene].h * 3;
    int rc = cuda_check(c, cudaMemcpyAsync(rgb, dev<float>(b->d_fb) + 3 * b->px_off[scene], n * sizeof(float),
                                           cudaMemcpyDeviceToHost, c->stream), "batch image");
    if (!rc) rc = cuda_check(c, cudaStreamSynchronize(c->stream), "batch image");
    return (hr_status)rc;
}

hr_status hr_batch_grid_info(hr_batch* b, uint32_t scene, hr_grid_info* info) {
    if (!valid_batch(b) || !info) return HR_ERR_INVALID_ARG;
    if (scene >= b->nsc) return (hr_status)set_error(b->c, HR_ERR_INVALID_ARG, "batch: scene %u out of range", scene);
    if (!b->planned) return (hr_status)set_error(b->c, HR_ERR_NOT_READY, "batch: run a step first");
    hr_ctx* c = b->c;
    DeviceGuard dg(c->device);
    GridDesc d;
    uint32_t co[2];
    int rc = cuda_check(c, cudaMemcpyAsync(&d, dev<GridDesc>(b->d_descs) + scene, sizeof(GridDesc), cudaMemcpyDeviceToHost,
                                           c->stream), "batch grid info");
    if (!rc) rc = cuda_check(c, cudaMemcpyAsync(co, dev<uint32_t>(b->d_cell_off) + scene, 2 * sizeof(uint32_t),
                                                cudaMemcpyDeviceToHost, c->stream), "batch grid info");
    if (!rc) rc = cuda_check(c, cudaStreamSynchronize(c->stream), "batch grid info");
    if (rc) return (hr_status)rc;
    // leaves and pairs of the scene: from the first leaf of its first top cell to the
    // first leaf of the next scene (or the end)
    const GridDesc& bd = *b->h_bdesc;
    uint2 first, next;
    rc = cuda_check(c, cudaMemcpy(&first, c->g.cells.as<uint2>() + co[0], sizeof(uint2), cudaMemcpyDeviceToHost), "cells");
    if (rc) return (hr_status)rc;
    uint32_t leaf_end = bd.nleaves;
    if (scene + 1 < b->nsc) {
        rc = cuda_check(c, cudaMemcpy(&next, c->g.cells.as<uint2>() + co[1], sizeof(uint2), cudaMemcpyDeviceToHost), "cells");
        if (rc) return (hr_status)rc;
        leaf_end = next.x;
    }
    // pairs: leaf ranges are ascending in leaf order; empty leaves are {0, 0}
    std::vector<uint2> lv(leaf_end - first.x);
    if (!lv.empty()) {
        rc = cuda_check(c, cudaMemcpy(lv.data(), c->g.leaves.as<uint2>() + first.x, lv.size() * sizeof(uint2),
                                      cudaMemcpyDeviceToHost), "leaves");
        if (rc) return (hr_status)rc;
    }
    uint32_t pmin = 0xffffffffu, pmax = 0;
    for (const uint2& r : lv)
        if (r.y > r.x) { pmin = std::min(pmin, r.x); pmax = std::max(pmax, r.y); }
    info->kind = HR_GRID_TWO_LEVEL;
    for (int k = 0; k < 3; ++k) {
        info->res[k] = d.res[k];
        info->bounds_min[k] = d.bmin[k]; info->bounds_max[k] = d.bmax[k];
        info->cell_size[k] = d.cs[k]; info->cell_size_rcp[k] = d.rcp[k];
    }
    info->num_cells = co[1] - co[0];
    info->num_leaves = leaf_end - first.x;
    info->num_pairs = pmax > pmin ? pmax - pmin : 0u;
    info->num_top_pairs = d.ntop_pairs;   // counted per scene by kb_count_pairs
    return HR_OK;
}

hr_status hr_batch_grid_download(hr_batch* b, uint32_t scene, uint32_t* cells, uint32_t* leaves, uint32_t* prims) {
    hr_grid_info info;
    hr_status st = hr_batch_grid_info(b, scene, &info);
    if (st != HR_OK) return st;
    hr_ctx* c = b->c;
    DeviceGuard dg(c->device);
    uint32_t co[2];
    int rc = cuda_check(c, cudaMemcpy(co, dev<uint32_t>(b->d_cell_off) + scene, 2 * sizeof(uint32_t),
                                      cudaMemcpyDeviceToHost), "batch grid");
    if (rc) return (hr_status)rc;
    std::vector<uint2> tc(info.num_cells);
    rc = cuda_check(c, cudaMemcpy(tc.data(), c->g.cells.as<uint2>() + co[0], tc.size() * sizeof(uint2),
                                  cudaMemcpyDeviceToHost), "batch cells");
    if (rc) return (hr_status)rc;
    const uint32_t leaf0 = tc.empty() ? 0u : tc[0].x;
    std::vector<uint2> lv(info.num_leaves);
    if (!lv.empty()) {
        rc = cuda_check(c, cudaMemcpy(lv.data(), c->g.leaves.as<uint2>() + leaf0, lv.size() * sizeof(uint2),
                                      cudaMemcpyDeviceToHost), "batch leaves");
        if (rc) return (hr_status)rc;
    }
    uint32_t pair0 = 0xffffffffu;
    for (const uint2& r : lv)
        if (r.y > r.x) pair0 = std::min(pair0, r.x);
    if (pair0 == 0xffffffffu) pair0 = 0;
    if (cells)
        for (size_t i = 0; i < tc.size(); ++i) { cells[2 * i] = tc[i].x - leaf0; cells[2 * i + 1] = tc[i].y; }
    if (leaves)
        for (size_t i = 0; i < lv.size(); ++i) {
            const bool empty = !(lv[i].y > lv[i].x);
            leaves[2 * i] = empty ? 0u : lv[i].x - pair0;
            leaves[2 * i + 1] = empty ? 0u : lv[i].y - pair0;
        }
    if (prims && info.num_pairs) {
        std::vector<uint32_t> pr(info.num_pairs);
        rc = cuda_check(c, cudaMemcpy(pr.data(), c->g.prims.as<uint32_t>() + pair0, pr.size() * sizeof(uint32_t),
                                      cudaMemcpyDeviceToHost), "batch prims");
        if (rc) return (hr_status)rc;
        const uint32_t t0 = b->sc[scene].tri_off;
        for (size_t i = 0; i < pr.size(); ++i) prims[i] = pr[i] - t0;
    }
    return HR_OK;
}

hr_status hr_batch_autotune(hr_batch* b, int32_t reps, hr_batch_tuning* best) {
    if (!valid_batch(b) || reps < 1) return HR_ERR_INVALID_ARG;
    if (b->nsc == 0) return (hr_status)set_error(b->c, HR_ERR_NOT_READY, "batch: no scenes");
    DeviceGuard dg(b->c->device);
    static const float tops[] = {1.0f / 32.0f, 1.0f / 16.0f, 1.0f / 8.0f, 1.0f / 4.0f};
    static const float leafs[] = {1.0f, 2.0f, 4.0f, 8.0f};
    static const int32_t blocks[] = {64, 128, 256};
    static const int32_t tiles[] = {4, 8, 16};
    hr_batch_tuning bt{};
    bt.ms_per_step = 1e30f;
    int trials = 0;
    auto measure = [&](float* ms) -> int {
        int rc;
        if ((rc = run_step(b, 0))) return rc;   // plan + warm
        float tot = 0.0f;
        for (int r = 0; r < reps; ++r) {
            if ((rc = run_step(b, 0))) return rc;
            tot += b->t_total;
        }
        *ms = tot / (float)reps;
        ++trials;
        return 0;
    };
    int rc;
    for (float t : tops)
        for (float l : leafs) {
            if ((rc = hr_batch_set_densities(b, 0xffffffffu, t, l))) return (hr_status)rc;
            float ms;
            if ((rc = measure(&ms))) return (hr_status)rc;
            if (ms < bt.ms_per_step) { bt.ms_per_step = ms; bt.top_density = t; bt.leaf_density = l; }
        }
    if ((rc = hr_batch_set_densities(b, 0xffffffffu, bt.top_density, bt.leaf_density))) return (hr_status)rc;
    bt.block_threads = b->block_threads;
    bt.tile_width = b->tile_w;
    for (int32_t nb : blocks)
        for (int32_t tw : tiles) {
            if ((rc = hr_batch_set_launch(b, nb, tw))) return (hr_status)rc;
            float ms;
            if ((rc = measure(&ms))) return (hr_status)rc;
            if (ms < bt.ms_per_step) { bt.ms_per_step = ms; bt.block_threads = nb; bt.tile_width = tw; }
        }
    if ((rc = hr_batch_set_launch(b, bt.block_threads, bt.tile_width))) return (hr_status)rc;
    if ((rc = run_step(b, 0))) return (hr_status)rc;
    bt.trials = trials;
    if (best) *best = bt;
    return HR_OK;
}

}  // extern "C"
