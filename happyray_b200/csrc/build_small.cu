// build_small.cu -- the uniform-grid build of a small scene as one launch.
//
// The build pipeline (build.cu, sort.cu) is a chain of about fifteen dependent kernels:
// bounds, resolution, pair count, scan, scatter, per radix pass a tile histogram, a digit
// row scan and a scatter, then the cell ranges.  For a scene of tens of thousands of
// triangles each is a few microseconds of work and the chain is paced by its launches.
// Here the build is one cooperative launch (every block resident at once) whose phases
// are separated by grid-wide barriers:
//   1  key-frame lerp + per-block bounds                            (k_lerp_bounds)
//   2  bounds of all blocks, resolution; per-triangle pair count    (k_grid_setup, k_count_pairs)
//   3  scan of the block counts, pair scatter (k_scan_block_sums, k_write_pairs); each
//      accepted pair also counted in its cell
//   4  per block: a chunk of cells (pair sum, longest list), a chunk of pairs (rejected)
//   5  cell starts by scan of the counts: cells[c] = (start, start), (0, 0) if empty
//   6  placement: an accepted pair at its cell's cursor (cells[c].y, an atomic add that
//      leaves .y at the cell's end), a rejected pair (exact test, key = ncells) after all
//      accepted ones in pair order
//   7  each cell's list sorted ascending in registers (a triangle is in a list at most
//      once, so this is the order the stable sort of the triangle-ordered pairs gives)
// Phases 5-7 replace the radix sort and the range pass when no cell holds more than
// kCountListMax triangles; otherwise (decided alike in every block from the phase-4
// maxima) the launch runs the pipeline's stable LSD radix passes (sort.cu) and cell ranges.
// Each phase computes what the pipeline computes, so the grid is bit-identical to it.
// Values written by one phase and read by another are read with L2-coherent loads (the
// read-only path may hold stale lines within a launch); block b keeps its triangles
// (b * 256 ...) in registers from phase 2 to phase 3.
// Every block meets every barrier or leaves at the same point: a block returns early only
// on conditions all blocks compute identically (overflow, bad index, the ordering choice).
// The barrier's wait is bounded: a block that gives up sets kDescErrBarrier in the
// descriptor's error word and returns, and the host builds the grid again through the
// pipeline (and keeps the context on it).
#include "build_dev.cuh"
#include "radix_tile.cuh"

#include <algorithm>

namespace hr {
namespace {

static_assert(kBT == kThreads, "the build block is the radix block");

constexpr uint32_t kBarrierPolls = 1u << 21;   // under a second of polling (one L2 round trip each)
constexpr uint32_t kCountListMax = 32;          // longest cell list placed by counting
constexpr int kRun = 8;                         // a thread's cells whose counts stay in registers

struct SmallUG {
    const float4* kf;            // key frames, or null: the vertices are only reduced
    const int4* sel;             // (frame a, frame b, coeff bits) of the lerp
    float4* verts;
    const uint32_t* idx;
    uint32_t nv, ntri;
    GridDesc* d;
    const uint32_t* bad_index_count;
    float density;
    uint32_t cap_cells, cap_pairs;
    int exact;
    float4* tris;
    uint32_t *keys_a, *vals_a, *keys_b, *vals_b, *sorted_keys, *prims;
    uint2* cells;
    uint32_t *tile_hist, *row_total;
    int passes, db;
    uint32_t* bar;               // {arrivals, generation}
    int32_t* blk_bounds;         // 6 encoded bounds per block
    uint32_t* blk_pairs;         // pair count per block
    uint32_t *blk_csum, *blk_cmax, *blk_rej;   // per block: its cells' pairs, longest list, rejected pairs
};

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ uint32_t atom_add_acq_rel(uint32_t* p, uint32_t x) {
    uint32_t old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(x) : "memory");
    return old;
}
__device__ __forceinline__ void red_add_release(uint32_t* p, uint32_t x) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" :: "l"(p), "r"(x) : "memory");
}

// Grid-wide barrier.  After the block barrier, one thread per block arrives with a
// release-acquire add (its block's writes, ordered before it by the block barrier, are
// released with it); the last block to arrive clears the arrival count and advances the
// generation with a release add, the others poll the generation with acquire loads.
// Returns false when the wait gave up.
__device__ bool grid_barrier(uint32_t* bar, GridDesc* d) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        const uint32_t gen0 = ld_acquire(bar + 1);
        int ok = 1;
        if (atom_add_acq_rel(bar, 1u) == gridDim.x - 1u) {
            bar[0] = 0u;
            red_add_release(bar + 1, 1u);
        } else {
            uint32_t polls = 0;
            while (ld_acquire(bar + 1) == gen0) {
                if (++polls > kBarrierPolls) {
                    ok = 0;
                    atomicOr(&d->error, kDescErrBarrier);
                    break;
                }
            }
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// maximum over the block (every thread gets it)
__device__ __forceinline__ uint32_t block_max_u32(uint32_t x) {
    __shared__ uint32_t s[kBT / 32];
    x = __reduce_max_sync(kFullMask, x);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = x;
    __syncthreads();
    uint32_t m = 0;
#pragma unroll
    for (int i = 0; i < kBT / 32; ++i) m = max(m, s[i]);
    __syncthreads();
    return m;
}

// sorts the L <= N words at a ascending, in registers (bitonic network over N, the slots
// past L padded with the largest word); the words were written by other blocks
template <int N>
__device__ __forceinline__ void sort_list(uint32_t* a, uint32_t L) {
    uint32_t v[N];
#pragma unroll
    for (int i = 0; i < N; ++i) v[i] = (uint32_t)i < L ? __ldcg(a + i) : 0xffffffffu;
#pragma unroll
    for (int k = 2; k <= N; k <<= 1)
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1)
#pragma unroll
            for (int i = 0; i < N; ++i) {
                const int l = i ^ j;
                if (l > i) {
                    const uint32_t x = v[i], y = v[l];
                    const bool up = (i & k) == 0;
                    v[i] = up ? min(x, y) : max(x, y);
                    v[l] = up ? max(x, y) : min(x, y);
                }
            }
#pragma unroll
    for (int i = 0; i < N; ++i)
        if ((uint32_t)i < L) a[i] = v[i];
}

// sum over the block, 64-bit (every thread gets it)
__device__ __forceinline__ uint64_t block_sum_u64(uint64_t x) {
    __shared__ uint64_t s[kBT / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(kFullMask, x, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) s[w] = x;
    __syncthreads();
    uint64_t t = 0;
#pragma unroll
    for (int i = 0; i < kBT / 32; ++i) t += s[i];
    __syncthreads();
    return t;
}

__global__ __launch_bounds__(kBT) void k_build_ug_small(SmallUG P) {
    __shared__ GridDesc s_d;
    __shared__ int32_t s_enc[6];
    const uint32_t G = gridDim.x, b = blockIdx.x, tid = threadIdx.x;
    const int lane = (int)(tid & 31u), w = (int)(tid >> 5);
    const uint32_t bad = *P.bad_index_count != 0u ? 1u : 0u;
    if (b == 0 && tid == 0) P.d->error = bad;

    // 1: key-frame lerp and this block's bounds
    {
        f3 lo = mk(FLT_MAX, FLT_MAX, FLT_MAX), hi = mk(-FLT_MAX, -FLT_MAX, -FLT_MAX);
        const float4* a = nullptr;
        const float4* c = nullptr;
        float coeff = 0.0f;
        if (P.kf) {
            const int4 q = *P.sel;
            a = P.kf + (size_t)q.x * P.nv;
            c = P.kf + (size_t)q.y * P.nv;
            coeff = __int_as_float(q.z);
        }
        const float w1 = 1.0f - coeff;
        for (uint32_t i = b * kBT + tid; i < P.nv; i += G * kBT) {
            f3 p;
            if (a) {
                const float4 qa = __ldg(a + i), qb = __ldg(c + i);
                p.x = qa.x * w1 + qb.x * coeff;
                p.y = qa.y * w1 + qb.y * coeff;
                p.z = qa.z * w1 + qb.z * coeff;
                P.verts[i] = make_float4(p.x, p.y, p.z, 0.0f);
            } else {
                const float4 q = __ldg(P.verts + i);
                p = mk(q.x, q.y, q.z);
            }
            lo = vmin(p, lo);
            hi = vmax(p, hi);
        }
        __shared__ float s_b[6][kBT / 32];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            lo.x = hmin(lo.x, __shfl_xor_sync(kFullMask, lo.x, o));
            lo.y = hmin(lo.y, __shfl_xor_sync(kFullMask, lo.y, o));
            lo.z = hmin(lo.z, __shfl_xor_sync(kFullMask, lo.z, o));
            hi.x = hmax(hi.x, __shfl_xor_sync(kFullMask, hi.x, o));
            hi.y = hmax(hi.y, __shfl_xor_sync(kFullMask, hi.y, o));
            hi.z = hmax(hi.z, __shfl_xor_sync(kFullMask, hi.z, o));
        }
        if (lane == 0) { s_b[0][w] = lo.x; s_b[1][w] = lo.y; s_b[2][w] = lo.z; s_b[3][w] = hi.x; s_b[4][w] = hi.y; s_b[5][w] = hi.z; }
        __syncthreads();
        if (tid < 6) {
            float v = s_b[tid][0];
            for (int i = 1; i < kBT / 32; ++i) v = tid < 3 ? hmin(v, s_b[tid][i]) : hmax(v, s_b[tid][i]);
            P.blk_bounds[6 * b + tid] = fenc(v);
        }
    }
    if (!grid_barrier(P.bar, P.d)) return;

    // 2: bounds of all blocks (the encoded min / max the pipeline's atomics take), padded
    // bounds and resolution in every block; block 0 publishes the descriptor
    if (w < 6) {
        int32_t v = w < 3 ? fenc(FLT_MAX) : fenc(-FLT_MAX);
        for (uint32_t j = (uint32_t)lane; j < G; j += 32) {
            const int32_t x = __ldcg(P.blk_bounds + 6 * j + w);
            v = w < 3 ? min(v, x) : max(v, x);
        }
        v = w < 3 ? __reduce_min_sync(kFullMask, v) : __reduce_max_sync(kFullMask, v);
        if (lane == 0) s_enc[w] = v;
    }
    __syncthreads();
    if (tid == 0) {
        uint32_t* z = reinterpret_cast<uint32_t*>(&s_d);
        for (uint32_t i = 0; i < sizeof(GridDesc) / sizeof(uint32_t); ++i) z[i] = 0u;
        for (int k = 0; k < 3; ++k) { s_d.bmin_enc[k] = s_enc[k]; s_d.bmax_enc[k] = s_enc[3 + k]; }
        s_d.kind = kUniform;
        s_d.ntri = P.ntri;
        s_d.error = bad;
        const uint64_t nc = grid_setup(&s_d, P.density);
        if (nc >= (uint64_t)P.cap_cells) {
            s_d.overflow |= kOvfCells;
            s_d.req_cells = nc > 0xfffffff0ull ? 0xfffffff0u : (uint32_t)nc;
            s_d.ncells = 0u;
        } else {
            s_d.ncells = (uint32_t)nc;
        }
        if (b == 0) {
            GridDesc* d = P.d;
            for (int k = 0; k < 3; ++k) {
                d->bmin[k] = s_d.bmin[k]; d->bmax[k] = s_d.bmax[k]; d->res[k] = s_d.res[k];
                d->cs[k] = s_d.cs[k]; d->rcp[k] = s_d.rcp[k];
                d->bmin_enc[k] = s_d.bmin_enc[k]; d->bmax_enc[k] = s_d.bmax_enc[k];
            }
            d->ncells = s_d.ncells;
            d->npairs = 0u; d->ntop_pairs = 0u; d->nleaves = 0u;
            d->overflow = s_d.overflow;
            d->kind = kUniform;
            d->ntri = P.ntri;
            d->req_cells = s_d.req_cells; d->req_pairs = 0u; d->req_leaf_pairs = 0u;
        }
    }
    __syncthreads();
    if (s_d.overflow | s_d.error) return;
    const DescRegs g = load_desc(&s_d);

    // pair count of this block's triangles (bounding-box cells), the per-triangle vertex array
    const uint32_t t = b * kBT + tid;
    uint32_t n = 0;
    f3 p[3];
    CRange r;
    if (t < P.ntri) {
        const uint32_t i0 = __ldg(P.idx + 3 * (size_t)t), i1 = __ldg(P.idx + 3 * (size_t)t + 1);
        const uint32_t i2 = __ldg(P.idx + 3 * (size_t)t + 2);
        const float4 q0 = __ldcg(P.verts + i0), q1 = __ldcg(P.verts + i1), q2 = __ldcg(P.verts + i2);
        p[0] = mk(q0.x, q0.y, q0.z); p[1] = mk(q1.x, q1.y, q1.z); p[2] = mk(q2.x, q2.y, q2.z);
        float4* q = P.tris + 3 * (size_t)t;
        q[0] = make_float4(p[0].x, p[0].y, p[0].z, 0.0f);
        q[1] = make_float4(p[1].x, p[1].y, p[1].z, 0.0f);
        q[2] = make_float4(p[2].x, p[2].y, p[2].z, 0.0f);
        f3 lo, hi;
        tri_bbox(p, &lo, &hi);
        n = cell_range(lo, hi, g.bmin, g.rcp, g.res, &r);
    }
    uint32_t btot;
    const uint32_t ex = block_excl_scan<uint32_t, kBT>(n, &btot);
    if (tid == 0) P.blk_pairs[b] = btot;
    // the cells' .y words count the accepted pairs of each cell in phase 3
    for (uint32_t c = b * kBT + tid; c < g.ncells; c += G * kBT) P.cells[c] = make_uint2(0u, 0u);
    if (!grid_barrier(P.bar, P.d)) return;

    // 3: this block's first pair and the pair total (the scan of the block counts); the
    // pairs go to their slots as k_write_pairs writes them, and every accepted pair is
    // counted in its cell
    uint64_t mine = 0, all = 0;
    for (uint32_t j = tid; j < G; j += kBT) {
        const uint32_t x = __ldcg(P.blk_pairs + j);
        all += x;
        if (j < b) mine += x;
    }
    const uint64_t pre64 = block_sum_u64(mine), total = block_sum_u64(all);
    if (total > (uint64_t)P.cap_pairs) {
        if (b == 0 && tid == 0) {
            atomicOr(&P.d->overflow, kOvfPairs);
            P.d->req_pairs = total > 0xffffffffull ? 0xffffffffu : (uint32_t)total;
        }
        return;
    }
    const uint32_t npairs = (uint32_t)total, pre = (uint32_t)pre64;
    if (b == 0 && tid == 0) P.d->npairs = npairs;
    const uint32_t C = g.ncells;
    uint32_t* const cnt = reinterpret_cast<uint32_t*>(P.cells) + 1;   // cells[c].y: stride 2 words
    const uint32_t rx = (uint32_t)g.res[0], rxy = (uint32_t)g.res[0] * (uint32_t)g.res[1];
    if (P.exact) {
        // each triangle's bounding-box cells in x, y, z order; a cell the SAT test rejects
        // gets key = ncells (sorted last, skipped by the ranges)
        if (n) {
            uint32_t slot = pre + ex;
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
                        const bool in = sat_overlap(nrm, c, p, h);
                        const uint32_t key = in ? (uint32_t)x + (uint32_t)y * rx + (uint32_t)z * rxy : C;
                        P.keys_a[slot] = key;
                        P.vals_a[slot] = t;
                        if (in) atomicAdd(cnt + 2 * (size_t)key, 1u);
                    }
                }
            }
        }
    } else {
        PairRun run;
        if (n) run = {(uint32_t)r.lo[0] + (uint32_t)r.lo[1] * rx + (uint32_t)r.lo[2] * rxy,
                      (uint32_t)(r.hi[0] - r.lo[0]), (uint32_t)(r.hi[1] - r.lo[1]), rx, rxy, t};
        block_write_runs<kBT, 2>(n, run, pre, P.keys_a, P.vals_a, cnt);
    }
    if (!grid_barrier(P.bar, P.d)) return;

    // 4: per block a chunk of the cells (their pair total and longest list) and a chunk of
    // the pairs (its rejected pairs, key = ncells); within a block every thread takes a
    // contiguous run of each, so that phases 5-7 visit them in cell and pair order
    const uint32_t cch = (C + G - 1) / G, c0 = min(b * cch, C), c1 = min(c0 + cch, C);
    const uint32_t pch = (npairs + G - 1) / G, p0 = min(b * pch, npairs), p1 = min(p0 + pch, npairs);
    const uint32_t cpt = (cch + kBT - 1) / kBT, tc0 = min(c0 + tid * cpt, c1), tc1 = min(tc0 + cpt, c1);
    const uint32_t ppt = (pch + kBT - 1) / kBT, tp0 = min(p0 + tid * ppt, p1), tp1 = min(tp0 + ppt, p1);
    {
        uint64_t sum = 0, rej = 0;
        uint32_t lmax = 0;
#pragma unroll 4
        for (uint32_t c = tc0; c < tc1; ++c) {
            const uint32_t k = __ldcg(cnt + 2 * (size_t)c);
            sum += k;
            lmax = max(lmax, k);
        }
#pragma unroll 4
        for (uint32_t i = tp0; i < tp1; ++i) rej += __ldcg(P.keys_a + i) >= C ? 1u : 0u;
        sum = block_sum_u64(sum);
        rej = block_sum_u64(rej);
        lmax = block_max_u32(lmax);
        if (tid == 0) {
            P.blk_csum[b] = (uint32_t)sum;
            P.blk_cmax[b] = lmax;
            P.blk_rej[b] = (uint32_t)rej;
        }
    }
    if (!grid_barrier(P.bar, P.d)) return;

    // 5: the longest list chooses the ordering for every block alike: lists of at most
    // kCountListMax triangles are placed by counting, longer ones take the radix sort
    uint64_t cpre = 0, ctot = 0, rpre = 0;
    uint32_t lmax = 0;
    for (uint32_t j = tid; j < G; j += kBT) {
        const uint32_t x = __ldcg(P.blk_csum + j), y = __ldcg(P.blk_rej + j);
        lmax = max(lmax, __ldcg(P.blk_cmax + j));
        ctot += x;
        if (j < b) { cpre += x; rpre += y; }
    }
    lmax = block_max_u32(lmax);
    cpre = block_sum_u64(cpre);
    ctot = block_sum_u64(ctot);
    rpre = block_sum_u64(rpre);
    if (lmax <= kCountListMax) {
        // cell starts: the exclusive scan of the counts; cells[c] = (start, start), and .y,
        // the cell's placement cursor, ends at the cell's end; an empty cell is (0, 0).  A
        // thread keeps the counts of its first kRun cells in registers for phase 7.
        uint32_t kc[kRun];
        uint32_t loc = 0;
#pragma unroll
        for (int q = 0; q < kRun; ++q) {
            kc[q] = tc0 + q < tc1 ? __ldcg(cnt + 2 * (size_t)(tc0 + q)) : 0u;
            loc += kc[q];
        }
        for (uint32_t c = tc0 + kRun; c < tc1; ++c) loc += __ldcg(cnt + 2 * (size_t)c);
        uint32_t tot;
        const uint32_t st0 = (uint32_t)cpre + block_excl_scan<uint32_t, kBT>(loc, &tot);
        uint32_t st = st0;
#pragma unroll
        for (int q = 0; q < kRun; ++q)
            if (tc0 + q < tc1) {
                P.cells[tc0 + q] = kc[q] ? make_uint2(st, st) : make_uint2(0u, 0u);
                st += kc[q];
            }
        for (uint32_t c = tc0 + kRun; c < tc1; ++c) {
            const uint32_t k = __ldcg(cnt + 2 * (size_t)c);
            P.cells[c] = k ? make_uint2(st, st) : make_uint2(0u, 0u);
            st += k;
        }
        if (!grid_barrier(P.bar, P.d)) return;

        // 6: accepted pairs at their cell's cursor (in any order), rejected pairs after all
        // accepted ones in pair order (where the stable sort puts them)
        {
            uint32_t nrej = 0;
#pragma unroll 4
            for (uint32_t i = tp0; i < tp1; ++i) nrej += __ldcg(P.keys_a + i) >= C ? 1u : 0u;
            uint32_t rtot;
            uint32_t rs = (uint32_t)(ctot + rpre) + block_excl_scan<uint32_t, kBT>(nrej, &rtot);
#pragma unroll 4
            for (uint32_t i = tp0; i < tp1; ++i) {
                const uint32_t key = __ldcg(P.keys_a + i), val = __ldcg(P.vals_a + i);
                if (key < C) P.prims[atomicAdd(cnt + 2 * (size_t)key, 1u)] = val;
                else P.prims[rs++] = val;
            }
        }
        if (!grid_barrier(P.bar, P.d)) return;

        // 7: each cell's list in ascending triangle order, the order the stable sort of the
        // triangle-ordered pairs gives (a triangle is in a cell's list once)
        st = st0;
#pragma unroll
        for (int q = 0; q < kRun; ++q) {
            const uint32_t L = kc[q];
            if (L >= 2u) {
                if (L <= 8u) sort_list<8>(P.prims + st, L);
                else if (L <= 16u) sort_list<16>(P.prims + st, L);
                else sort_list<32>(P.prims + st, L);
            }
            st += L;
        }
        for (uint32_t c = tc0 + kRun; c < tc1; ++c) {
            const uint2 cr = __ldcg(P.cells + c);
            const uint32_t L = cr.y - cr.x;
            if (L >= 2u) {
                if (L <= 8u) sort_list<8>(P.prims + cr.x, L);
                else if (L <= 16u) sort_list<16>(P.prims + cr.x, L);
                else sort_list<32>(P.prims + cr.x, L);
            }
        }
        return;
    }

    // 5 (long lists): stable LSD radix sort by cell (the passes and buffers of
    // radix_sort_pairs), then the cell ranges from the sorted keys
    for (uint32_t c = b * kBT + tid; c < C; c += G * kBT) P.cells[c] = make_uint2(0u, 0u);
    const uint32_t ntiles = (npairs + kTile - 1) / kTile;
    const uint32_t mask = (1u << P.db) - 1u;
    const uint32_t* src_k = P.keys_a;
    const uint32_t* src_v = P.vals_a;
    for (int pp = 0; pp < P.passes; ++pp) {
        const bool last = pp == P.passes - 1;
        uint32_t* dk = last ? P.sorted_keys : (pp % 2 == 0 ? P.keys_b : P.keys_a);
        uint32_t* dv = last ? P.prims : (pp % 2 == 0 ? P.vals_b : P.vals_a);
        const int shift = pp * P.db;
        for (uint32_t tile = b; tile < ntiles; tile += G)
            radix_upsweep_tile<true>(src_k, npairs, shift, mask, P.tile_hist, ntiles, tile);
        if (!grid_barrier(P.bar, P.d)) return;
        for (uint32_t dg = b; dg <= mask; dg += G)
            radix_scan_row<kBT, true>(P.tile_hist + (size_t)dg * ntiles, ntiles, P.row_total + dg);
        if (!grid_barrier(P.bar, P.d)) return;
        for (uint32_t tile = b; tile < ntiles; tile += G)
            radix_downsweep_tile<true>(src_k, src_v, dk, dv, npairs, shift, mask, P.tile_hist, ntiles, P.row_total,
                                       tile);
        if (!grid_barrier(P.bar, P.d)) return;
        src_k = dk;
        src_v = dv;
    }
    for (uint32_t i = b * kBT + tid; i < npairs; i += G * kBT) {
        const uint32_t k = __ldcg(P.sorted_keys + i);
        if (k >= C) continue;
        if (i == 0 || __ldcg(P.sorted_keys + i - 1) != k) P.cells[k].x = i;
        if (i + 1 == npairs || __ldcg(P.sorted_keys + i + 1) != k) P.cells[k].y = i + 1;
    }
}

}  // namespace

int build_small_uniform(hr_ctx* c, int32_t exact, int key_bits, bool* done) {
    *done = false;
    const uint32_t ntri = c->ntri;
    if (ntri == 0 || ntri > c->small_build_max_tris) return 0;
    if (c->small_build_bps < 0) {
        int bps = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_build_ug_small, kBT, 0) != cudaSuccess) {
            cudaGetLastError();
            bps = 0;
        }
        c->small_build_bps = bps;
    }
    // one block per SM at least (the sort phases), one per 256 triangles (phases 2-3), and
    // at most half the blocks the GPU holds at once, so that two such builds on different
    // streams always fit side by side
    const uint32_t G = std::max((ntri + kBT - 1) / kBT, (uint32_t)c->num_sms);
    if (c->small_build_bps <= 0 || 2 * G > (uint32_t)c->small_build_bps * (uint32_t)c->num_sms) return 0;
    const size_t bar_words = 4, bytes = sizeof(uint32_t) * (bar_words + 10 * (size_t)G);
    const void* before = c->build_bar.p;
    const size_t before_bytes = c->build_bar.bytes;
    int rc;
    if ((rc = ensure(c, c->build_bar, bytes))) return rc;
    // fresh memory: the barrier starts from zero arrivals (a completed launch leaves it so)
    if ((c->build_bar.p != before || c->build_bar.bytes != before_bytes) &&
        (rc = cuda_check(c, cudaMemsetAsync(c->build_bar.p, 0, sizeof(uint32_t) * bar_words, c->stream), "barrier")))
        return rc;
    GridBuffers& B = c->g;
    const int passes = radix_sort_passes(key_bits);
    SmallUG P;
    P.kf = c->lerp_pending ? c->keyframes.as<float4>() : nullptr;
    P.sel = c->frame_sel.as<int4>();
    P.verts = c->verts.as<float4>();
    P.idx = c->idx.as<uint32_t>();
    P.nv = c->nverts;
    P.ntri = ntri;
    P.d = B.desc.as<GridDesc>();
    P.bad_index_count = c->counters.as<uint32_t>() + 2;
    P.density = c->ug_density;
    P.cap_cells = (uint32_t)std::min(B.cap_cells, (size_t)0xffffffffu);
    P.cap_pairs = (uint32_t)std::min(B.cap_pairs, (size_t)0xffffffffu);
    P.exact = exact ? 1 : 0;
    P.tris = c->tris.as<float4>();
    P.keys_a = B.keys_a.as<uint32_t>();
    P.vals_a = B.vals_a.as<uint32_t>();
    P.keys_b = B.keys_b.as<uint32_t>();
    P.vals_b = B.vals_b.as<uint32_t>();
    P.sorted_keys = (passes % 2 == 1) ? P.keys_b : P.keys_a;
    P.prims = B.prims.as<uint32_t>();
    P.cells = B.cells.as<uint2>();
    P.tile_hist = B.tile_hist.as<uint32_t>();
    P.row_total = B.row_total.as<uint32_t>();
    P.passes = passes;
    P.db = (key_bits + passes - 1) / passes;
    uint32_t* w = c->build_bar.as<uint32_t>();
    P.bar = w;
    P.blk_bounds = reinterpret_cast<int32_t*>(w + bar_words);
    P.blk_pairs = w + bar_words + 6 * (size_t)G;
    P.blk_csum = P.blk_pairs + G;
    P.blk_cmax = P.blk_csum + G;
    P.blk_rej = P.blk_cmax + G;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(G);
    cfg.blockDim = dim3(kBT);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = c->stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    if (cudaLaunchKernelEx(&cfg, k_build_ug_small, P) != cudaSuccess) {
        // cooperative launches unavailable here: the pipeline from now on
        cudaGetLastError();
        c->small_build_max_tris = 0;
        return 0;
    }
    c->launches += 1;
    *done = true;
    return 0;
}

}  // namespace hr
