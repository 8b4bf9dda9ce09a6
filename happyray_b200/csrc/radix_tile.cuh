// radix_tile.cuh -- the per-tile steps of the stable LSD radix sort (sort.cu): the tile's
// digit histogram, the scan of one digit's row of tile counts, and the tile's stable rank
// and scatter.  Shared by the sort kernels (one kernel per step) and by the single-launch
// small-scene build (build_small.cu), which runs the same steps as phases of one kernel.
//
// CG selects the loads of the keys, values and counts: false reads them through the
// read-only path (__ldg: they were written by an earlier launch), true with L2-coherent
// loads (__ldcg: written by other blocks of the same launch before a grid barrier).
#pragma once

#include "hr_internal.h"
#include "hr_block.cuh"

namespace hr {
namespace {

constexpr int kThreads = 256;
constexpr int kItems = 8;
constexpr int kTile = kThreads * kItems;   // 2048 keys per tile
constexpr int kRadix = 512;                // max digit width 9 bits (two digits per thread below)
constexpr int kWarps = kThreads / 32;

template <bool CG>
__device__ __forceinline__ uint32_t rt_load(const uint32_t* p) {
    if (CG) return __ldcg(p);
    return __ldg(p);
}

// digit histogram of tile `tile` (kTile keys from tile * kTile, n keys in all) into column
// `tile` of tile_hist (digit-major rows of row_stride words); a tile past the count writes
// an empty column.  Block of kThreads threads.
template <bool CG>
__device__ __forceinline__ void radix_upsweep_tile(const uint32_t* keys, uint32_t n, int shift, uint32_t mask,
                                                   uint32_t* tile_hist, uint32_t row_stride, uint32_t tile) {
    __shared__ uint32_t h[kRadix];
    for (int d = threadIdx.x; d < kRadix; d += kThreads) h[d] = 0u;
    __syncthreads();
    const size_t base = (size_t)tile * kTile;
    const int lane = threadIdx.x & 31;
    if (base >= n) {
        for (uint32_t d = threadIdx.x; d <= mask; d += kThreads) tile_hist[(size_t)d * row_stride + tile] = 0u;
        return;
    }
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        size_t i = base + threadIdx.x + (size_t)k * kThreads;
        uint32_t dig = i < n ? (rt_load<CG>(keys + i) >> shift) & mask : 0xffffffffu;
        uint32_t peers = __match_any_sync(kFullMask, dig);
        if (dig != 0xffffffffu && lane == __ffs(peers) - 1) atomicAdd(&h[dig], __popc(peers));
    }
    __syncthreads();
    for (uint32_t d = threadIdx.x; d <= mask; d += kThreads) tile_hist[(size_t)d * row_stride + tile] = h[d];
    if (CG) __syncthreads();   // one launch takes many tiles per block: h is reused
}

// exclusive scan in place of one digit's row of tile counts; the row total to *total.
// Block of NT threads.
template <int NT, bool CG = false>
__device__ __forceinline__ void radix_scan_row(uint32_t* row, uint32_t len, uint32_t* total) {
    uint32_t carry = 0;
    for (uint32_t b = 0; b < len; b += NT) {
        uint32_t i = b + threadIdx.x;
        uint32_t x = i < len ? (CG ? __ldcg(row + i) : row[i]) : 0u;
        uint32_t tot;
        uint32_t ex = block_excl_scan<uint32_t, NT>(x, &tot);
        if (i < len) row[i] = carry + ex;
        carry += tot;
    }
    if (threadIdx.x == 0) *total = carry;
}

// stable rank and scatter of tile `tile`: each key goes to the start of its digit (digit
// totals row_total, scanned here) plus the tile's scanned count of that digit
// (tile_hist) plus its rank among the tile's keys of that digit in tile order.  Block of
// kThreads threads.
template <bool CG>
__device__ __forceinline__ void radix_downsweep_tile(const uint32_t* keys_in, const uint32_t* vals_in,
                                                     uint32_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out,
                                                     uint32_t n, int shift, uint32_t mask, const uint32_t* tile_hist,
                                                     uint32_t row_stride, const uint32_t* row_total, uint32_t tile) {
    __shared__ uint32_t s_whist[kWarps][kRadix];
    __shared__ uint32_t s_goff[kRadix];
    __shared__ uint32_t s_loff[kRadix];
    __shared__ uint32_t s_keys[kTile];
    __shared__ uint32_t s_vals[kTile];

    const size_t base = (size_t)tile * kTile;
    if (base >= n) return;
    const uint32_t nvalid = (uint32_t)min((size_t)kTile, n - base);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t lt_mask = (1u << lane) - 1u;

    for (int i = threadIdx.x; i < kWarps * kRadix; i += kThreads) (&s_whist[0][0])[i] = 0u;
    // digit start = exclusive scan of the digit totals (digits 2t and 2t + 1 on thread t)
    {
        const uint32_t d0 = 2u * threadIdx.x, d1 = d0 + 1u;
        const uint32_t t0 = d0 <= mask ? rt_load<CG>(row_total + d0) : 0u;
        const uint32_t t1 = d1 <= mask ? rt_load<CG>(row_total + d1) : 0u;
        uint32_t all;
        const uint32_t ex = block_excl_scan<uint32_t, kThreads>(t0 + t1, &all);
        if (d0 <= mask) s_goff[d0] = ex + rt_load<CG>(tile_hist + (size_t)d0 * row_stride + tile);
        if (d1 <= mask) s_goff[d1] = ex + t0 + rt_load<CG>(tile_hist + (size_t)d1 * row_stride + tile);
    }
    __syncthreads();

    uint32_t key[kItems], val[kItems], rank[kItems], dig[kItems];
#pragma unroll
    for (int r = 0; r < kItems; ++r) {
        const uint32_t li = (uint32_t)w * 32u * kItems + (uint32_t)r * 32u + (uint32_t)lane;
        const bool valid = li < nvalid;
        key[r] = valid ? rt_load<CG>(keys_in + base + li) : 0u;
        val[r] = valid ? rt_load<CG>(vals_in + base + li) : 0u;
        dig[r] = valid ? (key[r] >> shift) & mask : 0xffffffffu;
        const uint32_t peers = __match_any_sync(kFullMask, dig[r]);
        const int leader = __ffs(peers) - 1;
        uint32_t b = 0;
        if (valid && lane == leader) {
            b = s_whist[w][dig[r]];
            s_whist[w][dig[r]] = b + __popc(peers);
        }
        b = __shfl_sync(kFullMask, b, leader);
        rank[r] = b + __popc(peers & lt_mask);
        __syncwarp();
    }
    __syncthreads();
    // per digit: exclusive prefix over warps, tile-local digit totals (digits 2t, 2t + 1)
    uint32_t tcount[2] = {0u, 0u};
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        const uint32_t d = 2u * threadIdx.x + (uint32_t)j;
        if (d <= mask) {
            uint32_t run = 0;
#pragma unroll
            for (int ww = 0; ww < kWarps; ++ww) {
                uint32_t cnt = s_whist[ww][d];
                s_whist[ww][d] = run;
                run += cnt;
            }
            tcount[j] = run;
        }
    }
    {
        uint32_t all;
        const uint32_t ex = block_excl_scan<uint32_t, kThreads>(tcount[0] + tcount[1], &all);
        if (2u * threadIdx.x <= mask) s_loff[2u * threadIdx.x] = ex;
        if (2u * threadIdx.x + 1u <= mask) s_loff[2u * threadIdx.x + 1u] = ex + tcount[0];
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kItems; ++r) {
        if (dig[r] != 0xffffffffu) {
            uint32_t lp = s_loff[dig[r]] + s_whist[w][dig[r]] + rank[r];
            s_keys[lp] = key[r];
            s_vals[lp] = val[r];
        }
    }
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < nvalid; j += kThreads) {
        uint32_t k = s_keys[j];
        uint32_t d = (k >> shift) & mask;
        uint32_t g = s_goff[d] + (j - s_loff[d]);
        keys_out[g] = k;
        vals_out[g] = s_vals[j];
    }
    if (CG) __syncthreads();   // one launch takes many tiles per block: the arrays are reused
}

}  // namespace
}  // namespace hr
