// sort.cu -- device-wide exclusive scans and the stable LSD radix sort of (key, value)
// pairs used by the grid builders.
//
// Replaces the reference's CUB wrappers: ExclusiveScan (Scan.cu:39-58) and RadixSort
// (Sort.cu:31-53, cub::DeviceRadixSort::SortPairs over uint32 keys/values).
//
// Design: reduce-then-scan in every pass (upsweep tile histograms, one CTA per digit
// scans its row of tile counts, downsweep ranks and scatters), so no kernel waits on
// another CTA and nothing spins.  All element counts are read from device memory, so
// the whole pipeline is enqueued without a host round trip; grids are sized from the
// host-side capacity and surplus CTAs exit at once.
#include "hr_internal.h"
#include "hr_block.cuh"
#include "radix_tile.cuh"

namespace hr {

namespace {

// ----------------------------------------------------------------------------------
// generic exclusive scan: reduce -> scan partials -> apply

template <class T>
__global__ __launch_bounds__(kThreads) void k_scan_reduce(const T* __restrict__ data, const uint32_t* d_count,
                                                          T* partials) {
    const uint32_t n = *d_count;
    const size_t base = (size_t)blockIdx.x * kTile;
    T s = zero<T>();
    if (base < n) {
#pragma unroll
        for (int k = 0; k < kItems; ++k) {
            size_t i = base + threadIdx.x + (size_t)k * kThreads;
            if (i < n) s = s + data[i];
        }
    }
    T total;
    block_excl_scan<T, kThreads>(s, &total);
    if (threadIdx.x == 0) partials[blockIdx.x] = total;
}

// One CTA scans `n` partials (exclusive, in place); the grand total goes to d_total_*.
// If cap > 0 and the total exceeds it, `ovf_bit` is or-ed into *ovf.
template <class T>
__global__ __launch_bounds__(1024) void k_scan_partials(T* partials, uint32_t n, uint32_t* d_total_x,
                                                        uint32_t* d_total_y, uint32_t* ovf,
                                                        uint32_t cap_x, uint32_t ovf_bit_x,
                                                        uint32_t cap_y, uint32_t ovf_bit_y);

template <>
__global__ __launch_bounds__(1024) void k_scan_partials<uint32_t>(uint32_t* partials, uint32_t n,
                                                                  uint32_t* d_total_x, uint32_t*,
                                                                  uint32_t* ovf, uint32_t cap_x,
                                                                  uint32_t ovf_bit_x, uint32_t, uint32_t) {
    uint32_t carry = 0;
    for (uint32_t b = 0; b < n; b += 1024) {
        uint32_t i = b + threadIdx.x;
        uint32_t x = i < n ? partials[i] : 0u;
        uint32_t tot;
        uint32_t ex = block_excl_scan<uint32_t, 1024>(x, &tot);
        if (i < n) partials[i] = carry + ex;
        carry += tot;
    }
    if (threadIdx.x == 0) {
        if (d_total_x) *d_total_x = carry;
        if (ovf && cap_x && carry > cap_x) atomicOr(ovf, ovf_bit_x);
    }
}

template <>
__global__ __launch_bounds__(1024) void k_scan_partials<uint2>(uint2* partials, uint32_t n, uint32_t* d_total_x,
                                                               uint32_t* d_total_y, uint32_t* ovf,
                                                               uint32_t cap_x, uint32_t ovf_bit_x,
                                                               uint32_t cap_y, uint32_t ovf_bit_y) {
    uint2 carry = make_uint2(0u, 0u);
    for (uint32_t b = 0; b < n; b += 1024) {
        uint32_t i = b + threadIdx.x;
        uint2 x = i < n ? partials[i] : make_uint2(0u, 0u);
        uint2 tot;
        uint2 ex = block_excl_scan<uint2, 1024>(x, &tot);
        if (i < n) partials[i] = carry + ex;
        carry = carry + tot;
    }
    if (threadIdx.x == 0) {
        if (d_total_x) *d_total_x = carry.x;
        if (d_total_y) *d_total_y = carry.y;
        if (ovf && cap_x && carry.x > cap_x) atomicOr(ovf, ovf_bit_x);
        if (ovf && cap_y && carry.y > cap_y) atomicOr(ovf, ovf_bit_y);
    }
}

template <class T>
__global__ __launch_bounds__(kThreads) void k_scan_apply(T* data, const uint32_t* d_count, const T* partials) {
    const uint32_t n = *d_count;
    const size_t base = (size_t)blockIdx.x * kTile;
    if (base >= n) return;
    // blocked arrangement: thread j owns items base + j*kItems .. +kItems
    T v[kItems];
    T s = zero<T>();
    const size_t b0 = base + (size_t)threadIdx.x * kItems;
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        v[k] = (b0 + k < n) ? data[b0 + k] : zero<T>();
        s = s + v[k];
    }
    T total;
    T run = block_excl_scan<T, kThreads>(s, &total) + partials[blockIdx.x];
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        if (b0 + k < n) data[b0 + k] = run;
        run = run + v[k];
    }
}

// ----------------------------------------------------------------------------------
// radix sort kernels

__global__ __launch_bounds__(kThreads) void k_radix_upsweep(const uint32_t* __restrict__ keys, const uint32_t* d_count,
                                                            int shift, uint32_t mask, uint32_t* tile_hist,
                                                            uint32_t ntiles_cap) {
    radix_upsweep_tile<false>(keys, *d_count, shift, mask, tile_hist, ntiles_cap, blockIdx.x);
}

// one CTA per digit: exclusive scan of its row of tile counts, row total out
__global__ __launch_bounds__(1024) void k_radix_scan(uint32_t* tile_hist, uint32_t ntiles_cap, uint32_t* row_total) {
    radix_scan_row<1024>(tile_hist + (size_t)blockIdx.x * ntiles_cap, ntiles_cap, row_total + blockIdx.x);
}

__global__ __launch_bounds__(kThreads) void k_radix_downsweep(
    const uint32_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in, uint32_t* __restrict__ keys_out,
    uint32_t* __restrict__ vals_out, const uint32_t* d_count, int shift, uint32_t mask,
    const uint32_t* __restrict__ tile_hist, uint32_t ntiles_cap, const uint32_t* __restrict__ row_total) {
    radix_downsweep_tile<false>(keys_in, vals_in, keys_out, vals_out, *d_count, shift, mask, tile_hist, ntiles_cap,
                                row_total, blockIdx.x);
}

}  // namespace

// ----------------------------------------------------------------------------------
// host launchers

size_t scan_partials_words(size_t cap_count) { return (cap_count + kTile - 1) / kTile + 1; }

int exclusive_scan_u32(hr_ctx* c, uint32_t* data, const uint32_t* d_count, size_t cap_count,
                       uint32_t* d_total, uint32_t* partials, cudaStream_t s) {
    const uint32_t nb = (uint32_t)((cap_count + kTile - 1) / kTile);
    if (nb == 0) return 0;
    c->launches += 3;
    k_scan_reduce<uint32_t><<<nb, kThreads, 0, s>>>(data, d_count, partials);
    k_scan_partials<uint32_t><<<1, 1024, 0, s>>>(partials, nb, d_total, nullptr, nullptr, 0, 0, 0, 0);
    k_scan_apply<uint32_t><<<nb, kThreads, 0, s>>>(data, d_count, partials);
    return cuda_check(c, cudaGetLastError(), "exclusive_scan_u32");
}

int exclusive_scan_u32x2(hr_ctx* c, uint2* data, const uint32_t* d_count, size_t cap_count,
                         uint32_t* d_total_x, uint32_t* d_total_y, uint2* partials, cudaStream_t s) {
    const uint32_t nb = (uint32_t)((cap_count + kTile - 1) / kTile);
    if (nb == 0) return 0;
    c->launches += 3;
    k_scan_reduce<uint2><<<nb, kThreads, 0, s>>>(data, d_count, partials);
    k_scan_partials<uint2><<<1, 1024, 0, s>>>(partials, nb, d_total_x, d_total_y, nullptr, 0, 0, 0, 0);
    k_scan_apply<uint2><<<nb, kThreads, 0, s>>>(data, d_count, partials);
    return cuda_check(c, cudaGetLastError(), "exclusive_scan_u32x2");
}

// scan of per-block pair counts written by the count kernels (in place, exclusive).
// A total above `cap` sets `ovf_bit`, stores the total in *d_req and publishes a zero
// count, so every later stage of the build sees no work.
__global__ __launch_bounds__(1024) void k_scan_block_sums(uint32_t* sums, uint32_t n, uint32_t* d_total,
                                                          uint32_t* ovf, uint32_t cap, uint32_t ovf_bit,
                                                          uint32_t* d_req) {
    // 8 consecutive counts per thread, 8192 per round
    constexpr uint32_t kIpt = 8, kChunk = 1024 * kIpt;
    uint64_t carry = 0;
    for (uint32_t b = 0; b < n; b += kChunk) {
        const uint32_t i0 = b + threadIdx.x * kIpt;
        uint32_t x[kIpt], s = 0;
#pragma unroll
        for (uint32_t k = 0; k < kIpt; ++k) {
            x[k] = i0 + k < n ? sums[i0 + k] : 0u;
            s += x[k];
        }
        uint32_t tot;
        uint32_t run = (uint32_t)carry + block_excl_scan<uint32_t, 1024>(s, &tot);
#pragma unroll
        for (uint32_t k = 0; k < kIpt; ++k) {
            if (i0 + k < n) sums[i0 + k] = run;
            run += x[k];
        }
        carry += tot;
    }
    if (threadIdx.x == 0) {
        if (carry > cap) {
            atomicOr(ovf, ovf_bit);
            *d_req = carry > 0xffffffffull ? 0xffffffffu : (uint32_t)carry;
            *d_total = 0u;
        } else {
            *d_total = (uint32_t)carry;
        }
    }
}

int scan_block_sums(hr_ctx* c, uint32_t* sums, uint32_t n, uint32_t* d_total, uint32_t* ovf,
                    uint32_t cap, uint32_t ovf_bit, uint32_t* d_req, cudaStream_t s) {
    k_scan_block_sums<<<1, 1024, 0, s>>>(sums, n, d_total, ovf, cap, ovf_bit, d_req);
    return cuda_check(c, cudaGetLastError(), "scan_block_sums");
}

// fewest passes of at most max_db-bit digits, the bits spread evenly over them (the
// context path takes 9-bit digits: 17-18-bit cell keys sort in two passes, not three)
static void radix_plan(int key_bits, int max_db, int* passes, int* db) {
    if (key_bits < 1) key_bits = 1;
    if (key_bits > 32) key_bits = 32;
    *passes = (key_bits + max_db - 1) / max_db;
    *db = (key_bits + *passes - 1) / *passes;
}

constexpr int kMaxDigitBits = 9;   // context sorts; the allocation-free sort keeps 8 (its static scratch)

int radix_sort_passes(int key_bits) {
    int passes, db;
    radix_plan(key_bits, kMaxDigitBits, &passes, &db);
    return passes;
}

size_t radix_tile_hist_words(size_t cap_count, int key_bits) {
    int passes, db;
    radix_plan(key_bits, kMaxDigitBits, &passes, &db);
    size_t ntiles = (cap_count + kTile - 1) / kTile;
    if (ntiles == 0) ntiles = 1;
    return ntiles * ((size_t)1 << db);
}

int radix_sort_pairs(hr_ctx* c, const uint32_t* keys_in, const uint32_t* vals_in,
                     uint32_t* keys_tmp, uint32_t* vals_tmp, uint32_t* keys_out, uint32_t* vals_out,
                     const uint32_t* d_count, size_t cap_count, int key_bits,
                     uint32_t* tile_hist, size_t tile_hist_bytes, uint32_t* row_total, cudaStream_t s) {
    // the histogram holds 2^digit words per tile: fewer key bits can need more of them
    if (radix_tile_hist_words(cap_count, key_bits) * sizeof(uint32_t) > tile_hist_bytes)
        return set_error(c, 4, "radix sort: histogram of %zu bytes is too small for %zu keys of %d bits",
                         tile_hist_bytes, cap_count, key_bits);
    int passes, db;
    radix_plan(key_bits, kMaxDigitBits, &passes, &db);
    const uint32_t mask = (1u << db) - 1u;
    const uint32_t ntiles = (uint32_t)((cap_count + kTile - 1) / kTile);
    if (ntiles == 0) return 0;
    const uint32_t* src_k = keys_in;
    const uint32_t* src_v = vals_in;
    for (int p = 0; p < passes; ++p) {
        const bool last = p == passes - 1;
        uint32_t* dk = last ? keys_out : ((p % 2 == 0) ? keys_tmp : const_cast<uint32_t*>(keys_in));
        uint32_t* dv = last ? vals_out : ((p % 2 == 0) ? vals_tmp : const_cast<uint32_t*>(vals_in));
        const int shift = p * db;
        c->launches += 3;
        k_radix_upsweep<<<ntiles, kThreads, 0, s>>>(src_k, d_count, shift, mask, tile_hist, ntiles);
        k_radix_scan<<<mask + 1, 1024, 0, s>>>(tile_hist, ntiles, row_total);
        k_radix_downsweep<<<ntiles, kThreads, 0, s>>>(src_k, src_v, dk, dv, d_count, shift, mask, tile_hist,
                                                      ntiles, row_total);
        src_k = dk;
        src_v = dv;
    }
    return cuda_check(c, cudaGetLastError(), "radix_sort_pairs");
}

// Same pass sequence as radix_sort_pairs, without a context (no status text, no launch
// count); used by the allocation-free entry point.
cudaError_t radix_sort_pairs_raw(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_tmp,
                                 uint32_t* vals_tmp, uint32_t* keys_out, uint32_t* vals_out,
                                 const uint32_t* d_count, size_t cap_count, int key_bits, uint32_t* tile_hist,
                                 uint32_t* row_total, cudaStream_t s) {
    int passes, db;
    radix_plan(key_bits, 8, &passes, &db);
    const uint32_t mask = (1u << db) - 1u;
    const uint32_t ntiles = (uint32_t)((cap_count + kTile - 1) / kTile);
    if (ntiles == 0) return cudaSuccess;
    const uint32_t* src_k = keys_in;
    const uint32_t* src_v = vals_in;
    for (int p = 0; p < passes; ++p) {
        const bool last = p == passes - 1;
        uint32_t* dk = last ? keys_out : ((p % 2 == 0) ? keys_tmp : const_cast<uint32_t*>(keys_in));
        uint32_t* dv = last ? vals_out : ((p % 2 == 0) ? vals_tmp : const_cast<uint32_t*>(vals_in));
        const int shift = p * db;
        k_radix_upsweep<<<ntiles, kThreads, 0, s>>>(src_k, d_count, shift, mask, tile_hist, ntiles);
        k_radix_scan<<<mask + 1, 1024, 0, s>>>(tile_hist, ntiles, row_total);
        k_radix_downsweep<<<ntiles, kThreads, 0, s>>>(src_k, src_v, dk, dv, d_count, shift, mask, tile_hist,
                                                      ntiles, row_total);
        src_k = dk;
        src_v = dv;
    }
    return cudaGetLastError();
}

}  // namespace hr
