// hr_block.cuh -- CTA-wide scan helpers shared by the build and sort kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace hr {

constexpr unsigned kFullMask = 0xffffffffu;

__device__ __forceinline__ uint2 operator+(uint2 a, uint2 b) { return make_uint2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ uint2 operator-(uint2 a, uint2 b) { return make_uint2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ uint32_t shfl_up(uint32_t x, int o) { return __shfl_up_sync(kFullMask, x, o); }
__device__ __forceinline__ uint2 shfl_up(uint2 x, int o) {
    return make_uint2(__shfl_up_sync(kFullMask, x.x, o), __shfl_up_sync(kFullMask, x.y, o));
}
template <class T> __device__ __forceinline__ T zero();
template <> __device__ __forceinline__ uint32_t zero<uint32_t>() { return 0u; }
template <> __device__ __forceinline__ uint2 zero<uint2>() { return make_uint2(0u, 0u); }

// Exclusive scan of one value per thread across a CTA of NT threads; returns the
// exclusive prefix and writes the CTA total to *total.
template <class T, int NT>
__device__ __forceinline__ T block_excl_scan(T x, T* total) {
    __shared__ T s_w[NT / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    T inc = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T y = shfl_up(inc, o);
        if (lane >= o) inc = inc + y;
    }
    if (lane == 31) s_w[w] = inc;
    __syncthreads();
    if (w == 0) {
        T v = lane < NT / 32 ? s_w[lane] : zero<T>();
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            T y = shfl_up(v, o);
            if (lane >= o) v = v + y;
        }
        if (lane < NT / 32) s_w[lane] = v;
    }
    __syncthreads();
    T before = w > 0 ? s_w[w - 1] : zero<T>();
    *total = s_w[NT / 32 - 1];
    __syncthreads();
    return before + (inc - x);
}


}  // namespace hr

namespace hr {
// largest s in [0, n) with off[s] <= x, for ascending off with off[0] = 0
__device__ __forceinline__ uint32_t find_segment(const uint32_t* __restrict__ off, uint32_t n, uint32_t x) {
    uint32_t lo = 0, hi = n;
    while (hi - lo > 1u) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(off + mid) <= x) lo = mid;
        else hi = mid;
    }
    return lo;
}
}  // namespace hr
