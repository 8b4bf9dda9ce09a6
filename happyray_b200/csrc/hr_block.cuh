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

// Largest k in [0, NT) with off[k] <= j, for a non-decreasing off[] (off[0] = 0 <= j): the
// item whose output run [off[k], off[k + 1]) holds output j of a block.
template <int NT>
__device__ __forceinline__ int block_owner(const uint32_t* off, uint32_t j) {
    int k = 0;
#pragma unroll
    for (int step = NT / 2; step > 0; step >>= 1)
        if (off[k + step] <= j) k += step;
    return k;
}

// One item's run of (cell key, value) pairs: the cells of an ex x ey x ez box, x fastest,
// then y, then z, keyed key0 + dx + dy * sx + dz * sxy, all with value val.
struct PairRun { uint32_t key0, ex, ey, sx, sxy, val; };

// Writes a block's pairs with all its threads: the runs follow one another in thread order
// from out0, and pair j of the block is stored by thread j mod NT, so a run of thousands of
// cells costs its block a few strides instead of one thread a serial loop, and consecutive
// threads store consecutive slots.  n is this thread's run length, run is read when n > 0.
// Every thread of the block calls it.
// With `counts`, also adds every written key to counts[key * CS] (a histogram of the keys;
// the lanes of a warp holding the same key add once, so a crowded cell costs few atomics).
template <int NT, int CS = 1>
__device__ __forceinline__ void block_write_runs(uint32_t n, const PairRun& run, uint32_t out0,
                                                 uint32_t* __restrict__ keys, uint32_t* __restrict__ vals,
                                                 uint32_t* __restrict__ counts = nullptr) {
    __shared__ uint32_t s_off[NT];
    __shared__ PairRun s_run[NT];
    uint32_t tot;
    s_off[threadIdx.x] = block_excl_scan<uint32_t, NT>(n, &tot);
    if (n) s_run[threadIdx.x] = run;
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31u;
    // warp-uniform trip count, so that the whole warp meets the match below
    for (uint32_t j0 = threadIdx.x - lane; j0 < tot; j0 += NT) {
        const uint32_t j = j0 + lane;
        const bool valid = j < tot;
        uint32_t key = 0xffffffffu;
        if (valid) {
            const int k = block_owner<NT>(s_off, j);
            const PairRun q = s_run[k];
            const uint32_t l = j - s_off[k];
            key = q.key0;
            if (l) {
                const uint32_t a = l / q.ex, z = a / q.ey;
                key += (l - a * q.ex) + (a - z * q.ey) * q.sx + z * q.sxy;
            }
            keys[out0 + j] = key;
            vals[out0 + j] = q.val;
        }
        if (counts) {
            const uint32_t peers = __match_any_sync(0xffffffffu, key);
            if (valid && lane == (uint32_t)(__ffs(peers) - 1)) atomicAdd(counts + (size_t)key * CS, (uint32_t)__popc(peers));
        }
    }
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
