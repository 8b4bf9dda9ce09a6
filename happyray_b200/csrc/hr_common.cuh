// hr_common.cuh -- device-side arithmetic shared by the build and traversal kernels.
//
// Every float expression is written in a fixed evaluation order and the library is
// compiled with -fmad=false, IEEE division and IEEE square root, so each result is
// a deterministic function of its inputs (bit-identical to a strict binary32 host
// evaluation of the same expression).
#pragma once

#include <cstdint>
#include <cfloat>
#include <cuda_runtime.h>

namespace hr {

constexpr float kEps = 0.00001f;           // CUDAStdAfx.h:117 EPS
constexpr float kIsectEps = 0.0001f;       // RayTriangleIntersector.h:36 INTERSECTION_EPS
constexpr uint32_t kLeafRefsMax = 16u;     // TLGridBuildKernels.h:77
constexpr uint32_t kLeafMask = 0x10000000u;      // TwoLevelGrid.h:58
constexpr uint32_t kNotEmptyMask = 0x40000000u;  // TwoLevelGrid.h:60

enum GridKind : int32_t { kUniform = 0, kTwoLevel = 1 };

// overflow bits in GridDesc::overflow
enum : uint32_t {
    kOvfCells = 1u, kOvfPairs = 2u, kOvfTopPairs = 4u, kOvfLeaves = 8u, kOvfLeafPairs = 16u
};
// bits of GridDesc::error: a triangle index beyond the uploaded vertices (set from the
// upload's index check), a grid barrier of the single-launch build that gave up waiting
enum : uint32_t { kDescErrIndex = 1u, kDescErrBarrier = 2u };

// Grid descriptor kept in device memory and written by the build kernels, so no host
// round trip is needed between build stages.  Mirrors UniformGrid (UniformGrid.h:37-138)
// and TwoLevelGrid (TwoLevelGrid.h:163-230) parameters.
struct GridDesc {
    float bmin[3], bmax[3];
    int32_t res[3];
    float cs[3], rcp[3];
    uint32_t ncells;      // uniform: cells; two-level: top cells
    uint32_t npairs;      // uniform: pairs P; two-level: leaf pairs
    uint32_t ntop_pairs;  // two-level: top-level pairs
    uint32_t nleaves;     // two-level: leaf cells
    uint32_t overflow;    // kOvf* bits
    uint32_t error;
    int32_t kind;
    uint32_t ntri;
    int32_t bmin_enc[3], bmax_enc[3];  // ordered-int encoded running bounds
    uint32_t req_cells;   // cells needed when kOvfCells is set (ncells is then 0)
    uint32_t req_pairs;   // pairs needed when kOvfPairs / kOvfTopPairs is set (count is then 0)
    uint32_t req_leaf_pairs;   // leaf pairs needed when kOvfLeafPairs is set (count is then 0)
    uint32_t pad1;
};

// Area lights of the path tracer (AreaLightSource, LightSource.hpp:38-95): parallelogram
// c + s e1 + t e2 (s, t in [0, 1]) emitting radiance `emission` towards the side of its unit
// normal n, with the values formed once: nc = e1 x e2, inv_nn = 1 / |nc|^2, area = |nc|.
// A collection (AreaLightSourceCollection, LightSource.hpp:102-198) picks light k for a
// sample with probability w_k / W, w_k = area_k * emission_k, from the inclusive running
// sum cdf of the weights; it is built on the host (make_light_set) and read by the kernels
// from device memory.
constexpr int kMaxLights = 64;
struct LightQ {
    float c[3], e1[3], e2[3], n[3], nc[3];
    float inv_nn, area, emission;
};
struct LightSet {
    uint32_t count;
    uint32_t pad[3];
    float cdf[kMaxLights];
    LightQ q[kMaxLights];
};

__host__ __device__ __forceinline__ float hmin(float a, float b) { return (a != a) ? b : ((b < a) ? b : a); }
__host__ __device__ __forceinline__ float hmax(float a, float b) { return (a != a) ? b : ((b > a) ? b : a); }
__device__ __forceinline__ int32_t f2i(float x) { return __float2int_rz(x); }  // saturating, NaN -> 0

struct f3 { float x, y, z; };
__device__ __forceinline__ f3 mk(float x, float y, float z) { f3 r; r.x = x; r.y = y; r.z = z; return r; }
__device__ __forceinline__ f3 sub(f3 a, f3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ f3 add(f3 a, f3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ f3 mulf(f3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ f3 cross(f3 a, f3 b) {
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ f3 normalize(f3 a) { float inv = 1.0f / sqrtf(dot(a, a)); return mulf(a, inv); }
__device__ __forceinline__ f3 vmin(f3 a, f3 b) { return mk(hmin(a.x, b.x), hmin(a.y, b.y), hmin(a.z, b.z)); }
__device__ __forceinline__ f3 vmax(f3 a, f3 b) { return mk(hmax(a.x, b.x), hmax(a.y, b.y), hmax(a.z, b.z)); }
__device__ __forceinline__ float comp(f3 a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }
__device__ __forceinline__ f3 ldv(const float4* __restrict__ v, uint32_t i) {
    float4 q = __ldg(v + i);
    return mk(q.x, q.y, q.z);
}

// ordered-int encoding so that integer min/max equals float min/max
__device__ __forceinline__ int32_t fenc(float f) {
    int32_t b = __float_as_int(f);
    return b >= 0 ? b : (b ^ 0x7fffffff);
}
__host__ __device__ __forceinline__ float fdec(int32_t b) {
#ifdef __CUDA_ARCH__
    return __int_as_float(b >= 0 ? b : (b ^ 0x7fffffff));
#else
    int32_t v = b >= 0 ? b : (b ^ 0x7fffffff);
    float f;
    __builtin_memcpy(&f, &v, 4);
    return f;
#endif
}

// Triangle bounding box, BBox.hpp:89-93
__device__ __forceinline__ void tri_load(const float4* __restrict__ v, const uint32_t* __restrict__ idx,
                                         uint32_t t, f3* p) {
    uint32_t i0 = __ldg(idx + 3 * (size_t)t), i1 = __ldg(idx + 3 * (size_t)t + 1), i2 = __ldg(idx + 3 * (size_t)t + 2);
    p[0] = ldv(v, i0); p[1] = ldv(v, i1); p[2] = ldv(v, i2);
}
// Triangle vertices from the per-triangle array (3 float4 per triangle, written by the
// pair-count pass of every build): one contiguous 48-byte load instead of three
// index-dependent vertex gathers.
__device__ __forceinline__ void tri_fetch(const float4* __restrict__ tris, uint32_t t, f3* p) {
    const float4* q = tris + 3 * (size_t)t;
    const float4 a = __ldg(q), b = __ldg(q + 1), c = __ldg(q + 2);
    p[0] = mk(a.x, a.y, a.z); p[1] = mk(b.x, b.y, b.z); p[2] = mk(c.x, c.y, c.z);
}
__device__ __forceinline__ void tri_bbox(const f3* p, f3* lo, f3* hi) {
    f3 a = mk(FLT_MAX, FLT_MAX, FLT_MAX), b = mk(-FLT_MAX, -FLT_MAX, -FLT_MAX);
#pragma unroll
    for (int i = 0; i < 3; ++i) { a = vmin(a, p[i]); b = vmax(b, p[i]); }
    *lo = a; *hi = b;
}

struct CRange { int32_t lo[3], hi[3]; };

// bbox -> clamped cell range, UniformGridBuildKernels.h:56-73 (extents clamped at zero)
__device__ __forceinline__ uint32_t cell_range(f3 lo, f3 hi, f3 origin, const float* rcp, const int32_t* res, CRange* r) {
    f3 a = sub(lo, origin), b = sub(hi, origin);
    float af[3] = {a.x * rcp[0], a.y * rcp[1], a.z * rcp[2]};
    float bf[3] = {b.x * rcp[0] + 1.0f, b.y * rcp[1] + 1.0f, b.z * rcp[2] + 1.0f};
    uint32_t n = 1;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        r->lo[k] = max(0, f2i(af[k]));
        r->hi[k] = min(res[k], f2i(bf[k]));
        int32_t e = r->hi[k] - r->lo[k];
        n *= (uint32_t)(e > 0 ? e : 0);
    }
    return n;
}

// ---------------------------------------------------------------------------------
// PCG32 (M.E. O'Neill 2014, pcg32_random_r / pcg32_srandom_r)
struct Pcg32 { uint64_t state, inc; };
__device__ __forceinline__ uint32_t pcg_next(Pcg32& r) {
    uint64_t old = r.state;
    r.state = old * 6364136223846793005ULL + r.inc;
    uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = (uint32_t)(old >> 59u);
    return (xs >> rot) | (xs << ((0u - rot) & 31u));
}
__device__ __forceinline__ void pcg_seed(Pcg32& r, uint64_t initstate, uint64_t initseq) {
    r.state = 0u; r.inc = (initseq << 1u) | 1u;
    pcg_next(r); r.state += initstate; pcg_next(r);
}
__device__ __forceinline__ float pcg_float(Pcg32& r) { return (float)(pcg_next(r) >> 8) * (1.0f / 16777216.0f); }

// Advancing a PCG32 state n steps: the LCG's closed form state * a^n + inc * (1 + a + ... +
// a^(n-1)) (mod 2^64), so a pixel's AO sample k reaches its draws 2k and 2k + 1 in one
// multiply-add instead of 2k steps (the same state as stepping: integer arithmetic).
__host__ __device__ constexpr uint64_t pcg_pow(uint32_t n) {
    uint64_t a = 1u;
    for (uint32_t i = 0; i < n; ++i) a *= 6364136223846793005ULL;
    return a;
}
__host__ __device__ constexpr uint64_t pcg_geo(uint32_t n) {
    uint64_t g = 0u, a = 1u;
    for (uint32_t i = 0; i < n; ++i) { g += a; a *= 6364136223846793005ULL; }
    return g;
}
constexpr int kPcgJumps = 16;   // even step counts 0, 2, ..., 30 (AO samples 0..15)
__constant__ const uint64_t kPcgJumpA[kPcgJumps] = {
    pcg_pow(0), pcg_pow(2), pcg_pow(4), pcg_pow(6), pcg_pow(8), pcg_pow(10), pcg_pow(12), pcg_pow(14),
    pcg_pow(16), pcg_pow(18), pcg_pow(20), pcg_pow(22), pcg_pow(24), pcg_pow(26), pcg_pow(28), pcg_pow(30)};
__constant__ const uint64_t kPcgJumpG[kPcgJumps] = {
    pcg_geo(0), pcg_geo(2), pcg_geo(4), pcg_geo(6), pcg_geo(8), pcg_geo(10), pcg_geo(12), pcg_geo(14),
    pcg_geo(16), pcg_geo(18), pcg_geo(20), pcg_geo(22), pcg_geo(24), pcg_geo(26), pcg_geo(28), pcg_geo(30)};
// skip the 2k draws of AO samples 0..k-1
__device__ __forceinline__ void pcg_skip_pairs(Pcg32& r, uint32_t k) {
    if (k < (uint32_t)kPcgJumps) {
        r.state = r.state * kPcgJumpA[k] + r.inc * kPcgJumpG[k];
    } else {
        for (uint32_t j = 0; j < 2u * k; ++j) pcg_next(r);
    }
}

// sin/cos of 2*pi*u, u in [0,1): exact quadrant reduction + Maclaurin series of sin (to
// x^13) and cos (to x^14) on [0, pi/2) in Horner form; truncation error < 7e-10.
__device__ __forceinline__ void sincos2pi(float u, float* s, float* c) {
    float x4 = u * 4.0f;
    int32_t q = f2i(x4);
    float r = x4 - (float)q;
    float a = r * 1.57079632679489661923f;
    float a2 = a * a;
    float sn = a * (1.0f + a2 * (-0.166666667f + a2 * (0.00833333333f + a2 * (-0.000198412698f +
               a2 * (2.75573192e-06f + a2 * (-2.50521084e-08f + a2 * 1.60590438e-10f))))));
    float cs = 1.0f + a2 * (-0.5f + a2 * (0.0416666667f + a2 * (-0.00138888889f + a2 * (2.48015873e-05f +
               a2 * (-2.75573192e-07f + a2 * (2.08767570e-09f + a2 * -1.14707456e-11f))))));
    switch (q & 3) {
    case 0: *s = sn; *c = cs; break;
    case 1: *s = cs; *c = -sn; break;
    case 2: *s = -sn; *c = -cs; break;
    default: *s = -cs; *c = sn; break;
    }
}

// Natural logarithm of a positive normal float: x = m * 2^e with m in [sqrt(1/2), sqrt(2)),
// ln m = 2 atanh(s), s = (m - 1) / (m + 1), from the series 2 (s + s^3/3 + ... + s^11/11)
// (|s| <= 0.1716, truncation error < 1e-10), plus e ln 2.  The same binary32 operations on
// the host and the device.
__host__ __device__ __forceinline__ float log_series(float x) {
    uint32_t b;
#ifdef __CUDA_ARCH__
    b = __float_as_uint(x);
#else
    __builtin_memcpy(&b, &x, 4);
#endif
    int32_t e = (int32_t)((b >> 23) & 0xFFu) - 127;
    b = (b & 0x7FFFFFu) | 0x3F800000u;
    float m;
#ifdef __CUDA_ARCH__
    m = __uint_as_float(b);
#else
    __builtin_memcpy(&m, &b, 4);
#endif
    if (m > 1.41421356f) { m = m * 0.5f; e += 1; }
    const float sv = (m - 1.0f) / (m + 1.0f);
    const float s2 = sv * sv;
    const float lm = sv * (2.0f + s2 * (0.666666667f + s2 * (0.4f + s2 * (0.285714286f + s2 * (0.222222222f +
                     s2 * 0.181818182f)))));
    return lm + (float)e * 0.693147181f;
}

// Orthonormal basis, Duff et al., JCGT 6(1) 2017
__device__ __forceinline__ void onb(f3 n, f3* t, f3* b) {
    float sg = copysignf(1.0f, n.z);
    float a = -1.0f / (sg + n.z);
    float bb = n.x * n.y * a;
    *t = mk(1.0f + sg * n.x * n.x * a, sg * bb, -sg * n.x);
    *b = mk(bb, sg + n.y * n.y * a, -n.y);
}

// cosine-weighted hemisphere direction (HemisphereSamplers.hpp:54-72)
__device__ __forceinline__ f3 cosine_dir(f3 n, float u1, float u2) {
    float sn, cs;
    sincos2pi(u1, &sn, &cs);
    float r = sqrtf(1.0f - u2);
    float lx = cs * r, ly = sn * r, lz = sqrtf(u2);
    f3 t, b;
    onb(n, &t, &b);
    f3 w;
    w.x = n.x * lz + t.x * lx + b.x * ly;
    w.y = n.y * lz + t.y * lx + b.y * ly;
    w.z = n.z * lz + t.z * lx + b.z * ly;
    return normalize(w);
}

}  // namespace hr
