// trace.cu -- grid traversal (uniform and two-level 3D-DDA), Moller-Trumbore
// intersection and the primary / ambient-occlusion / path-tracing integrators.
//
// Reference path (javorkk/happyray):
//   uniform DDA            src/RT/Algorithm/UGridTraverser.h:44-177
//   two-level DDA          src/RT/Algorithm/TLGridTraverser.h:45-354
//   intersector            src/RT/Algorithm/RayTriangleIntersector.h:38-92
//   trace kernel           src/RT/Algorithm/RayTracingKernels.h:47-152
//   camera                 src/RT/Primitive/Camera.h:35-72
//   primary shading        src/RT/Integrator/SimpleIntegrator.h:41-126
//   ambient occlusion      src/RT/Integrator/AOIntegrator.h:64-191, 234-351; RayGenerators.h:286-342
//   path tracing           src/RT/Integrator/PathTracer.h:41-372
//
// Differences in arithmetic (all deterministic, bit-identical to the oracle):
//   * rays keep the direction and its IEEE reciprocal; the intersector and the entry
//     points use the direction itself instead of re-deriving it with __fdividef;
//   * primary ray directions are normalised, so t is a distance;
//   * no fast-math: IEEE division / square root, no FMA contraction.
//
// The traversal itself (warp-synchronous DDA + intersection) lives in traverse.cuh.
#include "traverse.cuh"

#include <type_traits>

#ifndef HR_AO_REFILL_MIN
#define HR_AO_REFILL_MIN 12   // idle lanes that make k_ao_samples_tl refill
#endif
#ifndef HR_AO_PRIMARY_REFILL_MIN
#define HR_AO_PRIMARY_REFILL_MIN 32   // idle lanes that make k_ao_primary_tl refill (> 32: k_ao_primary)
#endif
#ifndef HR_AO_LEAF_STEPS
#define HR_AO_LEAF_STEPS 6   // AO camera and sample rays: empty leaves stepped over per warp step
#endif
#ifndef HR_TRACE_MIN_BLOCKS
#define HR_TRACE_MIN_BLOCKS 8   // blocks of kTT per SM the ray kernels' register budget must allow (8: 64 registers)
#endif

namespace hr {

namespace {

template <int KIND, bool STATS>
__global__ __launch_bounds__(kTT, HR_TRACE_MIN_BLOCKS) void k_trace_rays(Scene s, const float* __restrict__ org, const float* __restrict__ dir,
                                                    uint32_t n, int32_t* __restrict__ oid, float* __restrict__ ot,
                                                    float* __restrict__ ou, float* __restrict__ ov,
                                                    uint32_t* __restrict__ stats) {
    const G g = load_g(s.desc);
    gate_scene(s);
    const uint32_t nl = round32(n);
    for (uint32_t i = blockIdx.x * kTT + threadIdx.x; i < nl; i += gridDim.x * kTT) {
        const bool valid = i < n;
        f3 o = mk(0.0f, 0.0f, 0.0f), d = mk(1.0f, 0.0f, 0.0f);
        if (valid) {
            o = mk(__ldg(org + 3 * (size_t)i), __ldg(org + 3 * (size_t)i + 1), __ldg(org + 3 * (size_t)i + 2));
            d = mk(__ldg(dir + 3 * (size_t)i), __ldg(dir + 3 * (size_t)i + 1), __ldg(dir + 3 * (size_t)i + 2));
        }
        Hit h;
        trace_one<KIND, false, STATS>(s, g, o, d, FLT_MAX, h, valid);
        if (valid) {
            if (h.hit) refine_uv(s, h.tri, o, d, &h.u, &h.v);
            oid[i] = h.hit ? (int32_t)h.tri : -1;
            ot[i] = h.hit ? h.t : FLT_MAX;
            ou[i] = h.u;
            ov[i] = h.v;
            if (STATS) { stats[2 * (size_t)i] = h.cells; stats[2 * (size_t)i + 1] = h.tests; }
        }
    }
}

template <int KIND, bool STATS>
__global__ __launch_bounds__(kTT, HR_TRACE_MIN_BLOCKS) void k_trace_primary(Scene s, Cam cam, int32_t* __restrict__ oid,
                                                       float* __restrict__ ot, float* __restrict__ ou,
                                                       float* __restrict__ ov, uint32_t* __restrict__ stats) {
    const G g = load_g(s.desc);
    gate_scene(s);
    const uint32_t slots = tile_slots(cam);
    const f3 o = mk(cam.pos[0], cam.pos[1], cam.pos[2]);
    for (uint32_t slot = blockIdx.x * kTT + threadIdx.x; slot < slots; slot += gridDim.x * kTT) {
        uint32_t i;
        const bool valid = tile_pixel(cam, slot, &i);
        Hit h;
        const f3 d = valid ? primary_dir(cam, i) : mk(1.0f, 0.0f, 0.0f);
        trace_one<KIND, false, STATS>(s, g, o, d, FLT_MAX, h, valid);
        if (valid) {
            if (h.hit) refine_uv(s, h.tri, o, d, &h.u, &h.v);
            oid[i] = h.hit ? (int32_t)h.tri : -1;
            ot[i] = h.hit ? h.t : FLT_MAX;
            ou[i] = h.u;
            ov[i] = h.v;
            if (STATS) { stats[2 * (size_t)i] = h.cells; stats[2 * (size_t)i + 1] = h.tests; }
        }
    }
}

// the ray-file form of render mode 0 (SimpleRayTraverser::integrate,
// SimpleRayTraverser.h:166-180): ray i traced (closest hit) and shaded by simpleShade into
// pixel i, progressive blend
template <int KIND>
__global__ __launch_bounds__(kTT, HR_TRACE_MIN_BLOCKS) void k_render_rays(Scene s, const float* __restrict__ org,
                                                                     const float* __restrict__ dir, uint32_t n,
                                                                     int32_t image_id, float* __restrict__ fb,
                                                                     unsigned long long* counter) {
    const G g = load_g(s.desc);
    gate_scene(s);
    const uint32_t nl = round32(n);
    for (uint32_t i = blockIdx.x * kTT + threadIdx.x; i < nl; i += gridDim.x * kTT) {
        const bool valid = i < n;
        f3 o = mk(0.0f, 0.0f, 0.0f), d = mk(1.0f, 0.0f, 0.0f);
        if (valid) {
            o = mk(__ldg(org + 3 * (size_t)i), __ldg(org + 3 * (size_t)i + 1), __ldg(org + 3 * (size_t)i + 2));
            d = mk(__ldg(dir + 3 * (size_t)i), __ldg(dir + 3 * (size_t)i + 1), __ldg(dir + 3 * (size_t)i + 2));
        }
        Hit h;
        trace_one<KIND, false, false>(s, g, o, d, FLT_MAX, h, valid);
        if (valid) {
            float rgb[3];
            simple_shade(s, h.hit, h.tri, o, d, rgb);
            for (int k = 0; k < 3; ++k) fb[3 * (size_t)i + k] = blend(fb[3 * (size_t)i + k], rgb[k], image_id);
        }
        add_rays<false>(counter, false, valid ? 1u : 0u);
    }
}

template <int KIND>
__global__ __launch_bounds__(kTT, HR_TRACE_MIN_BLOCKS) void k_occluded(Scene s, const float* __restrict__ org, const float* __restrict__ dir,
                                                  const float* __restrict__ tmax, uint32_t n, uint8_t* __restrict__ occ) {
    const G g = load_g(s.desc);
    gate_scene(s);
    const uint32_t nl = round32(n);
    for (uint32_t i = blockIdx.x * kTT + threadIdx.x; i < nl; i += gridDim.x * kTT) {
        const bool valid = i < n;
        f3 o = mk(0.0f, 0.0f, 0.0f), d = mk(1.0f, 0.0f, 0.0f);
        float tm = 0.0f;
        if (valid) {
            o = mk(org[3 * (size_t)i], org[3 * (size_t)i + 1], org[3 * (size_t)i + 2]);
            d = mk(dir[3 * (size_t)i], dir[3 * (size_t)i + 1], dir[3 * (size_t)i + 2]);
            tm = tmax[i];
        }
        Hit h;
        trace_one<KIND, true, false>(s, g, o, d, tm, h, valid);
        if (valid) occ[i] = h.hit ? 1 : 0;
    }
}

// mode 0: primary rays with barycentric false colour (SimpleIntegrator.h:41-126)
template <int KIND, bool STATS>
__global__ __launch_bounds__(kTT, HR_TRACE_MIN_BLOCKS) void k_render_primary(Scene s, Cam cam, int32_t image_id, uint64_t seed,
                                                        float* __restrict__ fb, unsigned long long* counter) {
    const G g = load_g(s.desc);
    gate_scene(s);
    const uint32_t slots = tile_slots(cam);
    const f3 o = mk(cam.pos[0], cam.pos[1], cam.pos[2]);
    for (uint32_t slot = blockIdx.x * kTT + threadIdx.x; slot < slots; slot += gridDim.x * kTT) {
        uint32_t i;
        const bool valid = tile_pixel(cam, slot, &i);
        const f3 d = valid ? primary_sample_dir(cam, i, image_id, seed) : mk(1.0f, 0.0f, 0.0f);
        Hit h;
        trace_one<KIND, false, STATS>(s, g, o, d, FLT_MAX, h, valid);
        if (valid) {
            float rgb[3];
            simple_shade(s, h.hit, h.tri, o, d, rgb);
            fb[3 * (size_t)i] = blend(fb[3 * (size_t)i], rgb[0], image_id);
            fb[3 * (size_t)i + 1] = blend(fb[3 * (size_t)i + 1], rgb[1], image_id);
            fb[3 * (size_t)i + 2] = blend(fb[3 * (size_t)i + 2], rgb[2], image_id);
        }
        add_rays<STATS>(counter, false, valid ? 1u : 0u, h.cells, h.tests);
    }
}

// mode 3, ambient occlusion (AOIntegrator.h:234-351: primary trace, AO rays, shading), as
// a wavefront of three kernels:
//   k_ao_primary  camera rays in pixel tiles; misses are shaded at once, hit pixels are
//                 appended (warp-aggregated) to a queue with their t and triangle;
//   k_ao_samples  one thread per (hit pixel, sample): AO ray generation as
//                 RayGenerators.h:286-342 with the configured radius and PCG32 stream of
//                 the pixel (sample k uses draws 2k and 2k+1), any-hit traversal, and the
//                 unoccluded count of the pixel (match_any-aggregated atomics);
//   k_ao_finish   visibility = unoccluded / samples, progressive blend (AOIntegrator.h:168-175).
template <int KIND, bool STATS>
__global__ __launch_bounds__(kTT, HR_TRACE_MIN_BLOCKS) void k_ao_primary(Scene s, Cam cam, int32_t image_id, float* __restrict__ fb,
                                                    float* __restrict__ hit_t, uint32_t* __restrict__ hit_tri,
                                                    uint32_t* __restrict__ unocc, uint32_t* __restrict__ queue,
                                                    uint32_t* qcount, unsigned long long* counter) {
    const G g = load_g(s.desc);
    gate_scene(s);
    const uint32_t slots = tile_slots(cam);
    const f3 o = mk(cam.pos[0], cam.pos[1], cam.pos[2]);
    const uint32_t lane = threadIdx.x & 31u, lt = (1u << lane) - 1u;
    for (uint32_t slot = blockIdx.x * kTT + threadIdx.x; slot < slots; slot += gridDim.x * kTT) {
        uint32_t pix;
        const bool valid = tile_pixel(cam, slot, &pix);
        Hit h;
        trace_one<KIND, false, STATS>(s, g, o, valid ? primary_dir(cam, pix) : mk(1.0f, 0.0f, 0.0f), FLT_MAX, h, valid);
        const bool hit = valid && h.hit;
        if (hit) {
            hit_t[pix] = h.t;
            hit_tri[pix] = h.tri;
            unocc[pix] = 0u;
        } else if (valid) {
            const float val = blend(fb[3 * (size_t)pix], 1.0f, image_id);
            fb[3 * (size_t)pix] = val;
            fb[3 * (size_t)pix + 1] = val;
            fb[3 * (size_t)pix + 2] = val;
        }
        const uint32_t m = __ballot_sync(kFullMask, hit);
        if (m) {
            const int leader = __ffs(m) - 1;
            uint32_t base = 0;
            if ((int)lane == leader) base = atomicAdd(qcount, (uint32_t)__popc(m));
            base = __shfl_sync(kFullMask, base, leader);
            if (hit) queue[base + __popc(m & lt)] = pix;
        }
        add_rays<STATS>(counter, false, valid ? 1u : 0u, h.cells, h.tests);
    }
}

template <int KIND, bool STATS>
__global__ __launch_bounds__(kTT, HR_TRACE_MIN_BLOCKS) void k_ao_samples(Scene s, Cam cam, int32_t spp, float alpha_frac, float alpha_abs,
                                                    uint64_t seed, int32_t image_id, const float* __restrict__ hit_t,
                                                    const uint32_t* __restrict__ hit_tri,
                                                    const uint32_t* __restrict__ queue, const uint32_t* qcount,
                                                    uint32_t* __restrict__ unocc, unsigned long long* counter) {
    const G g = load_g(s.desc);
    gate_scene(s);
    float alpha = alpha_abs;
    if (!(alpha > 0.0f)) {
        const f3 dd = mk(g.bmax[0] - g.bmin[0], g.bmax[1] - g.bmin[1], g.bmax[2] - g.bmin[2]);
        alpha = alpha_frac * sqrtf(dot(dd, dd));
    }
    const float off = 0.01f * alpha;
    const f3 o = mk(cam.pos[0], cam.pos[1], cam.pos[2]);
    const uint32_t nitems = *qcount * (uint32_t)spp;
    const uint32_t nloop = round32(nitems);
    for (uint32_t item = blockIdx.x * kTT + threadIdx.x; item < nloop; item += gridDim.x * kTT) {
        const bool valid = item < nitems;
        uint32_t pix = 0xffffffffu;
        f3 ao = mk(0.0f, 0.0f, 0.0f), w = mk(1.0f, 0.0f, 0.0f);
        if (valid) {
            const uint32_t q = item / (uint32_t)spp, k = item % (uint32_t)spp;
            pix = queue[q];
            const f3 d = primary_dir(cam, pix);
            const float t = hit_t[pix];
            const f3 p = mk(o.x + t * d.x, o.y + t * d.y, o.z + t * d.z);
            const f3 nrm = face_normal(s, hit_tri[pix], d);
            Pcg32 rng;
            pcg_seed(rng, ((uint64_t)(uint32_t)image_id << 32) | pix, seed);
            pcg_skip_pairs(rng, k);
            const float u1 = pcg_float(rng), u2 = pcg_float(rng);
            w = cosine_dir(nrm, u1, u2);
            ao = mk(p.x + off * w.x, p.y + off * w.y, p.z + off * w.z);
        }
        Hit hs;
        trace_one<KIND, true, STATS>(s, g, ao, w, alpha, hs, valid);
        const bool free = valid && !hs.hit;
        const uint32_t peers = __match_any_sync(kFullMask, pix);
        const uint32_t nfree = __popc(__ballot_sync(kFullMask, free) & peers);
        if (valid && nfree && (int)(threadIdx.x & 31u) == __ffs(peers) - 1) atomicAdd(unocc + pix, nfree);
        add_rays<STATS>(counter, true, valid ? 1u : 0u, hs.cells, hs.tests);
    }
}

// AO camera rays on a two-level grid with lanes refilled inside the traversal loop: once
// HR_AO_PRIMARY_REFILL_MIN lanes are done (their pixels shaded or queued as k_ao_primary
// does), they take that many consecutive pixel slots of the tile order from the pool.
template <bool STATS>
__global__ __launch_bounds__(kTT, HR_TRACE_MIN_BLOCKS) void k_ao_primary_tl(Scene s, Cam cam, int32_t image_id,
                                                              float* __restrict__ fb, float* __restrict__ hit_t,
                                                              uint32_t* __restrict__ hit_tri, uint32_t* __restrict__ unocc,
                                                              uint32_t* __restrict__ queue, uint32_t* qcount,
                                                              unsigned long long* counter, uint32_t* work) {
    const G g = load_g(s.desc);
    gate_scene(s);
    const uint32_t slots = tile_slots(cam);
    const f3 o = mk(cam.pos[0], cam.pos[1], cam.pos[2]);
    const uint32_t lane = threadIdx.x & 31u, lt = (1u << lane) - 1u;
    TL q;
    Hit h;
    h.t = FLT_MAX; h.u = 0.0f; h.v = 0.0f; h.tri = 0; h.hit = false; h.cells = 0; h.tests = 0;
    f3 d = mk(1.0f, 0.0f, 0.0f);
    uint32_t pix = 0, nrays = 0, ncells = 0, ntests = 0;
    bool has = false, valid = false, active = false, dry = false;
    while (true) {
        const uint32_t need = __ballot_sync(kFullMask, !has);
        if (need && !dry && (__popc(need) >= HR_AO_PRIMARY_REFILL_MIN || need == kFullMask ||
                             !__any_sync(kFullMask, active))) {   // warp-uniform
            const int leader = __ffs(need) - 1;
            uint32_t base = 0;
            if ((int)lane == leader) base = atomicAdd(work, (uint32_t)__popc(need));
            base = __shfl_sync(kFullMask, base, leader);
            if (base + (uint32_t)__popc(need) >= slots) dry = true;
            const uint32_t slot = base + __popc(need & lt);
            if (!has && slot < slots) {
                has = true;
                valid = tile_pixel(cam, slot, &pix);
                h.t = FLT_MAX; h.u = 0.0f; h.v = 0.0f; h.tri = 0; h.hit = false; h.cells = 0; h.tests = 0;
                active = false;
                if (valid) {
                    d = primary_dir(cam, pix);
                    if (s.ntri != 0u) active = tl_setup<STATS>(q, s, g, o, d, h);
                }
            }
        }
        if (!__any_sync(kFullMask, has)) break;   // the pool is dry and no ray is in flight
        uint32_t b = 0, e = 0;
        if (active) {
            const uint2 lr = __ldg(s.leaves + tl_leaf(q));
            b = lr.x; e = lr.y;
            if (STATS) h.cells++;
        }
        const bool done = test_lists<kHitClosest, STATS>(s, o, d, b, e, false, h);
        if (active) active = !done && tl_advance<STATS, false, HR_AO_LEAF_STEPS>(q, s, g, o, d, h);
        const bool fin = has && !active;
        const bool hit = fin && valid && h.hit;
        if (hit) {
            hit_t[pix] = h.t;
            hit_tri[pix] = h.tri;
            unocc[pix] = 0u;
        } else if (fin && valid) {
            const float val = blend(fb[3 * (size_t)pix], 1.0f, image_id);
            fb[3 * (size_t)pix] = val;
            fb[3 * (size_t)pix + 1] = val;
            fb[3 * (size_t)pix + 2] = val;
        }
        const uint32_t m = __ballot_sync(kFullMask, hit);
        if (m) {
            const int leader = __ffs(m) - 1;
            uint32_t qb = 0;
            if ((int)lane == leader) qb = atomicAdd(qcount, (uint32_t)__popc(m));
            qb = __shfl_sync(kFullMask, qb, leader);
            if (hit) queue[qb + __popc(m & lt)] = pix;
        }
        if (fin) {
            if (valid) {
                nrays += 1;
                ncells += h.cells;
                ntests += h.tests;
            }
            has = false;
        }
    }
    add_rays<STATS>(counter, false, nrays, ncells, ntests);
}

// AO samples on a two-level grid with lanes refilled inside the traversal loop: a lane
// whose ray is done (occluded, or out of the grid or past the radius) retires it and
// waits; once HR_AO_REFILL_MIN lanes wait (or no ray is left in flight) they take the next
// (hit pixel, sample) items from the pool together, so a warp keeps most of its lanes
// busy until the pool runs dry instead of waiting for its longest ray, and the divergent
// ray set-up runs for many lanes at once.  Per ray the generation, traversal and result
// are those of k_ao_samples.
template <bool STATS>
__global__ __launch_bounds__(kTT, HR_TRACE_MIN_BLOCKS) void k_ao_samples_tl(Scene s, Cam cam, int32_t spp, float alpha_frac,
                                                              float alpha_abs, uint64_t seed, int32_t image_id,
                                                              const float* __restrict__ hit_t,
                                                              const uint32_t* __restrict__ hit_tri,
                                                              const uint32_t* __restrict__ queue, const uint32_t* qcount,
                                                              uint32_t* __restrict__ unocc, unsigned long long* counter,
                                                              uint32_t* work) {
    const G g = load_g(s.desc);
    gate_scene(s);
    float alpha = alpha_abs;
    if (!(alpha > 0.0f)) {
        const f3 dd = mk(g.bmax[0] - g.bmin[0], g.bmax[1] - g.bmin[1], g.bmax[2] - g.bmin[2]);
        alpha = alpha_frac * sqrtf(dot(dd, dd));
    }
    const float off = 0.01f * alpha;
    const f3 cpos = mk(cam.pos[0], cam.pos[1], cam.pos[2]);
    const uint32_t nitems = *qcount * (uint32_t)spp;
    const uint32_t lane = threadIdx.x & 31u, lt = (1u << lane) - 1u;
    TL q;
    Hit h;
    h.t = alpha; h.u = 0.0f; h.v = 0.0f; h.tri = 0; h.hit = false; h.cells = 0; h.tests = 0;
    f3 o = mk(0.0f, 0.0f, 0.0f), w = mk(1.0f, 0.0f, 0.0f);
    uint32_t pix = 0xffffffffu, nrays = 0, ncells = 0, ntests = 0;
    bool has = false, active = false, dry = s.ntri == 0u;
    while (true) {
        const uint32_t need = __ballot_sync(kFullMask, !has);
        if (need && !dry && (__popc(need) >= HR_AO_REFILL_MIN || need == kFullMask ||
                             !__any_sync(kFullMask, active))) {   // warp-uniform
            const int leader = __ffs(need) - 1;
            uint32_t base = 0;
            if ((int)lane == leader) base = atomicAdd(work, (uint32_t)__popc(need));
            base = __shfl_sync(kFullMask, base, leader);
            if (base + (uint32_t)__popc(need) >= nitems) dry = true;
            const uint32_t item = base + __popc(need & lt);
            if (!has && item < nitems) {
                has = true;
                const uint32_t qi = item / (uint32_t)spp, k = item % (uint32_t)spp;
                pix = queue[qi];
                const f3 d = primary_dir(cam, pix);
                const float t = hit_t[pix];
                const f3 p = mk(cpos.x + t * d.x, cpos.y + t * d.y, cpos.z + t * d.z);
                const f3 nrm = face_normal(s, hit_tri[pix], d);
                Pcg32 rng;
                pcg_seed(rng, ((uint64_t)(uint32_t)image_id << 32) | pix, seed);
                pcg_skip_pairs(rng, k);
                const float u1 = pcg_float(rng), u2 = pcg_float(rng);
                w = cosine_dir(nrm, u1, u2);
                o = mk(p.x + off * w.x, p.y + off * w.y, p.z + off * w.z);
                h.t = alpha; h.hit = false; h.cells = 0; h.tests = 0;
                active = tl_setup<STATS>(q, s, g, o, w, h);
            }
        }
        if (!__any_sync(kFullMask, has)) break;   // the pool is dry and no ray is in flight
        uint32_t b = 0, e = 0;
        if (active) {
            const uint2 lr = __ldg(s.leaves + tl_leaf(q));
            b = lr.x; e = lr.y;
            if (STATS) h.cells++;
        }
        const bool done = test_lists<kHitAny, STATS>(s, o, w, b, e, true, h);
        if (active) active = !done && tl_advance<STATS, false, HR_AO_LEAF_STEPS>(q, s, g, o, w, h);
        const bool fin = has && !active;
        const uint32_t peers = __match_any_sync(kFullMask, fin ? pix : 0xffffffffu);
        const uint32_t nfree = __popc(__ballot_sync(kFullMask, fin && !h.hit) & peers);
        if (fin && nfree && (int)lane == __ffs(peers) - 1) atomicAdd(unocc + pix, nfree);
        if (fin) {
            nrays += 1;
            ncells += h.cells;
            ntests += h.tests;
            has = false;
        }
    }
    add_rays<STATS>(counter, true, nrays, ncells, ntests);
}

__global__ void k_ao_finish(const uint32_t* __restrict__ queue, const uint32_t* qcount, const uint32_t* __restrict__ unocc,
                            int32_t spp, int32_t image_id, float* __restrict__ fb) {
    const uint32_t n = *qcount;
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const uint32_t pix = queue[q];
        const float vis = (float)unocc[pix] / (float)spp;
        const float val = blend(fb[3 * (size_t)pix], vis, image_id);
        fb[3 * (size_t)pix] = val;
        fb[3 * (size_t)pix + 1] = val;
        fb[3 * (size_t)pix + 2] = val;
    }
}

#ifndef HR_AO_REFILL
#define HR_AO_REFILL 1   // two-level AO samples by k_ao_samples_tl (lanes refilled in the traversal loop)
#endif
#ifndef HR_PT_SMEM_STATE
#define HR_PT_SMEM_STATE 1   // path state in shared memory (registers left to the traversal)
#endif
#ifndef HR_PT_MIN_BLOCKS
#define HR_PT_MIN_BLOCKS 7   // blocks of kTT per SM the path tracer's register budget must allow (7: 72 registers)
#endif

// mode 1/2: path tracing with next-event estimation (PathTracer.h:41-372 structure), one
// path per pixel.  Persistent: each warp takes 32-pixel tiles from *work, and a lane whose
// path ends takes the next pixel at once (path_refill / path_step / path_retire), so lanes
// do not idle through the bounces of their warp's longest path.
template <int KIND, bool STATS>
__global__ __launch_bounds__(kTT, HR_PT_MIN_BLOCKS) void k_render_pt(Scene s, Cam cam, const LightSet* __restrict__ ls, int32_t bounces,
                                                                  float albedo, float eps_frac, uint64_t seed,
                                                                  int32_t image_id, float* __restrict__ fb,
                                                                  unsigned long long* counter, uint32_t* work) {
    const G g = load_g(s.desc);
    gate_scene(s);
    const PtConsts k = pt_consts(g, ls, bounces, albedo, eps_frac);
    const uint32_t ntiles = tile_slots(cam) >> 5;
    const uint32_t lane = threadIdx.x & 31u;
#if HR_PT_SMEM_STATE
    // the path state lives in shared memory, so the traversal has the registers to itself
    __shared__ __align__(16) unsigned char s_lanes[sizeof(PathLane) * kTT];
    PathLane& ln = reinterpret_cast<PathLane*>(s_lanes)[threadIdx.x];
    ln.pix = 0;
    ln.sample = 0;
    ln.val = 0.0f;
    ln.has = false;
#else
    PathLane ln;
#endif
    PtCounts n;
    uint32_t tile = 0, next = 32u;
    bool more = true;
    while (true) {
        while (more) {
            if (next >= 32u) {
                uint32_t t = 0;
                if (lane == 0) t = atomicAdd(work, 1u);
                t = __shfl_sync(kFullMask, t, 0);
                if (t >= ntiles) {
                    more = false;
                    break;
                }
                tile = t;
                next = 0;
            }
            if (path_refill(ln, cam, tile, &next, image_id, seed, fb) == 0u) break;
        }
        if (!__any_sync(kFullMask, ln.has)) break;
        const bool cont = path_step<KIND, STATS>(s, g, k, ln.p, ln.has, n);
        path_retire(ln, cont, cam, image_id, 1, seed, fb);
    }
    add_rays<STATS>(counter, false, n.rays, n.cells, n.tests);
    add_rays<STATS>(counter, true, n.srays, n.scells, n.stests);
}

Scene make_scene(hr_ctx* c) {
    Scene s;
    s.tris = c->tris.as<float4>();
    s.cells = c->g.cells.as<uint2>();
    s.leaves = c->g.leaves.as<uint2>();
    s.prims = c->g.prims.as<uint32_t>();
    s.desc = c->g.desc.as<GridDesc>();
    s.ntri = c->ntri;
    s.kind = c->built_kind;
    // shading normals and materials given for the current mesh
    s.nrm3 = c->nrm_ntri && c->nrm_ntri == c->ntri ? c->tri_nrm.as<float4>() : nullptr;
    s.alb = c->alb_ntri && c->alb_ntri == c->ntri ? c->tri_alb.as<float>() : nullptr;
    s.occ = c->built_kind == kTwoLevel ? c->g.occ.as<uint32_t>() : nullptr;
    s.occ_bit0 = 0;
    return s;
}

Cam make_cam(const hr_ctx* c) {
    Cam k;
    for (int i = 0; i < 3; ++i) {
        k.pos[i] = c->cam.pos[i]; k.tl[i] = c->cam.top_left[i];
        k.sx[i] = c->cam.step_x[i]; k.sy[i] = c->cam.step_y[i];
    }
    k.w = c->cam.w; k.h = c->cam.h;
    return k;
}

int grid_for(const hr_ctx* c, uint32_t n) {
    uint32_t b = (n + kTT - 1) / kTT;
    uint32_t cap = (uint32_t)c->num_sms * 16u;
    return (int)(b < 1 ? 1 : (b > cap ? cap : b));
}

uint32_t slots_for(const hr_ctx* c) {
    return (((uint32_t)c->cam.w + 7u) / 8u) * (((uint32_t)c->cam.h + 3u) / 4u) * 32u;
}

template <int V> using IntC = std::integral_constant<int, V>;
template <bool V> using BoolC = std::integral_constant<bool, V>;

// f(IntC<kind>, BoolC<stats>): picks the kernel instance of the built grid's kind
template <class F>
void by_kind(int32_t kind, bool stats, F&& f) {
    if (kind == kUniform) {
        if (stats) f(IntC<kUniform>{}, BoolC<true>{});
        else f(IntC<kUniform>{}, BoolC<false>{});
    } else {
        if (stats) f(IntC<kTwoLevel>{}, BoolC<true>{});
        else f(IntC<kTwoLevel>{}, BoolC<false>{});
    }
}

}  // namespace

int launch_trace_rays(hr_ctx* c, const float* org, const float* dir, uint32_t n, int32_t* id, float* t, float* u,
                      float* v, uint32_t* stats) {
    if (n == 0) return 0;
    Scene s = make_scene(c);
    c->launches += 1;
    by_kind(s.kind, stats != nullptr, [&](auto K, auto S) {
        k_trace_rays<K(), S()><<<grid_for(c, n), kTT, 0, c->stream>>>(s, org, dir, n, id, t, u, v, stats);
    });
    return cuda_check(c, cudaGetLastError(), "trace_rays launch");
}

int launch_trace_primary(hr_ctx* c, int32_t* id, float* t, float* u, float* v, uint32_t* stats) {
    Scene s = make_scene(c);
    Cam k = make_cam(c);
    const uint32_t n = (uint32_t)k.w * (uint32_t)k.h;
    if (n == 0) return 0;
    c->launches += 1;
    const int gb = grid_for(c, slots_for(c));
    by_kind(s.kind, stats != nullptr, [&](auto K, auto S) {
        k_trace_primary<K(), S()><<<gb, kTT, 0, c->stream>>>(s, k, id, t, u, v, stats);
    });
    return cuda_check(c, cudaGetLastError(), "trace_primary launch");
}

int launch_render_rays(hr_ctx* c, const float* org, const float* dir, uint32_t n, int32_t image_id, float* fb) {
    if (n == 0) return 0;
    c->launches += 1;
    const Scene s = make_scene(c);
    unsigned long long* ctr = c->counters.as<unsigned long long>();
    by_kind(s.kind, false, [&](auto K, auto) {
        k_render_rays<K()><<<grid_for(c, n), kTT, 0, c->stream>>>(s, org, dir, n, image_id, fb, ctr);
    });
    return cuda_check(c, cudaGetLastError(), "render_rays launch");
}

int launch_occluded(hr_ctx* c, const float* org, const float* dir, const float* tmax, uint32_t n, uint8_t* occ) {
    if (n == 0) return 0;
    c->launches += 1;
    const Scene s = make_scene(c);
    by_kind(s.kind, false, [&](auto K, auto) { k_occluded<K()><<<grid_for(c, n), kTT, 0, c->stream>>>(s, org, dir, tmax, n, occ); });
    return cuda_check(c, cudaGetLastError(), "occluded launch");
}

int launch_render(hr_ctx* c, int32_t mode, int32_t image_id, float* d_fb) {
    Scene s = make_scene(c);
    Cam k = make_cam(c);
    const uint32_t n = (uint32_t)k.w * (uint32_t)k.h;
    if (n == 0) return 0;
    unsigned long long* ctr = c->counters.as<unsigned long long>();
    const int gb = grid_for(c, slots_for(c));
    const bool st = c->collect_stats;
    cudaStream_t strm = c->stream;
    auto mark = [&](int i) { if (c->timing && i < 8) cudaEventRecord(c->rev[i], strm); };
    c->nrender_ev = 0;
    switch (mode) {
    case 0:
        c->launches += 1;
        mark(0);
        by_kind(s.kind, st, [&](auto K, auto S) { k_render_primary<K(), S()><<<gb, kTT, 0, strm>>>(s, k, image_id, c->ip.seed, d_fb, ctr); });
        mark(1);
        c->nrender_ev = 2;
        break;
    case 1:
    case 2: {
        const LightSet* l = c->lights_dev.as<LightSet>();
        uint32_t* work = reinterpret_cast<uint32_t*>(ctr + 7);
        int rc;
        if ((rc = cuda_check(c, cudaMemsetAsync(work, 0, sizeof(uint32_t), strm), "tile counter reset"))) return rc;
        c->launches += 1;
        mark(0);
        by_kind(s.kind, st, [&](auto K, auto S) {
            int nb = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_render_pt<K(), S()>, kTT, 0) != cudaSuccess || nb < 1) {
                cudaGetLastError();
                nb = 1;
            }
            const int gp = std::min(gb, nb * c->num_sms);
            k_render_pt<K(), S()><<<gp, kTT, 0, strm>>>(s, k, l, c->ip.pt_bounces, c->ip.albedo, c->ip.ray_eps_frac,
                                                        c->ip.seed, image_id, d_fb, ctr, work);
        });
        mark(1);
        c->nrender_ev = 2;
        break;
    }
    case 3: {
        int rc;
        if ((rc = ensure(c, c->hit_t, sizeof(float) * n)) || (rc = ensure(c, c->hit_tri, sizeof(uint32_t) * n)) ||
            (rc = ensure(c, c->unocc, sizeof(uint32_t) * n)) || (rc = ensure(c, c->queue, sizeof(uint32_t) * n)))
            return rc;
        // word 7: the hit-pixel queue length and the sample pool; word 8: the camera-ray pool
        uint32_t* qcount = reinterpret_cast<uint32_t*>(ctr + 7);
        if ((rc = cuda_check(c, cudaMemsetAsync(qcount, 0, 4 * sizeof(uint32_t), strm), "queue reset"))) return rc;
        const int spp = c->ip.ao_samples;
        c->launches += 3;
        mark(0);
        by_kind(s.kind, st, [&](auto K, auto S) {
            if (HR_AO_PRIMARY_REFILL_MIN <= 32 && K() == kTwoLevel) {
                int nb = 0;
                if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_ao_primary_tl<S()>, kTT, 0) != cudaSuccess ||
                    nb < 1) {
                    cudaGetLastError();
                    nb = 1;
                }
                k_ao_primary_tl<S()><<<std::min(gb, nb * c->num_sms), kTT, 0, strm>>>(
                    s, k, image_id, d_fb, c->hit_t.as<float>(), c->hit_tri.as<uint32_t>(), c->unocc.as<uint32_t>(),
                    c->queue.as<uint32_t>(), qcount, ctr, qcount + 2);
            } else {
                k_ao_primary<K(), S()><<<gb, kTT, 0, strm>>>(s, k, image_id, d_fb, c->hit_t.as<float>(),
                                                             c->hit_tri.as<uint32_t>(), c->unocc.as<uint32_t>(),
                                                             c->queue.as<uint32_t>(), qcount, ctr);
            }
        });
        mark(1);
        const int gs = c->num_sms * 16;
        by_kind(s.kind, st, [&](auto K, auto S) {
            if (HR_AO_REFILL && K() == kTwoLevel) {
                int nb = 0;
                if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_ao_samples_tl<S()>, kTT, 0) != cudaSuccess ||
                    nb < 1) {
                    cudaGetLastError();
                    nb = 1;
                }
                k_ao_samples_tl<S()><<<nb * c->num_sms, kTT, 0, strm>>>(
                    s, k, spp, c->ip.ao_radius_frac, c->ip.ao_radius_abs, c->ip.seed, image_id, c->hit_t.as<float>(),
                    c->hit_tri.as<uint32_t>(), c->queue.as<uint32_t>(), qcount, c->unocc.as<uint32_t>(), ctr,
                    qcount + 1);
            } else {
                k_ao_samples<K(), S()><<<gs, kTT, 0, strm>>>(s, k, spp, c->ip.ao_radius_frac, c->ip.ao_radius_abs,
                                                             c->ip.seed, image_id, c->hit_t.as<float>(),
                                                             c->hit_tri.as<uint32_t>(), c->queue.as<uint32_t>(), qcount,
                                                             c->unocc.as<uint32_t>(), ctr);
            }
        });
        mark(2);
        k_ao_finish<<<c->num_sms * 4, 256, 0, strm>>>(c->queue.as<uint32_t>(), qcount, c->unocc.as<uint32_t>(), spp,
                                                      image_id, d_fb);
        mark(3);
        c->nrender_ev = 4;
        break;
    }
    default:
        return set_error(c, 1, "render: unknown mode %d", mode);
    }
    return cuda_check(c, cudaGetLastError(), "render launch");
}

}  // namespace hr
