// jobs.cu -- persistent rendering of many jobs in one launch (batched and served forms).
//
// A job is one grid (two-level), a camera or a list of rays, an integrator and an output:
//   kJobPrimary  camera rays (mode 0 pixel samplers), simpleShade (SimpleIntegrator.h:41-126)
//   kJobAO       camera rays + spp AO samples per hit (AOIntegrator.h:234-351)
//   kJobPath     spp paths per pixel (PathTracer.h:41-372 structure), progressive blend
//   kJobRays     closest hit of a ray list (SimpleRayTraverser.h:168-261 query form)
// The reference runs one integrator over one scene per launch sequence; here the warps of
// one persistent launch take 32-pixel (32-ray) tiles of any job from a global work
// counter.  Every job's output is bit-identical to the per-scene kernels of trace.cu for
// the same grid, camera, samples, seed and image ids: the per-pixel random streams, ray
// construction and traversal are the same functions.
#include "traverse.cuh"
#include "../../include/happyray.h"

// Empty top cells a path or shadow ray of a job walks per warp step: fewer than in the
// per-scene path tracer (HR_PT_SEEK_STEPS), whose warps hold one image's paths; a job
// warp's lanes come from tiles of many requests and scenes (measured on the served
// workload: traversal per 1000 requests 1.77 s at 2, 1.86-1.90 s at 3).
#ifndef HR_JOB_PT_SEEK_STEPS
#define HR_JOB_PT_SEEK_STEPS 2
#endif

namespace hr {
namespace {

constexpr int kJobTT = 256;   // largest block of the persistent kernel
#ifndef HR_JOB_MIN_BLOCKS
#define HR_JOB_MIN_BLOCKS 3    // blocks of kJobTT per SM the register budget must allow (3: 80 registers)
#endif
#ifndef HR_JOB_PT_SMEM_STATE
#define HR_JOB_PT_SMEM_STATE 1   // path-tracing instance: path state in shared memory
#endif
#ifndef HR_JOB_PT_MIN_BLOCKS
#define HR_JOB_PT_MIN_BLOCKS 4   // the same for the path-tracing instance (4: 64 registers)
#endif

// position of the q-th (0-based) set bit of m; m has more than q set bits
__device__ __forceinline__ uint32_t nth_set_bit(uint32_t m, uint32_t q) {
    uint32_t pos = 0;
#pragma unroll
    for (uint32_t step = 16; step > 0; step >>= 1) {
        const uint32_t c = __popc(m & ((1u << step) - 1u));
        if (q >= c) { q -= c; m >>= step; pos += step; }
    }
    return pos;
}

// Per-warp state of the tile being rendered, in shared memory: the job's scene, grid and
// integrator parameters (which the per-scene kernels get from their launch parameters)
// and the hit points of the tile's camera rays, which the AO rounds read by lane.
struct TileCtx {
    Scene s;
    G g;
    Cam cam;
    PtConsts pk;
    float* fb;
    const float* org;
    const float* dir;
    int32_t* out_id;
    float *out_t, *out_u, *out_v;
    uint64_t seed;
    float alpha, off;
    uint32_t spp;
    int32_t image_id, mode;
    float px[32], py[32], pz[32], nx[32], ny[32], nz[32];
    uint32_t pix[32];
};

__device__ __forceinline__ void load_tile_ctx(TileCtx& T, const Job* __restrict__ J) {
    T.s.tris = J->tris;
    const uint32_t coff = J->cells_offset ? __ldg(J->cells_offset) : 0u;
    T.s.cells = J->cells + coff;
    T.s.occ = J->occ;
    T.s.occ_bit0 = coff;
    T.s.leaves = J->leaves;
    T.s.prims = J->prims;
    T.s.desc = J->desc;
    // a step whose build overflowed (or failed) renders on stale or partial arrays and is
    // redone by the host: its grid is not traversed
    const GridDesc* st = J->status ? J->status : J->desc;
    T.s.ntri = (__ldg(&st->overflow) | __ldg(&st->error)) ? 0u : J->ntri;
    T.s.kind = J->kind;
    T.s.nrm3 = nullptr;   // served scenes shade with geometric normals and the job's albedo
    T.s.alb = nullptr;
    T.g = load_g(J->desc);
    for (int q = 0; q < 3; ++q) {
        T.cam.pos[q] = J->cam_pos[q]; T.cam.tl[q] = J->cam_tl[q];
        T.cam.sx[q] = J->cam_sx[q]; T.cam.sy[q] = J->cam_sy[q];
    }
    T.cam.w = J->w;
    T.cam.h = J->h;
    T.fb = J->fb;
    T.org = J->org; T.dir = J->dir;
    T.out_id = J->out_id; T.out_t = J->out_t; T.out_u = J->out_u; T.out_v = J->out_v;
    T.seed = J->seed;
    T.spp = (uint32_t)J->spp;
    T.image_id = J->image_id;
    T.mode = J->mode;
    float alpha = J->alpha_abs;
    if (!(alpha > 0.0f)) {
        const f3 dd = mk(T.g.bmax[0] - T.g.bmin[0], T.g.bmax[1] - T.g.bmin[1], T.g.bmax[2] - T.g.bmin[2]);
        alpha = J->alpha_frac * sqrtf(dot(dd, dd));
    }
    T.alpha = alpha;
    T.off = 0.01f * alpha;
    if (J->mode == kJobPath) {
        T.pk = pt_consts(T.g, J->lights, J->bounces, J->albedo, J->eps_frac);
    }
}

// Persistent traversal over the tiles of all jobs.  A warp takes a tile from the work
// counter and, by the job's mode:
//   rays     traces 32 rays of the list (closest hit) and writes id, t, u, v;
//   primary  traces the tile's camera rays and shades them as k_render_primary;
//   AO       traces the camera rays, then the AO samples of the tile's hit pixels in
//            rounds of 32: item i of a round is sample (i mod spp) of the (i / spp)-th
//            hit pixel, with the PCG32 stream, direction, origin and radius of
//            k_ao_samples; each pixel's unoccluded count is summed from the round ballots
//            in its own lane's register;
//   path     runs spp paths per pixel, image ids image_id .. image_id + spp - 1, blended in
//            that order as k_render_pt frames; lanes regenerate paths (path_refill /
//            path_step / path_retire) so a warp stays full across bounces and samples.
// The PT variant runs path jobs only and the other variant every other mode: the host
// launches them over disjoint ranges of the job table.
template <bool PT>
__global__ __launch_bounds__(kJobTT, PT ? HR_JOB_PT_MIN_BLOCKS : HR_JOB_MIN_BLOCKS) void k_trace_jobs(const Job* __restrict__ jobs,
                                                                        const uint32_t* __restrict__ tile_off,
                                                                        uint32_t njobs, uint32_t* work,
                                                                        int32_t tile_w,
                                                                        unsigned long long* counter) {
    __shared__ TileCtx s_tile[kJobTT / 32];
    TileCtx& T = s_tile[threadIdx.x >> 5];
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t ntiles = __ldg(tile_off + njobs);
    const uint32_t tw = (uint32_t)tile_w, th = 32u / tw;
    if (PT) {
        // path jobs: lanes regenerate paths (next sample of the pixel, or the next pixel of
        // the warp's tiles); a tile of another job is taken once the warp's paths are done
        constexpr uint32_t kNone = 0xffffffffu;
        uint32_t cur_j = kNone, tile_local = 0, next = 32u, pend = kNone;
        bool more = true;
#if HR_JOB_PT_SMEM_STATE
        // the path state lives in shared memory, so the traversal has the registers to itself
        __shared__ __align__(16) unsigned char s_lanes[sizeof(PathLane) * kJobTT];
        PathLane& ln = reinterpret_cast<PathLane*>(s_lanes)[threadIdx.x];
        ln.pix = 0;
        ln.sample = 0;
        ln.val = 0.0f;
        ln.has = false;
#else
        PathLane ln;
#endif
        PtCounts n;
        while (true) {
            while (more) {
                if (next >= 32u) {
                    if (pend == kNone) {
                        uint32_t t = 0;
                        if (lane == 0) t = atomicAdd(work, 1u);
                        t = __shfl_sync(kFullMask, t, 0);
                        if (t >= ntiles) {
                            more = false;
                            break;
                        }
                        pend = t;
                    }
                    const uint32_t j = find_segment(tile_off, njobs, pend);
                    if (j != cur_j) {
                        if (__any_sync(kFullMask, ln.has)) break;   // finish this job's paths first
                        if (lane == 0) load_tile_ctx(T, jobs + j);
                        __syncwarp();
                        cur_j = j;
                    }
                    tile_local = pend - __ldg(tile_off + j);
                    pend = kNone;
                    next = 0;
                }
                if (path_refill(ln, T.cam, tile_local, &next, T.image_id, T.seed, T.fb) == 0u) break;
            }
            if (!__any_sync(kFullMask, ln.has)) break;   // the pool is dry and every path is done
            const bool cont = path_step<kTwoLevel, false, HR_JOB_PT_SEEK_STEPS>(T.s, T.g, T.pk, ln.p, ln.has, n);
            path_retire(ln, cont, T.cam, T.image_id, (int32_t)T.spp, T.seed, T.fb);
        }
        add_rays<false>(counter, false, n.rays);
        add_rays<false>(counter, true, n.srays);
        return;
    }
    while (true) {
        uint32_t tile = 0;
        if (lane == 0) tile = atomicAdd(work, 1u);
        tile = __shfl_sync(kFullMask, tile, 0);
        if (tile >= ntiles) break;
        const uint32_t j = find_segment(tile_off, njobs, tile);
        if (lane == 0) load_tile_ctx(T, jobs + j);
        __syncwarp();
        const uint32_t lt = tile - __ldg(tile_off + j);
        // one closest-hit call for ray-list and camera rays
        const bool rays = T.mode == kJobRays;
        bool valid;
        uint32_t pix;
        f3 o, d;
        if (rays) {
            pix = lt * 32u + lane;
            valid = pix < (uint32_t)T.cam.w;
            o = mk(0.0f, 0.0f, 0.0f);
            d = mk(1.0f, 0.0f, 0.0f);
            if (valid) {
                o = mk(__ldg(T.org + 3 * (size_t)pix), __ldg(T.org + 3 * (size_t)pix + 1), __ldg(T.org + 3 * (size_t)pix + 2));
                d = mk(__ldg(T.dir + 3 * (size_t)pix), __ldg(T.dir + 3 * (size_t)pix + 1), __ldg(T.dir + 3 * (size_t)pix + 2));
            }
        } else {
            const uint32_t cw = (uint32_t)T.cam.w, chh = (uint32_t)T.cam.h;
            const uint32_t tx = (cw + tw - 1u) / tw;
            const uint32_t x = (lt % tx) * tw + lane % tw, y = (lt / tx) * th + lane / tw;
            valid = x < cw && y < chh;
            pix = valid ? y * cw + x : 0u;
            o = mk(T.cam.pos[0], T.cam.pos[1], T.cam.pos[2]);
            d = !valid ? mk(1.0f, 0.0f, 0.0f)
                       : (T.mode == kJobPrimary ? primary_sample_dir(T.cam, pix, T.image_id, T.seed) : primary_dir(T.cam, pix));
        }
        Hit h;
        trace_one<kTwoLevel, false, false>(T.s, T.g, o, d, FLT_MAX, h, valid);
        add_rays<false>(counter, false, valid ? 1u : 0u);
        if (rays) {
            if (valid) {
                if (h.hit) refine_uv(T.s, h.tri, o, d, &h.u, &h.v);
                T.out_id[pix] = h.hit ? (int32_t)h.tri : -1;
                T.out_t[pix] = h.hit ? h.t : FLT_MAX;
                T.out_u[pix] = h.u;
                T.out_v[pix] = h.v;
            }
            __syncwarp();
            continue;
        }
        float* fb = T.fb + 3 * (size_t)pix;
        if (T.mode != kJobAO) {
            if (valid) {
                float rgb[3];
                simple_shade(T.s, h.hit, h.tri, o, d, rgb);
                fb[0] = blend(fb[0], rgb[0], T.image_id);
                fb[1] = blend(fb[1], rgb[1], T.image_id);
                fb[2] = blend(fb[2], rgb[2], T.image_id);
            }
            __syncwarp();
            continue;
        }
        const bool hit = valid && h.hit;
        if (valid && !hit) {
            const float val = blend(fb[0], 1.0f, T.image_id);
            fb[0] = val; fb[1] = val; fb[2] = val;
        }
        const uint32_t m = __ballot_sync(kFullMask, hit);
        if (m == 0u) {
            __syncwarp();
            continue;
        }
        if (hit) {
            const f3 p = mk(o.x + h.t * d.x, o.y + h.t * d.y, o.z + h.t * d.z);
            const f3 nrm = face_normal(T.s, h.tri, d);
            T.px[lane] = p.x; T.py[lane] = p.y; T.pz[lane] = p.z;
            T.nx[lane] = nrm.x; T.ny[lane] = nrm.y; T.nz[lane] = nrm.z;
            T.pix[lane] = pix;
        }
        __syncwarp();
        const uint32_t spp = T.spp;
        const uint32_t rank = __popc(m & ((1u << lane) - 1u));
        const uint32_t total = (uint32_t)__popc(m) * spp;
        uint32_t unocc = 0;
        for (uint32_t base = 0; base < total; base += 32u) {
            const uint32_t item = base + lane;
            const bool v2 = item < total;
            f3 ao = mk(0.0f, 0.0f, 0.0f), w = mk(1.0f, 0.0f, 0.0f);
            if (v2) {
                const uint32_t q = item / spp, k = item - q * spp;
                const uint32_t src = nth_set_bit(m, q);
                Pcg32 rng;
                pcg_seed(rng, ((uint64_t)(uint32_t)T.image_id << 32) | T.pix[src], T.seed);
                pcg_skip_pairs(rng, k);
                const float u1 = pcg_float(rng), u2 = pcg_float(rng);
                w = cosine_dir(mk(T.nx[src], T.ny[src], T.nz[src]), u1, u2);
                const float off = T.off;
                ao = mk(T.px[src] + off * w.x, T.py[src] + off * w.y, T.pz[src] + off * w.z);
            }
            Hit hs;
            trace_one<kTwoLevel, true, false>(T.s, T.g, ao, w, T.alpha, hs, v2);
            const uint32_t fm = __ballot_sync(kFullMask, v2 && !hs.hit);
            if (hit) {
                // this lane's samples are items [rank * spp, rank * spp + spp)
                const int32_t lo = max((int32_t)(rank * spp) - (int32_t)base, 0);
                const int32_t hi = min((int32_t)(rank * spp + spp) - (int32_t)base, 32);
                if (hi > lo) {
                    const uint32_t span = (uint32_t)(hi - lo);
                    const uint32_t rm = (span == 32u ? 0xffffffffu : ((1u << span) - 1u)) << lo;
                    unocc += __popc(fm & rm);
                }
            }
            add_rays<false>(counter, true, v2 ? 1u : 0u);
        }
        if (hit) {
            const float vis = (float)unocc / (float)spp;
            const float val = blend(fb[0], vis, T.image_id);
            fb[0] = val; fb[1] = val; fb[2] = val;
        }
        __syncwarp();   // the tile context is rewritten for the next tile
    }
}

}  // namespace

uint32_t job_tiles(const Job& j, int32_t tw) {
    if (j.mode == kJobRays) return ((uint32_t)j.w + 31u) / 32u;
    const uint32_t th = 32u / (uint32_t)tw;
    return (((uint32_t)j.w + (uint32_t)tw - 1u) / (uint32_t)tw) * (((uint32_t)j.h + th - 1u) / th);
}

int job_blocks_per_sm(int32_t block_threads, bool pt) {
    int nb = 0;
    cudaError_t e = pt ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_trace_jobs<true>, block_threads, 0)
                       : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_trace_jobs<false>, block_threads, 0);
    if (e != cudaSuccess) {
        cudaGetLastError();
        nb = 0;
    }
    return nb > 0 ? nb : 1;
}

int launch_jobs(hr_ctx* c, const Job* d_jobs, const uint32_t* d_tile_off, uint32_t njobs, uint32_t* d_work,
                int32_t tile_w, int32_t block_threads, int32_t nblocks, bool pt, cudaStream_t s) {
    if (block_threads < 32 || block_threads > kJobTT || block_threads % 32 != 0)
        return set_error(c, HR_ERR_INVALID_ARG, "jobs: block of %d threads", block_threads);
    c->launches += 1;
    unsigned long long* ctr = c->counters.as<unsigned long long>();
    if (pt) k_trace_jobs<true><<<nblocks, block_threads, 0, s>>>(d_jobs, d_tile_off, njobs, d_work, tile_w, ctr);
    else k_trace_jobs<false><<<nblocks, block_threads, 0, s>>>(d_jobs, d_tile_off, njobs, d_work, tile_w, ctr);
    return cuda_check(c, cudaGetLastError(), "jobs launch");
}

}  // namespace hr
