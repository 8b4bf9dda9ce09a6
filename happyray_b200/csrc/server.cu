// server.cu -- served rendering: continuous batching of render and ray-query requests over
// device-resident animated scenes (hr_server_* in include/happyray.h).
//
// The reference renders one scene per process from its own frame loop
// (src/Application/CUDAApplication.cu:116-160); this is the multi-request form of the same
// hot path.  Batched mode, per wave:
//   1. admission (FIFO, under the lock): queued requests join the wave while their device
//      buffers fit in (budget - resident scenes - requests in flight) and the wave has
//      slots; a scene takes part with one frame time per wave (a request for another frame
//      time of that scene waits for the next wave);
//   2. rebuilds: a scene whose resident grid has another frame time is rebuilt on its own
//      stream (build_grid_async: key-frame lerp fused into the build, no host sync) after
//      the last wave that read the old grid (stream wait on that wave's event); the
//      server stream waits for the rebuilds;
//   3. one persistent launch traces every request of the wave (jobs.cu), path-traced
//      requests in a second launch of the path-tracing variant; results are copied back
//      in stream order;
//   4. up to two waves are in flight: while one traces, the worker admits and enqueues the
//      next (its rebuilds of other scenes run concurrently on their streams); a finished
//      wave is retired in launch order, its buffers released, its requests completed.
// A grid rebuilt asynchronously is checked when its wave retires; if it overflowed its
// capacities (sized at add_scene by building every key frame), the capacities grow and
// every request that read it is queued again.
#include "hr_internal.h"
#include "../../include/happyray.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <set>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

using namespace hr;

namespace {

uint64_t now_ns() {
    return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
               std::chrono::steady_clock::now().time_since_epoch()).count();
}

size_t ctx_bytes(const hr_ctx* c) {
    const DevBuf* b[] = {&c->verts, &c->idx, &c->tris, &c->keyframes, &c->staging, &c->counters, &c->fb,
                         &c->out_id, &c->out_t, &c->out_u, &c->out_v, &c->ray_in, &c->g.desc, &c->g.cells,
                         &c->g.leaves, &c->g.prims, &c->g.keys_a, &c->g.vals_a, &c->g.keys_b, &c->g.vals_b,
                         &c->g.block_sums, &c->g.tile_hist, &c->g.row_total, &c->g.leaf_cnt, &c->g.occ, &c->g.lkeys_a, &c->g.lvals_a, &c->g.lkeys_b, &c->g.lvals_b,
                         &c->g.scan_partials, &c->g.tri_ranges, &c->g.ref_ranges, &c->hit_t, &c->hit_tri,
                         &c->unocc, &c->queue};
    size_t s = 0;
    for (const DevBuf* d : b) s += d->bytes;
    return s;
}

struct SrvScene {
    hr_ctx* ctx = nullptr;           // resident scene (batched and serial modes)
    std::vector<float> host_kf;      // plain mode: host key frames (xyz) and triangles
    std::vector<uint32_t> host_idx;
    float top = 0.0625f, leaf = 2.0f;   // grid densities
    uint32_t nverts = 0, ntri = 0, nkf = 0;
    float cur_time = -1.0f;          // frame time of the resident grid (< 0: none)
    uint64_t gen = 0;                // build generation of the resident grid
    std::set<uint64_t> bad_gens;     // generations whose asynchronous build overflowed
    cudaEvent_t last_read = nullptr; // after the last wave that read the grid
    cudaEvent_t built = nullptr;     // after the last rebuild
    bool ever_read = false, ever_built = false;
};

struct SrvReq {
    hr_request r{};
    Camera cam;
    int32_t status = 0;              // 0 queued, 1 in flight, 2 done, < 0 failed
    uint32_t wave = 0;
    uint64_t submit_ns = 0, admit_ns = 0, done_ns = 0;
    size_t bytes = 0;                // device bytes of its buffers
    void* dbuf = nullptr;
    bool pinned_out = false;
    uint64_t gen = 0;                // grid generation it was traced with
};

struct Wave {
    std::vector<uint64_t> reqs;
    std::vector<SrvReq*> rp;         // the same requests (stable addresses; the map may rehash)
    std::vector<uint32_t> rebuilt;
    cudaEvent_t done = nullptr;
    int slot = 0;
    uint32_t index = 0;
    uint64_t launched_ns = 0;        // host time of the launch (watchdog)
    int32_t stall_ms = 0;            // injected: treated as unfinished this long after the launch
    bool timed_out = false;          // the watchdog failed its requests; its buffers are held until it ends
};

constexpr int kSlots = 2;
constexpr size_t kMaxScenes = 4096;   // scenes of one server (the table never reallocates)

bool is_pinned(const void* p) {
    if (!p) return true;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

}  // namespace

struct hr_server {
    hr_ctx* c = nullptr;             // server stream, job-kernel ray counters, error text;
                                     // plain mode: the one context every request re-uploads into
    int32_t mode = HR_SERVER_BATCHED;
    uint64_t budget = 0;
    std::vector<std::unique_ptr<SrvScene>> scenes;
    uint64_t resident = 0;
    uint64_t inflight_bytes = 0, peak_inflight = 0;
    std::mutex m;
    std::condition_variable cv_work, cv_done;
    std::deque<uint64_t> queue;
    std::unordered_map<uint64_t, SrvReq> reqs;
    uint64_t next_id = 1;
    std::thread worker;
    bool stop = false;
    std::deque<Wave> inflight;
    DevBuf d_jobs[kSlots], d_tiles[kSlots], d_work[kSlots];
    Job* h_jobs[kSlots] = {};
    uint32_t* h_tiles[kSlots] = {};
    bool slot_busy[kSlots] = {};
    cudaEvent_t wave_ev[kSlots] = {};
    cudaEvent_t wave_start[kSlots] = {};   // before a wave's traversal launches
    cudaEvent_t wave_trace_end[kSlots] = {};
    double trace_ms = 0.0;
    int32_t max_jobs = 512;
    int32_t tile_w = 8, block_threads = 256;
    int blocks_main = 0, blocks_pt = 0;
    uint32_t waves = 0;
    uint64_t completed = 0, failed = 0, rebuilds = 0, host_rays = 0;
    int32_t watchdog_ms = 0;         // 0: no watchdog
    uint64_t watchdog_trips = 0;     // waves the watchdog declared stuck
    uint32_t inject_waves = 0;       // test hook: the next waves are held back ...
    int32_t inject_ms = 0;           // ... this long after their launch, on the host only
    std::string err;                 // last error (caller-visible)
};

namespace {

void fail_req(hr_server* S, SrvReq& R, int code) {
    R.status = -code;
    R.done_ns = now_ns();
    S->failed += 1;
}

size_t req_bytes(const hr_request& r) {
    if (r.kind == HR_REQUEST_RAYS) return (size_t)r.num_rays * 40u + 256u;
    return (size_t)r.width * (size_t)r.height * 12u + 256u;
}

// frame time of a scene's grid, set and rebuilt asynchronously on the scene's stream
// after the last wave that read it; the server stream waits for the new grid
int rebuild_async(hr_server* S, SrvScene& X, float t) {
    hr_ctx* c = X.ctx;
    if (X.ever_read) cudaStreamWaitEvent(c->stream, X.last_read, 0);
    if (hr_set_frame_time(c, t, 0.0f) != HR_OK) return HR_ERR_INVALID_ARG;
    int rc = build_grid_async(c, HR_GRID_TWO_LEVEL, 1);
    if (rc) return rc;
    X.cur_time = t;
    X.gen += 1;
    cudaEventRecord(X.built, c->stream);
    X.ever_built = true;
    S->rebuilds += 1;
    return 0;
}

void fill_render_job(Job& J, const SrvScene& X, const SrvReq& R) {
    std::memset(&J, 0, sizeof(Job));
    const hr_ctx* c = X.ctx;
    J.tris = c->tris.as<float4>();
    J.cells = c->g.cells.as<uint2>();
    J.occ = c->g.occ.as<uint32_t>();
    J.leaves = c->g.leaves.as<uint2>();
    J.prims = c->g.prims.as<uint32_t>();
    J.desc = c->g.desc.as<GridDesc>();
    J.ntri = X.ntri;
    J.kind = kTwoLevel;
    J.seed = R.r.seed;
    J.alpha_frac = c->ip.ao_radius_frac;
    J.eps_frac = c->ip.ray_eps_frac;
    J.bounces = c->ip.pt_bounces;
    J.albedo = c->ip.albedo;
    J.lights = c->lights_dev.as<LightSet>();
    if (R.r.kind == HR_REQUEST_RAYS) {
        float* base = static_cast<float*>(R.dbuf);
        const size_t n = R.r.num_rays;
        J.mode = kJobRays;
        J.org = base;
        J.dir = base + 3 * n;
        J.out_id = reinterpret_cast<int32_t*>(base + 6 * n);
        J.out_t = base + 7 * n;
        J.out_u = base + 8 * n;
        J.out_v = base + 9 * n;
        J.w = (int32_t)n;
        J.h = 1;
        return;
    }
    J.fb = static_cast<float*>(R.dbuf);
    for (int q = 0; q < 3; ++q) {
        J.cam_pos[q] = R.cam.pos[q]; J.cam_tl[q] = R.cam.top_left[q];
        J.cam_sx[q] = R.cam.step_x[q]; J.cam_sy[q] = R.cam.step_y[q];
    }
    J.w = R.cam.w;
    J.h = R.cam.h;
    J.mode = R.r.mode == HR_RENDER_AO ? kJobAO : (R.r.mode == HR_RENDER_PRIMARY ? kJobPrimary : kJobPath);
    J.spp = R.r.spp;
    J.image_id = 0;
}

// enqueue one wave (no lock held; the wave's requests are owned by the worker)
int launch_wave(hr_server* S, Wave& w, std::map<uint32_t, float>& times) {
    hr_ctx* c = S->c;
    cudaStream_t s = c->stream;
    int rc;
    // rebuilds, then the server stream waits for every grid the wave reads
    for (auto& kv : times) {
        SrvScene& X = *S->scenes[kv.first];
        if (X.cur_time != kv.second) {
            if ((rc = rebuild_async(S, X, kv.second))) return rc;
            w.rebuilt.push_back(kv.first);
        }
        if (X.ever_built) cudaStreamWaitEvent(s, X.built, 0);
    }
    // request buffers, inputs
    for (SrvReq* rq : w.rp) {
        SrvReq& R = *rq;
        R.gen = S->scenes[R.r.scene]->gen;
        if ((rc = cuda_check(c, cudaMallocAsync(&R.dbuf, R.bytes, s), "request buffer"))) return rc;
        if (R.r.kind == HR_REQUEST_RAYS) {
            const size_t n = R.r.num_rays;
            float* base = static_cast<float*>(R.dbuf);
            if ((rc = cuda_check(c, cudaMemcpyAsync(base, R.r.ray_org, 12 * n, cudaMemcpyHostToDevice, s), "rays")) ||
                (rc = cuda_check(c, cudaMemcpyAsync(base + 3 * n, R.r.ray_dir, 12 * n, cudaMemcpyHostToDevice, s), "rays")))
                return rc;
            R.pinned_out = is_pinned(R.r.out_id) && is_pinned(R.r.out_t) && is_pinned(R.r.out_u) && is_pinned(R.r.out_v);
        } else {
            if ((rc = cuda_check(c, cudaMemsetAsync(R.dbuf, 0, R.bytes, s), "framebuffer"))) return rc;
            R.pinned_out = is_pinned(R.r.out_rgb);
        }
    }
    // job table: path-traced requests last, each group with its own tile prefix and counter.
    // Within a group the requests with the most samples per pixel (the costliest tiles) come
    // first, so that the warps that take the last tiles of the pool take short ones.
    Job* hj = S->h_jobs[w.slot];
    uint32_t* ht = S->h_tiles[w.slot];
    uint32_t n_main = 0, n_pt = 0;
    std::vector<const SrvReq*> order(w.rp.begin(), w.rp.end());
    std::stable_sort(order.begin(), order.end(), [](const SrvReq* a, const SrvReq* b) {
        const int32_t sa = a->r.kind == HR_REQUEST_RENDER ? a->r.spp : 1;
        const int32_t sb = b->r.kind == HR_REQUEST_RENDER ? b->r.spp : 1;
        return sa > sb;
    });
    for (int pass = 0; pass < 2; ++pass)
        for (const SrvReq* rq : order) {
            const SrvReq& R = *rq;
            const bool pt = R.r.kind == HR_REQUEST_RENDER && R.r.mode == HR_RENDER_PATH;
            if (pt != (pass == 1)) continue;
            fill_render_job(hj[n_main + n_pt], *S->scenes[R.r.scene], R);
            (pt ? n_pt : n_main) += 1;
        }
    const size_t tiles_pt0 = (size_t)S->max_jobs + 1;   // second prefix array
    ht[0] = 0;
    for (uint32_t i = 0; i < n_main; ++i) ht[i + 1] = ht[i] + job_tiles(hj[i], S->tile_w);
    ht[tiles_pt0] = 0;
    for (uint32_t i = 0; i < n_pt; ++i) ht[tiles_pt0 + i + 1] = ht[tiles_pt0 + i] + job_tiles(hj[n_main + i], S->tile_w);
    Job* dj = S->d_jobs[w.slot].as<Job>();
    uint32_t* dt = S->d_tiles[w.slot].as<uint32_t>();
    uint32_t* dw = S->d_work[w.slot].as<uint32_t>();
    if ((rc = cuda_check(c, cudaMemcpyAsync(dj, hj, sizeof(Job) * (n_main + n_pt), cudaMemcpyHostToDevice, s), "jobs")) ||
        (rc = cuda_check(c, cudaMemcpyAsync(dt, ht, sizeof(uint32_t) * (2 * tiles_pt0), cudaMemcpyHostToDevice, s),
                         "tiles")) ||
        (rc = cuda_check(c, cudaMemsetAsync(dw, 0, 2 * sizeof(uint32_t), s), "work")))
        return rc;
    cudaEventRecord(S->wave_start[w.slot], s);
    if (n_main && (rc = launch_jobs(c, dj, dt, n_main, dw, S->tile_w, S->block_threads, S->blocks_main, false, s)))
        return rc;
    if (n_pt && (rc = launch_jobs(c, dj + n_main, dt + tiles_pt0, n_pt, dw + 1, S->tile_w, S->block_threads,
                                  S->blocks_pt, true, s)))
        return rc;
    cudaEventRecord(S->wave_trace_end[w.slot], s);
    for (auto& kv : times) {
        SrvScene& X = *S->scenes[kv.first];
        cudaEventRecord(X.last_read, s);
        X.ever_read = true;
    }
    // results to pinned host memory in stream order; pageable ones when the wave retires
    for (SrvReq* rq : w.rp) {
        SrvReq& R = *rq;
        if (!R.pinned_out) continue;
        if (R.r.kind == HR_REQUEST_RAYS) {
            const size_t n = R.r.num_rays;
            const float* base = static_cast<const float*>(R.dbuf);
            if ((rc = cuda_check(c, cudaMemcpyAsync(R.r.out_id, base + 6 * n, 4 * n, cudaMemcpyDeviceToHost, s), "out")) ||
                (rc = cuda_check(c, cudaMemcpyAsync(R.r.out_t, base + 7 * n, 4 * n, cudaMemcpyDeviceToHost, s), "out")) ||
                (rc = cuda_check(c, cudaMemcpyAsync(R.r.out_u, base + 8 * n, 4 * n, cudaMemcpyDeviceToHost, s), "out")) ||
                (rc = cuda_check(c, cudaMemcpyAsync(R.r.out_v, base + 9 * n, 4 * n, cudaMemcpyDeviceToHost, s), "out")))
                return rc;
        } else if ((rc = cuda_check(c, cudaMemcpyAsync(R.r.out_rgb, R.dbuf, (size_t)R.cam.w * R.cam.h * 12,
                                                       cudaMemcpyDeviceToHost, s), "out"))) {
            return rc;
        }
    }
    return cuda_check(c, cudaEventRecord(w.done, s), "wave event");
}

// a retired wave: check its rebuilds, copy pageable results, release buffers.  Returns
// the requests to queue again (their grid overflowed).
std::vector<uint64_t> retire_wave(hr_server* S, Wave& w) {
    hr_ctx* c = S->c;
    std::vector<uint64_t> redo;
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, S->wave_start[w.slot], S->wave_trace_end[w.slot]) == cudaSuccess) S->trace_ms += ms;
    cudaGetLastError();
    for (uint32_t sc : w.rebuilt) {
        SrvScene& X = *S->scenes[sc];
        bool fit = true;
        build_async_result(X.ctx, &fit);
        if (!fit) {
            X.bad_gens.insert(X.gen);
            X.cur_time = -1.0f;   // the next wave reading this scene rebuilds it (capacities grown)
        }
    }
    for (size_t i = 0; i < w.rp.size(); ++i) {
        SrvReq& R = *w.rp[i];
        if (w.timed_out) {
            // the caller was answered with a timeout: nothing is copied to its buffers
        } else if (S->scenes[R.r.scene]->bad_gens.count(R.gen)) {
            redo.push_back(w.reqs[i]);
        } else if (!R.pinned_out) {
            if (R.r.kind == HR_REQUEST_RAYS) {
                const size_t n = R.r.num_rays;
                const float* base = static_cast<const float*>(R.dbuf);
                cudaMemcpy(R.r.out_id, base + 6 * n, 4 * n, cudaMemcpyDeviceToHost);
                cudaMemcpy(R.r.out_t, base + 7 * n, 4 * n, cudaMemcpyDeviceToHost);
                cudaMemcpy(R.r.out_u, base + 8 * n, 4 * n, cudaMemcpyDeviceToHost);
                cudaMemcpy(R.r.out_v, base + 9 * n, 4 * n, cudaMemcpyDeviceToHost);
            } else {
                cudaMemcpy(R.r.out_rgb, R.dbuf, (size_t)R.cam.w * R.cam.h * 12, cudaMemcpyDeviceToHost);
            }
        }
        cudaFreeAsync(R.dbuf, c->stream);
        R.dbuf = nullptr;
    }
    return redo;
}

int serve_on(hr_server* S, hr_ctx* c, SrvReq& R);

// one request through the per-scene path: serial mode on the scene's resident context,
// plain mode on the one context after uploading the request's frame (RTEngine::upload)
int serve_serial(hr_server* S, SrvReq& R) {
    SrvScene& X = *S->scenes[R.r.scene];
    int rc;
    if (S->mode == HR_SERVER_PLAIN) {
        hr_ctx* c = S->c;
        const uint32_t k = (uint32_t)R.r.frame_time;
        const uint32_t k2 = (k + 1u) % X.nkf;
        const float coeff = R.r.frame_time - (float)k;
        const float* a = X.host_kf.data() + (size_t)k * X.nverts * 3;
        const float* b = X.host_kf.data() + (size_t)k2 * X.nverts * 3;
        if (hr_upload(c, a, b, X.nverts, X.host_idx.data(), X.ntri, coeff) != HR_OK) return HR_ERR_DEVICE;
        hr_set_grid_densities(c, X.top, X.leaf);
        if ((rc = build_grid(c, HR_GRID_TWO_LEVEL, 1))) return rc;
        S->rebuilds += 1;
        return serve_on(S, c, R);
    }
    hr_ctx* c = X.ctx;
    if (X.cur_time != R.r.frame_time) {
        if (hr_set_frame_time(c, R.r.frame_time, 0.0f) != HR_OK) return HR_ERR_INVALID_ARG;
        if ((rc = build_grid(c, HR_GRID_TWO_LEVEL, 1))) return rc;
        X.cur_time = R.r.frame_time;
        S->rebuilds += 1;
    }
    return serve_on(S, c, R);
}

// render or ray query of one request on a context whose grid is built
int serve_on(hr_server* S, hr_ctx* c, SrvReq& R) {
    int rc;
    c->ip.seed = R.r.seed;
    if (R.r.kind == HR_REQUEST_RAYS) {
        const size_t n = R.r.num_rays;
        if ((rc = ensure(c, c->ray_in, 24 * n)) || (rc = ensure(c, c->out_id, 4 * n)) || (rc = ensure(c, c->out_t, 4 * n)) ||
            (rc = ensure(c, c->out_u, 4 * n)) || (rc = ensure(c, c->out_v, 4 * n)))
            return rc;
        float* org = c->ray_in.as<float>();
        if ((rc = cuda_check(c, cudaMemcpyAsync(org, R.r.ray_org, 12 * n, cudaMemcpyHostToDevice, c->stream), "rays")) ||
            (rc = cuda_check(c, cudaMemcpyAsync(org + 3 * n, R.r.ray_dir, 12 * n, cudaMemcpyHostToDevice, c->stream),
                             "rays")))
            return rc;
        if ((rc = launch_trace_rays(c, org, org + 3 * n, (uint32_t)n, c->out_id.as<int32_t>(), c->out_t.as<float>(),
                                    c->out_u.as<float>(), c->out_v.as<float>(), nullptr)))
            return rc;
        if ((rc = cuda_check(c, cudaMemcpyAsync(R.r.out_id, c->out_id.p, 4 * n, cudaMemcpyDeviceToHost, c->stream), "out")) ||
            (rc = cuda_check(c, cudaMemcpyAsync(R.r.out_t, c->out_t.p, 4 * n, cudaMemcpyDeviceToHost, c->stream), "out")) ||
            (rc = cuda_check(c, cudaMemcpyAsync(R.r.out_u, c->out_u.p, 4 * n, cudaMemcpyDeviceToHost, c->stream), "out")) ||
            (rc = cuda_check(c, cudaMemcpyAsync(R.r.out_v, c->out_v.p, 4 * n, cudaMemcpyDeviceToHost, c->stream), "out")))
            return rc;
        S->host_rays += n;
    } else {
        const size_t bytes = (size_t)R.cam.w * R.cam.h * 12;
        if ((rc = ensure(c, c->fb, bytes))) return rc;
        if ((rc = cuda_check(c, cudaMemsetAsync(c->fb.p, 0, bytes, c->stream), "framebuffer"))) return rc;
        c->cam = R.cam;
        c->have_camera = true;
        if (R.r.mode == HR_RENDER_PATH) {
            for (int32_t k = 0; k < R.r.spp; ++k)
                if ((rc = launch_render(c, HR_RENDER_PATH, k, c->fb.as<float>()))) return rc;
        } else {
            c->ip.ao_samples = R.r.spp;
            if ((rc = launch_render(c, R.r.mode, 0, c->fb.as<float>()))) return rc;
        }
        if ((rc = cuda_check(c, cudaMemcpyAsync(R.r.out_rgb, c->fb.p, bytes, cudaMemcpyDeviceToHost, c->stream), "out")))
            return rc;
    }
    return cuda_check(c, cudaStreamSynchronize(c->stream), "serial request");
}

void worker_main(hr_server* S) {
    cudaSetDevice(S->c->device);
    std::unique_lock<std::mutex> lk(S->m);
    uint32_t next_slot = 0;
    while (true) {
        if (S->mode != HR_SERVER_BATCHED) {
            if (S->queue.empty()) {
                if (S->stop) break;
                S->cv_work.wait(lk, [&] { return S->stop || !S->queue.empty(); });
                continue;
            }
            const uint64_t id = S->queue.front();
            S->queue.pop_front();
            SrvReq& R = S->reqs[id];   // a stable reference (the map may rehash, elements stay)
            R.status = 1;
            R.admit_ns = now_ns();
            R.wave = S->waves++;
            lk.unlock();
            const int rc = serve_serial(S, R);
            lk.lock();
            if (rc) {
                fail_req(S, R, rc);
            } else {
                R.status = 2;
                R.done_ns = now_ns();
                S->completed += 1;
            }
            S->cv_done.notify_all();
            continue;
        }
        // retire finished waves in launch order; the watchdog answers the requests of a wave
        // still unfinished watchdog_ms after its launch with HR_ERR_TIMEOUT at once (its GPU
        // work cannot be recalled: its buffers stay held until it ends, and later waves on
        // the same stream wait behind it)
        bool retired = false;
        const uint64_t tnow = now_ns();
        auto finished = [&](Wave& w, cudaError_t* qq) {
            *qq = cudaEventQuery(w.done);
            if (*qq == cudaErrorNotReady) return false;
            return !(w.stall_ms > 0 && tnow - w.launched_ns < (uint64_t)w.stall_ms * 1000000ull);
        };
        if (S->watchdog_ms > 0) {
            for (Wave& w : S->inflight) {
                cudaError_t qq;
                if (w.timed_out || tnow - w.launched_ns < (uint64_t)S->watchdog_ms * 1000000ull || finished(w, &qq))
                    continue;
                w.timed_out = true;
                S->watchdog_trips += 1;
                set_error(S->c, HR_ERR_TIMEOUT, "wave %u unfinished after %d ms: its requests failed", w.index,
                          S->watchdog_ms);
                for (SrvReq* rq : w.rp)
                    if (rq->status == 1) fail_req(S, *rq, HR_ERR_TIMEOUT);
                retired = true;
            }
        }
        cudaError_t q;
        while (!S->inflight.empty() && finished(S->inflight.front(), &q)) {
            Wave w = std::move(S->inflight.front());
            S->inflight.pop_front();
            if (q != cudaSuccess) {
                // a device error: the wave's results are lost
                set_error(S->c, HR_ERR_DEVICE, "wave %u: %s", w.index, cudaGetErrorString(q));
                for (SrvReq* rq : w.rp) {
                    S->inflight_bytes -= rq->bytes;
                    if (rq->status == 1) fail_req(S, *rq, HR_ERR_DEVICE);
                }
                S->slot_busy[w.slot] = false;
                retired = true;
                continue;
            }
            lk.unlock();
            std::vector<uint64_t> redo = retire_wave(S, w);
            lk.lock();
            const uint64_t t = now_ns();
            for (size_t i = w.rp.size(); i-- > 0;) {
                SrvReq& R = *w.rp[i];
                S->inflight_bytes -= R.bytes;
                if (w.timed_out) continue;   // answered by the watchdog
                if (std::find(redo.begin(), redo.end(), w.reqs[i]) != redo.end()) {
                    R.status = 0;
                    S->queue.push_front(w.reqs[i]);
                } else {
                    R.status = 2;
                    R.done_ns = t;
                    S->completed += 1;
                }
            }
            S->slot_busy[w.slot] = false;
            retired = true;
        }
        if (retired) S->cv_done.notify_all();
        if (S->stop && S->queue.empty() && S->inflight.empty()) break;
        // admit and launch a wave when a slot is free
        if ((int)S->inflight.size() < kSlots && !S->queue.empty()) {
            Wave w;
            w.slot = S->slot_busy[next_slot] ? (int)(next_slot ^ 1u) : (int)next_slot;
            next_slot = (uint32_t)w.slot ^ 1u;
            std::map<uint32_t, float> times;
            const uint64_t avail = S->budget > S->resident + S->inflight_bytes ? S->budget - S->resident - S->inflight_bytes : 0;
            uint64_t used = 0;
            const uint64_t t = now_ns();
            for (auto it = S->queue.begin(); it != S->queue.end() && (int)w.reqs.size() < S->max_jobs;) {
                SrvReq& R = S->reqs[*it];
                auto f = times.find(R.r.scene);
                if (f != times.end() && f->second != R.r.frame_time) { ++it; continue; }
                if (used + R.bytes > avail) break;   // FIFO: wait for memory
                times[R.r.scene] = R.r.frame_time;
                used += R.bytes;
                R.status = 1;
                R.admit_ns = t;
                R.wave = S->waves;
                w.reqs.push_back(*it);
                w.rp.push_back(&R);
                it = S->queue.erase(it);
            }
            if (!w.reqs.empty()) {
                w.index = S->waves++;
                w.done = S->wave_ev[w.slot];
                w.launched_ns = now_ns();
                if (S->inject_waves > 0) {
                    S->inject_waves -= 1;
                    w.stall_ms = S->inject_ms;
                }
                S->slot_busy[w.slot] = true;
                S->inflight_bytes += used;
                S->peak_inflight = std::max(S->peak_inflight, S->inflight_bytes);
                lk.unlock();
                const int rc = launch_wave(S, w, times);
                lk.lock();
                if (rc) {
                    // the wave could not be enqueued: its requests fail, buffers are released
                    cudaStreamSynchronize(S->c->stream);
                    for (SrvReq* rq : w.rp) {
                        SrvReq& R = *rq;
                        if (R.dbuf) cudaFreeAsync(R.dbuf, S->c->stream);
                        R.dbuf = nullptr;
                        S->inflight_bytes -= R.bytes;
                        fail_req(S, R, rc);
                    }
                    S->slot_busy[w.slot] = false;
                    S->cv_done.notify_all();
                } else {
                    S->inflight.push_back(std::move(w));
                }
                continue;
            }
            if (S->inflight.empty()) {
                // nothing in flight and the queue head does not fit the budget: it never will
                SrvReq& R = S->reqs[S->queue.front()];
                S->queue.pop_front();
                fail_req(S, R, HR_ERR_OUT_OF_MEMORY);
                S->cv_done.notify_all();
                continue;
            }
        }
        // wait for a submission or a wave to finish
        if (!S->inflight.empty()) S->cv_work.wait_for(lk, std::chrono::microseconds(20));
        else S->cv_work.wait(lk, [&] { return S->stop || !S->queue.empty(); });
    }
}

bool valid_server(const hr_server* s) { return s && s->c; }

}  // namespace

extern "C" {

hr_status hr_server_create(hr_server** out, int32_t device, uint64_t budget, int32_t mode) {
    if (!out || (mode != HR_SERVER_BATCHED && mode != HR_SERVER_SERIAL && mode != HR_SERVER_PLAIN) || budget == 0)
        return HR_ERR_INVALID_ARG;
    *out = nullptr;
    hr_server* S = new (std::nothrow) hr_server();
    if (!S) return HR_ERR_OUT_OF_MEMORY;
    hr_status st = hr_create(&S->c, device, nullptr);
    if (st != HR_OK) { delete S; return st; }
    S->mode = mode;
    S->budget = budget;
    S->scenes.reserve(kMaxScenes);
    DeviceGuard dg(device);
    // keep freed request buffers in the stream-ordered pool for the next waves
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t thr = budget;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    cudaGetLastError();
    int rc = 0;
    const size_t ntiles = 2 * ((size_t)S->max_jobs + 1);
    for (int k = 0; k < kSlots && !rc; ++k) {
        if ((rc = ensure(S->c, S->d_jobs[k], sizeof(Job) * S->max_jobs)) ||
            (rc = ensure(S->c, S->d_tiles[k], sizeof(uint32_t) * ntiles)) || (rc = ensure(S->c, S->d_work[k], 16)))
            break;
        if (cudaMallocHost((void**)&S->h_jobs[k], sizeof(Job) * S->max_jobs) != cudaSuccess ||
            cudaMallocHost((void**)&S->h_tiles[k], sizeof(uint32_t) * ntiles) != cudaSuccess ||
            cudaEventCreateWithFlags(&S->wave_ev[k], cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreate(&S->wave_start[k]) != cudaSuccess || cudaEventCreate(&S->wave_trace_end[k]) != cudaSuccess) {
            cudaGetLastError();
            rc = HR_ERR_OUT_OF_MEMORY;
        }
    }
    if (rc) { hr_server_destroy(S); return (hr_status)rc; }
    S->blocks_main = job_blocks_per_sm(S->block_threads, false) * S->c->num_sms;
    S->blocks_pt = job_blocks_per_sm(S->block_threads, true) * S->c->num_sms;
    S->worker = std::thread(worker_main, S);
    *out = S;
    return HR_OK;
}

void hr_server_destroy(hr_server* S) {
    if (!S) return;
    if (S->worker.joinable()) {
        {
            std::lock_guard<std::mutex> g(S->m);
            S->stop = true;
        }
        S->cv_work.notify_all();
        S->worker.join();
    }
    if (S->c) {
        DeviceGuard dg(S->c->device);
        cudaStreamSynchronize(S->c->stream);
        for (auto& X : S->scenes) {
            if (X->last_read) cudaEventDestroy(X->last_read);
            if (X->built) cudaEventDestroy(X->built);
            if (X->ctx) hr_destroy(X->ctx);
        }
        for (int k = 0; k < kSlots; ++k) {
            if (S->h_jobs[k]) cudaFreeHost(S->h_jobs[k]);
            if (S->h_tiles[k]) cudaFreeHost(S->h_tiles[k]);
            if (S->wave_ev[k]) cudaEventDestroy(S->wave_ev[k]);
            if (S->wave_start[k]) cudaEventDestroy(S->wave_start[k]);
            if (S->wave_trace_end[k]) cudaEventDestroy(S->wave_trace_end[k]);
            if (S->d_jobs[k].p) cudaFreeAsync(S->d_jobs[k].p, S->c->stream);
            if (S->d_tiles[k].p) cudaFreeAsync(S->d_tiles[k].p, S->c->stream);
            if (S->d_work[k].p) cudaFreeAsync(S->d_work[k].p, S->c->stream);
        }
        hr_destroy(S->c);
    }
    delete S;
}

const char* hr_server_last_error(const hr_server* S) {
    if (!S) return "null server";
    return S->err.empty() && S->c ? S->c->err.c_str() : S->err.c_str();
}

hr_status hr_server_add_scene(hr_server* S, const float* kf, uint32_t nkf, uint32_t nv, const uint32_t* idx,
                              uint32_t ntri, float top, float leaf, uint32_t* scene_id) {
    if (!valid_server(S) || !kf || !idx || nkf == 0 || nv == 0 || ntri == 0 || !(top > 0.0f) || !(leaf > 0.0f) ||
        !scene_id)
        return HR_ERR_INVALID_ARG;
    DeviceGuard dg(S->c->device);
    std::unique_ptr<SrvScene> X(new SrvScene());
    if (S->mode == HR_SERVER_PLAIN) {
        // nothing resident: every request uploads its frame, as the per-frame path does
        X->host_kf.assign(kf, kf + (size_t)nkf * nv * 3);
        X->host_idx.assign(idx, idx + (size_t)ntri * 3);
        X->nverts = nv;
        X->ntri = ntri;
        X->nkf = nkf;
        X->top = top;
        X->leaf = leaf;
        std::lock_guard<std::mutex> g(S->m);
        if (S->scenes.size() >= kMaxScenes) return HR_ERR_OUT_OF_MEMORY;
        *scene_id = (uint32_t)S->scenes.size();
        S->scenes.push_back(std::move(X));
        return HR_OK;
    }
    hr_status st = hr_create(&X->ctx, S->c->device, nullptr);
    if (st != HR_OK) return st;
    hr_ctx* c = X->ctx;
    auto fail = [&](hr_status code, const char* what) {
        S->err = std::string(what) + ": " + c->err;
        hr_destroy(c);
        return code;
    };
    if ((st = hr_set_keyframes(c, kf, nkf, nv, idx, ntri)) != HR_OK) return fail(st, "add_scene");
    hr_set_grid_densities(c, top, leaf);
    // size the grid capacities for the whole animation: every key frame and the midpoints
    for (uint32_t k = 0; k < 2 * nkf; ++k) {
        if (hr_set_frame_time(c, 0.5f * (float)k, 0.0f) != HR_OK) return fail(HR_ERR_INVALID_ARG, "add_scene");
        if (int rc = build_grid(c, HR_GRID_TWO_LEVEL, 1)) return fail((hr_status)rc, "add_scene build");
    }
    X->cur_time = 0.5f * (float)(2 * nkf - 1);
    X->gen = 1;
    X->nverts = nv;
    X->ntri = ntri;
    X->nkf = nkf;
    if (cudaEventCreateWithFlags(&X->last_read, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&X->built, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        return fail(HR_ERR_DEVICE, "add_scene events");
    }
    cudaStreamSynchronize(c->stream);
    const uint64_t bytes = ctx_bytes(c);
    std::lock_guard<std::mutex> g(S->m);
    if (S->resident + bytes > S->budget || S->scenes.size() >= kMaxScenes) {
        S->err = "add_scene: the scene does not fit the HBM budget";
        cudaEventDestroy(X->last_read);
        cudaEventDestroy(X->built);
        hr_destroy(c);
        return HR_ERR_OUT_OF_MEMORY;
    }
    S->resident += bytes;
    *scene_id = (uint32_t)S->scenes.size();
    S->scenes.push_back(std::move(X));
    return HR_OK;
}

hr_status hr_server_submit(hr_server* S, const hr_request* r, uint64_t* id) {
    if (!valid_server(S) || !r || !id) return HR_ERR_INVALID_ARG;
    std::unique_lock<std::mutex> lk(S->m);
    if (r->scene >= S->scenes.size()) { S->err = "submit: unknown scene"; return HR_ERR_INVALID_ARG; }
    const SrvScene& X = *S->scenes[r->scene];
    if (!(r->frame_time >= 0.0f) || r->frame_time >= (float)X.nkf) { S->err = "submit: frame time outside the key frames"; return HR_ERR_INVALID_ARG; }
    SrvReq R;
    R.r = *r;
    if (r->kind == HR_REQUEST_RAYS) {
        if (!r->ray_org || !r->ray_dir || !r->out_id || !r->out_t || !r->out_u || !r->out_v || r->num_rays == 0) {
            S->err = "submit: ray request without rays or outputs";
            return HR_ERR_INVALID_ARG;
        }
    } else if (r->kind == HR_REQUEST_RENDER) {
        if (!r->out_rgb || r->width <= 0 || r->height <= 0 || !(r->cam_fov_deg > 0.0f && r->cam_fov_deg < 180.0f) ||
            r->spp < 1 || (r->mode != HR_RENDER_PRIMARY && r->mode != HR_RENDER_AO && r->mode != HR_RENDER_PATH)) {
            S->err = "submit: invalid render request";
            return HR_ERR_INVALID_ARG;
        }
        camera_init(&R.cam, r->cam_position, r->cam_orientation, r->cam_up, r->cam_fov_deg, r->width, r->height);
    } else {
        S->err = "submit: unknown request kind";
        return HR_ERR_INVALID_ARG;
    }
    R.bytes = req_bytes(*r);
    R.submit_ns = now_ns();
    const uint64_t rid = S->next_id++;
    S->reqs.emplace(rid, R);
    S->queue.push_back(rid);
    *id = rid;
    lk.unlock();
    S->cv_work.notify_one();
    return HR_OK;
}

hr_status hr_server_wait(hr_server* S, uint64_t id, int32_t timeout_ms) {
    if (!valid_server(S)) return HR_ERR_INVALID_ARG;
    std::unique_lock<std::mutex> lk(S->m);
    auto it = S->reqs.find(id);
    if (it == S->reqs.end()) return HR_ERR_INVALID_ARG;
    SrvReq& R = it->second;
    auto done = [&] { return R.status >= 2 || R.status < 0; };
    if (timeout_ms < 0) S->cv_done.wait(lk, done);
    else if (!S->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), done)) return HR_ERR_TIMEOUT;
    return R.status < 0 ? (hr_status)(-R.status) : HR_OK;
}

hr_status hr_server_drain(hr_server* S, int32_t timeout_ms) {
    if (!valid_server(S)) return HR_ERR_INVALID_ARG;
    std::unique_lock<std::mutex> lk(S->m);
    auto idle = [&] {
        if (!S->queue.empty() || !S->inflight.empty()) return false;
        for (auto& kv : S->reqs)
            if (kv.second.status == 1) return false;
        return true;
    };
    if (timeout_ms < 0) S->cv_done.wait(lk, idle);
    else if (!S->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), idle)) return HR_ERR_TIMEOUT;
    return HR_OK;
}

hr_status hr_server_request_info(hr_server* S, uint64_t id, hr_request_info* info) {
    if (!valid_server(S) || !info) return HR_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> g(S->m);
    auto it = S->reqs.find(id);
    if (it == S->reqs.end()) return HR_ERR_INVALID_ARG;
    const SrvReq& R = it->second;
    info->status = R.status;
    info->wave = R.wave;
    info->submit_ns = R.submit_ns;
    info->admit_ns = R.admit_ns;
    info->done_ns = R.done_ns;
    return HR_OK;
}

hr_status hr_server_get_stats(hr_server* S, hr_server_stats* st) {
    if (!valid_server(S) || !st) return HR_ERR_INVALID_ARG;
    DeviceGuard dg(S->c->device);
    std::lock_guard<std::mutex> g(S->m);
    uint64_t rays = S->host_rays;
    uint64_t launches = S->c->launches;
    std::vector<hr_ctx*> ctxs{S->c};
    for (auto& X : S->scenes)
        if (X->ctx) ctxs.push_back(X->ctx);
    for (hr_ctx* c : ctxs) {
        uint64_t w[8];
        if (cudaMemcpy(w, c->counters.p, sizeof(w), cudaMemcpyDeviceToHost) == cudaSuccess) rays += w[0] + w[4];
        cudaGetLastError();
        if (c != S->c) launches += c->launches;
    }
    st->completed = S->completed;
    st->failed = S->failed;
    st->waves = S->waves;
    st->rebuilds = S->rebuilds;
    st->rays = rays;
    st->resident_bytes = S->resident;
    st->peak_inflight_bytes = S->peak_inflight;
    st->launches = launches;
    st->trace_ms = S->trace_ms;
    st->watchdog_trips = S->watchdog_trips;
    return HR_OK;
}

hr_status hr_server_set_watchdog(hr_server* S, int32_t timeout_ms) {
    if (!valid_server(S) || timeout_ms < 0) return HR_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> g(S->m);
    S->watchdog_ms = timeout_ms;
    S->cv_work.notify_all();
    return HR_OK;
}

hr_status hr_server_inject_stall(hr_server* S, uint32_t waves, int32_t stall_ms) {
    if (!valid_server(S) || stall_ms < 0) return HR_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> g(S->m);
    S->inject_waves = waves;
    S->inject_ms = stall_ms;
    return HR_OK;
}

}  // extern "C"
