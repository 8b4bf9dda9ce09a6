// hr_internal.h -- host-side context and launcher declarations of libhappyray_b200.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstddef>
#include <string>
#include <vector>

#include "hr_common.cuh"

#ifndef HR_BUILD_GRAPH
#define HR_BUILD_GRAPH 1   // static rebuilds replay a captured CUDA graph of the build
#endif

namespace hr {

// Grow-only device allocation (MemoryManager.h:104-119 semantics: never shrinks).
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    template <class T> T* as() const { return static_cast<T*>(p); }
};

struct Camera {
    float pos[3], top_left[3], step_x[3], step_y[3];
    int32_t w = 0, h = 0;
};


struct IntegratorParams {
    int32_t ao_samples = 8;
    float ao_radius_frac = 0.1f;   // AO radius as a fraction of the bounds diagonal
    float ao_radius_abs = 0.0f;    // > 0 overrides the fraction
    int32_t pt_bounces = 4;
    float albedo = 0.7f;
    float ray_eps_frac = 1e-4f;    // PT ray offset as a fraction of the bounds diagonal
    uint64_t seed = 0x853c49e6748fea9bULL;
};

// Scratch and result buffers of one acceleration structure.
struct GridBuffers {
    DevBuf desc;          // GridDesc
    DevBuf cells;         // uint2 per cell (uniform) or packed top cell (two-level)
    DevBuf leaves;        // uint2 per leaf (two-level)
    DevBuf prims;         // uint32 per pair
    DevBuf keys_a, vals_a, keys_b, vals_b;   // pair ping-pong
    DevBuf block_sums;    // per-block counts of the pair-count pass
    DevBuf tile_hist;     // radix tile histograms
    DevBuf row_total;     // radix digit totals
    DevBuf leaf_cnt;      // two-level: references, then leaf cells per top cell, scanned in place to the first leaf
    DevBuf occ;           // two-level: one bit per top cell, set when the cell holds references
    DevBuf lkeys_a, lvals_a, lkeys_b, lvals_b;   // two-level: leaf pair ping-pong
    DevBuf scan_partials; // generic scan partial sums
    DevBuf tri_ranges;    // uint4 per triangle: its cell range (16-bit coordinates) and pair count
    DevBuf ref_ranges;    // two-level: uint4 per top-level reference: sub-cell range, first leaf, triangle
    size_t cap_cells = 0, cap_pairs = 0, cap_top_pairs = 0, cap_leaves = 0, cap_leaf_pairs = 0;
    // largest sizes seen by a completed build: the capacities (which size the count, scan
    // and sort launches) follow them with headroom instead of the first estimates
    size_t seen_pairs = 0, seen_leaves = 0, seen_leaf_pairs = 0;
};

struct Stats {
    uint64_t rays = 0;
};

}  // namespace hr

struct hr_ctx {
    int device = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::string err;

    // mesh
    uint32_t ntri = 0, nverts = 0, nkeyframes = 0;
    hr::DevBuf verts;      // float4 current frame
    hr::DevBuf idx;        // uint32 x3
    hr::DevBuf tris;       // float4 x3 per triangle: the current frame's vertices, written by each build
    hr::DevBuf keyframes;  // float4 x nverts x nkeyframes
    hr::DevBuf staging;    // float4 staging of host keyframes on upload
    int32_t frame_a = 0, frame_b = 0;
    float frame_coeff = 1.0f;
    hr::DevBuf frame_sel;  // int4 (frame a, frame b, coeff bits, 0) read by the build's lerp kernel
    int32_t frame_sel_host[3] = {0, 0, 0};   // what the last k_frame_select wrote there
    bool frame_sel_valid = false;
    bool have_frame = false;     // a frame (static or lerp request) is set
    bool lerp_pending = false;   // the next build interpolates resident keyframes

    // grid
    float top_density = 0.0625f, leaf_density = 2.0f, ug_density = 5.0f;
    int32_t built_kind = -1;
    bool built = false;
    hr::GridBuffers g;
    hr::GridDesc host_desc{};    // last downloaded descriptor
    hr::GridDesc* desc_pinned = nullptr;   // descriptor of an asynchronous build (pinned)
    bool async_pending = false;  // an asynchronous build awaits build_async_result
    hr::DevBuf counters;         // uint64 ray counters
    cudaGraphExec_t build_exec = nullptr;   // captured static rebuild, and what it was captured for
    std::vector<uint8_t> build_key, last_build_key;
    uint64_t build_graph_launches = 0;
    int build_graph_stages = 0;
    bool build_graph_ok = true;      // false once a capture failed: build directly
    bool build_capturing = false;
    // uniform builds of at most this many triangles run as one cooperative launch
    // (build_small.cu); HAPPYRAY_SMALL_BUILD_MAX_TRIS at context creation, 0: never
    uint32_t small_build_max_tris = 131072;
    int small_build_bps = -1;        // resident blocks per SM of that kernel (-1: not queried)
    hr::DevBuf build_bar;            // its grid barrier words
    uint64_t launches = 0;       // kernels enqueued by this context (host-side count)
    bool collect_stats = false;  // render kernels accumulate cells visited / triangle tests
    cudaEvent_t ev[16] = {};
    bool timing = false;
    float stage_ms[16] = {};
    int nstages = 0;

    // camera / integrators
    hr::Camera cam;
    bool have_camera = false;
    hr::LightSet lights;         // host copy of the light collection (default: one 0.2 x 0.2 quad at z = 1)
    hr::DevBuf lights_dev;       // its device copy, read by the path tracer
    hr::DevBuf tri_nrm;          // 3 vertex normals (float4) per triangle, for the path tracer
    hr::DevBuf tri_alb;          // diffuse albedo per triangle, for the path tracer
    uint32_t nrm_ntri = 0, alb_ntri = 0;   // triangle count they were given for (0: none)
    hr::IntegratorParams ip;
    hr::DevBuf fb;               // float3 framebuffer (device)
    hr::DevBuf out_id, out_t, out_u, out_v, ray_in;  // ray-query staging
    hr::DevBuf hit_t, hit_tri, unocc, queue;          // AO wavefront: per-pixel hits, hit-pixel queue
    cudaEvent_t rev[8] = {};     // render kernel boundaries (timing mode)
    int nrender_ev = 0;
    void* pinned = nullptr;      // pinned host staging
    size_t pinned_bytes = 0;
};

namespace hr {

// status helpers (capi.cu)
int set_error(hr_ctx* c, int code, const char* fmt, ...);
int cuda_check(hr_ctx* c, cudaError_t e, const char* what);
int ensure(hr_ctx* c, DevBuf& b, size_t bytes);
// xyz (3 floats per vertex, device) -> float4 with w = 0
void expand_xyz(const float* xyz, float4* out, size_t n, int grid, cudaStream_t s);
// Builds a light collection of n lights (LightSource.hpp:38-198) in binary32 on the host:
// corners, edges and normals are xyz triples; normals may be null (then n = unit e2 x e1).
// Returns 0, or 1 when n is outside 1..kMaxLights or a light is degenerate.
int make_light_set(LightSet* out, uint32_t n, const float* corners, const float* e1, const float* e2,
                   const float* normals, const float* emissions);
// Makes `n` lights the context's collection (host and device copies).
int set_lights(hr_ctx* c, uint32_t n, const float* corners, const float* e1, const float* e2, const float* normals,
               const float* emissions);
// Camera::init (Camera.h:40-64) in binary32 on the host
void camera_init(Camera* c, const float pos[3], const float fwd[3], const float up[3], float fov, int w, int h);

// makes `dev` current for the lifetime of the guard
struct DeviceGuard {
    explicit DeviceGuard(int dev) { cudaGetDevice(&prev); if (prev != dev) cudaSetDevice(dev); }
    ~DeviceGuard() { int cur; cudaGetDevice(&cur); if (cur != prev) cudaSetDevice(prev); }
    int prev = 0;
};

// build.cu
int build_grid(hr_ctx* c, int32_t kind, int32_t exact);
// Enqueue one build with the current capacities and no host sync (a grid kind not built
// before is built synchronously).  Once the stream has passed it, build_async_result
// reports whether it fit; if not, the capacities are grown and the grid must be rebuilt.
int build_grid_async(hr_ctx* c, int32_t kind, int32_t exact);
void drop_build_graph(hr_ctx* c);   // frees the captured rebuild (hr_destroy)
int build_async_result(hr_ctx* c, bool* fit);

// build_small.cu: the uniform build of a small scene as one cooperative launch.  Returns
// 0 with *done = false when the scene does not qualify (the caller runs the pipeline).
int build_small_uniform(hr_ctx* c, int32_t exact, int key_bits, bool* done);

// sort.cu
int radix_sort_pairs(hr_ctx* c, const uint32_t* keys_in, const uint32_t* vals_in,
                     uint32_t* keys_tmp, uint32_t* vals_tmp, uint32_t* keys_out, uint32_t* vals_out,
                     const uint32_t* d_count, size_t cap_count, int key_bits,
                     uint32_t* tile_hist, size_t tile_hist_bytes, uint32_t* row_total, cudaStream_t s);
size_t radix_tile_hist_words(size_t cap_count, int key_bits);
// passes radix_sort_pairs makes for keys of key_bits bits (the output of an odd count ends in
// the temporary buffers' pass parity: the caller picks keys_out accordingly)
int radix_sort_passes(int key_bits);
constexpr int kRadixRowWords = 512;   // row_total words radix_sort_pairs needs (9-bit digits)
int exclusive_scan_u32(hr_ctx* c, uint32_t* data, const uint32_t* d_count, size_t cap_count,
                       uint32_t* d_total, uint32_t* partials, cudaStream_t s);
int exclusive_scan_u32x2(hr_ctx* c, uint2* data, const uint32_t* d_count, size_t cap_count,
                         uint32_t* d_total_x, uint32_t* d_total_y, uint2* partials, cudaStream_t s);
size_t scan_partials_words(size_t cap_count);
// Exclusive scan of per-block counts in place; the total goes to *d_total, or, when it
// exceeds cap, ovf_bit is set in *ovf, the total to *d_req and *d_total becomes 0.
int scan_block_sums(hr_ctx* c, uint32_t* sums, uint32_t n, uint32_t* d_total, uint32_t* ovf,
                    uint32_t cap, uint32_t ovf_bit, uint32_t* d_req, cudaStream_t s);

// jobs.cu: persistent rendering of many jobs (batched and served forms).  One job is a
// grid, a camera or a ray list, an integrator and an output; the kernel's warps take
// 32-pixel (32-ray) tiles of any job from one work counter.
enum : int32_t { kJobPrimary = 0, kJobPath = 1, kJobAO = 3, kJobRays = 16 };
struct Job {
    const float4* tris;              // per-triangle vertices of the grid's mesh
    const uint2* cells;
    const uint2* leaves;
    const uint32_t* prims;
    const GridDesc* desc;
    const uint32_t* cells_offset;    // nullable: added to cells (grids of one batch share arrays)
    const uint32_t* occ;             // nullable: top-cell occupancy bits, indexed like cells before the offset
    const GridDesc* status;          // nullable (then desc): a grid whose build overflowed or failed is not traced
    float* fb;                       // render jobs: float RGB per pixel
    const float* org;                // ray jobs: 3 floats per ray
    const float* dir;
    int32_t* out_id;                 // ray jobs: closest hit (triangle id or -1), t, u, v
    float* out_t;
    float* out_u;
    float* out_v;
    float cam_pos[3], cam_tl[3], cam_sx[3], cam_sy[3];
    int32_t w, h;                    // render jobs: image size; ray jobs: w = ray count
    const LightSet* lights;          // path jobs: the light collection (device memory)
    uint32_t ntri;
    int32_t kind;                    // kTwoLevel
    int32_t mode;                    // kJob*
    int32_t spp;                     // AO samples per hit pixel, or paths per pixel
    int32_t image_id;                // first image id (progressive blend weight 1 / (id + 1))
    int32_t bounces;
    float albedo, alpha_frac, alpha_abs, eps_frac;
    uint64_t seed;
};
// tiles of one job for tile width tw (32 / tw rows)
uint32_t job_tiles(const Job& j, int32_t tw);
// resident blocks per SM of the job kernel for a block size (pt: the path-tracing variant)
int job_blocks_per_sm(int32_t block_threads, bool pt);
// launch the persistent job kernel over njobs jobs whose tile prefix sums are d_tile_off
// (njobs + 1 entries); *d_work must be zero.  pt selects the variant for kJobPath jobs,
// which runs only those; the other variant runs every other mode.
int launch_jobs(hr_ctx* c, const Job* d_jobs, const uint32_t* d_tile_off, uint32_t njobs, uint32_t* d_work,
                int32_t tile_w, int32_t block_threads, int32_t nblocks, bool pt, cudaStream_t s);

// trace.cu
int launch_trace_rays(hr_ctx* c, const float* org, const float* dir, uint32_t n, int32_t* id,
                      float* t, float* u, float* v, uint32_t* stats);
int launch_trace_primary(hr_ctx* c, int32_t* id, float* t, float* u, float* v, uint32_t* stats);
int launch_render(hr_ctx* c, int32_t mode, int32_t image_id, float* d_fb);
int launch_occluded(hr_ctx* c, const float* org, const float* dir, const float* tmax, uint32_t n,
                    uint8_t* occluded);
int launch_render_rays(hr_ctx* c, const float* org, const float* dir, uint32_t n, int32_t image_id, float* fb);

}  // namespace hr
