/*
 * happyray.h -- C-ABI of libhappyray_b200.so, the B200 (sm_100a) grid-build and
 * grid-traversal engine that is a drop-in for the javorkk/happyray hot path.
 *
 * All entry points take plain pointers and sizes.  "Host" pointers are ordinary
 * (pageable or pinned) CPU memory; entry points with the _device suffix take device
 * pointers of the context's GPU.  Every call returns an hr_status; hr_last_error()
 * gives the message of the last failing call.  No call exits the process.
 *
 * Threading: one hr_ctx per host thread (or stream).  Work is enqueued on the
 * context's stream; calls that return data to host memory synchronise that stream.
 *
 * Reference interfaces (paths inside the reference project):
 *   RTEngine static API         src/RT/RTEngine.h:36-68, src/RT/RTEngine.cu:190-474
 *   Builder concept             src/RT/Algorithm/UGridSortBuilder.h:64-120,
 *                               src/RT/Algorithm/TLGridSortBuilder.h:66-133
 *   Grid descriptors            src/RT/Structure/UniformGrid.h:37-138,
 *                               src/RT/Structure/TwoLevelGrid.h:38-230
 *   Ray query (binary rays)     src/RT/Integrator/SimpleRayTraverser.h:168-261
 *   Scan / radix sort helpers   src/Utils/Scan.cu:39-58, src/Utils/Sort.cu:29-53
 */
#ifndef HAPPYRAY_H
#define HAPPYRAY_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum hr_status {
    HR_OK = 0,
    HR_ERR_INVALID_ARG = 1,
    HR_ERR_OUT_OF_MEMORY = 2,
    HR_ERR_CAPACITY_RETRY = 3,
    HR_ERR_DEVICE = 4,
    HR_ERR_TIMEOUT = 5,
    HR_ERR_NOT_READY = 6
} hr_status;

/* grid kinds: the reference selects them at compile time (RTEngine.cu:62-89) */
#define HR_GRID_UNIFORM 0
#define HR_GRID_TWO_LEVEL 1

/* render modes, numbered as RTEngine::renderFrame's switch (RTEngine.cu:410-441) */
#define HR_RENDER_PRIMARY 0
#define HR_RENDER_PATH 1
#define HR_RENDER_PATH_SINGLE_KERNEL 2
#define HR_RENDER_AO 3

typedef struct hr_ctx hr_ctx;

/* Grid parameters after a build (UniformGrid / TwoLevelGrid POD fields). */
typedef struct hr_grid_info {
    int32_t kind;
    int32_t res[3];
    float bounds_min[3], bounds_max[3];
    float cell_size[3], cell_size_rcp[3];
    uint32_t num_cells;      /* uniform cells, or top-level cells */
    uint32_t num_leaves;     /* two-level: leaf cells */
    uint32_t num_pairs;      /* primitive references in the final `primitives` array */
    uint32_t num_top_pairs;  /* two-level: top-level references */
} hr_grid_info;

/* RTEngine::init (RTEngine.h:40).  device: CUDA ordinal; stream: a cudaStream_t to
 * run on, or NULL for a context-owned non-blocking stream. */
hr_status hr_create(hr_ctx **out, int32_t device, void *stream);
/* RTEngine::cleanup (RTEngine.h:62) */
void hr_destroy(hr_ctx *ctx);
const char *hr_last_error(const hr_ctx *ctx);

/* RTEngine::upload(frame1, frame2, coeff) (RTEngine.h:42-45, RTEngine.cu:194-215):
 * vertices v = frame1 * (1 - coeff) + frame2 * coeff (xyz float triples, host),
 * triangle indices (3 uint32 per triangle, host).  The interpolation and the
 * bounds run on the device inside the next hr_build. */
hr_status hr_upload(hr_ctx *ctx, const float *frame1_xyz, const float *frame2_xyz,
                    uint32_t num_vertices, const uint32_t *tri_idx, uint32_t num_tris,
                    float coeff);
/* Resident key frames (AnimationManager keyframes, AnimationManager.hpp:46-138):
 * num_keyframes * num_vertices xyz triples, host. */
hr_status hr_set_keyframes(hr_ctx *ctx, const float *xyz, uint32_t num_keyframes,
                           uint32_t num_vertices, const uint32_t *tri_idx, uint32_t num_tris);
/* Frame selection of AnimationManager::getFrameId / getNextFrameId /
 * getInterpolationCoefficient (AnimationManager.hpp:68-97): key frame floor(t), next
 * (floor(t) + 1 + (size_t)step) mod K, coefficient frac(t).  Interpolated in hr_build. */
hr_status hr_set_frame_time(hr_ctx *ctx, float frame_time, float step_size);
/* RTEngine::setGridDensities (RTEngine.h:60, RTEngine.cu:446-450); uniform density
 * separately (RTEngine.cu:87). */
hr_status hr_set_grid_densities(hr_ctx *ctx, float top_level, float leaf_level);
hr_status hr_set_uniform_density(hr_ctx *ctx, float density);
/* RTEngine::buildAccStruct (RTEngine.cu:354-368): grid_kind HR_GRID_*, exact = exact
 * triangle insertion for the uniform grid (RTEngine.cu:82-84). */
hr_status hr_build(hr_ctx *ctx, int32_t grid_kind, int32_t exact);
hr_status hr_grid_get_info(hr_ctx *ctx, hr_grid_info *info);
/* Copies the built structure to host: cells (2 uint32 per cell: uniform {begin,end},
 * two-level packed TwoLevelGridCell), leaves (2 uint32 per leaf, two-level only, may be
 * NULL), prims (num_pairs uint32). */
hr_status hr_grid_download(hr_ctx *ctx, uint32_t *cells, uint32_t *leaves, uint32_t *prims);
/* Per-stage build times in ms of the last build (enable with hr_set_timing). */
hr_status hr_set_timing(hr_ctx *ctx, int32_t enable);
int32_t hr_get_stage_times(hr_ctx *ctx, float *ms, int32_t max_stages);
/* Interpolated vertices of the current frame (float4 per vertex) to host. */
hr_status hr_download_vertices(hr_ctx *ctx, float *xyzw);

/* RTEngine::setCamera (RTEngine.h:49-55, Camera.h:40-64) */
hr_status hr_set_camera(hr_ctx *ctx, const float position[3], const float orientation[3],
                        const float up[3], float fov_deg, int32_t res_x, int32_t res_y);
/* RTEngine::setLights (RTEngine.h:57, RTEngine.cu:393-396) for one light: a parallelogram
 * corner + s * edge1 + t * edge2 (s, t in [0, 1]) emitting radiance `emission` towards the
 * side of edge2 x edge1 (-z for edges along +x and +y).  Replaces the collection. */
hr_status hr_set_light(hr_ctx *ctx, const float corner[3], const float edge1[3],
                       const float edge2[3], float emission);
/* RTEngine::setLights with an AreaLightSourceCollection (LightSource.hpp:102-198): n lights
 * (1..64), corner / edge / normal xyz triples and one scalar radiance each (host arrays).
 * normals may be NULL (then each light emits towards its edge2 x edge1); a given normal is
 * used as is (unit length, the emitting side).  The path tracer picks a light per
 * next-event sample with probability area * emission / total, by the collection's
 * inclusive running sum of those weights (getLight, LightSource.hpp:114-126, CDF built by
 * InclusiveSum, Scan.cu:81-100), and divides its contribution by that probability.
 * Takes effect for renders enqueued after it returns.  HR_ERR_INVALID_ARG for n outside
 * 1..64, a degenerate light or a negative emission. */
hr_status hr_set_lights(hr_ctx *ctx, uint32_t n, const float *corners, const float *edge1s,
                        const float *edge2s, const float *normals, const float *emissions);
/* Shading normals of the mesh for the path tracer (WFObject normals and the faces' normal
 * indices, WFObject.hpp:96-106; RTEngine::upload's uploadObjFrameNormalData,
 * RTEngine.cu:205-209): num_normals xyz triples and 3 normal indices per triangle of the
 * current mesh (host).  At a hit the path tracer shades with the vertex normals blended as
 * PathTracer.h:111-136 does (weights of simpleShade), normalised, facing the ray.  Null
 * arguments remove them (geometric normals); a new mesh upload with another triangle count
 * drops them. */
hr_status hr_set_normals(hr_ctx *ctx, const float *normals_xyz, uint32_t num_normals,
                         const uint32_t *tri_normal_idx);
/* Per-triangle materials for the path tracer (the per-triangle PhongMaterial array,
 * RTEngine.cu:211, PathTracer.h:138): a table of num_materials diffuse albedos (scalar: the
 * path tracer's radiance is grey) and one material index per triangle of the current mesh
 * (host).  Null arguments remove them (hr_set_integrator's albedo for every triangle). */
hr_status hr_set_materials(hr_ctx *ctx, const float *albedo, uint32_t num_materials,
                           const uint32_t *tri_material);
/* Integrator parameters: AO samples per hit and radius (fraction of the bounds diagonal
 * if ao_radius < 0, absolute otherwise), PT extension rays, Lambertian albedo, seed. */
hr_status hr_set_integrator(hr_ctx *ctx, int32_t ao_samples, float ao_radius,
                            int32_t pt_bounces, float albedo, uint64_t seed);
/* RTEngine::renderFrame (RTEngine.h:59, RTEngine.cu:398-444): progressive blend into a
 * float3-per-pixel frame buffer, new = old * (1 - 1/(image_id+1)) + value / (image_id+1).
 * Host buffer: copied in and out (image 0 starts from zeros).  Device buffer: blended in
 * place, so it must hold finite values (e.g. zeros) before image 0. */
hr_status hr_render(hr_ctx *ctx, int32_t mode, int32_t image_id, float *framebuffer_rgb);
hr_status hr_render_device(hr_ctx *ctx, int32_t mode, int32_t image_id, float *d_framebuffer_rgb);
/* Ray query (SimpleRayTraverser.h:168-181 + RayTracingKernels.h:47-152): closest hit per
 * ray; org/dir are xyz float triples; id = triangle id or -1, t (FLT_MAX on miss), u, v =
 * barycentric weights of the triangle's 2nd and 3rd vertex. */
hr_status hr_trace_rays(hr_ctx *ctx, const float *org, const float *dir, uint32_t n,
                        int32_t *id, float *t, float *u, float *v);
hr_status hr_trace_rays_device(hr_ctx *ctx, const float *d_org, const float *d_dir, uint32_t n,
                               int32_t *d_id, float *d_t, float *d_u, float *d_v);
/* Camera rays of the current camera (RegularPrimaryRayGenerator, RayGenerators.h:40-69). */
hr_status hr_trace_primary_device(hr_ctx *ctx, int32_t *d_id, float *d_t, float *d_u, float *d_v,
                                  uint32_t *d_stats);
/* The ray-file form of RTEngine::renderFrame mode 0 (RTEngine.cu:410-414,
 * SimpleRayTraverser.h:166-180): ray i (xyz origin and direction triples, device) is traced
 * and shaded as a mode-0 camera ray (simpleShade) into pixel i of the float3 frame buffer
 * (device, n pixels), blended with weight 1 / (image_id + 1). */
hr_status hr_render_rays_device(hr_ctx *ctx, const float *d_org, const float *d_dir, uint32_t n,
                                int32_t image_id, float *d_framebuffer_rgb);
/* Any-hit within (1e-4, tmax[i]) per ray (shadow / AO traversal, UGridTraverser.h:68-74). */
hr_status hr_occluded_device(hr_ctx *ctx, const float *d_org, const float *d_dir,
                             const float *d_tmax, uint32_t n, uint8_t *d_occluded);
/* Rays traced by the render calls since the last reset. */
hr_status hr_get_ray_count(hr_ctx *ctx, uint64_t *rays, int32_t reset);
/* Traversal statistics of the render calls (the reference's debug counters have no
 * equivalent; these size the algorithmic bytes of a frame): with enable != 0 the
 * render kernels also count grid cells visited and triangle tests.  out[0] rays,
 * out[1] cells visited, out[2] triangle tests, out[3] kernels launched by the context;
 * out[4..6] the rays / cells / tests of the secondary pass alone (AO samples, shadow
 * rays); out[7] reserved. */
hr_status hr_set_stats(hr_ctx *ctx, int32_t enable);
hr_status hr_get_counters(hr_ctx *ctx, uint64_t out[8], int32_t reset);
/* With timing enabled (hr_set_timing): device time in ms of each kernel of the last
 * render call, in launch order (AO: primary pass, AO samples, shading).  Returns the
 * number of kernels written. */
int32_t hr_get_render_times(hr_ctx *ctx, float *ms, int32_t max_kernels);
hr_status hr_sync(hr_ctx *ctx);
/* RTEngine::getBoundingBoxDiagonalLength (RTEngine.h:64, RTEngine.cu:190-193) */
float hr_bounds_diagonal(hr_ctx *ctx);

/* Stand-alone primitives of the build pipeline (device pointers):
 * ExclusiveScan (Scan.cu:39-58) and RadixSort (Sort.cu:31-53), stable, over the low
 * key_bits bits.  Scratch comes from the context (grow-only). */
hr_status hr_exclusive_scan_device(hr_ctx *ctx, uint32_t *d_data, uint32_t n);
hr_status hr_radix_sort_pairs_device(hr_ctx *ctx, uint32_t *d_keys, uint32_t *d_values,
                                     uint32_t n, int32_t key_bits);

/* Largest n accepted by hr_radix_sort_pairs_noalloc. */
#define HR_NOALLOC_MAX_PAIRS (1u << 20)
/* The same stable radix sort as hr_radix_sort_pairs_device, for callers that must not
 * allocate device memory: a renderer or serving process that reserves its whole HBM
 * budget up front cannot call cudaMalloc inside its frame / request loop, where an
 * allocation may stall the device or fail under memory pressure.  No counterpart in
 * the reference (its RadixSort allocates through CUB's caching allocator).
 * Needs no context and allocates nothing: the scratch is a static per-GPU array of about
 * 8.5 MiB, held by every GPU that loads the library until the process exits.  Sorts
 * d_keys / d_values (device pointers of the current device) in place on `stream`
 * (cudaStream_t, NULL = default stream).  Returns HR_ERR_INVALID_ARG if n exceeds
 * HR_NOALLOC_MAX_PAIRS or key_bits is outside 1..32.  The first call on a device looks up
 * the scratch address; make it before any stream capture.  The address is kept for the
 * process, so do not use this entry point across a cudaDeviceReset of a device it has run
 * on.  All calls share the one scratch array: calls that overlap on the GPU race, so
 * serialise them. */
hr_status hr_radix_sort_pairs_noalloc(void *stream, uint32_t *d_keys, uint32_t *d_values,
                                      uint32_t n, int32_t key_bits);

/* Diagnostics: the L2-resident read rate of the current device in GB/s.  One kernel reads
 * a 32 MiB buffer 50 times through L2 (ld.global.cg, bypassing L1), timed with CUDA
 * events on `stream` (cudaStream_t, NULL = default stream).  The traversal kernels' working
 * sets live mostly in L2; benchmarks report their algorithmic bytes against this rate as
 * well as against the HBM copy rate.  No counterpart in the reference. */
hr_status hr_probe_l2_read(void *stream, double *gbs);

/* ---------------------------------------------------------------------------------
 * Batched scenes.  No counterpart in the reference, whose RTEngine holds one scene in
 * static globals (RTEngine.cu:91-181); it is the per-scene path above run for many
 * independent scenes at once.  All scenes of a batch get a two-level grid
 * (TLGridSortBuilder.h:66-452) built by ONE segmented pipeline whose launch count does
 * not depend on the number of scenes, and are rendered by ONE persistent traversal
 * launch; the whole step is captured in a CUDA graph and replayed.  Each scene's grid
 * and image are bit-identical to what the per-scene path gives for the same scene,
 * densities, camera, samples and seed.
 */
typedef struct hr_batch hr_batch;

typedef struct hr_batch_scene {
    const float *vertices_xyz;      /* host, 3 floats per vertex */
    uint32_t num_vertices;
    const uint32_t *indices;        /* host, 3 scene-local vertex indices per triangle */
    uint32_t num_triangles;         /* >= 1 */
    float cam_position[3], cam_orientation[3], cam_up[3];
    float cam_fov_deg;
    int32_t width, height;
    int32_t ao_samples;             /* 0: primary rays only (HR_RENDER_PRIMARY shading);
                                       > 0: HR_RENDER_AO with this many samples per hit */
    float top_density, leaf_density;  /* <= 0: the batch defaults (1/16, 2) */
} hr_batch_scene;

typedef struct hr_batch_tuning {
    float top_density, leaf_density;  /* applied to every scene */
    int32_t block_threads;            /* persistent traversal block size: 64, 128 or 256 */
    int32_t tile_width;               /* pixel tile of one warp: tile_width x (32 / tile_width) */
    float ms_per_step;                /* measured build + render time of the batch */
    int32_t trials;                   /* configurations timed */
} hr_batch_tuning;

hr_status hr_batch_create(hr_batch **out, int32_t device, void *stream);
void hr_batch_destroy(hr_batch *batch);
const char *hr_batch_last_error(const hr_batch *batch);
/* Copies the scenes' meshes and cameras to the device (replacing any previous set). */
hr_status hr_batch_set_scenes(hr_batch *batch, const hr_batch_scene *scenes, uint32_t num_scenes);
/* Grid densities of one scene (scene < num_scenes) or of all (scene = UINT32_MAX). */
hr_status hr_batch_set_densities(hr_batch *batch, uint32_t scene, float top_density, float leaf_density);
/* Launch shape of the persistent traversal: block_threads in {32, 64, ..., 256}, tile_width
 * in {1, 2, 4, 8, 16, 32}. */
hr_status hr_batch_set_launch(hr_batch *batch, int32_t block_threads, int32_t tile_width);
/* AO radius as a fraction of each scene's bounds diagonal, and the PCG32 sequence seed. */
hr_status hr_batch_set_integrator(hr_batch *batch, float ao_radius_fraction, uint64_t seed);
/* use_graph != 0 (default): a step is one replay of a captured CUDA graph. */
hr_status hr_batch_set_graph(hr_batch *batch, int32_t use_graph);
/* New vertex positions for every scene, same meshes (host, 3 floats per vertex, scenes
 * concatenated in order; num_vertices = the batch total).  The next step uses them. */
hr_status hr_batch_set_vertices(hr_batch *batch, const float *vertices_xyz, uint32_t num_vertices);
/* One step: rebuild every scene's grid and render every scene into its framebuffer
 * (progressive blend with weight 1 / (image_id + 1), as hr_render).  Synchronous. */
hr_status hr_batch_run(hr_batch *batch, int32_t image_id);
/* Device time of the last step: build, render (ms; -1 when not measured) and total. */
hr_status hr_batch_get_times(hr_batch *batch, float *build_ms, float *render_ms, float *total_ms);
/* out[0] rays, out[1] kernels launched, out[2] scenes, out[3] pixels, out[4] secondary
 * rays, out[5..7] reserved; reset != 0 zeroes the ray counts. */
hr_status hr_batch_get_counters(hr_batch *batch, uint64_t out[8], int32_t reset);
/* The framebuffer (float RGB per pixel) of one scene: host copy, or its device address. */
hr_status hr_batch_get_image(hr_batch *batch, uint32_t scene, float *rgb);
hr_status hr_batch_image_device(hr_batch *batch, uint32_t scene, float **d_rgb);
/* Every scene's framebuffer, scenes concatenated in order (num_floats = 3 x total pixels). */
hr_status hr_batch_download_images(hr_batch *batch, float *rgb, uint64_t num_floats);
/* One scene's grid, in the per-scene layout of hr_grid_get_info / hr_grid_download
 * (scene-local cell, leaf, pair and triangle indices). */
hr_status hr_batch_grid_info(hr_batch *batch, uint32_t scene, hr_grid_info *info);
hr_status hr_batch_grid_download(hr_batch *batch, uint32_t scene, uint32_t *cells, uint32_t *leaves,
                                 uint32_t *prims);
/* Autotuner: times top x leaf densities {1/32, 1/16, 1/8, 1/4} x {1, 2, 4, 8}, then
 * block_threads {64, 128, 256} x tile_width {4, 8, 16} at the best densities, each on
 * `reps` graph replays of the current batch; applies and returns the fastest. */
hr_status hr_batch_autotune(hr_batch *batch, int32_t reps, hr_batch_tuning *best);

/* ---------------------------------------------------------------------------------
 * Served rendering.  No counterpart in the reference (its CUDAApplication renders one
 * scene per process, CUDAApplication.cu:116-160).  A server keeps animated scenes
 * resident (key frames + the grid of one frame time each, hr_set_keyframes /
 * hr_set_frame_time semantics) and answers render and ray-query requests from any host
 * thread.  In HR_SERVER_BATCHED mode a worker thread admits queued requests (FIFO) while
 * their buffers fit the HBM budget, groups them into waves (one frame time per scene per
 * wave), rebuilds the grids of scenes whose frame time changed -- asynchronously, on the
 * scene's own stream, after the last wave reading the old grid -- and traces every request
 * of the wave in one persistent launch (rays batched across requests), with up to two
 * waves in flight so that the next wave's admission, rebuilds and copies overlap the
 * current one.  HR_SERVER_SERIAL runs the same requests one at a time through the
 * per-scene path (hr_build + hr_render / hr_trace_rays) over the same resident scenes.
 * HR_SERVER_PLAIN is the drop-in per-frame path as the reference's application drives it
 * (one context holding one scene, CUDAApplication.cu:116-160): per request hr_upload of the
 * two key frames around the frame time and the triangles (host copies kept by the server),
 * hr_build, hr_render, read back.  A request's result depends only on the request: it is
 * bit-identical in every mode, alone or among others.
 */
typedef struct hr_server hr_server;
#define HR_SERVER_BATCHED 0
#define HR_SERVER_SERIAL 1
#define HR_SERVER_PLAIN 2
#define HR_REQUEST_RENDER 0
#define HR_REQUEST_RAYS 1

typedef struct hr_request {
    uint32_t scene;
    float frame_time;             /* key-frame units, as hr_set_frame_time (step 0) */
    int32_t kind;                 /* HR_REQUEST_RENDER or HR_REQUEST_RAYS */
    /* render requests */
    int32_t mode;                 /* HR_RENDER_PRIMARY, HR_RENDER_AO or HR_RENDER_PATH */
    int32_t spp;                  /* AO samples per hit, or paths per pixel (image ids 0..spp-1) */
    float cam_position[3], cam_orientation[3], cam_up[3];
    float cam_fov_deg;
    int32_t width, height;
    uint64_t seed;
    float *out_rgb;               /* host, 3 floats per pixel; pinned memory lets the copy overlap */
    /* ray-query requests: closest hit of each ray (hr_trace_rays) */
    const float *ray_org, *ray_dir;   /* host, 3 floats per ray */
    uint32_t num_rays;
    int32_t *out_id;
    float *out_t, *out_u, *out_v;
} hr_request;

typedef struct hr_request_info {
    int32_t status;               /* 0 queued, 1 in flight, 2 done, < 0 failed (-hr_status) */
    uint32_t wave;                /* wave that traced it (batched mode) */
    uint64_t submit_ns, admit_ns, done_ns;   /* steady-clock times */
} hr_request_info;

typedef struct hr_server_stats {
    uint64_t completed, failed, waves, rebuilds, rays;
    uint64_t resident_bytes;      /* scenes: key frames, grids, vertex arrays */
    uint64_t peak_inflight_bytes; /* request buffers */
    uint64_t launches;
    double trace_ms;              /* device time of the waves' traversal launches (batched) */
    uint64_t watchdog_trips;      /* waves the watchdog declared stuck */
} hr_server_stats;

hr_status hr_server_create(hr_server **out, int32_t device, uint64_t hbm_budget_bytes, int32_t mode);
/* Finishes every queued request, then stops the worker and frees the scenes. */
void hr_server_destroy(hr_server *server);
const char *hr_server_last_error(const hr_server *server);
/* Makes a scene resident: key frames (host, num_keyframes x num_vertices xyz) and
 * triangles, two-level grid densities.  The grid capacities are sized by building every
 * key frame once.  Fails with HR_ERR_OUT_OF_MEMORY above the budget.  Call before the
 * first request of that scene. */
hr_status hr_server_add_scene(hr_server *server, const float *keyframes_xyz, uint32_t num_keyframes,
                              uint32_t num_vertices, const uint32_t *indices, uint32_t num_triangles,
                              float top_density, float leaf_density, uint32_t *scene_id);
/* Queues a request; the caller's buffers must stay valid until it is done. */
hr_status hr_server_submit(hr_server *server, const hr_request *request, uint64_t *request_id);
/* Waits until the request is done (HR_OK), failed (its error) or timeout_ms passed
 * (HR_ERR_TIMEOUT; timeout_ms < 0 waits without limit). */
hr_status hr_server_wait(hr_server *server, uint64_t request_id, int32_t timeout_ms);
/* Waits until no request is queued or in flight. */
hr_status hr_server_drain(hr_server *server, int32_t timeout_ms);
hr_status hr_server_request_info(hr_server *server, uint64_t request_id, hr_request_info *info);
hr_status hr_server_get_stats(hr_server *server, hr_server_stats *stats);
/* Watchdog (batched mode; no counterpart in the reference): a wave whose GPU work has not
 * finished timeout_ms after its launch is declared stuck and its requests fail at once
 * with HR_ERR_TIMEOUT, so that callers waiting on them are answered; the server keeps
 * admitting and launching.  GPU work cannot be recalled: a stuck wave's device buffers stay
 * held until it ends, later waves on the server's stream wait behind it, and its requests'
 * output buffers may still be written until then -- hr_server_drain returns only after
 * that.  0 turns the watchdog off (the default). */
hr_status hr_server_set_watchdog(hr_server *server, int32_t timeout_ms);
/* Test hook for the watchdog: the worker treats each of the next `waves` waves as
 * unfinished until stall_ms after its launch.  Host side only: the GPU work is untouched. */
hr_status hr_server_inject_stall(hr_server *server, uint32_t waves, int32_t stall_ms);

/* ---------------------------------------------------------------------------------
 * Scene input, ray files and images (host side; no GPU needed).
 *   scene.cfg            SceneConfigurationReader.cpp:29-190 ("obj", "frame prefix",
 *                        "frame suffix", "number of frames", "frame step", "camera",
 *                        "light", with their aliases; '#' comments)
 *   key-frame sequences  AnimationManager::read (AnimationLoader.cpp:50-101): frame i is
 *                        prefix + i zero-padded to the digits of (frames - 1) + suffix
 *   OBJ                  WFObject::read (WFObjectReader.cpp:320-560): v / f (v, v/t, v//n,
 *                        v/t/n; polygons fanned from their first vertex); vn, vt, o, g, s,
 *                        usemtl, mtllib are skipped; parsed in parallel over line chunks
 *   camera.cfg           CameraManager::read (CameraManager.cpp:33-168): position,
 *                        orientation, up, rotation (degrees), resX, resY, FOV
 *   light.cfg            LightSourceLoader::loadFromFile (LightSourceLoader.cpp:29-110)
 *   .rays                SimpleRayTraverser::loadRaysFromFile (SimpleRayTraverser.h:200-261):
 *                        headerless float32, 6 per ray (origin xyz, direction xyz)
 *   images               Image::writePNG (ImagePNG.cpp:160-215): each channel clamped to
 *                        [0, 1] and truncated to 8 bits; or PFM (float)
 */
typedef struct hr_scene hr_scene;

typedef struct hr_scene_info {
    uint32_t num_vertices, num_triangles, num_keyframes;
    float frame_step;
    int32_t has_camera;
    float cam_position[3], cam_orientation[3], cam_up[3];
    float cam_fov_deg;
    int32_t width, height;
    uint32_t num_lights;
    uint32_t num_normals;    /* shading normals (0: the OBJ had no vn) */
    uint32_t num_materials;  /* material table incl. "Default" (0: no usemtl / mtllib) */
} hr_scene_info;

#define HR_IMAGE_PNG 0
#define HR_IMAGE_PFM 1

/* A scene.cfg (animated or static, with its camera and lights), or one OBJ file as a
 * one-key-frame scene.  Paths inside scene.cfg are taken relative to the working
 * directory, else to the scene.cfg's directory.  threads <= 0: all hardware threads. */
hr_status hr_scene_load(const char *scene_cfg_path, int32_t threads, hr_scene **out);
hr_status hr_scene_load_obj(const char *obj_path, int32_t threads, hr_scene **out);
void hr_scene_free(hr_scene *scene);
/* Message of the last failing hr_scene_* / file call of the calling thread. */
const char *hr_io_last_error(void);
hr_status hr_scene_get_info(const hr_scene *scene, hr_scene_info *info);
/* num_keyframes x num_vertices x 3 floats, and num_triangles x 3 indices; owned by the scene. */
const float *hr_scene_keyframes(const hr_scene *scene);
const uint32_t *hr_scene_indices(const hr_scene *scene);
hr_status hr_scene_get_light(const hr_scene *scene, uint32_t light, float position[3], float edge1[3],
                             float edge2[3], float normal[3], float intensity[3]);
/* The OBJ's shading normals (num_normals x 3 floats: its vn, then one geometric normal per
 * face that lacks a normal index, as WFObjectReader.cpp:583-614) and num_triangles x 3
 * normal indices; null when num_normals is 0.  Key-frame scenes keep the first frame's
 * (RTEngine::upload's normals come from its first frame, RTEngine.cu:205-209). */
const float *hr_scene_normals(const hr_scene *scene);
const uint32_t *hr_scene_normal_indices(const hr_scene *scene);
/* The material table (num_materials diffuse albedos: "Default" 0.6774 first, then each
 * usemtl name in order of first use, its .mtl Kd as mean(min(Kd, 0.99)),
 * WFObjectReader.cpp:49-57, 135-258) and num_triangles material indices; null when
 * num_materials is 0.  Key-frame scenes keep the last frame's. */
const float *hr_scene_material_albedo(const hr_scene *scene);
const uint32_t *hr_scene_triangle_materials(const hr_scene *scene);
/* hr_set_keyframes with the scene's frames; its camera (hr_set_camera) if it has one; its
 * lights (hr_set_lights: corner = position, the file's normal, emission = mean intensity;
 * the first 64) if any; its shading normals (hr_set_normals) and materials
 * (hr_set_materials), or none of either. */
hr_status hr_scene_upload(hr_ctx *ctx, const hr_scene *scene);

hr_status hr_rays_file_count(const char *path, uint32_t *num_rays);
hr_status hr_rays_file_read(const char *path, float *org_dir, uint32_t num_rays);
hr_status hr_rays_file_write(const char *path, const float *org, const float *dir, uint32_t num_rays);
/* Closest hits of a ray query: per ray int32 id, then float32 t, u, v (16 bytes). */
hr_status hr_hits_file_write(const char *path, const int32_t *id, const float *t, const float *u,
                             const float *v, uint32_t num_rays);
/* A float RGB framebuffer (row 0 first) as PNG (8-bit RGB) or PFM (float RGB). */
hr_status hr_image_write(const char *path, const float *rgb, int32_t width, int32_t height, int32_t format);

/* ---------------------------------------------------------------------------------------
 * Instanced two-level grid hierarchy (reference: TwoLevelGridHierarchy.h,
 * TLGridHierarchySortBuilder.cu, TLGridHierarchyTraverser.h; RTEngine.cu:68-73 selects it
 * with densities 1.2 / 1.2).  Objects are consecutive triangle ranges of one mesh in their
 * own coordinates, each with its own uniform grid; instances place objects in the world
 * and are binned into a uniform grid over their world boxes.  A rigid-body frame only
 * changes the instances: hr_hier_build then rebuilds the instance grid alone.
 * ------------------------------------------------------------------------------------- */
typedef struct hr_hier hr_hier;

/* One instance: object index, the world -> object map as the three rows of the
 * reference's instances file (m_row_0..2: x' = m[0] x + m[1] y + m[2] z + m[3], y' from
 * m[4..7], z' from m[8..11]) and the instance's world-space box (AABB_min / AABB_max),
 * which must hold the transformed object. */
typedef struct hr_instance {
    uint32_t object;
    float m[12];
    float bmin[3], bmax[3];
} hr_instance;

typedef struct hr_hier_info {
    uint32_t num_objects, num_instances, num_triangles;
    uint32_t num_object_cells;   /* cells of all object grids */
    uint32_t num_pairs;          /* (cell, triangle) references of the object grids */
    int32_t top_res[3];          /* instance grid */
    uint32_t num_top_cells, num_top_pairs;
    float top_bmin[3], top_bmax[3];
    uint64_t launches;           /* kernels enqueued by this hierarchy so far */
} hr_hier_info;

/* Per-object grid as built (72 bytes, the layout hr_hier_download returns). */
typedef struct hr_hier_object {
    float bmin[3], bmax[3], cell_size[3], cell_size_rcp[3];
    int32_t res[3];
    uint32_t first_cell, first_triangle, num_triangles;
} hr_hier_object;

hr_status hr_hier_create(hr_hier **out, int32_t device, void *stream);
void hr_hier_destroy(hr_hier *h);
const char *hr_hier_last_error(const hr_hier *h);
/* Object-space mesh: nv xyz vertices, ntri index triples, object k = the next
 * object_tri_counts[k] triangles (every count > 0, the counts sum to ntri). */
hr_status hr_hier_set_objects(hr_hier *h, const float *verts_xyz, uint32_t nv, const uint32_t *idx, uint32_t ntri,
                              const uint32_t *object_tri_counts, uint32_t num_objects);
hr_status hr_hier_set_instances(hr_hier *h, const hr_instance *inst, uint32_t n);
/* instance-grid and object-grid densities (defaults 1.2, 1.2) */
hr_status hr_hier_set_densities(hr_hier *h, float top_density, float object_density);
/* Builds what changed: the object grids after hr_hier_set_objects / set_densities, the
 * instance grid always.  Synchronous. */
hr_status hr_hier_build(hr_hier *h);
hr_status hr_hier_get_info(hr_hier *h, hr_hier_info *info);
/* Host copies of the built arrays (any may be NULL): objects (num_objects records),
 * object cells (2 x num_object_cells), triangle lists (num_pairs), instance-grid cells
 * (2 x num_top_cells), instance lists (num_top_pairs). */
hr_status hr_hier_download(hr_hier *h, hr_hier_object *objects, uint32_t *object_cells, uint32_t *triangles,
                           uint32_t *top_cells, uint32_t *instances);
/* Closest hit through the hierarchy: instance id and triangle id (-1 on a miss), t, u, v.
 * Host buffers; the _device form takes device pointers and runs on the hierarchy's
 * stream without a sync. */
hr_status hr_hier_trace_rays(hr_hier *h, const float *org, const float *dir, uint32_t n, int32_t *inst_id,
                             int32_t *tri_id, float *t, float *u, float *v);
hr_status hr_hier_trace_rays_device(hr_hier *h, const float *org, const float *dir, uint32_t n, int32_t *inst_id,
                                    int32_t *tri_id, float *t, float *u, float *v);
/* hr_hier_trace_rays_device that also writes 5 counters per ray to stats (device):
 * instance-grid cells visited, instance boxes tested, instances entered, object-grid
 * cells visited, triangle tests. */
hr_status hr_hier_trace_stats_device(hr_hier *h, const float *org, const float *dir, uint32_t n, int32_t *inst_id,
                                     int32_t *tri_id, float *t, float *u, float *v, uint32_t *stats);
/* Any hit below tmax[i]: occluded[i] = 1 / 0 (host buffers). */
hr_status hr_hier_occluded(hr_hier *h, const float *org, const float *dir, const float *tmax, uint32_t n,
                           uint8_t *occluded);
/* The reference's instances file (WFObjectReader.cpp:762-825, WFObjWriter.cpp:94-111):
 * per instance "obj_id", "m_row_0..2" and "AABB_min / AABB_max" lines.  read: n_out gets
 * the count; up to cap records are stored (inst may be NULL to count). */
hr_status hr_instances_file_read(const char *path, hr_instance *inst, uint32_t cap, uint32_t *n_out);
hr_status hr_instances_file_write(const char *path, const hr_instance *inst, uint32_t n);

#ifdef __cplusplus
}
#endif
#endif
