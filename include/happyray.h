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
/* RTEngine::setLights (RTEngine.h:57): one quad light, corner + edges, emits along -z */
hr_status hr_set_light(hr_ctx *ctx, const float corner[3], const float edge1[3],
                       const float edge2[3], float emission);
/* Integrator parameters: AO samples per hit and radius (fraction of the bounds diagonal
 * if ao_radius < 0, absolute otherwise), PT extension rays, Lambertian albedo, seed. */
hr_status hr_set_integrator(hr_ctx *ctx, int32_t ao_samples, float ao_radius,
                            int32_t pt_bounces, float albedo, uint64_t seed);
/* RTEngine::renderFrame (RTEngine.h:59, RTEngine.cu:398-444): progressive blend into a
 * float3-per-pixel frame buffer.  Host buffer: copied in and out. */
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
 * the scratch address; make it before any stream capture.  All calls share the one
 * scratch array: calls that overlap on the GPU race, so serialise them. */
hr_status hr_radix_sort_pairs_noalloc(void *stream, uint32_t *d_keys, uint32_t *d_values,
                                      uint32_t n, int32_t key_bits);

#ifdef __cplusplus
}
#endif
#endif
