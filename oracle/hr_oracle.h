/*
 * hr_oracle.h -- CPU oracle for the happyray grid-build + grid-traversal hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a CPU restatement of the reference algorithm
 * (javorkk/happyray) used by the tests, by smoke() and by the bench's CPU-baseline
 * leg as the checker.  It is never linked into, called by, or shipped with the
 * product library (happyray_b200/libhappyray_b200.so).
 *
 * Arithmetic contract: strict IEEE-754 binary32, every expression evaluated in the
 * order written, no FMA contraction (-ffp-contract=off), no fast-math.  The CUDA
 * kernels follow the same operation order, so integer results (cells, leaves,
 * primitive lists, hit ids) and float results (t, u, v) compare bit-exact.
 * A separate FP64 brute-force closest-hit routine checks t/u/v against exact
 * arithmetic with tie / near-edge flags.
 *
 * Reference files restated here (paths inside the reference project):
 *   src/Application/WFObjectUploader.h:48-119       keyframe lerp + padded bounds
 *   src/RT/Algorithm/UGridSortBuilder.h:64-407      uniform grid resolution + build order
 *   src/RT/Algorithm/UniformGridBuildKernels.h:40-105, 180-252, 384-487
 *   src/RT/Algorithm/UniformGridBuildKernels.cu:8-48, 224-383   exact triangle/box SAT
 *   src/RT/Algorithm/TLGridSortBuilder.h:66-452     two-level grid build order
 *   src/RT/Algorithm/TLGridBuildKernels.h:45-147, 304-409, 536-663, 750-834
 *   src/RT/Structure/TwoLevelGrid.h:38-161          top-cell packing
 *   src/RT/Algorithm/UGridTraverser.h:44-177        uniform-grid DDA
 *   src/RT/Algorithm/TLGridTraverser.h:45-354       two-level DDA
 *   src/RT/Algorithm/RayTriangleIntersector.h:38-92 Moller-Trumbore
 *   src/RT/Primitive/Camera.h:35-72                 pinhole camera
 */
#ifndef HR_ORACLE_H
#define HR_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    float    bmin[3], bmax[3];
    int32_t  res[3];
    float    cs[3], rcp[3];
    uint32_t ncells;
} orc_grid;

/* Grid kinds */
#define ORC_UG 0
#define ORC_TL 1

typedef struct {
    const float    *v4;      /* float4 vertices (x,y,z,w) */
    const uint32_t *idx;     /* 3 indices per triangle */
    uint32_t        ntri;
    int32_t         kind;    /* ORC_UG or ORC_TL */
    orc_grid        g;
    const uint32_t *cells;   /* UG: uint2 cell ranges; TL: packed top cells */
    const uint32_t *leaves;  /* TL: uint2 leaf ranges */
    const uint32_t *prims;   /* primitive (triangle id) lists */
    const float    *nrm3;    /* path tracer: 9 floats (3 vertex normals) per triangle, or NULL */
    const float    *alb;     /* path tracer: diffuse albedo per triangle, or NULL */
} orc_scene;

typedef struct {
    float   pos[3], top_left[3], step_x[3], step_y[3];
    int32_t w, h;
} orc_camera;

/* Area lights for the path tracer (AreaLightSource, LightSource.hpp:38-95): a parallelogram
 * corner + s*e1 + t*e2 (s, t in [0, 1]) emitting radiance `emission` towards the side its
 * unit normal points to.  A collection of lights (AreaLightSourceCollection,
 * LightSource.hpp:102-198) picks light k for a sample with probability w_k / W, w_k =
 * area_k * emission_k, from the inclusive running sum of the weights. */
#define ORC_MAX_LIGHTS 64
typedef struct {
    float corner[3], e1[3], e2[3], normal[3];
    float emission;
} orc_light;

/* ---- build ---- */
void orc_lerp_bounds(const float *f1, const float *f2, uint32_t nv, float coeff,
                     float *out4, float bmin[3], float bmax[3]);
void orc_grid_setup(const float bmin[3], const float bmax[3], uint32_t nprims,
                    float density, orc_grid *g);
float orc_pow_third(float x);

/* Uniform grid.  *cells gets 2*ncells uint32, *prims gets npairs uint32 (malloc'd). */
int orc_build_ug(const float *v4, const uint32_t *idx, uint32_t ntri,
                 const float bmin[3], const float bmax[3], float density, int exact,
                 orc_grid *g, uint32_t **cells, uint32_t **prims, uint32_t *npairs);

/* Two-level grid. */
int orc_build_tl(const float *v4, const uint32_t *idx, uint32_t ntri,
                 const float bmin[3], const float bmax[3], float top_density,
                 float leaf_density, orc_grid *g, uint32_t **top_cells,
                 uint32_t **leaves, uint32_t *nleaves, uint32_t **prims,
                 uint32_t *npairs, uint32_t *ntop_pairs);

void orc_free(void *p);

/* ---- camera / rays ---- */
void orc_camera_init(orc_camera *c, const float pos[3], const float fwd[3],
                     const float up[3], float fov_deg, int32_t w, int32_t h);
void orc_primary_rays(const orc_camera *c, float *org, float *dir);

/* ---- traversal (closest hit); stats may be NULL (2 uint32 per ray: cells, tests) ---- */
void orc_trace(const orc_scene *s, const float *org, const float *dir, uint32_t n,
               int32_t *id, float *t, float *u, float *v, uint32_t *stats);
void orc_trace_primary(const orc_scene *s, const orc_camera *c, int32_t *id,
                       float *t, float *u, float *v, uint32_t *stats);
/* any-hit within (1e-4, tmax): occluded[i] = 1/0 */
void orc_occluded(const orc_scene *s, const float *org, const float *dir,
                  const float *tmax, uint32_t n, uint8_t *occluded);

/* ---- integrators ---- */
/* AO: per pixel visibility in [0,1] averaged over spp cosine rays, progressive
 * blend into fb (float per pixel); counts[0] += rays traced.  pixel_stride
 * lets the baseline time a bounded sample (every k-th pixel). */
void orc_render_ao(const orc_scene *s, const orc_camera *c, int32_t spp, float alpha,
                   uint64_t seed, int32_t image_id, float *fb, uint32_t pixel_stride,
                   uint64_t *counts);
/* PT: scalar radiance per pixel, `bounces` extension rays, NEE per hit. */
/* render mode 0 (RTEngine.cu:409-424): regular 2 x 2 / Gaussian pixel samples, simpleShade
 * (SimpleIntegrator.h:41-126), progressive blend into fb (3 floats per pixel) */
void orc_render_primary(const orc_scene *s, const orc_camera *c, int32_t image_id, uint64_t seed, float *fb);
float orc_log_series(float x);
/* the ray-file form of render mode 0 (SimpleRayTraverser.h:166-180): ray i shaded into pixel i */
void orc_render_rays(const orc_scene *s, const float *org, const float *dir, uint32_t n, int32_t image_id,
                     float *fb);
void orc_render_pt(const orc_scene *s, const orc_camera *c, const orc_light *l, int32_t nlights,
                   int32_t bounces, float albedo, float ray_eps, uint64_t seed,
                   int32_t image_id, float *fb, uint32_t pixel_stride, uint64_t *counts);

/* ---- FP64 brute-force closest hit (flags: 1 t-tie, 2 near edge, 4 grazing) ---- */
void orc_brute_f64(const float *v4, const uint32_t *idx, uint32_t ntri,
                   const float *org, const float *dir, uint32_t n, int32_t *id,
                   double *t, double *u, double *v, uint8_t *flags);

/* ---- helpers shared with tests ---- */
void  orc_sincos2pi(float u, float *s, float *c);
float orc_pcg32_first_floats(uint64_t initstate, uint64_t initseq, int32_t k, float *out);
int   orc_num_threads(void);

/* ---- instanced two-level grid hierarchy ----
 * Objects are consecutive triangle ranges of one mesh (object-space vertices), each
 * with its own uniform grid (TLGridHierarchySortBuilder.cu:522-682 buildLevelTwo); the
 * instances (object, world -> object transform, world AABB) are binned into a uniform
 * grid over the instance boxes (TLGridHierarchySortBuilder.cu:373-520).  Traversal as
 * TLGridHierarchyTraverser.h:45-405. */
typedef struct {
    float    bmin[3], bmax[3], cs[3], rcp[3];
    int32_t  res[3];
    uint32_t cell_off, tri_begin, tri_count;
} orc_obj;

typedef struct {
    uint32_t obj;
    float    m[12];          /* world -> object rows: x' = m0 x + m1 y + m2 z + m3, y' = m4.., z' = m8.. */
    float    bmin[3], bmax[3];   /* world-space box of the instance */
} orc_inst;

typedef struct {
    const float    *v4;      /* object-space vertices (float4) */
    const uint32_t *idx;
    uint32_t        ntri, nobj, ninst;
    const orc_obj  *objs;
    const orc_inst *inst;
    orc_grid        top;     /* instance grid */
    const uint32_t *top_cells;   /* uint2 ranges into inst_ids */
    const uint32_t *inst_ids;
    const uint32_t *obj_cells;   /* uint2 ranges into prims; object k's cells start at cell_off */
    const uint32_t *prims;
} orc_hier;

/* objs (nobj) and top are filled; the arrays are malloc'd (orc_free). */
int orc_hier_build(const float *v4, const uint32_t *idx, uint32_t ntri, const uint32_t *obj_tri_counts,
                   uint32_t nobj, const orc_inst *inst, uint32_t ninst, float top_density, float leaf_density,
                   orc_obj *objs, orc_grid *top, uint32_t **obj_cells, uint32_t *nobj_cells, uint32_t **prims,
                   uint32_t *npairs, uint32_t **top_cells, uint32_t **inst_ids, uint32_t *ntop_pairs);
/* closest hit (tmax NULL: unbounded), or any hit below tmax[i] (anyhit = 1: inst_id >= 0
 * marks an occluded ray); inst_id / tri_id -1 on a miss */
void orc_hier_trace(const orc_hier *H, const float *org, const float *dir, const float *tmax, uint32_t n,
                    int anyhit, int32_t *inst_id, int32_t *tri_id, float *t, float *u, float *v);

#ifdef __cplusplus
}
#endif
#endif
