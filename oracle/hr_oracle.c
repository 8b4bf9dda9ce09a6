/*
 * hr_oracle.c -- CPU restatement of the happyray build + traversal hot path.
 *
 * TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the bench's
 * CPU-baseline / reference arm as the checker.  Not part of the product library.
 *
 * Compile with: gcc -O2 -fopenmp -ffp-contract=off -fno-fast-math (see oracle/Makefile).
 * Every float expression below is written in the evaluation order the CUDA kernels use.
 * Each function cites the reference file:line it follows (paths inside the reference).
 */
#include "hr_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_EPS 0.00001f             /* CUDAStdAfx.h:117 EPS */
#define ORC_ISECT_EPS 0.0001f        /* RayTriangleIntersector.h:36 INTERSECTION_EPS */
#define ORC_LEAF_REFS_MAX 16u        /* TLGridBuildKernels.h:77 numCellRefs <= 16 */
#define ORC_LEAFMASK 0x10000000u     /* TwoLevelGrid.h:58 LARGELEAFMASK */
#define ORC_NOTEMPTYMASK 0x40000000u /* TwoLevelGrid.h:60 LARGENOTEMPTYMASK */

/* ------------------------------------------------------------------------- */
/* scalar helpers: identical semantics to the device helpers (NaN-ignoring
 * min/max like fminf/fmaxf; ties return the first argument; saturating
 * float->int conversion with NaN -> 0, as cvt.rzi.s32.f32 does). */
static inline float hmin(float a, float b) { return (a != a) ? b : ((b < a) ? b : a); }
static inline float hmax(float a, float b) { return (a != a) ? b : ((b > a) ? b : a); }
static inline int32_t f2i(float x) {
    if (x != x) return 0;
    if (x >= 2147483648.0f) return 2147483647;
    if (x <= -2147483648.0f) return (int32_t)0x80000000u;
    return (int32_t)x;
}
static inline int32_t imax(int32_t a, int32_t b) { return a > b ? a : b; }
static inline int32_t imin(int32_t a, int32_t b) { return a < b ? a : b; }

typedef struct { float x, y, z; } f3;
static inline f3 mk(float x, float y, float z) { f3 r; r.x = x; r.y = y; r.z = z; return r; }
static inline f3 sub(f3 a, f3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline f3 add(f3 a, f3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline f3 mulf(f3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
static inline float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
/* Algebra.hpp:301-304 operator% (cross product) */
static inline f3 cross(f3 a, f3 b) {
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
/* Algebra.hpp:307-310 operator~ (normalise); 1/sqrt is correctly rounded here */
static inline f3 normalize(f3 a) { float inv = 1.0f / sqrtf(dot(a, a)); return mulf(a, inv); }
static inline f3 vmin(f3 a, f3 b) { return mk(hmin(a.x, b.x), hmin(a.y, b.y), hmin(a.z, b.z)); }
static inline f3 vmax(f3 a, f3 b) { return mk(hmax(a.x, b.x), hmax(a.y, b.y), hmax(a.z, b.z)); }
static inline float comp(f3 a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }
static inline f3 ld3(const float *p) { return mk(p[0], p[1], p[2]); }
static inline f3 vtx(const float *v4, uint32_t i) { return ld3(v4 + 4 * (size_t)i); }

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_free(void *p) { free(p); }

/* powf(x, 0.3333333f) as used by UGridSortBuilder.h:82-83 and TLGridBuildKernels.h:62-63,
 * evaluated in double and rounded once to float (the CUDA side does the same). */
float orc_pow_third(float x) { return (float)pow((double)x, (double)0.3333333f); }

/* ------------------------------------------------------------------------- */
/* a1: keyframe interpolation + bounds, WFObjectUploader.h:82-114 */
void orc_lerp_bounds(const float *f1, const float *f2, uint32_t nv, float coeff,
                     float *out4, float bmin[3], float bmax[3]) {
    f3 lo = mk(FLT_MAX, FLT_MAX, FLT_MAX), hi = mk(-FLT_MAX, -FLT_MAX, -FLT_MAX);
    const float w1 = 1.0f - coeff;
    for (uint32_t i = 0; i < nv; ++i) {
        f3 p;
        p.x = f1[3 * (size_t)i + 0] * w1 + f2[3 * (size_t)i + 0] * coeff;
        p.y = f1[3 * (size_t)i + 1] * w1 + f2[3 * (size_t)i + 1] * coeff;
        p.z = f1[3 * (size_t)i + 2] * w1 + f2[3 * (size_t)i + 2] * coeff;
        if (out4) {
            out4[4 * (size_t)i + 0] = p.x; out4[4 * (size_t)i + 1] = p.y;
            out4[4 * (size_t)i + 2] = p.z; out4[4 * (size_t)i + 3] = 0.0f;
        }
        lo = vmin(p, lo);  /* cudastd::min(verticesHost[it].x, oMinBound.x) */
        hi = vmax(p, hi);
    }
    f3 d = sub(hi, lo);
    float diag = sqrtf(dot(d, d));
    float pad = 0.001f * diag;
    bmin[0] = lo.x - pad; bmin[1] = lo.y - pad; bmin[2] = lo.z - pad;
    bmax[0] = hi.x + pad; bmax[1] = hi.y + pad; bmax[2] = hi.z + pad;
}

/* a2: grid resolution, UGridSortBuilder.h:78-92; fallback UGridMemoryManager.cu:338-345;
 * cell size / reciprocal UGridMemoryManager.h:93-101 (host IEEE division). */
void orc_grid_setup(const float bmin[3], const float bmax[3], uint32_t nprims,
                    float density, orc_grid *g) {
    f3 d = mk(bmax[0] - bmin[0], bmax[1] - bmin[1], bmax[2] - bmin[2]);
    float vol = d.x * d.y * d.z;
    float m = orc_pow_third(density * (float)nprims / vol);
    d = mulf(d, m);
    g->res[0] = f2i(d.x); g->res[1] = f2i(d.y); g->res[2] = f2i(d.z);
    if (g->res[0] <= 0 || g->res[1] <= 0 || g->res[2] <= 0)
        g->res[0] = g->res[1] = g->res[2] = 32;
    for (int k = 0; k < 3; ++k) {
        g->bmin[k] = bmin[k]; g->bmax[k] = bmax[k];
        float dk = bmax[k] - bmin[k];
        g->cs[k] = dk / (float)g->res[k];
        g->rcp[k] = (float)g->res[k] / dk;
    }
    g->ncells = (uint32_t)g->res[0] * (uint32_t)g->res[1] * (uint32_t)g->res[2];
}

/* triangle bbox -> clamped cell range, UniformGridBuildKernels.h:56-73.
 * Each extent is clamped at zero so the count always equals the pairs written. */
typedef struct { int32_t lo[3], hi[3]; } crange;
static inline void tri_bbox(const float *v4, const uint32_t *idx, uint32_t t, f3 *lo, f3 *hi, f3 *p) {
    p[0] = vtx(v4, idx[3 * (size_t)t + 0]);
    p[1] = vtx(v4, idx[3 * (size_t)t + 1]);
    p[2] = vtx(v4, idx[3 * (size_t)t + 2]);
    f3 a = mk(FLT_MAX, FLT_MAX, FLT_MAX), b = mk(-FLT_MAX, -FLT_MAX, -FLT_MAX);
    for (int i = 0; i < 3; ++i) { a = vmin(a, p[i]); b = vmax(b, p[i]); }  /* BBox.hpp:89-93 */
    *lo = a; *hi = b;
}
static inline uint32_t cell_range(f3 lo, f3 hi, f3 origin, const float rcp[3], const int32_t res[3], crange *r) {
    f3 a = sub(lo, origin), b = sub(hi, origin);
    float af[3] = {a.x * rcp[0], a.y * rcp[1], a.z * rcp[2]};
    float bf[3] = {b.x * rcp[0] + 1.0f, b.y * rcp[1] + 1.0f, b.z * rcp[2] + 1.0f};
    uint32_t n = 1;
    for (int k = 0; k < 3; ++k) {
        r->lo[k] = imax(0, f2i(af[k]));
        r->hi[k] = imin(res[k], f2i(bf[k]));
        int32_t e = r->hi[k] - r->lo[k];
        n *= (uint32_t)(e > 0 ? e : 0);
    }
    return n;
}

/* exact triangle/box overlap, UniformGridBuildKernels.cu:8-48 axisTest and 299-366 */
static inline int axis_test(float a, float b, float fa, float fb, float v0a, float v0b,
                            float v1a, float v1b, float ha, float hb) {
    float p0 = a * v0a + b * v0b;
    float p1 = a * v1a + b * v1b;
    float mn = hmin(p0, p1), mx = hmax(p0, p1);
    float rad = fa * ha + fb * hb;
    return !(mn > rad + ORC_EPS || mx + ORC_EPS < -rad);
}
static int sat_overlap(f3 nrm, f3 c, const f3 *tv, f3 h) {
    f3 v0 = sub(tv[0], c), v1 = sub(tv[1], c), v2 = sub(tv[2], c);
    f3 e0 = sub(v1, v0), e1 = sub(v2, v1), e2 = sub(v0, v2);
    int pass = 1;
    f3 mn, mx;
    mn.x = (nrm.x > 0.0f) ? -h.x : h.x;
    mn.y = (nrm.y > 0.0f) ? -h.y : h.y;
    mn.z = (nrm.z > 0.0f) ? -h.z : h.z;
    mx = mk(-mn.x, -mn.y, -mn.z);
    mx = sub(mx, v0);
    mn = sub(mn, v0);
    pass = pass && dot(nrm, mn) <= 0.0f && dot(nrm, mx) > 0.0f;
    f3 fe;
    fe = mk(fabsf(e0.x), fabsf(e0.y), fabsf(e0.z));
    pass = pass && axis_test(e0.z, -e0.y, fe.z, fe.y, v0.y, v0.z, v2.y, v2.z, h.y, h.z); /* X01 */
    pass = pass && axis_test(-e0.z, e0.x, fe.z, fe.x, v0.x, v0.z, v2.x, v2.z, h.x, h.z); /* Y02 */
    pass = pass && axis_test(e0.y, -e0.x, fe.y, fe.x, v1.x, v1.y, v2.x, v2.y, h.x, h.y); /* Z12 */
    fe = mk(fabsf(e1.x), fabsf(e1.y), fabsf(e1.z));
    pass = pass && axis_test(e1.z, -e1.y, fe.z, fe.y, v0.y, v0.z, v2.y, v2.z, h.y, h.z); /* X01 */
    pass = pass && axis_test(-e1.z, e1.x, fe.z, fe.x, v0.x, v0.z, v2.x, v2.z, h.x, h.z); /* Y02 */
    pass = pass && axis_test(e1.y, -e1.x, fe.y, fe.x, v0.x, v0.y, v1.x, v1.y, h.x, h.y); /* Z0 */
    fe = mk(fabsf(e2.x), fabsf(e2.y), fabsf(e2.z));
    pass = pass && axis_test(e2.z, -e2.y, fe.z, fe.y, v0.y, v0.z, v1.y, v1.z, h.y, h.z); /* X2 */
    pass = pass && axis_test(-e2.z, e2.x, fe.z, fe.x, v0.x, v0.z, v1.x, v1.z, h.x, h.z); /* Y1 */
    pass = pass && axis_test(e2.y, -e2.x, fe.y, fe.x, v1.x, v1.y, v2.x, v2.y, h.x, h.y); /* Z12 */
    return pass;
}

/* write the pairs of one triangle in z,y,x order starting at `slot`,
 * UniformGridBuildKernels.h:237-249 (bbox) and .cu:285-381 (exact) */
static void write_tri_pairs(const orc_grid *g, uint32_t tri, const f3 *tv, const crange *r,
                            int exact, uint32_t *keys, uint32_t *vals, size_t slot) {
    const uint32_t rx = (uint32_t)g->res[0], rxy = (uint32_t)g->res[0] * (uint32_t)g->res[1];
    if (!exact) {
        for (int32_t z = r->lo[2]; z < r->hi[2]; ++z)
            for (int32_t y = r->lo[1]; y < r->hi[1]; ++y)
                for (int32_t x = r->lo[0]; x < r->hi[0]; ++x, ++slot) {
                    keys[slot] = (uint32_t)x + (uint32_t)y * rx + (uint32_t)z * rxy;
                    vals[slot] = tri;
                }
        return;
    }
    f3 nrm = normalize(cross(sub(tv[1], tv[0]), sub(tv[2], tv[0])));
    f3 cs = ld3(g->cs), bmin = ld3(g->bmin);
    f3 h = mulf(cs, 0.505f);
    f3 mc = mk((float)r->lo[0], (float)r->lo[1], (float)r->lo[2]);
    mc = mk(mc.x * cs.x, mc.y * cs.y, mc.z * cs.z);
    mc = add(add(mc, bmin), h);
    f3 c;
    c.z = mc.z - cs.z;
    for (int32_t z = r->lo[2]; z < r->hi[2]; ++z) {
        c.z += cs.z;
        c.y = mc.y - cs.y;
        for (int32_t y = r->lo[1]; y < r->hi[1]; ++y) {
            c.y += cs.y;
            c.x = mc.x - cs.x;
            for (int32_t x = r->lo[0]; x < r->hi[0]; ++x, ++slot) {
                c.x += cs.x;
                keys[slot] = sat_overlap(nrm, c, tv, h)
                                 ? (uint32_t)x + (uint32_t)y * rx + (uint32_t)z * rxy
                                 : g->ncells;
                vals[slot] = tri;
            }
        }
    }
}

/* Stable counting sort of (key, value) pairs with keys < nbuckets: the result equals
 * the stable LSD radix sort of Sort.cu:31-53 applied to the same pair order. */
static void stable_sort_pairs(const uint32_t *keys, const uint32_t *vals, size_t n,
                              uint32_t nbuckets, uint32_t *okeys, uint32_t *ovals) {
    int nt = orc_num_threads();
    if (nt > 1 && n > 65536 && (size_t)nt * (nbuckets + 1) <= (size_t)64 << 20) {
        size_t *hist = (size_t *)calloc((size_t)nt * (nbuckets + 1), sizeof(size_t));
#pragma omp parallel num_threads(nt)
        {
#ifdef _OPENMP
            int tid = omp_get_thread_num();
#else
            int tid = 0;
#endif
            size_t b = n * tid / nt, e = n * (tid + 1) / nt;
            size_t *h = hist + (size_t)tid * (nbuckets + 1);
            for (size_t i = b; i < e; ++i) h[keys[i]]++;
#pragma omp barrier
#pragma omp single
            {
                size_t run = 0;
                for (uint32_t k = 0; k < nbuckets; ++k)
                    for (int t = 0; t < nt; ++t) {
                        size_t c = hist[(size_t)t * (nbuckets + 1) + k];
                        hist[(size_t)t * (nbuckets + 1) + k] = run;
                        run += c;
                    }
            }
            for (size_t i = b; i < e; ++i) {
                size_t p = h[keys[i]]++;
                okeys[p] = keys[i];
                ovals[p] = vals[i];
            }
        }
        free(hist);
        return;
    }
    size_t *off = (size_t *)calloc((size_t)nbuckets + 1, sizeof(size_t));
    for (size_t i = 0; i < n; ++i) off[keys[i] + 1]++;
    for (uint32_t k = 0; k < nbuckets; ++k) off[k + 1] += off[k];
    for (size_t i = 0; i < n; ++i) {
        size_t p = off[keys[i]]++;
        okeys[p] = keys[i];
        ovals[p] = vals[i];
    }
    free(off);
}

/* cell ranges from sorted keys, UniformGridBuildKernels.h:384-487 (keys >= ncells skipped) */
static void cell_ranges(const uint32_t *skeys, size_t n, uint32_t ncells, uint32_t *cells) {
    memset(cells, 0, sizeof(uint32_t) * 2 * (size_t)ncells);
#pragma omp parallel for schedule(static)
    for (long long ii = 0; ii < (long long)n; ++ii) {
        size_t i = (size_t)ii;
        uint32_t k = skeys[i];
        if (k >= ncells) continue;
        if (i > 0 && skeys[i - 1] != k) cells[2 * (size_t)k] = (uint32_t)i;
        if (i + 1 == n || skeys[i + 1] != k) cells[2 * (size_t)k + 1] = (uint32_t)(i + 1);
    }
}

/* count -> scan -> write -> stable sort: UGridSortBuilder.h:130-342.  Returns sorted
 * keys/values (malloc'd) and the pair count. */
static int sorted_pairs(const float *v4, const uint32_t *idx, uint32_t ntri, const orc_grid *g,
                        int exact, uint32_t **okeys, uint32_t **ovals, size_t *onp) {
    size_t *off = (size_t *)malloc(sizeof(size_t) * ((size_t)ntri + 1));
    if (!off) return -1;
    f3 bmin = ld3(g->bmin);
#pragma omp parallel for schedule(static)
    for (long long t = 0; t < (long long)ntri; ++t) {
        f3 lo, hi, p[3];
        crange r;
        tri_bbox(v4, idx, (uint32_t)t, &lo, &hi, p);
        off[t + 1] = cell_range(lo, hi, bmin, g->rcp, g->res, &r);
    }
    off[0] = 0;
    for (uint32_t t = 0; t < ntri; ++t) off[t + 1] += off[t];
    size_t np = off[ntri];
    uint32_t *keys = (uint32_t *)malloc(sizeof(uint32_t) * (np + 1));
    uint32_t *vals = (uint32_t *)malloc(sizeof(uint32_t) * (np + 1));
    uint32_t *sk = (uint32_t *)malloc(sizeof(uint32_t) * (np + 1));
    uint32_t *sv = (uint32_t *)malloc(sizeof(uint32_t) * (np + 1));
    if (!keys || !vals || !sk || !sv) { free(off); free(keys); free(vals); free(sk); free(sv); return -1; }
#pragma omp parallel for schedule(dynamic, 256)
    for (long long t = 0; t < (long long)ntri; ++t) {
        f3 lo, hi, p[3];
        crange r;
        tri_bbox(v4, idx, (uint32_t)t, &lo, &hi, p);
        cell_range(lo, hi, bmin, g->rcp, g->res, &r);
        write_tri_pairs(g, (uint32_t)t, p, &r, exact, keys, vals, off[t]);
    }
    stable_sort_pairs(keys, vals, np, g->ncells + 1, sk, sv);
    free(keys); free(vals); free(off);
    *okeys = sk; *ovals = sv; *onp = np;
    return 0;
}

int orc_build_ug(const float *v4, const uint32_t *idx, uint32_t ntri,
                 const float bmin[3], const float bmax[3], float density, int exact,
                 orc_grid *g, uint32_t **cells, uint32_t **prims, uint32_t *npairs) {
    orc_grid_setup(bmin, bmax, ntri, density, g);
    uint32_t *sk, *sv;
    size_t np;
    if (sorted_pairs(v4, idx, ntri, g, exact, &sk, &sv, &np)) return -1;
    uint32_t *c = (uint32_t *)malloc(sizeof(uint32_t) * 2 * (size_t)g->ncells);
    if (!c) { free(sk); free(sv); return -1; }
    cell_ranges(sk, np, g->ncells, c);
    free(sk);
    *cells = c; *prims = sv; *npairs = (uint32_t)np;
    return 0;
}

/* a8: leaf resolution of one top cell, TLGridBuildKernels.h:55-87 */
static void leaf_res(const orc_grid *g, uint32_t refs, float leaf_density, uint32_t res[3], int *is_leaf) {
    float vol = g->cs[0] * g->cs[1] * g->cs[2];
    float m = orc_pow_third(leaf_density * (float)refs / vol);
    *is_leaf = refs <= ORC_LEAF_REFS_MAX;
    for (int k = 0; k < 3; ++k) {
        float r = hmin(255.0f, hmax(1.0f, g->cs[k] * m));
        res[k] = *is_leaf ? 1u : (uint32_t)r;
    }
}

/* sub-cell range of a triangle inside top cell (cx,cy,cz), TLGridBuildKernels.h:338-377 */
static uint32_t leaf_range(const orc_grid *g, const uint32_t lres[3], const int32_t cc[3],
                           f3 lo, f3 hi, crange *r) {
    f3 org;
    org.x = (float)cc[0] * g->cs[0] + g->bmin[0];
    org.y = (float)cc[1] * g->cs[1] + g->bmin[1];
    org.z = (float)cc[2] * g->cs[2] + g->bmin[2];
    float srcp[3];
    int32_t ires[3];
    for (int k = 0; k < 3; ++k) { srcp[k] = (float)lres[k] / g->cs[k]; ires[k] = (int32_t)lres[k]; }
    return cell_range(lo, hi, org, srcp, ires, r);
}

int orc_build_tl(const float *v4, const uint32_t *idx, uint32_t ntri,
                 const float bmin[3], const float bmax[3], float top_density,
                 float leaf_density, orc_grid *g, uint32_t **top_cells,
                 uint32_t **leaves, uint32_t *nleaves, uint32_t **prims,
                 uint32_t *npairs, uint32_t *ntop_pairs) {
    /* top level: TLGridSortBuilder.h:146-245 (bounding-box insertion) */
    orc_grid_setup(bmin, bmax, ntri, top_density, g);
    uint32_t *sk, *sv;
    size_t np;
    if (sorted_pairs(v4, idx, ntri, g, 0, &sk, &sv, &np)) return -1;
    const uint32_t C = g->ncells;
    uint32_t *rng = (uint32_t *)malloc(sizeof(uint32_t) * 2 * (size_t)C);
    uint32_t *tc = (uint32_t *)malloc(sizeof(uint32_t) * 2 * (size_t)C);
    size_t *lcnt = (size_t *)malloc(sizeof(size_t) * ((size_t)C + 1));
    size_t *rcnt = (size_t *)malloc(sizeof(size_t) * ((size_t)C + 1));
    if (!rng || !tc || !lcnt || !rcnt) return -1;
    cell_ranges(sk, np, C, rng);
    free(sk);
    const uint32_t rx = (uint32_t)g->res[0], rxy = (uint32_t)g->res[0] * (uint32_t)g->res[1];
    /* a8 + a10: leaf cell counts and leaf pair counts per top cell */
#pragma omp parallel for schedule(dynamic, 64)
    for (long long cl = 0; cl < (long long)C; ++cl) {
        uint32_t c = (uint32_t)cl;
        uint32_t b = rng[2 * (size_t)c], e = rng[2 * (size_t)c + 1];
        uint32_t refs = e - b, lres[3];
        int is_leaf;
        leaf_res(g, refs, leaf_density, lres, &is_leaf);
        int32_t cc[3] = {(int32_t)(c % rx), (int32_t)((c % rxy) / rx), (int32_t)(c / rxy)};
        size_t cnt = 0;
        for (uint32_t i = b; i < e; ++i) {
            f3 lo, hi, p[3];
            crange r;
            tri_bbox(v4, idx, sv[i], &lo, &hi, p);
            cnt += leaf_range(g, lres, cc, lo, hi, &r);
        }
        lcnt[c + 1] = (size_t)lres[0] * lres[1] * lres[2];
        rcnt[c + 1] = cnt;
        uint32_t y = (lres[0] & 0xFFu) | ((lres[1] & 0xFFu) << 8) | ((lres[2] & 0xFFu) << 16);
        if (is_leaf) y |= ORC_LEAFMASK;
        if (refs != 0) y |= ORC_NOTEMPTYMASK;
        tc[2 * (size_t)c + 1] = y;
    }
    /* a9: scans, TLGridSortBuilder.h:277-294 and 320-345 */
    lcnt[0] = 0; rcnt[0] = 0;
    for (uint32_t c = 0; c < C; ++c) { lcnt[c + 1] += lcnt[c]; rcnt[c + 1] += rcnt[c]; }
    const size_t CL = lcnt[C], PL = rcnt[C];
    uint32_t *lv = (uint32_t *)calloc(2 * CL + 2, sizeof(uint32_t));
    uint32_t *pr = (uint32_t *)malloc(sizeof(uint32_t) * (PL + 1));
    if (!lv || !pr) return -1;
    /* a11-a13: per top cell, leaf pairs in reference order, stable sort, leaf ranges */
#pragma omp parallel for schedule(dynamic, 64)
    for (long long cl = 0; cl < (long long)C; ++cl) {
        uint32_t c = (uint32_t)cl;
        tc[2 * (size_t)c] = (uint32_t)lcnt[c];  /* prepareTopLevelCellRanges */
        uint32_t b = rng[2 * (size_t)c], e = rng[2 * (size_t)c + 1];
        if (b == e) continue;
        uint32_t y = tc[2 * (size_t)c + 1];
        uint32_t lres[3] = {y & 0xFFu, (y >> 8) & 0xFFu, (y >> 16) & 0xFFu};
        uint32_t nl = lres[0] * lres[1] * lres[2];
        int32_t cc[3] = {(int32_t)(c % rx), (int32_t)((c % rxy) / rx), (int32_t)(c / rxy)};
        size_t n = rcnt[c + 1] - rcnt[c];
        uint32_t *k = (uint32_t *)malloc(sizeof(uint32_t) * (n + 1));
        uint32_t *v = (uint32_t *)malloc(sizeof(uint32_t) * (n + 1));
        uint32_t *cnt = (uint32_t *)calloc((size_t)nl + 1, sizeof(uint32_t));
        size_t w = 0;
        for (uint32_t i = b; i < e; ++i) {
            f3 lo, hi, p[3];
            crange r;
            uint32_t tri = sv[i];
            tri_bbox(v4, idx, tri, &lo, &hi, p);
            leaf_range(g, lres, cc, lo, hi, &r);
            for (int32_t z = r.lo[2]; z < r.hi[2]; ++z)
                for (int32_t yy = r.lo[1]; yy < r.hi[1]; ++yy)
                    for (int32_t x = r.lo[0]; x < r.hi[0]; ++x) {
                        uint32_t key = (uint32_t)x + (uint32_t)yy * lres[0] + (uint32_t)z * lres[0] * lres[1];
                        k[w] = key; v[w] = tri; ++w; cnt[key + 1]++;
                    }
        }
        for (uint32_t q = 0; q < nl; ++q) cnt[q + 1] += cnt[q];
        const size_t rb = rcnt[c];
        const size_t lb = lcnt[c];
        for (uint32_t q = 0; q < nl; ++q) {
            if (cnt[q + 1] > cnt[q]) {
                lv[2 * (lb + q)] = (uint32_t)(rb + cnt[q]);
                lv[2 * (lb + q) + 1] = (uint32_t)(rb + cnt[q + 1]);
            }
        }
        for (size_t i = 0; i < w; ++i) pr[rb + cnt[k[i]]++] = v[i];
        free(k); free(v); free(cnt);
    }
    free(rng); free(sv); free(lcnt); free(rcnt);
    *top_cells = tc; *leaves = lv; *nleaves = (uint32_t)CL; *prims = pr;
    *npairs = (uint32_t)PL; *ntop_pairs = (uint32_t)np;
    return 0;
}

/* ------------------------------------------------------------------------- */
/* camera, Camera.h:40-64 (host-side init) */
void orc_camera_init(orc_camera *c, const float pos[3], const float fwd[3],
                     const float up[3], float fov_deg, int32_t w, int32_t h) {
    f3 f = normalize(ld3(fwd));
    f3 r = normalize(cross(f, ld3(up)));
    f3 u = normalize(cross(f, r));
    float aspect = (float)w / (float)h;
    float ang = fov_deg * 3.14159265358979323846f / 180.0f;
    float tn = tanf(ang / 2.0f);
    f3 row = mulf(mulf(mulf(r, 2.0f), tn), aspect);
    f3 col = mulf(mulf(u, 2.0f), tn);
    f3 sx = mk(row.x / (float)w, row.y / (float)w, row.z / (float)w);
    f3 sy = mk(col.x / (float)h, col.y / (float)h, col.z / (float)h);
    f3 tl = sub(sub(f, mk(row.x / 2.0f, row.y / 2.0f, row.z / 2.0f)),
                mk(col.x / 2.0f, col.y / 2.0f, col.z / 2.0f));
    for (int k = 0; k < 3; ++k) {
        c->pos[k] = pos[k]; c->top_left[k] = comp(tl, k);
        c->step_x[k] = comp(sx, k); c->step_y[k] = comp(sy, k);
    }
    c->w = w; c->h = h;
}

/* pixel centre ray, normalised direction */
static inline f3 primary_dir(const orc_camera *c, uint32_t pix) {
    float px = (float)(pix % (uint32_t)c->w) + 0.5f;
    float py = (float)(pix / (uint32_t)c->w) + 0.5f;
    f3 d;
    d.x = c->top_left[0] + px * c->step_x[0] + py * c->step_y[0];
    d.y = c->top_left[1] + px * c->step_x[1] + py * c->step_y[1];
    d.z = c->top_left[2] + px * c->step_x[2] + py * c->step_y[2];
    return normalize(d);
}

void orc_primary_rays(const orc_camera *c, float *org, float *dir) {
    uint32_t n = (uint32_t)c->w * (uint32_t)c->h;
    for (uint32_t i = 0; i < n; ++i) {
        f3 d = primary_dir(c, i);
        org[3 * (size_t)i] = c->pos[0]; org[3 * (size_t)i + 1] = c->pos[1]; org[3 * (size_t)i + 2] = c->pos[2];
        dir[3 * (size_t)i] = d.x; dir[3 * (size_t)i + 1] = d.y; dir[3 * (size_t)i + 2] = d.z;
    }
}

/* ------------------------------------------------------------------------- */
/* traversal */
typedef struct {
    float t, u, v;
    uint32_t tri;
    int hit;
    uint32_t cells, tests;
} hitrec;

/* a16: Moller-Trumbore, RayTriangleIntersector.h:52-90 (first-tested wins ties) */
static inline int isect_range(const orc_scene *s, f3 o, f3 d, uint32_t b, uint32_t e,
                              int anyhit, hitrec *h) {
    for (uint32_t it = b; it < e; ++it) {
        uint32_t tri = s->prims[it];
        f3 v0 = vtx(s->v4, s->idx[3 * (size_t)tri]);
        f3 v1 = vtx(s->v4, s->idx[3 * (size_t)tri + 1]);
        f3 v2 = vtx(s->v4, s->idx[3 * (size_t)tri + 2]);
        f3 e1 = sub(v1, v0), e2 = sub(v2, v0);
        f3 p = cross(d, e2);
        float det = dot(e1, p);
        float inv = 1.0f / det;
        f3 sv = sub(o, v0);
        float u = dot(sv, p) * inv;
        f3 q = cross(sv, e1);
        float v = dot(q, d) * inv;
        float t = dot(e2, q) * inv;
        h->tests++;
        if (u >= 0.0f && v >= 0.0f && u + v <= 1.0f && t > ORC_ISECT_EPS && t < h->t) {
            h->t = t; h->u = u; h->v = v; h->tri = tri; h->hit = 1;
            if (anyhit) return 1;
        }
    }
    return 0;
}

#define MIN_DIM(a, b, c) ((a) < (b) ? ((a) < (c) ? 0 : 2) : ((b) < (c) ? 1 : 2))

/* slab test shared by both traversers, UGridTraverser.h:76-92 */
static inline int clip(const orc_grid *g, f3 o, const float rcp[3], float *t0, float *t1) {
    float tn[3], tf[3];
    for (int k = 0; k < 3; ++k) {
        float a = (g->bmin[k] - comp(o, k)) * rcp[k];
        float b = (g->bmax[k] - comp(o, k)) * rcp[k];
        tn[k] = hmin(a, b); tf[k] = hmax(a, b);
    }
    *t0 = hmax(hmax(tn[0], tn[1]), tn[2]);
    *t1 = hmin(hmin(tf[0], tf[1]), tf[2]);
    return (*t1 > *t0 && *t1 >= 0.0f);
}

/* a14: uniform grid DDA, UGridTraverser.h:76-172 */
static void trace_ug(const orc_scene *s, f3 o, f3 d, int anyhit, hitrec *h) {
    const orc_grid *g = &s->g;
    float rcp[3] = {1.0f / d.x, 1.0f / d.y, 1.0f / d.z};
    float t0, t1;
    if (!clip(g, o, rcp, &t0, &t1)) return;
    f3 ep = o;
    if (t0 >= 0.0f) { float te = t0 + ORC_EPS; ep = mk(o.x + te * d.x, o.y + te * d.y, o.z + te * d.z); }
    float tmax[3];
    int32_t cell[3];
    for (int k = 0; k < 3; ++k) {
        float cf = floorf((comp(ep, k) - g->bmin[k]) * g->rcp[k]);
        cf = hmin((float)g->res[k] - 1.0f, hmax(cf, 0.0f));
        float stp = rcp[k] > 0.0f ? 1.0f : 0.0f;
        tmax[k] = ((cf + stp) * g->cs[k] + g->bmin[k] - comp(o, k)) * rcp[k];
        cell[k] = f2i(cf);
    }
    int active = cell[0] < g->res[0] && cell[0] > -1 && cell[1] < g->res[1] && cell[1] > -1 &&
                 cell[2] < g->res[2] && cell[2] > -1;
    const uint32_t rx = (uint32_t)g->res[0], rxy = (uint32_t)g->res[0] * (uint32_t)g->res[1];
    while (active) {
        uint32_t c = (uint32_t)cell[0] + (uint32_t)cell[1] * rx + (uint32_t)cell[2] * rxy;
        h->cells++;
        if (isect_range(s, o, d, s->cells[2 * (size_t)c], s->cells[2 * (size_t)c + 1], anyhit, h)) return;
        int k = MIN_DIM(tmax[0], tmax[1], tmax[2]);
        active = h->t > tmax[k];
        cell[k] += rcp[k] > 0.0f ? 1 : -1;
        tmax[k] += g->cs[k] * fabsf(rcp[k]);
        active = active && cell[k] < g->res[k] && cell[k] > -1;
    }
}

/* a15: two-level grid DDA, TLGridTraverser.h:79-349 */
static void trace_tl(const orc_scene *s, f3 o, f3 d, int anyhit, hitrec *h) {
    const orc_grid *g = &s->g;
    float rcp[3] = {1.0f / d.x, 1.0f / d.y, 1.0f / d.z};
    float t0, t1;
    if (!clip(g, o, rcp, &t0, &t1)) return;
    float tentry = hmax(0.0f, t0);
    f3 ep = mk(o.x + tentry * d.x, o.y + tentry * d.y, o.z + tentry * d.z);
    float tmax[3];
    int32_t cell[3];
    for (int k = 0; k < 3; ++k) {
        float cf = floorf((comp(ep, k) - g->bmin[k]) * g->rcp[k]);
        cf = hmin((float)g->res[k] - 1.0f, hmax(cf, 0.0f));
        float stp = rcp[k] > 0.0f ? 1.0f : 0.0f;
        tmax[k] = ((cf + stp) * g->cs[k] + g->bmin[k] - comp(o, k)) * rcp[k];
        cell[k] = f2i(cf);
    }
    int active = cell[0] < g->res[0] && cell[0] > -1 && cell[1] < g->res[1] && cell[1] > -1 &&
                 cell[2] < g->res[2] && cell[2] > -1;
    const uint32_t rx = (uint32_t)g->res[0], rxy = (uint32_t)g->res[0] * (uint32_t)g->res[1];
    while (active) {
        uint32_t c = (uint32_t)cell[0] + (uint32_t)cell[1] * rx + (uint32_t)cell[2] * rxy;
        uint32_t lbeg = s->cells[2 * (size_t)c], y = s->cells[2 * (size_t)c + 1];
        h->cells++;
        if (y & ORC_NOTEMPTYMASK) {
            uint32_t lres[3] = {y & 0xFFu, (y >> 8) & 0xFFu, (y >> 16) & 0xFFu};
            f3 e2 = mk(o.x + tentry * d.x, o.y + tentry * d.y, o.z + tentry * d.z);
            float srcp[3], scs[3], mb[3], tm2[3];
            int32_t c2[3];
            for (int k = 0; k < 3; ++k) {
                float cres = (float)lres[k];
                srcp[k] = g->rcp[k] * cres;
                mb[k] = (float)cell[k] * g->cs[k] + g->bmin[k];
                float cf = floorf((comp(e2, k) - mb[k]) * srcp[k]);
                scs[k] = 1.0f / srcp[k];
                cf = hmin(cres - 1.0f, hmax(cf, 0.0f));
                float stp = rcp[k] > 0.0f ? 1.0f : 0.0f;
                tm2[k] = ((cf + stp) * scs[k] + mb[k] - comp(o, k)) * rcp[k];
                c2[k] = f2i(cf);
            }
            int inner = 1;
            while (inner) {
                uint32_t li = lbeg + (uint32_t)c2[0] + lres[0] * (uint32_t)c2[1] +
                              lres[0] * lres[1] * (uint32_t)c2[2];
                h->cells++;
                if (isect_range(s, o, d, s->leaves[2 * (size_t)li], s->leaves[2 * (size_t)li + 1], anyhit, h))
                    return;
                int k = MIN_DIM(tm2[0], tm2[1], tm2[2]);
                if (h->t < tm2[k]) { inner = 0; active = 0; }
                c2[k] += rcp[k] > 0.0f ? 1 : -1;
                tm2[k] += scs[k] * fabsf(rcp[k]);
                inner = inner && c2[k] != (int32_t)lres[k] && c2[k] != -1;
            }
        }
        if (active) {
            int k = MIN_DIM(tmax[0], tmax[1], tmax[2]);
            active = h->t > tmax[k];
            tentry = tmax[k];
            cell[k] += rcp[k] > 0.0f ? 1 : -1;
            tmax[k] += g->cs[k] * fabsf(rcp[k]);
            active = active && cell[k] != g->res[k] && cell[k] != -1;
        }
    }
}

static inline void trace_one(const orc_scene *s, f3 o, f3 d, float tmax, int anyhit, hitrec *h) {
    h->t = tmax; h->u = 0.0f; h->v = 0.0f; h->tri = 0; h->hit = 0; h->cells = 0; h->tests = 0;
    if (s->ntri == 0) return;
    if (s->kind == ORC_UG) trace_ug(s, o, d, anyhit, h);
    else trace_tl(s, o, d, anyhit, h);
}

/* (u, v) of the hit of ray (o, d) on triangle tri reported by the ray queries:
 * Moller-Trumbore in binary64 from the binary32 inputs, in the library's operation order */
static inline void refine_uv(const orc_scene *s, uint32_t tri, f3 o, f3 d, float *ou, float *ov) {
    const f3 p0 = vtx(s->v4, s->idx[3 * (size_t)tri]), p1 = vtx(s->v4, s->idx[3 * (size_t)tri + 1]),
             p2 = vtx(s->v4, s->idx[3 * (size_t)tri + 2]);
    const double ax = p0.x, ay = p0.y, az = p0.z;
    const double e1x = (double)p1.x - ax, e1y = (double)p1.y - ay, e1z = (double)p1.z - az;
    const double e2x = (double)p2.x - ax, e2y = (double)p2.y - ay, e2z = (double)p2.z - az;
    const double dx = d.x, dy = d.y, dz = d.z;
    const double px = dy * e2z - dz * e2y, py = dz * e2x - dx * e2z, pz = dx * e2y - dy * e2x;
    const double det = e1x * px + e1y * py + e1z * pz;
    const double sx = (double)o.x - ax, sy = (double)o.y - ay, sz = (double)o.z - az;
    const double u = (sx * px + sy * py + sz * pz) / det;
    const double qx = sy * e1z - sz * e1y, qy = sz * e1x - sx * e1z, qz = sx * e1y - sy * e1x;
    const double v = (qx * dx + qy * dy + qz * dz) / det;
    *ou = (float)u;
    *ov = (float)v;
}

void orc_trace(const orc_scene *s, const float *org, const float *dir, uint32_t n,
               int32_t *id, float *t, float *u, float *v, uint32_t *stats) {
#pragma omp parallel for schedule(dynamic, 256)
    for (long long ii = 0; ii < (long long)n; ++ii) {
        size_t i = (size_t)ii;
        hitrec h;
        trace_one(s, ld3(org + 3 * i), ld3(dir + 3 * i), FLT_MAX, 0, &h);
        if (h.hit) refine_uv(s, h.tri, ld3(org + 3 * i), ld3(dir + 3 * i), &h.u, &h.v);
        id[i] = h.hit ? (int32_t)h.tri : -1;
        t[i] = h.hit ? h.t : FLT_MAX;
        u[i] = h.u; v[i] = h.v;
        if (stats) { stats[2 * i] = h.cells; stats[2 * i + 1] = h.tests; }
    }
}

void orc_trace_primary(const orc_scene *s, const orc_camera *c, int32_t *id,
                       float *t, float *u, float *v, uint32_t *stats) {
    uint32_t n = (uint32_t)c->w * (uint32_t)c->h;
    f3 o = ld3(c->pos);
#pragma omp parallel for schedule(dynamic, 256)
    for (long long ii = 0; ii < (long long)n; ++ii) {
        size_t i = (size_t)ii;
        hitrec h;
        const f3 d = primary_dir(c, (uint32_t)i);
        trace_one(s, o, d, FLT_MAX, 0, &h);
        if (h.hit) refine_uv(s, h.tri, o, d, &h.u, &h.v);
        id[i] = h.hit ? (int32_t)h.tri : -1;
        t[i] = h.hit ? h.t : FLT_MAX;
        u[i] = h.u; v[i] = h.v;
        if (stats) { stats[2 * i] = h.cells; stats[2 * i + 1] = h.tests; }
    }
}

void orc_occluded(const orc_scene *s, const float *org, const float *dir,
                  const float *tmax, uint32_t n, uint8_t *occluded) {
#pragma omp parallel for schedule(dynamic, 256)
    for (long long ii = 0; ii < (long long)n; ++ii) {
        size_t i = (size_t)ii;
        hitrec h;
        trace_one(s, ld3(org + 3 * i), ld3(dir + 3 * i), tmax[i], 1, &h);
        occluded[i] = (uint8_t)h.hit;
    }
}

/* ------------------------------------------------------------------------- */
/* PCG32 (M.E. O'Neill, "PCG: A Family of Simple Fast Space-Efficient Statistically
 * Good Algorithms for Random Number Generation", 2014): pcg32_random_r / srandom_r. */
typedef struct { uint64_t state, inc; } pcg32;
static inline uint32_t pcg32_next(pcg32 *r) {
    uint64_t old = r->state;
    r->state = old * 6364136223846793005ULL + r->inc;
    uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = (uint32_t)(old >> 59u);
    return (xs >> rot) | (xs << ((0u - rot) & 31u));
}
static inline void pcg32_seed(pcg32 *r, uint64_t initstate, uint64_t initseq) {
    r->state = 0u; r->inc = (initseq << 1u) | 1u;
    pcg32_next(r); r->state += initstate; pcg32_next(r);
}
static inline float pcg32_float(pcg32 *r) { return (float)(pcg32_next(r) >> 8) * (1.0f / 16777216.0f); }

float orc_pcg32_first_floats(uint64_t initstate, uint64_t initseq, int32_t k, float *out) {
    pcg32 r;
    pcg32_seed(&r, initstate, initseq);
    for (int32_t i = 0; i < k; ++i) out[i] = pcg32_float(&r);
    return k > 0 ? out[0] : 0.0f;
}

/* sin(2 pi u), cos(2 pi u) for u in [0,1): quadrant reduction (exact: u*4 is exact)
 * followed by the Maclaurin series of sin (to x^13) and cos (to x^14) on [0, pi/2),
 * Horner form, no FMA.  Truncation error < 7e-10. */
void orc_sincos2pi(float u, float *s, float *c) {
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

/* Orthonormal basis from a unit normal: Duff et al., "Building an Orthonormal Basis,
 * Revisited", JCGT 6(1), 2017. */
static inline void onb(f3 n, f3 *t, f3 *b) {
    float sg = copysignf(1.0f, n.z);
    float a = -1.0f / (sg + n.z);
    float bb = n.x * n.y * a;
    *t = mk(1.0f + sg * n.x * n.x * a, sg * bb, -sg * n.x);
    *b = mk(bb, sg + n.y * n.y * a, -n.y);
}

/* cosine-weighted direction around n, HemisphereSamplers.hpp:54-72 */
static inline f3 cosine_dir(f3 n, float u1, float u2) {
    float sn, cs;
    orc_sincos2pi(u1, &sn, &cs);
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

static inline f3 face_normal(const orc_scene *s, uint32_t tri, f3 d) {
    f3 v0 = vtx(s->v4, s->idx[3 * (size_t)tri]);
    f3 v1 = vtx(s->v4, s->idx[3 * (size_t)tri + 1]);
    f3 v2 = vtx(s->v4, s->idx[3 * (size_t)tri + 2]);
    f3 n = normalize(cross(sub(v1, v0), sub(v2, v0)));
    if (dot(n, d) > 0.0f) n = mk(-n.x, -n.y, -n.z);
    return n;
}

static inline void blend(float *fb, size_t i, float val, int32_t image_id) {
    float nw = 1.0f / (float)(image_id + 1);
    float ow = 1.0f - nw;
    fb[i] = fb[i] * ow + val * nw;   /* AOIntegrator.h:168-175 progressive average */
}

/* a19: ambient occlusion, AOIntegrator.h:234-351 and RayGenerators.h:286-342 with the
 * configured sample count, AO radius and PCG32 stream keyed by (image, pixel, seed). */
/* natural logarithm of a positive normal float (atanh series of m in [sqrt(1/2), sqrt(2))),
 * the same binary32 operations as the library's */
static inline float log_series(float x) {
    uint32_t b;
    memcpy(&b, &x, 4);
    int32_t e = (int32_t)((b >> 23) & 0xFFu) - 127;
    b = (b & 0x7FFFFFu) | 0x3F800000u;
    float m;
    memcpy(&m, &b, 4);
    if (m > 1.41421356f) { m = m * 0.5f; e += 1; }
    const float sv = (m - 1.0f) / (m + 1.0f);
    const float s2 = sv * sv;
    const float lm = sv * (2.0f + s2 * (0.666666667f + s2 * (0.4f + s2 * (0.285714286f + s2 * (0.222222222f +
                     s2 * 0.181818182f)))));
    return lm + (float)e * 0.693147181f;
}

float orc_log_series(float x) { return log_series(x); }

/* camera ray of render mode 0 for progressive image image_id (RTEngine.cu:409-424): the
 * 2 x 2 regular in-pixel pattern for images 0-3 (RegularPixelSampler<2,2>, Camera.h:75-98),
 * a Gaussian offset around the pixel corner for later ones (GaussianPixelSampler,
 * Camera.h:116-132) from two PCG32 draws keyed by (image, pixel, seed); normalised */
static inline f3 primary_sample_dir(const orc_camera *c, uint32_t pix, int32_t image_id, uint64_t seed) {
    float ox, oy;
    if (image_id < 4) {
        const float tmp = (float)(image_id % 4) / 2.0f;
        oy = (truncf(tmp) + 0.5f) / 2.0f;
        ox = tmp - truncf(tmp) + 0.5f / 2.0f;
    } else {
        pcg32 r;
        pcg32_seed(&r, ((uint64_t)(uint32_t)image_id << 32) | pix, seed);
        const float u1 = pcg32_float(&r), u2 = pcg32_float(&r);
        const float rad = 0.5f * sqrtf(-log_series(1.0f - u1));
        float sn, cs;
        orc_sincos2pi(u2, &sn, &cs);
        ox = rad * cs;
        oy = rad * sn;
    }
    const float px = (float)(pix % (uint32_t)c->w) + ox;
    const float py = (float)(pix / (uint32_t)c->w) + oy;
    f3 d;
    d.x = c->top_left[0] + px * c->step_x[0] + py * c->step_y[0];
    d.y = c->top_left[1] + px * c->step_x[1] + py * c->step_y[1];
    d.z = c->top_left[2] + px * c->step_x[2] + py * c->step_y[2];
    return normalize(d);
}

/* simpleShade (SimpleIntegrator.h:41-126) of a closest hit: weights from the ray origin's
 * cross products, colour (u, v, 1 - u - v) times |cos|; background on a miss */
static inline void simple_shade(const orc_scene *s, const hitrec *h, f3 o, f3 d, float *rgb) {
    rgb[0] = 0.15f; rgb[1] = 0.2f; rgb[2] = 0.3f;
    if (!h->hit) return;
    const f3 p0 = vtx(s->v4, s->idx[3 * (size_t)h->tri]), p1 = vtx(s->v4, s->idx[3 * (size_t)h->tri + 1]),
             p2 = vtx(s->v4, s->idx[3 * (size_t)h->tri + 2]);
    const f3 nr = cross(sub(p1, p0), sub(p2, p0));
    const f3 a0 = sub(p0, o), a1 = sub(p1, o), a2 = sub(p2, o);
    const f3 n0 = cross(a1, a2), n1 = cross(a2, a0);
    const float inv = 1.0f / sqrtf(dot(nr, nr));
    const float u = sqrtf(dot(n0, n0)) * inv;
    const float v = sqrtf(dot(n1, n1)) * inv;
    const f3 nrm = normalize(nr);
    const f3 dn = normalize(d);
    const float cs = fmaxf(0.0f, fabsf(dot(mk(-nrm.x, -nrm.y, -nrm.z), dn)));
    rgb[0] = u * cs;
    rgb[1] = v * cs;
    rgb[2] = (1.0f - u - v) * cs;
}

/* render mode 0: camera rays of the mode-0 samplers, simpleShade, progressive blend of the
 * 3 channels into fb (3 floats per pixel) */
void orc_render_primary(const orc_scene *s, const orc_camera *c, int32_t image_id, uint64_t seed, float *fb) {
    const uint32_t n = (uint32_t)c->w * (uint32_t)c->h;
    const f3 o = ld3(c->pos);
    const float nw = 1.0f / (float)(image_id + 1);
    const float ow = 1.0f - nw;
#pragma omp parallel for schedule(dynamic, 256)
    for (long long ii = 0; ii < (long long)n; ++ii) {
        const uint32_t pix = (uint32_t)ii;
        const f3 d = primary_sample_dir(c, pix, image_id, seed);
        hitrec h;
        trace_one(s, o, d, FLT_MAX, 0, &h);
        float rgb[3];
        simple_shade(s, &h, o, d, rgb);
        for (int k = 0; k < 3; ++k) fb[3 * (size_t)pix + k] = fb[3 * (size_t)pix + k] * ow + rgb[k] * nw;
    }
}

/* the ray-file form of render mode 0 (SimpleRayTraverser.h:166-180): ray i shaded into pixel i */
void orc_render_rays(const orc_scene *s, const float *org, const float *dir, uint32_t n, int32_t image_id,
                     float *fb) {
    const float nw = 1.0f / (float)(image_id + 1);
    const float ow = 1.0f - nw;
#pragma omp parallel for schedule(dynamic, 256)
    for (long long ii = 0; ii < (long long)n; ++ii) {
        const size_t i = (size_t)ii;
        const f3 o = ld3(org + 3 * i), d = ld3(dir + 3 * i);
        hitrec h;
        trace_one(s, o, d, FLT_MAX, 0, &h);
        float rgb[3];
        simple_shade(s, &h, o, d, rgb);
        for (int k = 0; k < 3; ++k) fb[3 * i + k] = fb[3 * i + k] * ow + rgb[k] * nw;
    }
}

void orc_render_ao(const orc_scene *s, const orc_camera *c, int32_t spp, float alpha,
                   uint64_t seed, int32_t image_id, float *fb, uint32_t pixel_stride,
                   uint64_t *counts) {
    uint32_t n = (uint32_t)c->w * (uint32_t)c->h;
    if (pixel_stride == 0) pixel_stride = 1;
    f3 o = ld3(c->pos);
    uint64_t rays = 0;
    const float off = 0.01f * alpha;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : rays)
    for (long long ii = 0; ii < (long long)n; ii += pixel_stride) {
        uint32_t pix = (uint32_t)ii;
        f3 d = primary_dir(c, pix);
        hitrec h;
        trace_one(s, o, d, FLT_MAX, 0, &h);
        rays += 1;
        float vis = 1.0f;
        if (h.hit) {
            f3 p = mk(o.x + h.t * d.x, o.y + h.t * d.y, o.z + h.t * d.z);
            f3 nrm = face_normal(s, h.tri, d);
            pcg32 rng;
            pcg32_seed(&rng, ((uint64_t)(uint32_t)image_id << 32) | pix, seed);
            int32_t unocc = 0;
            for (int32_t k = 0; k < spp; ++k) {
                float u1 = pcg32_float(&rng), u2 = pcg32_float(&rng);
                f3 w = cosine_dir(nrm, u1, u2);
                f3 ao = mk(p.x + off * w.x, p.y + off * w.y, p.z + off * w.z);
                hitrec hs;
                trace_one(s, ao, w, alpha, 1, &hs);
                unocc += hs.hit ? 0 : 1;
            }
            rays += (uint64_t)spp;
            vis = (float)unocc / (float)spp;
        }
        blend(fb, pix, vis, image_id);
    }
    if (counts) counts[0] += rays;
}

/* shading normal of a path tracer hit (PathTracer.h:111-136): vertex normals blended with the
 * simpleShade weights from the ray origin, normalised, turned to face the ray */
static inline f3 shading_normal(const orc_scene *s, uint32_t tri, f3 o, f3 d) {
    const f3 p0 = vtx(s->v4, s->idx[3 * (size_t)tri]), p1 = vtx(s->v4, s->idx[3 * (size_t)tri + 1]),
             p2 = vtx(s->v4, s->idx[3 * (size_t)tri + 2]);
    const f3 nr = cross(sub(p1, p0), sub(p2, p0));
    const f3 a0 = sub(p0, o), a1 = sub(p1, o), a2 = sub(p2, o);
    const f3 n0 = cross(a1, a2), n1 = cross(a2, a0);
    const float inv = 1.0f / sqrtf(dot(nr, nr));
    const float u = sqrtf(dot(n0, n0)) * inv;
    const float v = sqrtf(dot(n1, n1)) * inv;
    const float w = 1.0f - u - v;
    const float *m = s->nrm3 + 9 * (size_t)tri;
    f3 n = mk(u * m[0] + v * m[3] + w * m[6], u * m[1] + v * m[4] + w * m[7], u * m[2] + v * m[5] + w * m[8]);
    n = normalize(n);
    if (dot(n, d) > 0.0f) n = mk(-n.x, -n.y, -n.z);
    return n;
}

/* A light of the collection with the values the path tracer forms once: the edge cross
 * product nc, 1 / |nc|^2 (for the parallelogram coordinates), area |nc|, sampling weight
 * area * emission.  cdf: inclusive running sum of the weights (LightSource.hpp:185-190). */
typedef struct { f3 c, e1, e2, nrm, nc; float inv_nn, emission, area, w; } light_q;

static void lights_prep(const orc_light *l, int32_t n, light_q *q, float *cdf) {
    float run = 0.0f;
    for (int32_t k = 0; k < n; ++k) {
        q[k].c = ld3(l[k].corner);
        q[k].e1 = ld3(l[k].e1);
        q[k].e2 = ld3(l[k].e2);
        q[k].nrm = ld3(l[k].normal);
        q[k].nc = cross(q[k].e1, q[k].e2);
        const float nn = dot(q[k].nc, q[k].nc);
        q[k].inv_nn = 1.0f / nn;
        q[k].area = sqrtf(nn);
        q[k].emission = l[k].emission;
        q[k].w = q[k].area * q[k].emission;
        run = run + q[k].w;
        cdf[k] = run;
    }
}

/* AreaLightSourceCollection::getLight (LightSource.hpp:114-126): the first light whose
 * normalised running weight exceeds u, else the last */
static inline int32_t light_pick(const float *cdf, int32_t n, float u) {
    for (int32_t i = 0; i < n - 1; ++i)
        if (u < cdf[i] / cdf[n - 1]) return i;
    return n - 1;
}

/* distance along (o, d) to the emitting side of parallelogram light q, or -1 */
static inline float light_hit(const light_q *q, f3 o, f3 d) {
    const float den = dot(d, q->nrm);
    if (!(den < 0.0f)) return -1.0f;
    const float tl = dot(sub(q->c, o), q->nrm) / den;
    const f3 r = sub(mk(o.x + tl * d.x, o.y + tl * d.y, o.z + tl * d.z), q->c);
    const float a = dot(cross(r, q->e2), q->nc) * q->inv_nn;
    const float b = dot(cross(q->e1, r), q->nc) * q->inv_nn;
    return (a >= 0.0f && a <= 1.0f && b >= 0.0f && b <= 1.0f) ? tl : -1.0f;
}

/* a20: path tracing with next-event estimation towards a light collection (PathTracer.h
 * pathTrace 41-372 / tracePath 374-747 structure, configured as a fixed number of
 * extension rays, Lambertian albedo, no Russian roulette). */
void orc_render_pt(const orc_scene *s, const orc_camera *c, const orc_light *l, int32_t nlights,
                   int32_t bounces, float albedo, float ray_eps, uint64_t seed,
                   int32_t image_id, float *fb, uint32_t pixel_stride, uint64_t *counts) {
    uint32_t n = (uint32_t)c->w * (uint32_t)c->h;
    if (pixel_stride == 0) pixel_stride = 1;
    if (nlights < 1 || nlights > ORC_MAX_LIGHTS) return;
    uint64_t rays = 0;
    light_q lq[ORC_MAX_LIGHTS];
    float cdf[ORC_MAX_LIGHTS];
    lights_prep(l, nlights, lq, cdf);
    const float a_pi = albedo * 0.318309886f;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : rays)
    for (long long ii = 0; ii < (long long)n; ii += pixel_stride) {
        uint32_t pix = (uint32_t)ii;
        pcg32 rng;
        pcg32_seed(&rng, ((uint64_t)(uint32_t)image_id << 32) | pix, seed);
        f3 o = ld3(c->pos);
        f3 d = primary_dir(c, pix);
        float L = 0.0f, beta = 1.0f;
        for (int32_t bounce = 0; bounce < bounces; ++bounce) {
            hitrec h;
            trace_one(s, o, d, FLT_MAX, 0, &h);
            rays += 1;
            if (bounce == 0) {
                /* camera ray against the emitters: the nearest one in front of the hit ends the path */
                float best = h.t;
                int32_t hit_light = -1;
                for (int32_t k = 0; k < nlights; ++k) {
                    const float tl = light_hit(&lq[k], o, d);
                    if (tl > ORC_ISECT_EPS && tl < best) { best = tl; hit_light = k; }
                }
                if (hit_light >= 0) {
                    L = L + lq[hit_light].emission;
                    break;
                }
            }
            if (!h.hit) break;
            f3 p = mk(o.x + h.t * d.x, o.y + h.t * d.y, o.z + h.t * d.z);
            f3 nrm = face_normal(s, h.tri, d);
            if (s->nrm3) nrm = shading_normal(s, h.tri, o, d);
            const float alb = s->alb ? s->alb[h.tri] : albedo;
            const float hit_a_pi = s->alb ? alb * 0.318309886f : a_pi;
            /* next-event estimation: one light of the collection (by weight when there are
             * several; its radiance divided by the probability of picking it), one point on it */
            int32_t k = 0;
            float scale = 1.0f;
            if (nlights > 1) {
                k = light_pick(cdf, nlights, pcg32_float(&rng));
                scale = cdf[nlights - 1] / lq[k].w;
            }
            const light_q *q = &lq[k];
            float u1 = pcg32_float(&rng), u2 = pcg32_float(&rng);
            f3 lp = mk(q->c.x + u1 * q->e1.x + u2 * q->e2.x, q->c.y + u1 * q->e1.y + u2 * q->e2.y,
                       q->c.z + u1 * q->e1.z + u2 * q->e2.z);
            f3 wi = sub(lp, p);
            float dist2 = dot(wi, wi);
            float dist = sqrtf(dist2);
            wi = mulf(wi, 1.0f / dist);
            float cos_s = dot(nrm, wi), cos_l = -dot(q->nrm, wi);
            if (cos_s > 0.0f && cos_l > 0.0f) {
                f3 so = mk(p.x + ray_eps * wi.x, p.y + ray_eps * wi.y, p.z + ray_eps * wi.z);
                hitrec hs;
                trace_one(s, so, wi, dist - ray_eps, 1, &hs);
                rays += 1;
                if (!hs.hit) {
                    float cl = beta * hit_a_pi * q->emission * cos_s * cos_l * q->area / dist2;
                    if (nlights > 1) cl = cl * scale;
                    L = L + cl;
                }
            }
            /* Lambertian bounce: f * cos / pdf = albedo */
            beta = beta * alb;
            float u3 = pcg32_float(&rng), u4 = pcg32_float(&rng);
            d = cosine_dir(nrm, u3, u4);
            o = mk(p.x + ray_eps * d.x, p.y + ray_eps * d.y, p.z + ray_eps * d.z);
        }
        blend(fb, pix, L, image_id);
    }
    if (counts) counts[0] += rays;
}

/* ------------------------------------------------------------------------- */
/* FP64 brute-force closest hit with tie / edge / grazing flags */
void orc_brute_f64(const float *v4, const uint32_t *idx, uint32_t ntri,
                   const float *org, const float *dir, uint32_t n, int32_t *id,
                   double *t, double *u, double *v, uint8_t *flags) {
#pragma omp parallel for schedule(dynamic, 16)
    for (long long ii = 0; ii < (long long)n; ++ii) {
        size_t i = (size_t)ii;
        double o[3] = {org[3 * i], org[3 * i + 1], org[3 * i + 2]};
        double d[3] = {dir[3 * i], dir[3 * i + 1], dir[3 * i + 2]};
        double bt = INFINITY, bu = 0, bv = 0, bdet = 0;
        int32_t best = -1;
        double second = INFINITY;   /* closest t of another triangle */
        double nearmiss = INFINITY; /* closest t of a near-miss (margin > -1e-5) */
        for (uint32_t tr = 0; tr < ntri; ++tr) {
            const float *a = v4 + 4 * (size_t)idx[3 * (size_t)tr];
            const float *b = v4 + 4 * (size_t)idx[3 * (size_t)tr + 1];
            const float *cc = v4 + 4 * (size_t)idx[3 * (size_t)tr + 2];
            double e1[3] = {(double)b[0] - a[0], (double)b[1] - a[1], (double)b[2] - a[2]};
            double e2[3] = {(double)cc[0] - a[0], (double)cc[1] - a[1], (double)cc[2] - a[2]};
            double p[3] = {d[1] * e2[2] - d[2] * e2[1], d[2] * e2[0] - d[0] * e2[2], d[0] * e2[1] - d[1] * e2[0]};
            double det = e1[0] * p[0] + e1[1] * p[1] + e1[2] * p[2];
            if (det == 0.0) continue;
            double inv = 1.0 / det;
            double sv[3] = {o[0] - a[0], o[1] - a[1], o[2] - a[2]};
            double uu = (sv[0] * p[0] + sv[1] * p[1] + sv[2] * p[2]) * inv;
            double q[3] = {sv[1] * e1[2] - sv[2] * e1[1], sv[2] * e1[0] - sv[0] * e1[2], sv[0] * e1[1] - sv[1] * e1[0]};
            double vv = (q[0] * d[0] + q[1] * d[1] + q[2] * d[2]) * inv;
            double tt = (e2[0] * q[0] + e2[1] * q[1] + e2[2] * q[2]) * inv;
            double margin = fmin(uu, fmin(vv, 1.0 - uu - vv));
            if (tt <= 1e-4) continue;
            if (margin >= 0.0) {
                if (tt < bt) {
                    if (best >= 0) second = fmin(second, bt);
                    bt = tt; bu = uu; bv = vv; best = (int32_t)tr; bdet = det;
                } else {
                    second = fmin(second, tt);
                }
            } else if (margin > -1e-5) {
                nearmiss = fmin(nearmiss, tt);
            }
        }
        uint8_t f = 0;
        if (best >= 0) {
            if (second <= bt * (1.0 + 1e-5)) f |= 1;
            if (fmin(bu, fmin(bv, 1.0 - bu - bv)) < 1e-5) f |= 2;
            const float *a = v4 + 4 * (size_t)idx[3 * (size_t)best];
            const float *b = v4 + 4 * (size_t)idx[3 * (size_t)best + 1];
            const float *cc = v4 + 4 * (size_t)idx[3 * (size_t)best + 2];
            double e1[3] = {(double)b[0] - a[0], (double)b[1] - a[1], (double)b[2] - a[2]};
            double e2[3] = {(double)cc[0] - a[0], (double)cc[1] - a[1], (double)cc[2] - a[2]};
            double nx = e1[1] * e2[2] - e1[2] * e2[1], ny = e1[2] * e2[0] - e1[0] * e2[2], nz = e1[0] * e2[1] - e1[1] * e2[0];
            double nl = sqrt(nx * nx + ny * ny + nz * nz), dl = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
            if (fabs(bdet) < 1e-3 * nl * dl) f |= 4;
        }
        if (nearmiss < (best >= 0 ? bt * (1.0 + 1e-5) : INFINITY)) f |= 2;
        id[i] = best; t[i] = best >= 0 ? bt : INFINITY; u[i] = bu; v[i] = bv; flags[i] = f;
    }
}

/* ------------------------------------------------------------------------- */
/* Instanced two-level grid hierarchy.                                        */

/* object grid cell range of a triangle box: countPairsMultiUniformGrid,
 * TLGridHierarchySortBuilder.cu:122-145 (both ends clamped into [0, res)) */
static inline uint32_t obj_cell_range(f3 lo, f3 hi, const orc_obj *g, crange *r) {
    float af[3] = {(lo.x - g->bmin[0]) * g->rcp[0], (lo.y - g->bmin[1]) * g->rcp[1], (lo.z - g->bmin[2]) * g->rcp[2]};
    float bf[3] = {(hi.x - g->bmin[0]) * g->rcp[0] + 1.0f, (hi.y - g->bmin[1]) * g->rcp[1] + 1.0f,
                   (hi.z - g->bmin[2]) * g->rcp[2] + 1.0f};
    uint32_t n = 1;
    for (int k = 0; k < 3; ++k) {
        r->lo[k] = imin(g->res[k] - 1, imax(0, f2i(af[k])));
        r->hi[k] = imax(1, imin(g->res[k], f2i(bf[k])));
        int32_t e = r->hi[k] - r->lo[k];
        n *= (uint32_t)(e > 0 ? e : 0);
    }
    return n;
}

/* object grid geometry: bounds padded by 10 EPS (RTEngine.cu:268-300) and the
 * resolution of countGridCellsMultiUniformGrid (TLGridHierarchySortBuilder.cu:31-57) */
static void obj_setup(orc_obj *g, f3 lo, f3 hi, float density) {
    const float pad = 10.0f * ORC_EPS;
    g->bmin[0] = lo.x - pad; g->bmin[1] = lo.y - pad; g->bmin[2] = lo.z - pad;
    g->bmax[0] = hi.x + pad; g->bmax[1] = hi.y + pad; g->bmax[2] = hi.z + pad;
    f3 d = mk(g->bmax[0] - g->bmin[0], g->bmax[1] - g->bmin[1], g->bmax[2] - g->bmin[2]);
    float vol = d.x * d.y * d.z;
    float m = orc_pow_third(density * (float)g->tri_count / vol);
    f3 r = mulf(d, m);
    int32_t ri[3] = {f2i(r.x), f2i(r.y), f2i(r.z)};
    for (int k = 0; k < 3; ++k) {
        g->res[k] = ri[k] > 0 ? ri[k] : 1;
        float dk = comp(d, k), rk = (float)g->res[k];
        g->cs[k] = dk / rk;
        g->rcp[k] = rk / dk;
    }
}

/* instance grid: union of the instance boxes padded as the scene bounds
 * (WFObjectUploader.h:112-114), resolution of TLGridHierarchySortBuilder.cu:275-286,
 * cell size diagonal / res (TLGridHierarchyMemoryManager.h:111-119) */
static void top_setup(orc_grid *g, const orc_inst *inst, uint32_t ninst, float density) {
    f3 lo = mk(FLT_MAX, FLT_MAX, FLT_MAX), hi = mk(-FLT_MAX, -FLT_MAX, -FLT_MAX);
    for (uint32_t i = 0; i < ninst; ++i) {
        lo = vmin(lo, ld3(inst[i].bmin));
        hi = vmax(hi, ld3(inst[i].bmax));
    }
    f3 dd = sub(hi, lo);
    float pad = 0.001f * sqrtf(dot(dd, dd));
    g->bmin[0] = lo.x - pad; g->bmin[1] = lo.y - pad; g->bmin[2] = lo.z - pad;
    g->bmax[0] = hi.x + pad; g->bmax[1] = hi.y + pad; g->bmax[2] = hi.z + pad;
    f3 d = mk(g->bmax[0] - g->bmin[0], g->bmax[1] - g->bmin[1], g->bmax[2] - g->bmin[2]);
    float vol = d.x * d.y * d.z;
    float m = orc_pow_third(density * (float)ninst / vol);
    f3 r = mulf(d, m);
    g->res[0] = imax(1, f2i(r.x)); g->res[1] = imax(1, f2i(r.y)); g->res[2] = imax(1, f2i(r.z));
    for (int k = 0; k < 3; ++k) {
        float dk = comp(d, k), rk = (float)g->res[k];
        g->cs[k] = dk / rk;
        g->rcp[k] = rk / dk;
    }
    g->ncells = (uint32_t)g->res[0] * (uint32_t)g->res[1] * (uint32_t)g->res[2];
}

int orc_hier_build(const float *v4, const uint32_t *idx, uint32_t ntri, const uint32_t *obj_tri_counts,
                   uint32_t nobj, const orc_inst *inst, uint32_t ninst, float top_density, float leaf_density,
                   orc_obj *objs, orc_grid *top, uint32_t **obj_cells, uint32_t *nobj_cells, uint32_t **prims,
                   uint32_t *npairs, uint32_t **top_cells, uint32_t **inst_ids, uint32_t *ntop_pairs) {
    /* level two: one uniform grid per object, cells of all objects in one array */
    uint32_t begin = 0, cells = 0;
    for (uint32_t k = 0; k < nobj; ++k) {
        orc_obj *g = &objs[k];
        g->tri_begin = begin;
        g->tri_count = obj_tri_counts[k];
        f3 lo = mk(FLT_MAX, FLT_MAX, FLT_MAX), hi = mk(-FLT_MAX, -FLT_MAX, -FLT_MAX);
        for (uint32_t t = begin; t < begin + g->tri_count; ++t)
            for (int c = 0; c < 3; ++c) {
                f3 p = vtx(v4, idx[3 * (size_t)t + c]);
                lo = vmin(lo, p);
                hi = vmax(hi, p);
            }
        obj_setup(g, lo, hi, leaf_density);
        g->cell_off = cells;
        cells += (uint32_t)g->res[0] * (uint32_t)g->res[1] * (uint32_t)g->res[2];
        begin += g->tri_count;
    }
    if (begin != ntri) return -1;
    /* pairs in triangle order (writeKeysAndValuesMultiUniformGrid, .cu:151-225), keys
     * offset by the object's first cell, then a stable sort by key */
    size_t *off = (size_t *)malloc(sizeof(size_t) * ((size_t)ntri + 1));
    uint32_t *tobj = (uint32_t *)malloc(sizeof(uint32_t) * ((size_t)ntri + 1));
    if (!off || !tobj) { free(off); free(tobj); return -1; }
    for (uint32_t k = 0; k < nobj; ++k)
        for (uint32_t t = objs[k].tri_begin; t < objs[k].tri_begin + objs[k].tri_count; ++t) tobj[t] = k;
    off[0] = 0;
    for (uint32_t t = 0; t < ntri; ++t) {
        f3 lo, hi, p[3];
        crange r;
        tri_bbox(v4, idx, t, &lo, &hi, p);
        off[t + 1] = off[t] + obj_cell_range(lo, hi, &objs[tobj[t]], &r);
    }
    size_t np = off[ntri];
    uint32_t *keys = (uint32_t *)malloc(sizeof(uint32_t) * (np + 1));
    uint32_t *vals = (uint32_t *)malloc(sizeof(uint32_t) * (np + 1));
    uint32_t *sk = (uint32_t *)malloc(sizeof(uint32_t) * (np + 1));
    uint32_t *sv = (uint32_t *)malloc(sizeof(uint32_t) * (np + 1));
    uint32_t *oc = (uint32_t *)malloc(sizeof(uint32_t) * 2 * ((size_t)cells + 1));
    if (!keys || !vals || !sk || !sv || !oc) {
        free(off); free(tobj); free(keys); free(vals); free(sk); free(sv); free(oc);
        return -1;
    }
    for (uint32_t t = 0; t < ntri; ++t) {
        const orc_obj *g = &objs[tobj[t]];
        f3 lo, hi, p[3];
        crange r;
        tri_bbox(v4, idx, t, &lo, &hi, p);
        obj_cell_range(lo, hi, g, &r);
        size_t w = off[t];
        const uint32_t rx = (uint32_t)g->res[0], rxy = (uint32_t)g->res[0] * (uint32_t)g->res[1];
        for (int32_t z = r.lo[2]; z < r.hi[2]; ++z)
            for (int32_t y = r.lo[1]; y < r.hi[1]; ++y)
                for (int32_t x = r.lo[0]; x < r.hi[0]; ++x) {
                    keys[w] = (uint32_t)x + (uint32_t)y * rx + (uint32_t)z * rxy + g->cell_off;
                    vals[w] = t;
                    ++w;
                }
    }
    stable_sort_pairs(keys, vals, np, cells + 1, sk, sv);
    cell_ranges(sk, np, cells, oc);
    free(off); free(tobj); free(keys); free(vals); free(sk);
    *obj_cells = oc; *nobj_cells = cells; *prims = sv; *npairs = (uint32_t)np;

    /* level one: instance boxes into a uniform grid (countPairs / writeKeysAndValues
     * over GeometryInstance boxes, UniformGridBuildKernels.h:40-105, 180-252) */
    top_setup(top, inst, ninst, top_density);
    size_t *ioff = (size_t *)malloc(sizeof(size_t) * ((size_t)ninst + 1));
    if (!ioff) return -1;
    ioff[0] = 0;
    for (uint32_t i = 0; i < ninst; ++i) {
        crange r;
        ioff[i + 1] = ioff[i] + cell_range(ld3(inst[i].bmin), ld3(inst[i].bmax), ld3(top->bmin), top->rcp, top->res, &r);
    }
    size_t ntp = ioff[ninst];
    uint32_t *ik = (uint32_t *)malloc(sizeof(uint32_t) * (ntp + 1));
    uint32_t *iv = (uint32_t *)malloc(sizeof(uint32_t) * (ntp + 1));
    uint32_t *isk = (uint32_t *)malloc(sizeof(uint32_t) * (ntp + 1));
    uint32_t *isv = (uint32_t *)malloc(sizeof(uint32_t) * (ntp + 1));
    uint32_t *tc = (uint32_t *)malloc(sizeof(uint32_t) * 2 * ((size_t)top->ncells + 1));
    if (!ik || !iv || !isk || !isv || !tc) {
        free(ioff); free(ik); free(iv); free(isk); free(isv); free(tc);
        return -1;
    }
    const uint32_t rx = (uint32_t)top->res[0], rxy = (uint32_t)top->res[0] * (uint32_t)top->res[1];
    for (uint32_t i = 0; i < ninst; ++i) {
        crange r;
        cell_range(ld3(inst[i].bmin), ld3(inst[i].bmax), ld3(top->bmin), top->rcp, top->res, &r);
        size_t w = ioff[i];
        for (int32_t z = r.lo[2]; z < r.hi[2]; ++z)
            for (int32_t y = r.lo[1]; y < r.hi[1]; ++y)
                for (int32_t x = r.lo[0]; x < r.hi[0]; ++x) {
                    ik[w] = (uint32_t)x + (uint32_t)y * rx + (uint32_t)z * rxy;
                    iv[w] = i;
                    ++w;
                }
    }
    stable_sort_pairs(ik, iv, ntp, top->ncells + 1, isk, isv);
    cell_ranges(isk, ntp, top->ncells, tc);
    free(ioff); free(ik); free(iv); free(isk);
    *top_cells = tc; *inst_ids = isv; *ntop_pairs = (uint32_t)ntp;
    return 0;
}

/* slab test against a box (BBox.hpp:64-79 fastClip) */
static inline void box_clip(const float *bmin, const float *bmax, f3 o, const float rcp[3], float *t0, float *t1) {
    float tn[3], tf[3];
    for (int k = 0; k < 3; ++k) {
        float a = (bmin[k] - comp(o, k)) * rcp[k];
        float b = (bmax[k] - comp(o, k)) * rcp[k];
        tn[k] = hmin(a, b); tf[k] = hmax(a, b);
    }
    *t0 = hmax(hmax(tn[0], tn[1]), tn[2]);
    *t1 = hmin(hmin(tf[0], tf[1]), tf[2]);
}

typedef struct { float t, u, v; int32_t inst, tri; } hhit;

/* one instance: world box test, ray into object space, object grid DDA
 * (GeometryInstanceTraverser, TLGridHierarchyTraverser.h:45-205).  Returns 1 when the
 * instance's hit is accepted. */
static int hier_instance(const orc_hier *H, uint32_t ii, f3 o, f3 d, const float rcp[3], hhit *h) {
    const orc_inst *I = &H->inst[ii];
    float te1, tx1;
    box_clip(I->bmin, I->bmax, o, rcp, &te1, &tx1);
    if (!(tx1 > te1 && tx1 >= 0.0f && te1 < h->t)) return 0;
    const float *m = I->m;
    /* transformRay (TwoLevelGridHierarchy.h:636-646): rows of the world -> object map;
     * the direction is carried, not re-derived from its reciprocal */
    f3 ot = mk(m[0] * o.x + m[1] * o.y + m[2] * o.z + m[3], m[4] * o.x + m[5] * o.y + m[6] * o.z + m[7],
               m[8] * o.x + m[9] * o.y + m[10] * o.z + m[11]);
    f3 dt = mk(m[0] * d.x + m[1] * d.y + m[2] * d.z, m[4] * d.x + m[5] * d.y + m[6] * d.z,
               m[8] * d.x + m[9] * d.y + m[10] * d.z);
    float rt[3] = {1.0f / dt.x, 1.0f / dt.y, 1.0f / dt.z};
    const orc_obj *g = &H->objs[I->obj];
    float rayT = h->t, bu = 0.0f, bv = 0.0f;
    int32_t best = -1;
    float te, tx;
    box_clip(g->bmin, g->bmax, ot, rt, &te, &tx);
    int flag = tx > te && tx >= 0.0f && te < rayT;
    f3 ep = ot;
    if (te >= 0.0f) { float s = te + ORC_EPS; ep = mk(ot.x + s * dt.x, ot.y + s * dt.y, ot.z + s * dt.z); }
    float tmax[3];
    int32_t cell[3];
    for (int k = 0; k < 3; ++k) {
        float cf = floorf((comp(ep, k) - g->bmin[k]) * g->rcp[k]);
        cf = rt[k] > 0.0f ? hmin((float)g->res[k] - 1.0f, cf) : hmax(cf, 0.0f);
        float stp = rt[k] > 0.0f ? 1.0f : 0.0f;
        tmax[k] = ((cf + stp) * g->cs[k] + g->bmin[k] - comp(ot, k)) * rt[k];
        cell[k] = f2i(cf);
        flag = flag && (rt[k] > 0.0f ? cell[k] < g->res[k] : cell[k] > -1);
    }
    const uint32_t rx = (uint32_t)g->res[0], rxy = (uint32_t)g->res[0] * (uint32_t)g->res[1];
    while (flag) {
        if (cell[0] < g->res[0] && cell[0] > -1 && cell[1] < g->res[1] && cell[1] > -1 && cell[2] < g->res[2] &&
            cell[2] > -1) {
            size_t c = g->cell_off + (uint32_t)cell[0] + (uint32_t)cell[1] * rx + (uint32_t)cell[2] * rxy;
            for (uint32_t it = H->obj_cells[2 * c]; it < H->obj_cells[2 * c + 1]; ++it) {
                uint32_t tri = H->prims[it];
                f3 v0 = vtx(H->v4, H->idx[3 * (size_t)tri]);
                f3 v1 = vtx(H->v4, H->idx[3 * (size_t)tri + 1]);
                f3 v2 = vtx(H->v4, H->idx[3 * (size_t)tri + 2]);
                f3 e1 = sub(v1, v0), e2 = sub(v2, v0);
                f3 p = cross(dt, e2);
                float det = dot(e1, p);
                float inv = 1.0f / det;
                f3 sv = sub(ot, v0);
                float u = dot(sv, p) * inv;
                f3 q = cross(sv, e1);
                float v = dot(q, dt) * inv;
                float t = dot(e2, q) * inv;
                if (u >= 0.0f && v >= 0.0f && u + v <= 1.0f && t > ORC_ISECT_EPS && t < rayT) {
                    rayT = t; bu = u; bv = v; best = (int32_t)tri;
                }
            }
        }
        int k = MIN_DIM(tmax[0], tmax[1], tmax[2]);
        flag = flag && rayT > tmax[k];
        cell[k] += rt[k] > 0.0f ? 1 : -1;
        tmax[k] += g->cs[k] * fabsf(rt[k]);
        flag = flag && (rt[k] > 0.0f ? cell[k] < g->res[k] : cell[k] > -1);
    }
    if (best >= 0 && rayT < h->t && rayT >= te1 && rayT < tx1) {
        h->t = rayT; h->u = bu; h->v = bv; h->inst = (int32_t)ii; h->tri = best;
        return 1;
    }
    return 0;
}

/* instance-grid DDA, TLGridHierarchyTraverser.h:220-405 */
static void trace_hier(const orc_hier *H, f3 o, f3 d, int anyhit, hhit *h) {
    const orc_grid *g = &H->top;
    float rcp[3] = {1.0f / d.x, 1.0f / d.y, 1.0f / d.z};
    float t0, t1;
    box_clip(g->bmin, g->bmax, o, rcp, &t0, &t1);
    if (!(t1 > t0 && t1 >= 0.0f)) return;
    f3 ep = o;
    if (t0 >= 0.0f) { float s = t0 + ORC_EPS; ep = mk(o.x + s * d.x, o.y + s * d.y, o.z + s * d.z); }
    float tmax[3];
    int32_t cell[3];
    int active = 1;
    for (int k = 0; k < 3; ++k) {
        float cf = floorf((comp(ep, k) - g->bmin[k]) * g->rcp[k]);
        float stp = rcp[k] > 0.0f ? 1.0f : 0.0f;
        tmax[k] = ((cf + stp) * g->cs[k] + g->bmin[k] - comp(o, k)) * rcp[k];
        cell[k] = f2i(cf);
        active = active && (rcp[k] > 0.0f ? cell[k] < g->res[k] : cell[k] > -1);
    }
    const uint32_t rx = (uint32_t)g->res[0], rxy = (uint32_t)g->res[0] * (uint32_t)g->res[1];
    while (active) {
        if (cell[0] < g->res[0] && cell[0] > -1 && cell[1] < g->res[1] && cell[1] > -1 && cell[2] < g->res[2] &&
            cell[2] > -1) {
            size_t c = (uint32_t)cell[0] + (uint32_t)cell[1] * rx + (uint32_t)cell[2] * rxy;
            for (uint32_t it = H->top_cells[2 * c]; it < H->top_cells[2 * c + 1]; ++it)
                if (hier_instance(H, H->inst_ids[it], o, d, rcp, h) && anyhit) return;
        }
        int k = MIN_DIM(tmax[0], tmax[1], tmax[2]);
        active = h->t > tmax[k];
        cell[k] += rcp[k] > 0.0f ? 1 : -1;
        tmax[k] += g->cs[k] * fabsf(rcp[k]);
        active = active && (rcp[k] > 0.0f ? cell[k] < g->res[k] : cell[k] > -1);
    }
}

void orc_hier_trace(const orc_hier *H, const float *org, const float *dir, const float *tmax, uint32_t n,
                    int anyhit, int32_t *inst_id, int32_t *tri_id, float *t, float *u, float *v) {
#pragma omp parallel for schedule(dynamic, 64)
    for (long long ii = 0; ii < (long long)n; ++ii) {
        size_t i = (size_t)ii;
        hhit h;
        h.t = tmax ? tmax[i] : FLT_MAX; h.u = 0.0f; h.v = 0.0f; h.inst = -1; h.tri = -1;
        trace_hier(H, ld3(org + 3 * i), ld3(dir + 3 * i), anyhit, &h);
        inst_id[i] = h.inst; tri_id[i] = h.tri;
        t[i] = h.inst >= 0 ? h.t : FLT_MAX; u[i] = h.u; v[i] = h.v;
    }
}
