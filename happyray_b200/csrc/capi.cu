// capi.cu -- the extern "C" boundary of libhappyray_b200.so (declared in include/happyray.h).
//
// Mirrors the reference engine facade RTEngine (src/RT/RTEngine.h:36-68,
// src/RT/RTEngine.cu:190-474) over an explicit context instead of static globals, with
// status codes instead of exit(1) (src/Utils/CUDAUtil.h:199-206).
#include "hr_internal.h"
#include "../../include/happyray.h"

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

namespace hr {

int set_error(hr_ctx* c, int code, const char* fmt, ...) {
    if (c) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof(buf), fmt, ap);
        va_end(ap);
        c->err = buf;
    }
    return code;
}

int cuda_check(hr_ctx* c, cudaError_t e, const char* what) {
    if (e == cudaSuccess) return 0;
    int code = (e == cudaErrorMemoryAllocation) ? HR_ERR_OUT_OF_MEMORY : HR_ERR_DEVICE;
    return set_error(c, code, "%s: %s", what, cudaGetErrorString(e));
}

int ensure(hr_ctx* c, DevBuf& b, size_t bytes) {
    if (bytes == 0) bytes = 16;
    if (b.bytes >= bytes) return 0;
    if (b.p) {
        cudaError_t e = cudaFreeAsync(b.p, c->stream);
        if (e != cudaSuccess) cudaFree(b.p);
        b.p = nullptr;
        b.bytes = 0;
    }
    size_t want = bytes + bytes / 8;   // grow-only with headroom
    cudaError_t e = cudaMallocAsync(&b.p, want, c->stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return set_error(c, HR_ERR_OUT_OF_MEMORY, "device allocation of %zu bytes failed: %s", want,
                         cudaGetErrorString(e));
    }
    b.bytes = want;
    return 0;
}

int make_light_set(LightSet* out, uint32_t n, const float* corners, const float* e1, const float* e2,
                   const float* normals, const float* emissions) {
    if (n < 1 || n > (uint32_t)kMaxLights || !corners || !e1 || !e2 || !emissions) return 1;
    std::memset(out, 0, sizeof(LightSet));
    out->count = n;
    float run = 0.0f;
    for (uint32_t k = 0; k < n; ++k) {
        LightQ& q = out->q[k];
        for (int i = 0; i < 3; ++i) { q.c[i] = corners[3 * k + i]; q.e1[i] = e1[3 * k + i]; q.e2[i] = e2[3 * k + i]; }
        q.nc[0] = q.e1[1] * q.e2[2] - q.e1[2] * q.e2[1];
        q.nc[1] = q.e1[2] * q.e2[0] - q.e1[0] * q.e2[2];
        q.nc[2] = q.e1[0] * q.e2[1] - q.e1[1] * q.e2[0];
        const float nn = q.nc[0] * q.nc[0] + q.nc[1] * q.nc[1] + q.nc[2] * q.nc[2];
        if (!(nn > 0.0f) || !(emissions[k] >= 0.0f)) return 1;
        q.inv_nn = 1.0f / nn;
        q.area = sqrtf(nn);
        q.emission = emissions[k];
        if (normals) {
            for (int i = 0; i < 3; ++i) q.n[i] = normals[3 * k + i];
        } else {   // the side of e2 x e1 = -nc
            const float inv = 1.0f / q.area;
            for (int i = 0; i < 3; ++i) q.n[i] = -q.nc[i] * inv;
        }
        run = run + q.area * q.emission;
        out->cdf[k] = run;
    }
    return 0;
}

int set_lights(hr_ctx* c, uint32_t n, const float* corners, const float* e1, const float* e2, const float* normals,
               const float* emissions) {
    LightSet ls;
    if (make_light_set(&ls, n, corners, e1, e2, normals, emissions))
        return set_error(c, HR_ERR_INVALID_ARG, "set_lights: %u lights (1..%d, non-degenerate, emission >= 0)", n,
                         kMaxLights);
    int rc;
    if ((rc = ensure(c, c->lights_dev, sizeof(LightSet)))) return rc;
    // stream order: renders enqueued before this call still read the previous collection
    c->lights = ls;
    if ((rc = cuda_check(c, cudaMemcpyAsync(c->lights_dev.p, &c->lights, sizeof(LightSet), cudaMemcpyHostToDevice,
                                            c->stream), "light upload")))
        return rc;
    return cuda_check(c, cudaStreamSynchronize(c->stream), "light upload");
}

// Camera::init (Camera.h:40-64), evaluated on the host in binary32
void camera_init(Camera* c, const float pos[3], const float fwd[3], const float up[3], float fov, int w, int h) {
    auto norm = [](float v[3]) {
        float inv = 1.0f / sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        v[0] = v[0] * inv; v[1] = v[1] * inv; v[2] = v[2] * inv;
    };
    auto crs = [](const float a[3], const float b[3], float r[3]) {
        r[0] = a[1] * b[2] - a[2] * b[1];
        r[1] = a[2] * b[0] - a[0] * b[2];
        r[2] = a[0] * b[1] - a[1] * b[0];
    };
    float f[3] = {fwd[0], fwd[1], fwd[2]};
    norm(f);
    float r[3], u[3];
    crs(f, up, r);
    norm(r);
    crs(f, r, u);
    norm(u);
    const float aspect = (float)w / (float)h;
    const float ang = fov * 3.14159265358979323846f / 180.0f;
    const float tn = tanf(ang / 2.0f);
    for (int k = 0; k < 3; ++k) {
        float row = r[k] * 2.0f * tn * aspect;
        float col = u[k] * 2.0f * tn;
        c->pos[k] = pos[k];
        c->step_x[k] = row / (float)w;
        c->step_y[k] = col / (float)h;
        c->top_left[k] = f[k] - row / 2.0f - col / 2.0f;
    }
    c->w = w;
    c->h = h;
}

namespace {

void free_buf(hr_ctx* c, DevBuf& b) {
    if (b.p) cudaFreeAsync(b.p, c->stream);
    b.p = nullptr;
    b.bytes = 0;
}

__global__ void k_expand_xyz(const float* __restrict__ xyz, float4* __restrict__ out, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        out[i] = make_float4(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], 0.0f);
}

}  // namespace

void expand_xyz(const float* xyz, float4* out, size_t n, int grid, cudaStream_t s) {
    k_expand_xyz<<<grid, 256, 0, s>>>(xyz, out, n);
}

namespace {


int ensure_pinned(hr_ctx* c, size_t bytes) {
    if (c->pinned_bytes >= bytes) return 0;
    if (c->pinned) cudaFreeHost(c->pinned);
    c->pinned = nullptr;
    c->pinned_bytes = 0;
    if (cudaMallocHost(&c->pinned, bytes) != cudaSuccess) {
        cudaGetLastError();
        return set_error(c, HR_ERR_OUT_OF_MEMORY, "pinned host allocation of %zu bytes failed", bytes);
    }
    c->pinned_bytes = bytes;
    return 0;
}

// copy `frames` xyz frames from host to float4 device storage
int upload_frames(hr_ctx* c, const float* const* frames, uint32_t nframes, uint32_t nv, DevBuf& dst) {
    const size_t fbytes = (size_t)nv * 3 * sizeof(float);
    int rc;
    if ((rc = ensure(c, dst, (size_t)nv * nframes * sizeof(float4)))) return rc;
    if ((rc = ensure(c, c->staging, fbytes * nframes))) return rc;
    for (uint32_t f = 0; f < nframes; ++f) {
        if ((rc = cuda_check(c, cudaMemcpyAsync(c->staging.as<char>() + f * fbytes, frames[f], fbytes,
                                                cudaMemcpyHostToDevice, c->stream), "frame upload")))
            return rc;
    }
    const size_t n = (size_t)nv * nframes;
    int grid = (int)std::min<size_t>((n + 255) / 256, (size_t)c->num_sms * 16);
    if (grid < 1) grid = 1;
    k_expand_xyz<<<grid, 256, 0, c->stream>>>(c->staging.as<float>(), dst.as<float4>(), n);
    return cuda_check(c, cudaGetLastError(), "frame expand");
}

// counts indices >= nv; the count lands in counters word 2 and makes the next build fail
__global__ void k_check_indices(const uint32_t* __restrict__ idx, size_t n, uint32_t nv, uint32_t* bad) {
    uint32_t cnt = 0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        cnt += idx[i] >= nv ? 1u : 0u;
    if (cnt) atomicAdd(bad, cnt);
}

int upload_indices(hr_ctx* c, const uint32_t* idx, uint32_t ntri, uint32_t nv) {
    int rc;
    if ((rc = ensure(c, c->idx, (size_t)ntri * 3 * sizeof(uint32_t)))) return rc;
    uint32_t* bad = c->counters.as<uint32_t>() + 2;
    if ((rc = cuda_check(c, cudaMemsetAsync(bad, 0, sizeof(uint32_t), c->stream), "index check"))) return rc;
    if (ntri == 0) return 0;
    if ((rc = cuda_check(c, cudaMemcpyAsync(c->idx.p, idx, (size_t)ntri * 3 * sizeof(uint32_t), cudaMemcpyHostToDevice,
                                            c->stream), "index upload")))
        return rc;
    const size_t n = (size_t)ntri * 3;
    int grid = (int)std::min<size_t>((n + 255) / 256, (size_t)c->num_sms * 8);
    k_check_indices<<<grid, 256, 0, c->stream>>>(c->idx.as<uint32_t>(), n, nv, bad);
    return cuda_check(c, cudaGetLastError(), "index check");
}

bool bad(hr_ctx* c) { return c == nullptr; }

}  // namespace
}  // namespace hr

using namespace hr;

extern "C" {

hr_status hr_create(hr_ctx** out, int32_t device, void* stream) {
    if (!out) return HR_ERR_INVALID_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return HR_ERR_DEVICE;
    }
    if (device < 0 || device >= ndev) return HR_ERR_INVALID_ARG;
    hr_ctx* c = new (std::nothrow) hr_ctx();
    if (!c) return HR_ERR_OUT_OF_MEMORY;
    c->device = device;
    if (cudaSetDevice(device) != cudaSuccess) { delete c; return HR_ERR_DEVICE; }
    cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device);
    if (const char* e = std::getenv("HAPPYRAY_SMALL_BUILD_MAX_TRIS")) c->small_build_max_tris = (uint32_t)std::strtoul(e, nullptr, 10);
    if (stream) {
        c->stream = (cudaStream_t)stream;
    } else {
        if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) { delete c; return HR_ERR_DEVICE; }
        c->own_stream = true;
    }
    for (auto& e : c->ev) cudaEventCreate(&e);
    for (auto& e : c->rev) cudaEventCreate(&e);
    if (ensure(c, c->counters, 80)) { hr_destroy(c); return HR_ERR_OUT_OF_MEMORY; }   // 8 counter words, 2 pool words
    cudaMemsetAsync(c->counters.p, 0, 80, c->stream);
    {   // default light: a 0.2 x 0.2 quad at z = 1 centred over (0.5, 0.5), emitting along -z
        const float corner[3] = {0.4f, 0.4f, 1.0f}, e1[3] = {0.2f, 0.0f, 0.0f}, e2[3] = {0.0f, 0.2f, 0.0f};
        const float em = 20.0f;
        if (set_lights(c, 1, corner, e1, e2, nullptr, &em)) { hr_destroy(c); return HR_ERR_OUT_OF_MEMORY; }
    }
    *out = c;
    return HR_OK;
}

void hr_destroy(hr_ctx* c) {
    if (!c) return;
    DeviceGuard dg(c->device);
    cudaStreamSynchronize(c->stream);
    drop_build_graph(c);
    DevBuf* bufs[] = {&c->verts, &c->idx, &c->tris, &c->keyframes, &c->frame_sel, &c->staging, &c->counters, &c->fb, &c->out_id,
                      &c->out_t, &c->out_u, &c->out_v, &c->ray_in, &c->g.desc, &c->g.cells, &c->g.leaves,
                      &c->g.prims, &c->g.keys_a, &c->g.vals_a, &c->g.keys_b, &c->g.vals_b, &c->g.block_sums,
                      &c->g.tile_hist, &c->g.row_total, &c->g.leaf_cnt, &c->g.occ,
                      &c->g.lkeys_a, &c->g.lvals_a, &c->g.lkeys_b, &c->g.lvals_b, &c->g.scan_partials,
                      &c->g.tri_ranges, &c->g.ref_ranges, &c->lights_dev, &c->tri_nrm, &c->tri_alb,
                      &c->hit_t, &c->hit_tri, &c->unocc, &c->queue, &c->build_bar};
    for (DevBuf* b : bufs) free_buf(c, *b);
    cudaStreamSynchronize(c->stream);
    for (auto& e : c->ev) if (e) cudaEventDestroy(e);
    for (auto& e : c->rev) if (e) cudaEventDestroy(e);
    if (c->pinned) cudaFreeHost(c->pinned);
    if (c->desc_pinned) cudaFreeHost(c->desc_pinned);
    if (c->own_stream) cudaStreamDestroy(c->stream);
    delete c;
}

const char* hr_last_error(const hr_ctx* c) { return c ? c->err.c_str() : "null context"; }

hr_status hr_upload(hr_ctx* c, const float* f1, const float* f2, uint32_t nv, const uint32_t* idx, uint32_t ntri,
                    float coeff) {
    if (bad(c)) return HR_ERR_INVALID_ARG;
    if ((nv && (!f1 || !f2)) || (ntri && !idx)) return (hr_status)set_error(c, HR_ERR_INVALID_ARG, "upload: null input");
    DeviceGuard dg(c->device);
    const float* frames[2] = {f1, f2};
    int rc;
    if ((rc = upload_frames(c, frames, 2, nv, c->keyframes))) return (hr_status)rc;
    if ((rc = upload_indices(c, idx, ntri, nv))) return (hr_status)rc;
    if ((rc = ensure(c, c->verts, (size_t)nv * sizeof(float4)))) return (hr_status)rc;
    c->nverts = nv;
    c->ntri = ntri;
    c->nkeyframes = 2;
    c->frame_a = 0;
    c->frame_b = 1;
    c->frame_coeff = coeff;
    c->lerp_pending = true;
    c->have_frame = true;
    c->built = false;
    return HR_OK;
}

hr_status hr_set_keyframes(hr_ctx* c, const float* xyz, uint32_t nk, uint32_t nv, const uint32_t* idx, uint32_t ntri) {
    if (bad(c)) return HR_ERR_INVALID_ARG;
    if (nk == 0 || (nv && !xyz) || (ntri && !idx)) return (hr_status)set_error(c, HR_ERR_INVALID_ARG, "set_keyframes: bad input");
    DeviceGuard dg(c->device);
    int rc;
    const float* frames[1] = {xyz};
    // one contiguous block of nk frames
    const size_t bytes = (size_t)nv * nk * 3 * sizeof(float);
    if ((rc = ensure(c, c->keyframes, (size_t)nv * nk * sizeof(float4)))) return (hr_status)rc;
    if ((rc = ensure(c, c->staging, bytes))) return (hr_status)rc;
    if (bytes && (rc = cuda_check(c, cudaMemcpyAsync(c->staging.p, frames[0], bytes, cudaMemcpyHostToDevice, c->stream),
                                  "keyframe upload")))
        return (hr_status)rc;
    const size_t n = (size_t)nv * nk;
    int grid = (int)std::min<size_t>((n + 255) / 256, (size_t)c->num_sms * 16);
    if (grid < 1) grid = 1;
    k_expand_xyz<<<grid, 256, 0, c->stream>>>(c->staging.as<float>(), c->keyframes.as<float4>(), n);
    if ((rc = cuda_check(c, cudaGetLastError(), "keyframe expand"))) return (hr_status)rc;
    if ((rc = upload_indices(c, idx, ntri, nv))) return (hr_status)rc;
    if ((rc = ensure(c, c->verts, (size_t)nv * sizeof(float4)))) return (hr_status)rc;
    c->nverts = nv;
    c->ntri = ntri;
    c->nkeyframes = nk;
    c->frame_a = 0;
    c->frame_b = 0;
    c->frame_coeff = 1.0f;
    c->lerp_pending = true;
    c->have_frame = true;
    c->built = false;
    return HR_OK;
}

hr_status hr_set_frame_time(hr_ctx* c, float t, float step) {
    if (bad(c)) return HR_ERR_INVALID_ARG;
    if (c->nkeyframes == 0) return (hr_status)set_error(c, HR_ERR_NOT_READY, "set_frame_time: no key frames");
    if (!(t >= 0.0f) || !(step >= 0.0f)) return (hr_status)set_error(c, HR_ERR_INVALID_ARG, "set_frame_time: negative time");
    const size_t k = (size_t)t;
    if (k >= c->nkeyframes) return (hr_status)set_error(c, HR_ERR_INVALID_ARG, "set_frame_time: time beyond key frames");
    c->frame_a = (int32_t)k;
    c->frame_b = (int32_t)((k + 1u + (size_t)step) % c->nkeyframes);
    c->frame_coeff = t - (float)k;
    c->lerp_pending = true;
    return HR_OK;
}

hr_status hr_set_grid_densities(hr_ctx* c, float top, float leaf) {
    if (bad(c) || !(top > 0.0f) || !(leaf > 0.0f)) return HR_ERR_INVALID_ARG;
    c->top_density = top;
    c->leaf_density = leaf;
    return HR_OK;
}

hr_status hr_set_uniform_density(hr_ctx* c, float d) {
    if (bad(c) || !(d > 0.0f)) return HR_ERR_INVALID_ARG;
    c->ug_density = d;
    return HR_OK;
}

hr_status hr_build(hr_ctx* c, int32_t kind, int32_t exact) {
    if (bad(c)) return HR_ERR_INVALID_ARG;
    if (kind != HR_GRID_UNIFORM && kind != HR_GRID_TWO_LEVEL)
        return (hr_status)set_error(c, HR_ERR_INVALID_ARG, "build: unknown grid kind %d", kind);
    if (!c->have_frame) return (hr_status)set_error(c, HR_ERR_NOT_READY, "build: no mesh uploaded");
    DeviceGuard dg(c->device);
    return (hr_status)build_grid(c, kind, exact);
}

hr_status hr_grid_get_info(hr_ctx* c, hr_grid_info* info) {
    if (bad(c) || !info) return HR_ERR_INVALID_ARG;
    if (!c->built) return (hr_status)set_error(c, HR_ERR_NOT_READY, "grid_get_info: no grid built");
    const GridDesc& d = c->host_desc;
    info->kind = c->built_kind;
    for (int k = 0; k < 3; ++k) {
        info->res[k] = d.res[k];
        info->bounds_min[k] = d.bmin[k]; info->bounds_max[k] = d.bmax[k];
        info->cell_size[k] = d.cs[k]; info->cell_size_rcp[k] = d.rcp[k];
    }
    info->num_cells = d.ncells;
    info->num_leaves = c->built_kind == HR_GRID_TWO_LEVEL ? d.nleaves : 0u;
    info->num_pairs = d.npairs;
    info->num_top_pairs = c->built_kind == HR_GRID_TWO_LEVEL ? d.ntop_pairs : 0u;
    return HR_OK;
}

hr_status hr_grid_download(hr_ctx* c, uint32_t* cells, uint32_t* leaves, uint32_t* prims) {
    if (bad(c)) return HR_ERR_INVALID_ARG;
    if (!c->built) return (hr_status)set_error(c, HR_ERR_NOT_READY, "grid_download: no grid built");
    DeviceGuard dg(c->device);
    const GridDesc& d = c->host_desc;
    int rc;
    if (cells && d.ncells &&
        (rc = cuda_check(c, cudaMemcpyAsync(cells, c->g.cells.p, (size_t)d.ncells * 8, cudaMemcpyDeviceToHost, c->stream), "cells")))
        return (hr_status)rc;
    if (leaves && c->built_kind == HR_GRID_TWO_LEVEL && d.nleaves &&
        (rc = cuda_check(c, cudaMemcpyAsync(leaves, c->g.leaves.p, (size_t)d.nleaves * 8, cudaMemcpyDeviceToHost, c->stream), "leaves")))
        return (hr_status)rc;
    if (prims && d.npairs &&
        (rc = cuda_check(c, cudaMemcpyAsync(prims, c->g.prims.p, (size_t)d.npairs * 4, cudaMemcpyDeviceToHost, c->stream), "prims")))
        return (hr_status)rc;
    return (hr_status)cuda_check(c, cudaStreamSynchronize(c->stream), "grid_download");
}

hr_status hr_set_timing(hr_ctx* c, int32_t enable) {
    if (bad(c)) return HR_ERR_INVALID_ARG;
    c->timing = enable != 0;
    return HR_OK;
}

int32_t hr_get_stage_times(hr_ctx* c, float* ms, int32_t max_stages) {
    if (bad(c) || !ms) return 0;
    int32_t n = c->nstages > 0 ? c->nstages - 1 : 0;
    if (n > max_stages) n = max_stages;
    for (int32_t i = 0; i < n; ++i) ms[i] = c->stage_ms[i];
    return n;
}

hr_status hr_download_vertices(hr_ctx* c, float* xyzw) {
    if (bad(c) || !xyzw) return HR_ERR_INVALID_ARG;
    if (!c->built) return (hr_status)set_error(c, HR_ERR_NOT_READY, "download_vertices: build first");
    DeviceGuard dg(c->device);
    int rc = cuda_check(c, cudaMemcpyAsync(xyzw, c->verts.p, (size_t)c->nverts * 16, cudaMemcpyDeviceToHost, c->stream), "vertices");
    if (rc) return (hr_status)rc;
    return (hr_status)cuda_check(c, cudaStreamSynchronize(c->stream), "download_vertices");
}

hr_status hr_set_camera(hr_ctx* c, const float pos[3], const float orient[3], const float up[3], float fov, int32_t w,
                        int32_t h) {
    if (bad(c) || !pos || !orient || !up || w <= 0 || h <= 0 || !(fov > 0.0f && fov < 180.0f))
        return c ? (hr_status)set_error(c, HR_ERR_INVALID_ARG, "set_camera: bad arguments") : HR_ERR_INVALID_ARG;
    camera_init(&c->cam, pos, orient, up, fov, w, h);
    c->have_camera = true;
    return HR_OK;
}

hr_status hr_set_light(hr_ctx* c, const float corner[3], const float e1[3], const float e2[3], float emission) {
    if (bad(c) || !corner || !e1 || !e2) return HR_ERR_INVALID_ARG;
    DeviceGuard dg(c->device);
    return (hr_status)set_lights(c, 1, corner, e1, e2, nullptr, &emission);
}

hr_status hr_set_lights(hr_ctx* c, uint32_t n, const float* corners, const float* edge1s, const float* edge2s,
                        const float* normals, const float* emissions) {
    if (bad(c)) return HR_ERR_INVALID_ARG;
    DeviceGuard dg(c->device);
    return (hr_status)set_lights(c, n, corners, edge1s, edge2s, normals, emissions);
}

hr_status hr_set_normals(hr_ctx* c, const float* normals, uint32_t num_normals, const uint32_t* tri_normal_idx) {
    if (bad(c)) return HR_ERR_INVALID_ARG;
    if (!normals || !tri_normal_idx || num_normals == 0) {
        c->nrm_ntri = 0;
        return HR_OK;
    }
    if (c->ntri == 0) return (hr_status)set_error(c, HR_ERR_NOT_READY, "set_normals: upload the mesh first");
    DeviceGuard dg(c->device);
    std::vector<float> g((size_t)c->ntri * 12);
    for (size_t i = 0; i < 3 * (size_t)c->ntri; ++i) {
        const uint32_t k = tri_normal_idx[i];
        if (k >= num_normals) return (hr_status)set_error(c, HR_ERR_INVALID_ARG, "set_normals: index %u of %u", k, num_normals);
        g[4 * i] = normals[3 * (size_t)k]; g[4 * i + 1] = normals[3 * (size_t)k + 1];
        g[4 * i + 2] = normals[3 * (size_t)k + 2]; g[4 * i + 3] = 0.0f;
    }
    int rc;
    if ((rc = ensure(c, c->tri_nrm, g.size() * sizeof(float)))) return (hr_status)rc;
    if ((rc = cuda_check(c, cudaMemcpyAsync(c->tri_nrm.p, g.data(), g.size() * sizeof(float), cudaMemcpyHostToDevice,
                                            c->stream), "normal upload")) ||
        (rc = cuda_check(c, cudaStreamSynchronize(c->stream), "normal upload")))
        return (hr_status)rc;
    c->nrm_ntri = c->ntri;
    return HR_OK;
}

hr_status hr_set_materials(hr_ctx* c, const float* albedo, uint32_t num_materials, const uint32_t* tri_material) {
    if (bad(c)) return HR_ERR_INVALID_ARG;
    if (!albedo || !tri_material || num_materials == 0) {
        c->alb_ntri = 0;
        return HR_OK;
    }
    if (c->ntri == 0) return (hr_status)set_error(c, HR_ERR_NOT_READY, "set_materials: upload the mesh first");
    DeviceGuard dg(c->device);
    std::vector<float> g(c->ntri);
    for (size_t i = 0; i < c->ntri; ++i) {
        const uint32_t k = tri_material[i];
        if (k >= num_materials) return (hr_status)set_error(c, HR_ERR_INVALID_ARG, "set_materials: index %u of %u", k, num_materials);
        g[i] = albedo[k];
    }
    int rc;
    if ((rc = ensure(c, c->tri_alb, g.size() * sizeof(float)))) return (hr_status)rc;
    if ((rc = cuda_check(c, cudaMemcpyAsync(c->tri_alb.p, g.data(), g.size() * sizeof(float), cudaMemcpyHostToDevice,
                                            c->stream), "material upload")) ||
        (rc = cuda_check(c, cudaStreamSynchronize(c->stream), "material upload")))
        return (hr_status)rc;
    c->alb_ntri = c->ntri;
    return HR_OK;
}

hr_status hr_set_integrator(hr_ctx* c, int32_t ao_samples, float ao_radius, int32_t pt_bounces, float albedo,
                            uint64_t seed) {
    if (bad(c) || ao_samples < 0 || pt_bounces < 0) return HR_ERR_INVALID_ARG;
    c->ip.ao_samples = ao_samples;
    if (ao_radius < 0.0f) { c->ip.ao_radius_frac = -ao_radius; c->ip.ao_radius_abs = 0.0f; }
    else c->ip.ao_radius_abs = ao_radius;
    c->ip.pt_bounces = pt_bounces;
    c->ip.albedo = albedo;
    c->ip.seed = seed;
    return HR_OK;
}

static int render_check(hr_ctx* c) {
    if (!c->built) return set_error(c, HR_ERR_NOT_READY, "render: build a grid first");
    if (!c->have_camera) return set_error(c, HR_ERR_NOT_READY, "render: no camera");
    return 0;
}

hr_status hr_render_device(hr_ctx* c, int32_t mode, int32_t image_id, float* d_fb) {
    if (bad(c) || !d_fb || image_id < 0) return HR_ERR_INVALID_ARG;
    int rc;
    if ((rc = render_check(c))) return (hr_status)rc;
    DeviceGuard dg(c->device);
    return (hr_status)launch_render(c, mode, image_id, d_fb);
}

hr_status hr_render(hr_ctx* c, int32_t mode, int32_t image_id, float* fb) {
    if (bad(c) || !fb || image_id < 0) return HR_ERR_INVALID_ARG;
    int rc;
    if ((rc = render_check(c))) return (hr_status)rc;
    DeviceGuard dg(c->device);
    const size_t bytes = (size_t)c->cam.w * c->cam.h * 3 * sizeof(float);
    if ((rc = ensure(c, c->fb, bytes))) return (hr_status)rc;
    // image 0 weighs the old content by 0: start from zeros (the reused buffer may hold anything)
    if (image_id > 0) rc = cuda_check(c, cudaMemcpyAsync(c->fb.p, fb, bytes, cudaMemcpyHostToDevice, c->stream), "fb upload");
    else rc = cuda_check(c, cudaMemsetAsync(c->fb.p, 0, bytes, c->stream), "fb clear");
    if (rc) return (hr_status)rc;
    if ((rc = launch_render(c, mode, image_id, c->fb.as<float>()))) return (hr_status)rc;
    if ((rc = cuda_check(c, cudaMemcpyAsync(fb, c->fb.p, bytes, cudaMemcpyDeviceToHost, c->stream), "fb download")))
        return (hr_status)rc;
    return (hr_status)cuda_check(c, cudaStreamSynchronize(c->stream), "render");
}

hr_status hr_trace_rays_device(hr_ctx* c, const float* org, const float* dir, uint32_t n, int32_t* id, float* t,
                               float* u, float* v) {
    if (bad(c) || (n && (!org || !dir || !id || !t || !u || !v))) return HR_ERR_INVALID_ARG;
    if (!c->built) return (hr_status)set_error(c, HR_ERR_NOT_READY, "trace_rays: build a grid first");
    DeviceGuard dg(c->device);
    return (hr_status)launch_trace_rays(c, org, dir, n, id, t, u, v, nullptr);
}

hr_status hr_trace_rays(hr_ctx* c, const float* org, const float* dir, uint32_t n, int32_t* id, float* t, float* u,
                        float* v) {
    if (bad(c) || (n && (!org || !dir || !id || !t || !u || !v))) return HR_ERR_INVALID_ARG;
    if (!c->built) return (hr_status)set_error(c, HR_ERR_NOT_READY, "trace_rays: build a grid first");
    if (n == 0) return HR_OK;
    DeviceGuard dg(c->device);
    int rc;
    const size_t b3 = (size_t)n * 3 * sizeof(float), b1 = (size_t)n * sizeof(float);
    if ((rc = ensure(c, c->ray_in, 2 * b3))) return (hr_status)rc;
    if ((rc = ensure(c, c->out_id, b1)) || (rc = ensure(c, c->out_t, b1)) || (rc = ensure(c, c->out_u, b1)) ||
        (rc = ensure(c, c->out_v, b1)))
        return (hr_status)rc;
    float* dorg = c->ray_in.as<float>();
    float* ddir = dorg + (size_t)n * 3;
    if ((rc = cuda_check(c, cudaMemcpyAsync(dorg, org, b3, cudaMemcpyHostToDevice, c->stream), "ray upload")) ||
        (rc = cuda_check(c, cudaMemcpyAsync(ddir, dir, b3, cudaMemcpyHostToDevice, c->stream), "ray upload")))
        return (hr_status)rc;
    if ((rc = launch_trace_rays(c, dorg, ddir, n, c->out_id.as<int32_t>(), c->out_t.as<float>(), c->out_u.as<float>(),
                                c->out_v.as<float>(), nullptr)))
        return (hr_status)rc;
    if ((rc = cuda_check(c, cudaMemcpyAsync(id, c->out_id.p, b1, cudaMemcpyDeviceToHost, c->stream), "hit download")) ||
        (rc = cuda_check(c, cudaMemcpyAsync(t, c->out_t.p, b1, cudaMemcpyDeviceToHost, c->stream), "hit download")) ||
        (rc = cuda_check(c, cudaMemcpyAsync(u, c->out_u.p, b1, cudaMemcpyDeviceToHost, c->stream), "hit download")) ||
        (rc = cuda_check(c, cudaMemcpyAsync(v, c->out_v.p, b1, cudaMemcpyDeviceToHost, c->stream), "hit download")))
        return (hr_status)rc;
    return (hr_status)cuda_check(c, cudaStreamSynchronize(c->stream), "trace_rays");
}

hr_status hr_trace_primary_device(hr_ctx* c, int32_t* id, float* t, float* u, float* v, uint32_t* stats) {
    if (bad(c) || !id || !t || !u || !v) return HR_ERR_INVALID_ARG;
    int rc;
    if ((rc = render_check(c))) return (hr_status)rc;
    DeviceGuard dg(c->device);
    return (hr_status)launch_trace_primary(c, id, t, u, v, stats);
}

hr_status hr_render_rays_device(hr_ctx* c, const float* org, const float* dir, uint32_t n, int32_t image_id,
                                float* fb) {
    if (bad(c) || (n && (!org || !dir || !fb)) || image_id < 0) return HR_ERR_INVALID_ARG;
    if (!c->built) return (hr_status)set_error(c, HR_ERR_NOT_READY, "render_rays: build a grid first");
    DeviceGuard dg(c->device);
    return (hr_status)launch_render_rays(c, org, dir, n, image_id, fb);
}

hr_status hr_occluded_device(hr_ctx* c, const float* org, const float* dir, const float* tmax, uint32_t n, uint8_t* occ) {
    if (bad(c) || (n && (!org || !dir || !tmax || !occ))) return HR_ERR_INVALID_ARG;
    if (!c->built) return (hr_status)set_error(c, HR_ERR_NOT_READY, "occluded: build a grid first");
    DeviceGuard dg(c->device);
    return (hr_status)launch_occluded(c, org, dir, tmax, n, occ);
}

// device counter words: [0] rays, [2] cells, [3] tests of the primary pass; [4] rays,
// [5] cells, [6] tests of the secondary pass; [1] index check; [7] AO queue length
static int read_counters(hr_ctx* c, uint64_t w[8], int32_t reset) {
    int rc;
    if ((rc = cuda_check(c, cudaMemcpyAsync(w, c->counters.p, 64, cudaMemcpyDeviceToHost, c->stream), "counters")))
        return rc;
    if (reset) {
        // word 1 holds the index-check result of the last upload and is kept
        cudaMemsetAsync(c->counters.p, 0, 8, c->stream);
        cudaMemsetAsync(c->counters.as<uint64_t>() + 2, 0, 40, c->stream);
    }
    return cuda_check(c, cudaStreamSynchronize(c->stream), "counters");
}

hr_status hr_get_ray_count(hr_ctx* c, uint64_t* rays, int32_t reset) {
    if (bad(c) || !rays) return HR_ERR_INVALID_ARG;
    DeviceGuard dg(c->device);
    uint64_t w[8];
    int rc;
    if ((rc = read_counters(c, w, reset))) return (hr_status)rc;
    *rays = w[0] + w[4];
    return HR_OK;
}

hr_status hr_set_stats(hr_ctx* c, int32_t enable) {
    if (bad(c)) return HR_ERR_INVALID_ARG;
    c->collect_stats = enable != 0;
    return HR_OK;
}

hr_status hr_get_counters(hr_ctx* c, uint64_t out[8], int32_t reset) {
    if (bad(c) || !out) return HR_ERR_INVALID_ARG;
    DeviceGuard dg(c->device);
    uint64_t w[8];
    int rc;
    if ((rc = read_counters(c, w, reset))) return (hr_status)rc;
    out[0] = w[0] + w[4];
    out[1] = w[2] + w[5];
    out[2] = w[3] + w[6];
    out[3] = c->launches;
    out[4] = w[4];
    out[5] = w[5];
    out[6] = w[6];
    out[7] = 0;
    return HR_OK;
}

int32_t hr_get_render_times(hr_ctx* c, float* ms, int32_t max_kernels) {
    if (bad(c) || !ms || !c->timing) return 0;
    DeviceGuard dg(c->device);
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return 0;
    int32_t n = c->nrender_ev > 0 ? c->nrender_ev - 1 : 0;
    if (n > max_kernels) n = max_kernels;
    for (int32_t i = 0; i < n; ++i) {
        if (cudaEventElapsedTime(&ms[i], c->rev[i], c->rev[i + 1]) != cudaSuccess) return 0;
    }
    return n;
}

hr_status hr_sync(hr_ctx* c) {
    if (bad(c)) return HR_ERR_INVALID_ARG;
    DeviceGuard dg(c->device);
    return (hr_status)cuda_check(c, cudaStreamSynchronize(c->stream), "sync");
}

float hr_bounds_diagonal(hr_ctx* c) {
    if (bad(c) || !c->built) return 0.0f;
    const GridDesc& d = c->host_desc;
    const float x = d.bmax[0] - d.bmin[0], y = d.bmax[1] - d.bmin[1], z = d.bmax[2] - d.bmin[2];
    return sqrtf(x * x + y * y + z * z);
}

hr_status hr_exclusive_scan_device(hr_ctx* c, uint32_t* data, uint32_t n) {
    if (bad(c) || (n && !data)) return HR_ERR_INVALID_ARG;
    if (n == 0) return HR_OK;
    DeviceGuard dg(c->device);
    int rc;
    if ((rc = ensure(c, c->g.scan_partials, sizeof(uint2) * (scan_partials_words(n) + 2)))) return (hr_status)rc;
    uint32_t* cnt = c->g.scan_partials.as<uint32_t>();
    uint32_t* parts = cnt + 2;
    if ((rc = cuda_check(c, cudaMemcpyAsync(cnt, &n, 4, cudaMemcpyHostToDevice, c->stream), "scan count"))) return (hr_status)rc;
    if ((rc = exclusive_scan_u32(c, data, cnt, n, cnt + 1, parts, c->stream))) return (hr_status)rc;
    return (hr_status)cuda_check(c, cudaStreamSynchronize(c->stream), "exclusive_scan");
}

hr_status hr_radix_sort_pairs_device(hr_ctx* c, uint32_t* keys, uint32_t* vals, uint32_t n, int32_t key_bits) {
    if (bad(c) || (n && (!keys || !vals)) || key_bits < 1 || key_bits > 32) return HR_ERR_INVALID_ARG;
    if (n == 0) return HR_OK;
    DeviceGuard dg(c->device);
    int rc;
    GridBuffers& B = c->g;
    if ((rc = ensure(c, B.keys_b, (size_t)n * 4)) || (rc = ensure(c, B.vals_b, (size_t)n * 4)) ||
        (rc = ensure(c, B.tile_hist, 4 * radix_tile_hist_words(n, key_bits))) || (rc = ensure(c, B.row_total, 4 * kRadixRowWords)) ||
        (rc = ensure(c, B.scan_partials, 64)))
        return (hr_status)rc;
    uint32_t* cnt = B.scan_partials.as<uint32_t>();
    if ((rc = cuda_check(c, cudaMemcpyAsync(cnt, &n, 4, cudaMemcpyHostToDevice, c->stream), "sort count"))) return (hr_status)rc;
    const int passes = radix_sort_passes(key_bits);
    // the final pass lands in (keys, vals): odd pass counts go through the scratch pair first
    if (passes % 2 == 1) {
        if ((rc = cuda_check(c, cudaMemcpyAsync(B.keys_b.p, keys, (size_t)n * 4, cudaMemcpyDeviceToDevice, c->stream), "sort copy")) ||
            (rc = cuda_check(c, cudaMemcpyAsync(B.vals_b.p, vals, (size_t)n * 4, cudaMemcpyDeviceToDevice, c->stream), "sort copy")))
            return (hr_status)rc;
        // passes: b -> keys(tmp) ... ends in `keys`
        if ((rc = ensure(c, B.keys_a, (size_t)n * 4)) || (rc = ensure(c, B.vals_a, (size_t)n * 4))) return (hr_status)rc;
        rc = radix_sort_pairs(c, B.keys_b.as<uint32_t>(), B.vals_b.as<uint32_t>(), B.keys_a.as<uint32_t>(),
                              B.vals_a.as<uint32_t>(), keys, vals, cnt, n, key_bits, B.tile_hist.as<uint32_t>(), B.tile_hist.bytes,
                              B.row_total.as<uint32_t>(), c->stream);
    } else {
        rc = radix_sort_pairs(c, keys, vals, B.keys_b.as<uint32_t>(), B.vals_b.as<uint32_t>(), keys, vals, cnt, n,
                              key_bits, B.tile_hist.as<uint32_t>(), B.tile_hist.bytes, B.row_total.as<uint32_t>(), c->stream);
    }
    if (rc) return (hr_status)rc;
    return (hr_status)cuda_check(c, cudaStreamSynchronize(c->stream), "radix_sort");
}

}  // extern "C"
