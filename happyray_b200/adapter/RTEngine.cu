// RTEngine.cu -- the reference engine facade (RTEngine, src/RT/RTEngine.h:36-68) implemented
// on libhappyray_b200.  It is built in place of the reference's src/RT/RTEngine.cu: compile it
// with the reference's src/ and this repository's include/ on the include path and link
// -lhappyray_b200; CUDAApplication and the rest of the application keep calling RTEngine
// unchanged.  happyray_b200/adapter/Makefile compiles it against the reference's own headers.
//
// Every method of RTEngine.h maps to the C-ABI (include/happyray.h):
//   init                      hr_create on device 0, the reference's grid densities
//                             (RTEngine.cu:76-77: 1.2 top, 2.2 leaf) and AO settings
//                             (4 samples, radius 0.05 x bounds diagonal: AOIntegrator.h:45,
//                             RTEngine.cu:259)
//   upload(f1, f2, coeff)     hr_upload of both frames' vertices and frame 2's faces
//                             (ObjUploader, WFObjectUploader.h:48-119)
//   buildAccStruct            hr_build (two-level grid, as the reference's TLGRID build;
//                             define HAPPYRAY_UNIFORM_GRID for its uniform-grid build)
//   setCamera                 hr_set_camera
//   setLights(collection)     hr_set_lights with every light of the collection
//   renderFrame(fb, id, mode) hr_render_device into fb.deviceData, or, after
//                             setInputRayFileName, the file's rays shaded by
//                             hr_render_rays_device (mode 0, RTEngine.cu:410-414)
//   setGridDensities          hr_set_grid_densities
//   getBoundingBoxDiagonalLength  hr_bounds_diagonal
//   setInputRayFileName       hr_rays_file_count / hr_rays_file_read, rays kept on the device
//   cleanup                   hr_destroy
// A failing call is reported and ends the process, as the reference's MY_CUDA_SAFE_CALL
// does (CUDAUtil.h:199-206).
#include "RT/RTEngine.h"
#include "happyray.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace {

hr_ctx* gCtx = nullptr;
float* gRays = nullptr;        // device: origins then directions of the ray file
uint32_t gNumRays = 0;
bool gUseInputRays = false;

void check(hr_status st, const char* what) {
    if (st == HR_OK) return;
    std::fprintf(stderr, "RTEngine (happyray): %s failed (status %d): %s\n", what, (int)st,
                 gCtx ? hr_last_error(gCtx) : hr_io_last_error());
    std::exit(1);
}

void checkCuda(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return;
    std::fprintf(stderr, "RTEngine (happyray): %s failed: %s\n", what, cudaGetErrorString(e));
    std::exit(1);
}

// AreaLightSourceCollection keeps its size and device arrays private
// (LightSource.hpp:102-108); its layout is read through this mirror of the same members.
struct CollectionView {
    int size;
    float* cdf;
    float* weights;
    AreaLightSource* lights;
};
static_assert(sizeof(CollectionView) == sizeof(AreaLightSourceCollection),
              "AreaLightSourceCollection layout changed");

}  // namespace

void RTEngine::init() {
    check(hr_create(&gCtx, 0, nullptr), "hr_create");
    check(hr_set_grid_densities(gCtx, 1.2f, 2.2f), "hr_set_grid_densities");
    check(hr_set_integrator(gCtx, 4, -0.05f, 4, 0.7f, 0x853c49e6748fea9bULL), "hr_set_integrator");
}

void RTEngine::upload(const WFObject& aFrame1, const WFObject& aFrame2, const float aCoeff) {
    const size_t nv = aFrame2.getNumVertices(), nt = aFrame2.getNumFaces();
    if (aFrame1.getNumVertices() != nv) check(HR_ERR_INVALID_ARG, "upload: key frames differ in vertex count");
    std::vector<float> a(3 * nv), b(3 * nv);
    for (size_t i = 0; i < nv; ++i) {
        const float3 p = aFrame1.getVertex(i), q = aFrame2.getVertex(i);
        a[3 * i] = p.x; a[3 * i + 1] = p.y; a[3 * i + 2] = p.z;
        b[3 * i] = q.x; b[3 * i + 1] = q.y; b[3 * i + 2] = q.z;
    }
    std::vector<uint32_t> idx(3 * nt);
    for (size_t i = 0; i < nt; ++i) {
        const WFObject::Face f = aFrame2.getFace(i);
        idx[3 * i] = (uint32_t)f.vert1;
        idx[3 * i + 1] = (uint32_t)f.vert2;
        idx[3 * i + 2] = (uint32_t)f.vert3;
    }
    check(hr_upload(gCtx, a.data(), b.data(), (uint32_t)nv, idx.data(), (uint32_t)nt, aCoeff), "hr_upload");
}

void RTEngine::buildAccStruct() {
#ifdef HAPPYRAY_UNIFORM_GRID
    check(hr_build(gCtx, HR_GRID_UNIFORM, 1), "hr_build");
#else
    check(hr_build(gCtx, HR_GRID_TWO_LEVEL, 1), "hr_build");
#endif
}

void RTEngine::setCamera(const float3& aPosition, const float3& aOrientation, const float3& aUp, const float aFOV,
                         const int aX, const int aY) {
    const float p[3] = {aPosition.x, aPosition.y, aPosition.z};
    const float o[3] = {aOrientation.x, aOrientation.y, aOrientation.z};
    const float u[3] = {aUp.x, aUp.y, aUp.z};
    check(hr_set_camera(gCtx, p, o, u, aFOV, aX, aY), "hr_set_camera");
}

void RTEngine::setLights(const AreaLightSourceCollection& aLights) {
    CollectionView v;
    std::memcpy(&v, &aLights, sizeof(v));
    if (v.size <= 0) return;
    std::vector<AreaLightSource> ls((size_t)v.size);
    checkCuda(cudaMemcpy(ls.data(), v.lights, sizeof(AreaLightSource) * ls.size(), cudaMemcpyDeviceToHost),
              "light collection download");
    const size_t n = ls.size() < 64 ? ls.size() : 64;
    std::vector<float> c(3 * n), e1(3 * n), e2(3 * n), nrm(3 * n), em(n);
    for (size_t k = 0; k < n; ++k) {
        const AreaLightSource& L = ls[k];
        c[3 * k] = L.position.x; c[3 * k + 1] = L.position.y; c[3 * k + 2] = L.position.z;
        e1[3 * k] = L.edge1.x; e1[3 * k + 1] = L.edge1.y; e1[3 * k + 2] = L.edge1.z;
        e2[3 * k] = L.edge2.x; e2[3 * k + 1] = L.edge2.y; e2[3 * k + 2] = L.edge2.z;
        nrm[3 * k] = L.normal.x; nrm[3 * k + 1] = L.normal.y; nrm[3 * k + 2] = L.normal.z;
        em[k] = (L.intensity.x + L.intensity.y + L.intensity.z) / 3.0f;   // scalar radiance
    }
    check(hr_set_lights(gCtx, (uint32_t)n, c.data(), e1.data(), e2.data(), nrm.data(), em.data()), "hr_set_lights");
}

void RTEngine::renderFrame(FrameBuffer& aFrameBuffer, const int aImageId, const int aRenderMode) {
    float* fb = reinterpret_cast<float*>(aFrameBuffer.deviceData);
    if (aRenderMode == 0 && gUseInputRays) {
        const uint32_t n = gNumRays < aFrameBuffer.resX * aFrameBuffer.resY ? gNumRays
                                                                            : aFrameBuffer.resX * aFrameBuffer.resY;
        check(hr_render_rays_device(gCtx, gRays, gRays + 3 * (size_t)gNumRays, n, 0, fb), "hr_render_rays_device");
    } else {
        check(hr_render_device(gCtx, aRenderMode, aImageId, fb), "hr_render_device");
    }
    check(hr_sync(gCtx), "hr_sync");
}

void RTEngine::setGridDensities(float aTopLvl, float aLeafLvl) {
    check(hr_set_grid_densities(gCtx, aTopLvl, aLeafLvl), "hr_set_grid_densities");
}

void RTEngine::cleanup() {
    if (gRays) cudaFree(gRays);
    gRays = nullptr;
    gNumRays = 0;
    gUseInputRays = false;
    hr_destroy(gCtx);
    gCtx = nullptr;
}

float RTEngine::getBoundingBoxDiagonalLength() { return hr_bounds_diagonal(gCtx); }

// The reference's ray loader reads the whole file at the first frame (SimpleRayTraverser.h:
// 200-261); here it is read once, now, and kept on the device in the library's layout.
void RTEngine::setInputRayFileName(const std::string& aFileName) {
    uint32_t n = 0;
    check(hr_rays_file_count(aFileName.c_str(), &n), "hr_rays_file_count");
    std::vector<float> od(6 * (size_t)n);
    if (n) check(hr_rays_file_read(aFileName.c_str(), od.data(), n), "hr_rays_file_read");
    std::vector<float> soa(6 * (size_t)n);   // origins, then directions
    for (size_t i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) {
            soa[3 * i + k] = od[6 * i + k];
            soa[3 * (size_t)n + 3 * i + k] = od[6 * i + 3 + k];
        }
    if (gRays) cudaFree(gRays);
    gRays = nullptr;
    if (n) {
        checkCuda(cudaMalloc((void**)&gRays, sizeof(float) * soa.size()), "ray buffer");
        checkCuda(cudaMemcpy(gRays, soa.data(), sizeof(float) * soa.size(), cudaMemcpyHostToDevice), "ray upload");
    }
    gNumRays = n;
    gUseInputRays = true;
}
