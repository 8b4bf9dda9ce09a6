// harness.cu -- drives the RTEngine adapter (RTEngine.cu) the way the reference's
// CUDAApplication drives RTEngine (CUDAApplication.cu:63-71, 78-114, 116-160): the scene goes
// in as WFObject key frames, the lights as an AreaLightSourceCollection, frames come back
// through FrameBuffer -- all the reference's own classes.  Test infrastructure: the tests
// run it and compare its frames with the library's own calls on the same inputs.
//
// Input (little-endian): "HRA1"; nv, nt (u32); coeff, top density, leaf density (f32);
// camera position, orientation, up (3 f32 each), fov (f32), resX, resY (i32); nlights
// (u32); ray-file path length (u32) and bytes; frame 1 and frame 2 vertices (nv x 3 f32
// each); faces (nt x 3 u32); per light position, edge1, edge2, normal, intensity (3 f32
// each).
// Output: diagonal (f32); mode-0 frame after images 0..5; AO frame (mode 3, image 0); path
// traced frame (mode 1, image 0); with a ray file, the ray-file frame (mode 0) -- each
// resX x resY x 3 f32.
#include "RT/RTEngine.h"

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace {

bool rd(FILE* f, void* p, size_t n) { return std::fread(p, 1, n, f) == n; }

template <class T> bool rd_vec(FILE* f, std::vector<T>& v, size_t n) {
    v.resize(n);
    return n == 0 || rd(f, v.data(), sizeof(T) * n);
}

void put_frame(FILE* out, FrameBuffer& fb) {
    std::vector<float3> h(fb.resX * fb.resY);
    fb.download(h.data());
    std::fwrite(h.data(), sizeof(float3), h.size(), out);
}

}  // namespace

int main(int argc, char** argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: %s input output\n", argv[0]);
        return 2;
    }
    FILE* in = std::fopen(argv[1], "rb");
    if (!in) return 2;
    char magic[4];
    uint32_t nv = 0, nt = 0, nl = 0, plen = 0;
    float coeff = 1.0f, top = 0.0f, leaf = 0.0f, fov = 60.0f;
    float cam[9];
    int32_t res[2];
    bool ok = rd(in, magic, 4) && std::memcmp(magic, "HRA1", 4) == 0 && rd(in, &nv, 4) && rd(in, &nt, 4) &&
              rd(in, &coeff, 4) && rd(in, &top, 4) && rd(in, &leaf, 4) && rd(in, cam, 36) && rd(in, &fov, 4) &&
              rd(in, res, 8) && rd(in, &nl, 4) && rd(in, &plen, 4);
    std::string ray_file(plen, '\0');
    std::vector<float> v1, v2, lights;
    std::vector<uint32_t> faces;
    ok = ok && (plen == 0 || rd(in, &ray_file[0], plen)) && rd_vec(in, v1, 3 * (size_t)nv) &&
         rd_vec(in, v2, 3 * (size_t)nv) && rd_vec(in, faces, 3 * (size_t)nt) && rd_vec(in, lights, 15 * (size_t)nl);
    std::fclose(in);
    if (!ok) {
        std::fprintf(stderr, "bad input\n");
        return 2;
    }
    WFObject f1, f2;
    for (uint32_t i = 0; i < nv; ++i) {
        f1.insertVertex(make_float3(v1[3 * i], v1[3 * i + 1], v1[3 * i + 2]));
        f2.insertVertex(make_float3(v2[3 * i], v2[3 * i + 1], v2[3 * i + 2]));
    }
    for (uint32_t i = 0; i < nt; ++i) {
        WFObject::Face fa(&f2);
        fa.material = 0;
        fa.vert1 = faces[3 * i]; fa.vert2 = faces[3 * i + 1]; fa.vert3 = faces[3 * i + 2];
        fa.tex1 = fa.tex2 = fa.tex3 = 0;
        fa.norm1 = fa.norm2 = fa.norm3 = 0;
        f1.insertFace(fa);
        f2.insertFace(fa);
    }
    AreaLightSourceCollection collection;
    for (uint32_t k = 0; k < nl; ++k) {
        const float* L = &lights[15 * (size_t)k];
        AreaLightSource ls;
        ls.position = make_float3(L[0], L[1], L[2]);
        ls.edge1 = make_float3(L[3], L[4], L[5]);
        ls.edge2 = make_float3(L[6], L[7], L[8]);
        ls.normal = make_float3(L[9], L[10], L[11]);
        ls.intensity = make_float3(L[12], L[13], L[14]);
        collection.upload(ls.getArea() * len(ls.intensity), ls);   // as SceneLoader.cpp:288
    }

    RTEngine::init();
    RTEngine::upload(f1, f2, coeff);
    RTEngine::setGridDensities(top, leaf);
    RTEngine::buildAccStruct();
    RTEngine::setCamera(make_float3(cam[0], cam[1], cam[2]), make_float3(cam[3], cam[4], cam[5]),
                        make_float3(cam[6], cam[7], cam[8]), fov, res[0], res[1]);
    if (nl) RTEngine::setLights(collection);
    FILE* out = std::fopen(argv[2], "wb");
    if (!out) return 2;
    const float diag = RTEngine::getBoundingBoxDiagonalLength();
    std::fwrite(&diag, 4, 1, out);
    FrameBuffer fb;
    fb.init((uint)res[0], (uint)res[1]);
    for (int im = 0; im < 6; ++im) RTEngine::renderFrame(fb, im, 0);
    put_frame(out, fb);
    fb.setZero();
    RTEngine::renderFrame(fb, 0, 3);
    put_frame(out, fb);
    fb.setZero();
    RTEngine::renderFrame(fb, 0, 1);
    put_frame(out, fb);
    if (plen) {
        fb.setZero();
        RTEngine::setInputRayFileName(ray_file);
        RTEngine::renderFrame(fb, 0, 0);
        put_frame(out, fb);
    }
    std::fclose(out);
    fb.cleanup();
    collection.cleanup();
    RTEngine::cleanup();
    return 0;
}
