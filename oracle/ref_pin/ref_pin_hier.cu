// ref_pin_hier.cu -- runs the reference's OWN instanced two-level grid hierarchy
// (javorkk/happyray: TLGridHierarchyMemoryManager, TLGridHierarchySortBuilder,
// TLGridHierarchyTraverser, compiled in place from its sources by oracle/ref_pin/Makefile)
// on small inputs, so that the CPU oracle's restatement can be checked against the
// reference itself.  Test infrastructure only: the product library never links or calls it.
//
// The host side sets the memory manager up as RTEngine::upload does in its
// TLGRIDHIERARCHY branch (RTEngine.cu:261-352: per-object grid bounds and resolution,
// instance table) and then calls the reference's builder (TLGridHierarchySortBuilder::init
// and build, as RTEngine::buildAccStruct, RTEngine.cu:356-358).  One input differs, on
// purpose: the instance grid's bounds are the union of the instance boxes padded by
// 0.001 x |diagonal| (the bounds the library and the oracle use), where RTEngine takes the
// uploaded vertices' bounds -- so that the two structures can be compared cell by cell.
// Rays are traced by TLGridHierarchyTraverser with the reciprocal direction in shared
// memory, as the reference's trace kernel keeps it (RayTracingKernels.h:109-127).
//
// Input (little-endian): "HRH1", nv, nt, nobj, ninst, nrays (u32); top and object
// densities (f32); nv x 3 f32 vertices; nt x 3 u32 indices; nobj u32 triangle counts;
// ninst x (u32 object, 12 f32 rows m_row_0..2, 3 f32 box min, 3 f32 box max);
// nrays x 6 f32 (origin, direction).
// Output: per object res (3 i32), box (6 f32), cell size (3 f32), cell size rcp (3 f32),
// first cell (u32); object cells (count, 2 u32 each); triangle lists (count, u32 each);
// instance grid res (3 i32), box (6 f32), cell size, rcp (3 f32 each); cells (count, 2 u32
// each); instance lists (count, u32 each); nrays x (instance u32, triangle u32, t f32).
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "CUDAStdAfx.h"
#undef ANY
#undef ALL
#define ANY(p) __any_sync(0xffffffffu, (p))
#define ALL(p) __all_sync(0xffffffffu, (p))
#include "Core/Algebra.hpp"
#include "RT/Primitive/Triangle.hpp"
#include "RT/Primitive/BBox.hpp"
#include "RT/Structure/PrimitiveArray.h"
#include "RT/Structure/TwoLevelGridHierarchy.h"
#include "RT/Structure/TLGridHierarchyMemoryManager.h"
#include "RT/Algorithm/TLGridHierarchySortBuilder.h"
#include "RT/Algorithm/RayTriangleIntersector.h"
#include "RT/Algorithm/TLGridHierarchyTraverser.h"

#define CK(x)                                                                                   \
    do {                                                                                        \
        cudaError_t e_ = (x);                                                                   \
        if (e_ != cudaSuccess) {                                                                \
            std::fprintf(stderr, "%s:%d %s: %s\n", __FILE__, __LINE__, #x, cudaGetErrorString(e_)); \
            std::exit(2);                                                                       \
        }                                                                                       \
    } while (0)

namespace {

struct Inst {
    uint32_t obj;
    float m[12], lo[3], hi[3];
};

struct Input {
    uint32_t nv = 0, nt = 0, nobj = 0, ninst = 0, nrays = 0;
    float top = 0.f, leaf = 0.f;
    std::vector<float> v, rays;
    std::vector<uint32_t> idx, counts;
    std::vector<Inst> inst;
};

bool read_input(const char* path, Input& in) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return false;
    char magic[4];
    bool ok = std::fread(magic, 1, 4, f) == 4 && std::memcmp(magic, "HRH1", 4) == 0;
    uint32_t h[5];
    float d[2];
    ok = ok && std::fread(h, 4, 5, f) == 5 && std::fread(d, 4, 2, f) == 2;
    if (ok) {
        in.nv = h[0]; in.nt = h[1]; in.nobj = h[2]; in.ninst = h[3]; in.nrays = h[4];
        in.top = d[0]; in.leaf = d[1];
        in.v.resize((size_t)in.nv * 3);
        in.idx.resize((size_t)in.nt * 3);
        in.counts.resize(in.nobj);
        in.inst.resize(in.ninst);
        in.rays.resize((size_t)in.nrays * 6);
        ok = std::fread(in.v.data(), 4, in.v.size(), f) == in.v.size() &&
             std::fread(in.idx.data(), 4, in.idx.size(), f) == in.idx.size() &&
             std::fread(in.counts.data(), 4, in.counts.size(), f) == in.counts.size() &&
             std::fread(in.inst.data(), sizeof(Inst), in.inst.size(), f) == in.inst.size() &&
             std::fread(in.rays.data(), 4, in.rays.size(), f) == in.rays.size();
    }
    std::fclose(f);
    return ok;
}

std::vector<uint32_t> read_pitched(const cudaPitchedPtr& p, int rx, int ry, int rz) {
    std::vector<uint32_t> out((size_t)rx * ry * rz * 2);
    cudaMemcpy3DParms m = {};
    m.srcPtr = p;
    m.dstPtr = make_cudaPitchedPtr(out.data(), (size_t)rx * sizeof(uint2), (size_t)rx, (size_t)ry);
    m.extent = make_cudaExtent((size_t)rx * sizeof(uint2), (size_t)ry, (size_t)rz);
    m.kind = cudaMemcpyDeviceToHost;
    CK(cudaMemcpy3D(&m));
    return out;
}

__global__ void k_trace(PrimitiveArray<Triangle> pa, TwoLevelGridHierarchy grid, const float* rays, uint n,
                        uint* oinst, uint* otri, float* ot) {
    extern __shared__ uint smem[];
    const uint i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < n;
    float3& rcp = ((float3*)smem)[threadId1D32()];
    float3 org = make_float3(0.f, 0.f, 0.f);
    rcp = make_float3(1.f, 1.f, 1.f);
    if (valid) {
        org = make_float3(rays[6 * i], rays[6 * i + 1], rays[6 * i + 2]);
        rcp = make_float3(1.f / rays[6 * i + 3], 1.f / rays[6 * i + 4], 1.f / rays[6 * i + 5]);
    }
    float rayT = FLT_MAX;
    uint bestHit = (uint)pa.numPrimitives;
    TLGridHierarchyTraverser<Triangle, MollerTrumboreIntersectionTest, false> traverse;
    traverse(pa, grid, org, rcp, rayT, bestHit, valid, smem);
    if (valid) {
        const bool hit = rayT < FLT_MAX;
        otri[i] = hit ? grid.primitives[bestHit] : 0xffffffffu;
        oinst[i] = hit ? traverse.getBestHitInstance() : 0xffffffffu;
        ot[i] = rayT;
    }
}

void write_all(FILE* f, const void* p, size_t bytes) {
    if (bytes && std::fwrite(p, 1, bytes, f) != bytes) { std::perror("write"); std::exit(3); }
}

}  // namespace

int main(int argc, char** argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: %s input.bin output.bin\n", argv[0]);
        return 1;
    }
    Input in;
    if (!read_input(argv[1], in)) {
        std::fprintf(stderr, "cannot read %s\n", argv[1]);
        return 1;
    }
    std::vector<float4> v4(in.nv);
    for (uint32_t i = 0; i < in.nv; ++i) v4[i] = make_float4(in.v[3 * i], in.v[3 * i + 1], in.v[3 * i + 2], 0.f);
    PrimitiveArray<Triangle> pa;
    CK(cudaMalloc(&pa.vertexBufferDevicePtr, v4.size() * sizeof(float4)));
    CK(cudaMalloc(&pa.indicesBufferDevicePtr, in.idx.size() * 4));
    CK(cudaMemcpy(pa.vertexBufferDevicePtr, v4.data(), v4.size() * sizeof(float4), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(pa.indicesBufferDevicePtr, in.idx.data(), in.idx.size() * 4, cudaMemcpyHostToDevice));
    pa.numPrimitives = in.nt;

    TLGridHierarchyMemoryManager mm;
    // instance-grid bounds: the union of the instance boxes, padded as WFObjectUploader.h:112-114
    float3 lo = make_float3(FLT_MAX, FLT_MAX, FLT_MAX), hi = make_float3(-FLT_MAX, -FLT_MAX, -FLT_MAX);
    for (const Inst& I : in.inst) {
        lo = make_float3(fminf(lo.x, I.lo[0]), fminf(lo.y, I.lo[1]), fminf(lo.z, I.lo[2]));
        hi = make_float3(fmaxf(hi.x, I.hi[0]), fmaxf(hi.y, I.hi[1]), fmaxf(hi.z, I.hi[2]));
    }
    const float3 dd = make_float3(hi.x - lo.x, hi.y - lo.y, hi.z - lo.z);
    const float pad = 0.001f * sqrtf(dd.x * dd.x + dd.y * dd.y + dd.z * dd.z);
    mm.bounds.vtx[0] = make_float3(lo.x - pad, lo.y - pad, lo.z - pad);
    mm.bounds.vtx[1] = make_float3(hi.x + pad, hi.y + pad, hi.z + pad);

    // per-object grids, RTEngine.cu:267-330
    mm.allocateGrids(in.nobj);
    uint32_t begin = 0;
    for (uint32_t k = 0; k < in.nobj; ++k) {
        mm.primitiveCounts[k] = in.counts[k];
        float3 mn = make_float3(FLT_MAX, FLT_MAX, FLT_MAX), mx = make_float3(-FLT_MAX, -FLT_MAX, -FLT_MAX);
        for (uint32_t t = begin; t < begin + in.counts[k]; ++t)
            for (int c = 0; c < 3; ++c) {
                const float* p = &in.v[3 * (size_t)in.idx[3 * (size_t)t + c]];
                mn = make_float3(fminf(mn.x, p[0]), fminf(mn.y, p[1]), fminf(mn.z, p[2]));
                mx = make_float3(fmaxf(mx.x, p[0]), fmaxf(mx.y, p[1]), fmaxf(mx.z, p[2]));
            }
        begin += in.counts[k];
        UniformGrid& g = mm.gridsHost[k];
        g.vtx[0] = make_float3(mn.x - 10.f * EPS, mn.y - 10.f * EPS, mn.z - 10.f * EPS);
        g.vtx[1] = make_float3(mx.x + 10.f * EPS, mx.y + 10.f * EPS, mx.z + 10.f * EPS);
        const float3 diag = g.vtx[1] - g.vtx[0];
        const float volume = diag.x * diag.y * diag.z;
        const float magic = powf(in.leaf * static_cast<float>(in.counts[k]) / volume, 0.3333333f);
        const float3 r = diag * magic;
        g.res[0] = (int)r.x > 0 ? (int)r.x : 1;
        g.res[1] = (int)r.y > 0 ? (int)r.y : 1;
        g.res[2] = (int)r.z > 0 ? (int)r.z : 1;
        const float3 rf = make_float3((float)g.res[0], (float)g.res[1], (float)g.res[2]);
        g.setCellSize(diag / rf);
        g.setCellSizeRCP(rf / diag);
    }
    mm.copyGridsHostToDevice();
    // instances, RTEngine.cu:333-349
    mm.allocateDeviceInstances(in.ninst);
    mm.allocateHostInstances(in.ninst);
    for (uint32_t i = 0; i < in.ninst; ++i) {
        const Inst& I = in.inst[i];
        mm.instancesHost[i].setIndex(I.obj);
        mm.instancesHost[i].setTransformation(I.m[0], I.m[1], I.m[2], I.m[3], I.m[4], I.m[5], I.m[6], I.m[7], I.m[8],
                                              I.m[9], I.m[10], I.m[11]);
        mm.instancesHost[i].vtx[0] = make_float3(I.lo[0], I.lo[1], I.lo[2]);
        mm.instancesHost[i].vtx[1] = make_float3(I.hi[0], I.hi[1], I.hi[2]);
    }
    mm.copyInstancesHostToDevice();

    TLGridHierarchySortBuilder builder;
    builder.init(mm, in.ninst, in.top, in.leaf);
    builder.build(mm, in.nobj, mm.primitiveCounts, pa);
    CK(cudaDeviceSynchronize());
    mm.copyGridsDeviceToHost();

    // traversal
    const size_t nr = in.nrays;
    float* drays;
    uint *dinst, *dtri;
    float* dt;
    CK(cudaMalloc(&drays, (nr + 1) * 24));
    CK(cudaMalloc(&dinst, (nr + 1) * 4));
    CK(cudaMalloc(&dtri, (nr + 1) * 4));
    CK(cudaMalloc(&dt, (nr + 1) * 4));
    if (nr) CK(cudaMemcpy(drays, in.rays.data(), nr * 24, cudaMemcpyHostToDevice));
    TwoLevelGridHierarchy grid = mm.getParameters();
    const uint tb = 128, gb = (uint)((nr + tb - 1) / tb);
    if (nr) k_trace<<<gb, tb, tb * sizeof(float3)>>>(pa, grid, drays, (uint)nr, dinst, dtri, dt);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());

    const size_t nleaves = mm.leavesSize / sizeof(uint2), nprims = mm.primitiveIndicesSize / 4,
                 ninstidx = mm.instanceIndicesSize / 4;
    std::vector<uint32_t> leaves(2 * nleaves), prims(nprims), instidx(ninstidx), hinst(nr), htri(nr);
    std::vector<float> ht(nr);
    if (nleaves) CK(cudaMemcpy(leaves.data(), mm.leavesDevice, nleaves * 8, cudaMemcpyDeviceToHost));
    if (nprims) CK(cudaMemcpy(prims.data(), mm.primitiveIndices, nprims * 4, cudaMemcpyDeviceToHost));
    if (ninstidx) CK(cudaMemcpy(instidx.data(), mm.instanceIndicesDevice, ninstidx * 4, cudaMemcpyDeviceToHost));
    if (nr) {
        CK(cudaMemcpy(hinst.data(), dinst, nr * 4, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(htri.data(), dtri, nr * 4, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(ht.data(), dt, nr * 4, cudaMemcpyDeviceToHost));
    }
    std::vector<uint32_t> topcells = read_pitched(mm.cellsPtrDevice, mm.resX, mm.resY, mm.resZ);

    FILE* f = std::fopen(argv[2], "wb");
    if (!f) { std::perror(argv[2]); return 3; }
    for (uint32_t k = 0; k < in.nobj; ++k) {
        const UniformGrid& g = mm.gridsHost[k];
        write_all(f, g.res, 12);
        const float3 cs = g.getCellSize(), rcp = g.getCellSizeRCP();
        const float geo[12] = {g.vtx[0].x, g.vtx[0].y, g.vtx[0].z, g.vtx[1].x, g.vtx[1].y, g.vtx[1].z,
                               cs.x, cs.y, cs.z, rcp.x, rcp.y, rcp.z};
        write_all(f, geo, 48);
        const uint32_t first = (uint32_t)((uint2*)g.cells.ptr - (uint2*)mm.leavesDevice);
        write_all(f, &first, 4);
    }
    const uint32_t nl = (uint32_t)nleaves, np = (uint32_t)nprims, ni = (uint32_t)ninstidx;
    write_all(f, &nl, 4);
    write_all(f, leaves.data(), leaves.size() * 4);
    write_all(f, &np, 4);
    write_all(f, prims.data(), prims.size() * 4);
    const int tres[3] = {mm.resX, mm.resY, mm.resZ};
    write_all(f, tres, 12);
    const float3 tcs = mm.getCellSize(), trcp = mm.getCellSizeRCP();
    const float tgeo[12] = {mm.bounds.vtx[0].x, mm.bounds.vtx[0].y, mm.bounds.vtx[0].z, mm.bounds.vtx[1].x,
                            mm.bounds.vtx[1].y, mm.bounds.vtx[1].z, tcs.x, tcs.y, tcs.z, trcp.x, trcp.y, trcp.z};
    write_all(f, tgeo, 48);
    const uint32_t ntc = (uint32_t)(topcells.size() / 2);
    write_all(f, &ntc, 4);
    write_all(f, topcells.data(), topcells.size() * 4);
    write_all(f, &ni, 4);
    write_all(f, instidx.data(), instidx.size() * 4);
    for (size_t i = 0; i < nr; ++i) {
        write_all(f, &hinst[i], 4);
        write_all(f, &htri[i], 4);
        write_all(f, &ht[i], 4);
    }
    std::fclose(f);
    std::printf("ok objects %u object cells %zu pairs %zu instance grid %d %d %d lists %zu rays %zu\n", in.nobj,
                nleaves, nprims, mm.resX, mm.resY, mm.resZ, ninstidx, nr);
    return 0;
}
