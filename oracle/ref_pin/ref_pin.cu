// ref_pin.cu -- runs the reference's OWN grid-build kernels and grid traversers
// (javorkk/happyray, compiled in place from its sources by oracle/ref_pin/Makefile) on
// small inputs, so that the CPU oracle can be checked against the reference itself.
// Test infrastructure only: the product library never links or calls it.
//
// The host side below is this harness's own orchestration of the reference kernels, in
// the order the reference's builders launch them:
//   uniform grid    UGridSortBuilder.h:64-99 (resolution), 122-345 (countPairs, scan,
//                   writeKeysAndValues, sort by key, prepareCellRanges)
//   two-level grid  TLGridSortBuilder.h:66-105, 130-420 (top level as above, then
//                   countLeafLevelCells, scan, prepareTopLevelCellRanges,
//                   countLeafLevelPairs, scan, writeLeafLevelKeysAndValues, sort,
//                   prepareLeafCellRanges)
//   bounds          WFObjectUploader.h:82-114 (min / max of the vertices, padded by
//                   0.001 x |diagonal|)
//   rays            RayTracingKernels.h:103-149 (reciprocal direction, traverse,
//                   primitives[bestHit])
// The exclusive scans run on the host (the reference reads their totals from mapped
// host memory, MemoryManager.h:38-61); the pair sorts use thrust::sort_by_key as the
// reference does without CUB_SORT.
//
// Input (little-endian): "HRP1", kind (0 uniform, 1 two-level), exact, nv, nt, nrays,
// density (uniform or top), leaf density; nv x 3 f32 vertices; nt x 3 u32 indices;
// nrays x 6 f32 (origin, direction).
// Output: res i32 x 3; bmin, bmax, cell size, cell size rcp (f32 x 3 each); ncells, cells
// (2 u32 each; two-level: packed top cells); nleaves, leaves (2 u32 each); nprims, prims;
// nrays x (u32 hit id or 0xffffffff, f32 t).
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include <thrust/device_ptr.h>
#include <thrust/sort.h>

#include "CUDAStdAfx.h"
// The reference's warp votes are the pre-Volta __any / __all (CUDAStdAfx.h:76-82), which
// sm_70+ no longer assembles.  Every vote the harness reaches is executed by all 32 lanes
// of the warp (k_trace runs one ray per lane with whole warps), so the full-mask _sync
// forms are equivalent there.
#undef ANY
#undef ALL
#define ANY(p) __any_sync(0xffffffffu, (p))
#define ALL(p) __all_sync(0xffffffffu, (p))
#include "Core/Algebra.hpp"
#include "RT/Primitive/Triangle.hpp"
#include "RT/Primitive/BBox.hpp"
#include "RT/Structure/PrimitiveArray.h"
#include "RT/Structure/UniformGrid.h"
#include "RT/Structure/TwoLevelGrid.h"
#include "RT/Algorithm/UniformGridBuildKernels.h"
#include "RT/Algorithm/TLGridBuildKernels.h"
#include "RT/Algorithm/RayTriangleIntersector.h"
#include "RT/Algorithm/UGridTraverser.h"
#include "RT/Algorithm/TLGridTraverser.h"

#define CK(x)                                                                                   \
    do {                                                                                        \
        cudaError_t e_ = (x);                                                                   \
        if (e_ != cudaSuccess) {                                                                \
            std::fprintf(stderr, "%s:%d %s: %s\n", __FILE__, __LINE__, #x, cudaGetErrorString(e_)); \
            std::exit(2);                                                                       \
        }                                                                                       \
    } while (0)

namespace {

constexpr size_t kPad = 1024;   // spare elements after every array the reference kernels index

struct Input {
    uint32_t kind = 0, exact = 0, nv = 0, nt = 0, nrays = 0;
    float dens = 0.f, leaf = 0.f;
    std::vector<float> v;
    std::vector<uint32_t> idx;
    std::vector<float> rays;
};

bool read_input(const char* path, Input& in) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return false;
    char magic[4];
    bool ok = std::fread(magic, 1, 4, f) == 4 && std::memcmp(magic, "HRP1", 4) == 0;
    uint32_t h[5];
    ok = ok && std::fread(h, 4, 5, f) == 5;
    float d[2];
    ok = ok && std::fread(d, 4, 2, f) == 2;
    if (ok) {
        in.kind = h[0]; in.exact = h[1]; in.nv = h[2]; in.nt = h[3]; in.nrays = h[4];
        in.dens = d[0]; in.leaf = d[1];
        in.v.resize((size_t)in.nv * 3);
        in.idx.resize((size_t)in.nt * 3);
        in.rays.resize((size_t)in.nrays * 6);
        ok = std::fread(in.v.data(), 4, in.v.size(), f) == in.v.size() &&
             std::fread(in.idx.data(), 4, in.idx.size(), f) == in.idx.size() &&
             std::fread(in.rays.data(), 4, in.rays.size(), f) == in.rays.size();
    }
    std::fclose(f);
    return ok;
}

// exclusive scan of n device counters on the host; returns the total (the last entry)
uint32_t host_scan(uint32_t* d, size_t n) {
    std::vector<uint32_t> h(n);
    CK(cudaMemcpy(h.data(), d, n * 4, cudaMemcpyDeviceToHost));
    uint32_t run = 0;
    for (size_t i = 0; i < n; ++i) { const uint32_t x = h[i]; h[i] = run; run += x; }
    CK(cudaMemcpy(d, h.data(), n * 4, cudaMemcpyHostToDevice));
    return h[n - 1];
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

template <class tGrid, class tTraverser>
__global__ void k_trace(PrimitiveArray<Triangle> pa, tGrid grid, const float* rays, uint n, uint* oid, float* ot) {
    // one ray per thread; the launch covers whole warps, lanes past n pass traversalFlag = false
    const uint i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < n;
    float3 org = make_float3(0.f, 0.f, 0.f), rcp = make_float3(1.f, 1.f, 1.f);
    if (valid) {
        org = make_float3(rays[6 * i], rays[6 * i + 1], rays[6 * i + 2]);
        rcp = make_float3(1.f / rays[6 * i + 3], 1.f / rays[6 * i + 4], 1.f / rays[6 * i + 5]);
    }
    float rayT = FLT_MAX;
    uint bestHit = (uint)pa.numPrimitives;
    tTraverser traverse;
    traverse(pa, grid, org, rcp, rayT, bestHit, valid, nullptr);
    if (valid) {
        const bool hit = rayT < FLT_MAX;
        oid[i] = hit ? grid.primitives[bestHit] : 0xffffffffu;
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
    // bounds, WFObjectUploader.h:82-114
    float3 lo = make_float3(FLT_MAX, FLT_MAX, FLT_MAX), hi = make_float3(-FLT_MAX, -FLT_MAX, -FLT_MAX);
    std::vector<float4> v4(in.nv);
    for (uint32_t i = 0; i < in.nv; ++i) {
        const float x = in.v[3 * i], y = in.v[3 * i + 1], z = in.v[3 * i + 2];
        v4[i] = make_float4(x, y, z, 0.f);
        lo.x = x < lo.x ? x : lo.x; lo.y = y < lo.y ? y : lo.y; lo.z = z < lo.z ? z : lo.z;
        hi.x = x > hi.x ? x : hi.x; hi.y = y > hi.y ? y : hi.y; hi.z = z > hi.z ? z : hi.z;
    }
    const float3 dg = make_float3(hi.x - lo.x, hi.y - lo.y, hi.z - lo.z);
    const float diag = sqrtf(dg.x * dg.x + dg.y * dg.y + dg.z * dg.z);
    lo = make_float3(lo.x - 0.001f * diag, lo.y - 0.001f * diag, lo.z - 0.001f * diag);
    hi = make_float3(hi.x + 0.001f * diag, hi.y + 0.001f * diag, hi.z + 0.001f * diag);
    // resolution, UGridSortBuilder.h:78-92 / TLGridSortBuilder.h:80-92
    float3 e = make_float3(hi.x - lo.x, hi.y - lo.y, hi.z - lo.z);
    const float vol = e.x * e.y * e.z;
    const float magic = powf(in.dens * (float)in.nt / vol, 0.3333333f);
    const int res[3] = {(int)(e.x * magic), (int)(e.y * magic), (int)(e.z * magic)};
    const float3 resf = make_float3((float)res[0], (float)res[1], (float)res[2]);
    const float3 cs = make_float3(e.x / resf.x, e.y / resf.y, e.z / resf.z);
    const float3 rcp = make_float3(resf.x / e.x, resf.y / e.y, resf.z / e.z);
    const uint ncells = (uint)res[0] * (uint)res[1] * (uint)res[2];

    PrimitiveArray<Triangle> pa;
    CK(cudaMalloc(&pa.vertexBufferDevicePtr, v4.size() * sizeof(float4)));
    CK(cudaMalloc(&pa.indicesBufferDevicePtr, in.idx.size() * 4));
    CK(cudaMemcpy(pa.vertexBufferDevicePtr, v4.data(), v4.size() * sizeof(float4), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(pa.indicesBufferDevicePtr, in.idx.data(), in.idx.size() * 4, cudaMemcpyHostToDevice));
    pa.numPrimitives = in.nt;

    const bool tl = in.kind == 1;
    const uint cthreads = tl ? 512u : 128u, cblocks = tl ? 256u : 90u;
    const uint sthreads = tl ? 512u : 256u, sblocks = tl ? 256u : 90u;
    uint* counts;
    CK(cudaMalloc(&counts, (cblocks + 1) * 4));
    CK(cudaMemset(counts, 0, (cblocks + 1) * 4));
    if (tl)
        countPairs<Triangle, PrimitiveArray<Triangle>, 512><<<cblocks, cthreads, cthreads * (4 + 12)>>>(
            pa, in.nt, resf, lo, cs, rcp, counts);
    else
        countPairs<Triangle, PrimitiveArray<Triangle>, 128><<<cblocks, cthreads, cthreads * (4 + 12)>>>(
            pa, in.nt, resf, lo, cs, rcp, counts);
    CK(cudaGetLastError());
    const uint npairs = host_scan(counts, cblocks + 1);
    uint *keys, *vals, *prims;
    CK(cudaMalloc(&keys, (size_t)(npairs + kPad) * 4));
    CK(cudaMalloc(&vals, (size_t)(npairs + kPad) * 4));
    if (!tl && in.exact)
        writeKeysAndValues<Triangle, PrimitiveArray<Triangle>, true><<<cblocks, cthreads, 4>>>(
            pa, keys, vals, in.nt, counts, resf, lo, cs, rcp);
    else
        writeKeysAndValues<Triangle, PrimitiveArray<Triangle>, false><<<cblocks, cthreads, 4>>>(
            pa, keys, vals, in.nt, counts, resf, lo, cs, rcp);
    CK(cudaGetLastError());
    thrust::sort_by_key(thrust::device_ptr<uint>(keys), thrust::device_ptr<uint>(keys) + npairs,
                        thrust::device_ptr<uint>(vals));
    cudaPitchedPtr cells;
    CK(cudaMalloc3D(&cells, make_cudaExtent((size_t)res[0] * sizeof(uint2), (size_t)res[1], (size_t)res[2])));
    CK(cudaMemset3D(cells, 0, make_cudaExtent((size_t)res[0] * sizeof(uint2), (size_t)res[1], (size_t)res[2])));
    CK(cudaMalloc(&prims, (size_t)(npairs + kPad) * 4));
    if (tl)
        prepareCellRanges<512><<<sblocks, sthreads, (2 + sthreads) * 4>>>(prims, keys, vals, npairs, cells,
                                                                          (uint)res[0], (uint)res[1], (uint)res[2]);
    else
        prepareCellRanges<256><<<sblocks, sthreads, (2 + sthreads) * 4>>>(prims, keys, vals, npairs, cells,
                                                                          (uint)res[0], (uint)res[1], (uint)res[2]);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());

    uint nleaves = 0, nprims = npairs;
    uint2* leaves = nullptr;
    uint* final_prims = prims;
    if (tl) {
        uint* ccount;
        CK(cudaMalloc(&ccount, (size_t)(ncells + 1) * 4));
        CK(cudaMemset(ccount, 0, (size_t)(ncells + 1) * 4));
        countLeafLevelCells<false><<<dim3(res[1], res[2]), res[0]>>>(cs, in.leaf, cells, ccount);
        CK(cudaGetLastError());
        nleaves = host_scan(ccount, (size_t)ncells + 1);
        prepareTopLevelCellRanges<0><<<dim3(res[1], res[2]), res[0]>>>(ccount, cells);
        CK(cudaGetLastError());
        CK(cudaMemset(counts, 0, (cblocks + 1) * 4));
        countLeafLevelPairs<Triangle, PrimitiveArray, 512><<<cblocks, cthreads, cthreads * 4>>>(
            pa, npairs, keys, vals, cells, (uint)res[0], (uint)res[1], (uint)res[2], lo, cs, counts);
        CK(cudaGetLastError());
        const uint nleafpairs = host_scan(counts, cblocks + 1);
        uint *lkeys, *lvals;
        CK(cudaMalloc(&lkeys, (size_t)(nleafpairs + kPad) * 4));
        CK(cudaMalloc(&lvals, (size_t)(nleafpairs + kPad) * 4));
        writeLeafLevelKeysAndValues<Triangle, PrimitiveArray><<<cblocks, cthreads, 4>>>(
            pa, npairs, keys, vals, cells, nleaves, counts, (uint)res[0], (uint)res[1], (uint)res[2], lo, cs, lkeys,
            lvals);
        CK(cudaGetLastError());
        thrust::sort_by_key(thrust::device_ptr<uint>(lkeys), thrust::device_ptr<uint>(lkeys) + nleafpairs,
                            thrust::device_ptr<uint>(lvals));
        CK(cudaMalloc(&leaves, (size_t)(nleaves + kPad) * sizeof(uint2)));
        CK(cudaMemset(leaves, 0, (size_t)(nleaves + kPad) * sizeof(uint2)));
        CK(cudaMalloc(&final_prims, (size_t)(nleafpairs + kPad) * 4));
        prepareLeafCellRanges<512><<<sblocks, sthreads, (2 + sthreads) * 4>>>(final_prims, lkeys, lvals, nleafpairs,
                                                                              leaves);
        CK(cudaGetLastError());
        CK(cudaDeviceSynchronize());
        nprims = nleafpairs;
    }

    // traversal, RayTracingKernels.h:103-149
    float* drays;
    uint* did;
    float* dt;
    const size_t nr = in.nrays;
    CK(cudaMalloc(&drays, (nr + 1) * 24));
    CK(cudaMalloc(&did, (nr + 1) * 4));
    CK(cudaMalloc(&dt, (nr + 1) * 4));
    if (nr) CK(cudaMemcpy(drays, in.rays.data(), nr * 24, cudaMemcpyHostToDevice));
    const uint tb = 128, gb = (uint)((nr + tb - 1) / tb);
    if (nr && tl) {
        TwoLevelGrid g;
        g.vtx[0] = lo;
        g.vtx[1] = hi;
        for (int k = 0; k < 3; ++k) g.res[k] = res[k];
        g.setCellSize(cs);
        g.setCellSizeRCP(rcp);
        g.cells = cells;
        g.leaves = (TwoLevelGrid::t_Leaf*)leaves;
        g.primitives = final_prims;
        k_trace<TwoLevelGrid, TLGridTraverser<Triangle, MollerTrumboreIntersectionTest, false>>
            <<<gb, tb>>>(pa, g, drays, (uint)nr, did, dt);
    } else if (nr) {
        UniformGrid g;
        g.vtx[0] = lo;
        g.vtx[1] = hi;
        for (int k = 0; k < 3; ++k) g.res[k] = res[k];
        g.setCellSize(cs);
        g.setCellSizeRCP(rcp);
        g.cells = cells;
        g.primitives = final_prims;
        k_trace<UniformGrid, UGridTraverser<Triangle, MollerTrumboreIntersectionTest, false>>
            <<<gb, tb>>>(pa, g, drays, (uint)nr, did, dt);
    }
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());

    std::vector<uint32_t> hcells = read_pitched(cells, res[0], res[1], res[2]);
    std::vector<uint32_t> hleaves((size_t)nleaves * 2), hprims(nprims), hid(nr);
    std::vector<float> ht(nr);
    if (nleaves) CK(cudaMemcpy(hleaves.data(), leaves, (size_t)nleaves * 8, cudaMemcpyDeviceToHost));
    if (nprims) CK(cudaMemcpy(hprims.data(), final_prims, (size_t)nprims * 4, cudaMemcpyDeviceToHost));
    if (nr) {
        CK(cudaMemcpy(hid.data(), did, nr * 4, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(ht.data(), dt, nr * 4, cudaMemcpyDeviceToHost));
    }
    FILE* f = std::fopen(argv[2], "wb");
    if (!f) { std::perror(argv[2]); return 3; }
    write_all(f, res, 12);
    const float geo[12] = {lo.x, lo.y, lo.z, hi.x, hi.y, hi.z, cs.x, cs.y, cs.z, rcp.x, rcp.y, rcp.z};
    write_all(f, geo, 48);
    write_all(f, &ncells, 4);
    write_all(f, hcells.data(), hcells.size() * 4);
    write_all(f, &nleaves, 4);
    write_all(f, hleaves.data(), hleaves.size() * 4);
    write_all(f, &nprims, 4);
    write_all(f, hprims.data(), hprims.size() * 4);
    for (size_t i = 0; i < nr; ++i) {
        write_all(f, &hid[i], 4);
        write_all(f, &ht[i], 4);
    }
    std::fclose(f);
    std::printf("ok res %d %d %d pairs %u leaves %u prims %u rays %zu\n", res[0], res[1], res[2], npairs, nleaves,
                nprims, nr);
    return 0;
}
