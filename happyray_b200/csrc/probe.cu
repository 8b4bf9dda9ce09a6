// probe.cu -- measured cache bandwidth for the traversal roofline.
//
// The traversal kernels read leaf ranges, primitive lists and triangle vertices whose
// working sets mostly stay in the 126 MB L2, so their algorithmic bytes are reported
// against an L2 read rate measured on the same device, next to the HBM copy rate.  No
// counterpart in the reference.
#include "hr_internal.h"
#include "happyray.h"

namespace hr {
namespace {

// reps passes over n16 16-byte words loaded through L2 only (ld.global.cg), folded into
// one word per thread so that the loads are kept
__global__ __launch_bounds__(256) void k_l2_read(const uint4* __restrict__ a, size_t n16, int reps,
                                                 uint32_t* __restrict__ sink) {
    uint32_t acc = 0;
    for (int r = 0; r < reps; ++r)
        for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n16; i += (size_t)gridDim.x * blockDim.x) {
            const uint4 v = __ldcg(a + i);
            acc ^= v.x ^ v.y ^ v.z ^ v.w;
        }
    if (acc == 0x9e3779b9u) sink[0] = acc;   // never true for the zero-filled buffer
}

}  // namespace
}  // namespace hr

using namespace hr;

extern "C" hr_status hr_probe_l2_read(void* stream, double* gbs) {
    if (!gbs) return HR_ERR_INVALID_ARG;
    *gbs = 0.0;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        cudaGetLastError();
        return HR_ERR_DEVICE;
    }
    constexpr size_t kBytes = 32u << 20;   // a quarter of L2
    constexpr int kReps = 50;
    void* buf = nullptr;
    if (cudaMallocAsync(&buf, kBytes + 16, s) != cudaSuccess) {
        cudaGetLastError();
        return HR_ERR_OUT_OF_MEMORY;
    }
    uint32_t* sink = reinterpret_cast<uint32_t*>(static_cast<char*>(buf) + kBytes);
    cudaEvent_t a = nullptr, b = nullptr;
    hr_status st = HR_OK;
    const uint4* p = static_cast<const uint4*>(buf);
    const size_t n16 = kBytes / 16;
    const int grid = sms * 8;
    float ms = 0.0f;
    if (cudaMemsetAsync(buf, 0, kBytes + 16, s) != cudaSuccess || cudaEventCreate(&a) != cudaSuccess ||
        cudaEventCreate(&b) != cudaSuccess) {
        st = HR_ERR_DEVICE;
    } else {
        k_l2_read<<<grid, 256, 0, s>>>(p, n16, 2, sink);   // warm-up: the buffer into L2
        cudaEventRecord(a, s);
        k_l2_read<<<grid, 256, 0, s>>>(p, n16, kReps, sink);
        cudaEventRecord(b, s);
        if (cudaEventSynchronize(b) != cudaSuccess || cudaEventElapsedTime(&ms, a, b) != cudaSuccess || ms <= 0.0f)
            st = HR_ERR_DEVICE;
        else
            *gbs = (double)kBytes * kReps / (ms * 1e-3) / 1e9;
    }
    cudaGetLastError();
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    cudaFreeAsync(buf, s);
    cudaStreamSynchronize(s);
    return st;
}
