// noalloc.cu -- a radix sort of (key, value) pairs that allocates no memory.
//
// Who needs it: callers whose device memory is fully reserved before their frame or
// request loop starts -- a renderer that budgets its whole HBM at start-up, or a serving
// process that admits work against a fixed memory budget.  They cannot call cudaMalloc
// inside the loop: an allocation may block on the device, may fail under memory
// pressure half-way through a frame, and escapes the caller's accounting.  Everything
// else in this library draws its scratch from a context that grows its buffers with
// cudaMallocAsync; this entry point needs neither a context nor an allocation.
//
// Scratch: one file-scope __device__ array of kScratchWords words (about 8.5 MiB)
// per GPU.  It exists on every GPU that loads this library, from module load until the
// process exits.  Its device address is looked up once per device, with that device
// current, through cudaGetSymbolAddress (host code must not take the array's address
// directly: on the host the symbol is only a stand-in).  The first call on a device does
// this lookup, so make that first call before any stream capture.
//
// Every call shares the one array and leaves the last call's data in it.  No part of the
// array is accumulated into, so nothing needs clearing: the pair count is written by
// every call before its first pass reads it, each pass's digit-total scan rewrites the
// totals it reads, and every histogram and ping-pong word a pass reads was written
// earlier in the same call.  Two calls whose work overlaps on the GPU (two streams, or
// two host threads) race on the array and corrupt each other's results: serialise them,
// e.g. on one stream.
//
// The cached address belongs to the device's current context: after cudaDeviceReset the
// module is loaded again and the array may move, so this entry point must not be used
// across a cudaDeviceReset of a device it has already run on.
#include "hr_internal.h"
#include "../../include/happyray.h"

#include <mutex>

namespace hr {
cudaError_t radix_sort_pairs_raw(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_tmp,
                                 uint32_t* vals_tmp, uint32_t* keys_out, uint32_t* vals_out,
                                 const uint32_t* d_count, size_t cap_count, int key_bits, uint32_t* tile_hist,
                                 uint32_t* row_total, cudaStream_t s);
}

namespace {

constexpr size_t kMaxPairs = HR_NOALLOC_MAX_PAIRS;
constexpr size_t kTileKeys = 2048;                               // keys per radix tile (sort.cu)
constexpr size_t kMaxTiles = (kMaxPairs + kTileKeys - 1) / kTileKeys;
constexpr size_t kCtlOff = 0;                                    // [0] pair count
constexpr size_t kRowOff = 64;                                   // 256 digit totals
constexpr size_t kKeysOff = kRowOff + 256;                       // ping-pong keys
constexpr size_t kValsOff = kKeysOff + kMaxPairs;                // ping-pong values
constexpr size_t kHistOff = kValsOff + kMaxPairs;                // tile histograms, 256 per tile
constexpr size_t kScratchWords = kHistOff + kMaxTiles * 256;

static __device__ __align__(256) uint32_t g_sort_scratch[kScratchWords];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
uint32_t* g_scratch[kMaxDevices] = {};

// the pair count, which the sort kernels read from device memory
__global__ void k_noalloc_count(uint32_t* scratch, uint32_t n) { scratch[kCtlOff] = n; }

// device address of the scratch on the current device (looked up once per device)
cudaError_t scratch_address(uint32_t** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_sort_scratch);
        if (e != cudaSuccess) return e;
        g_scratch[dev] = static_cast<uint32_t*>(p);
    }
    *out = g_scratch[dev];
    return cudaSuccess;
}

}  // namespace

extern "C" hr_status hr_radix_sort_pairs_noalloc(void* stream, uint32_t* d_keys, uint32_t* d_values, uint32_t n,
                                                 int32_t key_bits) {
    if (key_bits < 1 || key_bits > 32) return HR_ERR_INVALID_ARG;
    if (n > kMaxPairs) return HR_ERR_INVALID_ARG;   // beyond the static scratch
    if (n == 0) return HR_OK;
    if (!d_keys || !d_values) return HR_ERR_INVALID_ARG;
    uint32_t* scratch = nullptr;
    if (scratch_address(&scratch) != cudaSuccess) {
        cudaGetLastError();
        return HR_ERR_DEVICE;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    uint32_t* count = scratch + kCtlOff;
    uint32_t* row = scratch + kRowOff;
    uint32_t* tk = scratch + kKeysOff;
    uint32_t* tv = scratch + kValsOff;
    uint32_t* hist = scratch + kHistOff;
    k_noalloc_count<<<1, 1, 0, s>>>(scratch, n);
    const int passes = (key_bits + 7) / 8;
    cudaError_t e;
    if (passes % 2 == 0) {
        // even pass count: caller's arrays -> scratch -> ... -> caller's arrays
        e = hr::radix_sort_pairs_raw(d_keys, d_values, tk, tv, d_keys, d_values, count, n, key_bits, hist, row, s);
    } else {
        // odd pass count ends in the scratch pair, which is then copied back
        e = hr::radix_sort_pairs_raw(d_keys, d_values, tk, tv, tk, tv, count, n, key_bits, hist, row, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(d_keys, tk, (size_t)n * 4, cudaMemcpyDeviceToDevice, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(d_values, tv, (size_t)n * 4, cudaMemcpyDeviceToDevice, s);
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        return HR_ERR_DEVICE;
    }
    return HR_OK;
}
