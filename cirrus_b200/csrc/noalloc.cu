// cirrus_leaf_dot_noalloc: the LEAF-tile dot product of cirrus_dot (same kernel, same block
// count, so the same bits) for callers that must not allocate.  Its reduction scratch -- the
// per-block partial sums, the ticket counter and the result slot -- lives in one fixed static
// device array of this file instead of memory allocated with a grid; the call makes no
// cudaMalloc/cudaFree or other allocating call.
#include "cirrus_b200.h"
#include "solver_internal.hpp"

#include <algorithm>
#include <mutex>

namespace cirrus {
namespace {

// Scratch layout (bytes): per-block partials, 2 doubles per block (k_leaf_reduce's layout), for
// CIRRUS_NOALLOC_MAX_BLOCKS blocks; the Scalars record whose `gamma` receives the sum; the ticket
// counter, which must be 0 when the kernel starts (each call zeroes it on its stream first).
constexpr size_t kPartialsBytes = sizeof(double) * 2 * CIRRUS_NOALLOC_MAX_BLOCKS;
constexpr size_t kScalarsOffset = kPartialsBytes;
constexpr size_t kCounterOffset = (kScalarsOffset + sizeof(Scalars) + 255) & ~size_t(255);
constexpr size_t kScratchBytes = kCounterOffset + 256;

// One copy per device (a __device__ variable exists in every context the library is loaded in).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_lock;
unsigned char* g_scratch_of[kMaxDevices] = {};

// Device address of this device's scratch, looked up once per device.
cirrus_status scratch_of_device(int dev, unsigned char** out) {
    if (dev < 0 || dev >= kMaxDevices) return CIRRUS_ERR_NO_DEVICE;
    std::lock_guard<std::mutex> lk(g_lock);
    if (!g_scratch_of[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr) {
            cudaGetLastError();
            return CIRRUS_ERR_CUDA;
        }
        g_scratch_of[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_scratch_of[dev];
    return CIRRUS_OK;
}

cirrus_status leaf_dot_noalloc(const float* a, const float* b, const int32_t* leaf_tiles, int n_leaf, double* result,
                               cudaStream_t s) {
    if (!a || !b || !result || n_leaf < 0 || (n_leaf > 0 && !leaf_tiles)) return CIRRUS_ERR_INVALID_ARGUMENT;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return CIRRUS_ERR_NO_DEVICE;
    }
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        cudaGetLastError();
        return CIRRUS_ERR_CUDA;
    }
    // the block count of the grid's own reductions: one 256-thread block per 256 vectors of 4
    // cells, at most 4 per SM
    const long long want = ((long long)n_leaf * 128 + 255) / 256;
    const long long blocks = std::max(1LL, std::min(want, 4LL * sms));
    if (blocks > CIRRUS_NOALLOC_MAX_BLOCKS) return CIRRUS_ERR_INVALID_ARGUMENT;
    unsigned char* base = nullptr;
    cirrus_status st = scratch_of_device(dev, &base);
    if (st != CIRRUS_OK) return st;
    double* partials = reinterpret_cast<double*>(base);
    Scalars* S = reinterpret_cast<Scalars*>(base + kScalarsOffset);
    unsigned int* counter = reinterpret_cast<unsigned int*>(base + kCounterOffset);
    if (cudaMemsetAsync(counter, 0, sizeof(unsigned int), s) != cudaSuccess) {
        cudaGetLastError();
        return CIRRUS_ERR_CUDA;
    }
    launch::leaf_dot_raw(a, b, leaf_tiles, n_leaf, (int)blocks, partials, counter, S, s);
    if (cudaGetLastError() != cudaSuccess) return CIRRUS_ERR_CUDA;
    if (cudaMemcpyAsync(result, &S->gamma, sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
        cudaGetLastError();
        return CIRRUS_ERR_CUDA;
    }
    return CIRRUS_OK;
}

}  // namespace
}  // namespace cirrus

extern "C" cirrus_status cirrus_leaf_dot_noalloc(const float* a, const float* b, const int32_t* leaf_tiles, int n_leaf,
                                                 double* result, void* stream) {
    try {
        return cirrus::leaf_dot_noalloc(a, b, leaf_tiles, n_leaf, result, static_cast<cudaStream_t>(stream));
    } catch (...) {
        return CIRRUS_ERR_CUDA;
    }
}
