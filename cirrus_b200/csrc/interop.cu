// Zero-copy interop with array-of-tiles storage (the reference keeps each tile as one
// allocation holding all channels, src/PoissonTile.h:51-56): gather one channel of every tile
// into the SoA pool and scatter it back, on the device, through a table of tile pointers; and
// check the tiles' cell types (mCellType, rewritten by CalcCellTypesFromLeafs every step,
// src/FluidEuler.h:934) against the ones the pool was built from.
#include "kernels.cuh"
#include "solver_internal.hpp"

namespace cirrus {

namespace {

__global__ void __launch_bounds__(128) k_gather_tiles(const char* const* __restrict__ ptrs, size_t off, float* dst, int n) {
    const int tile = blockIdx.x;
    if (tile >= n) return;
    const float* src = reinterpret_cast<const float*>(ptrs[tile] + off);
    st4(dst + (size_t)tile * kTileCells + threadIdx.x * 4, ld4(src + threadIdx.x * 4));
}

__global__ void __launch_bounds__(128) k_scatter_tiles(char* const* __restrict__ ptrs, size_t off, const float* src, int n) {
    const int tile = blockIdx.x;
    if (tile >= n) return;
    float* dst = reinterpret_cast<float*>(ptrs[tile] + off);
    st4(dst + threadIdx.x * 4, ld4(src + (size_t)tile * kTileCells + threadIdx.x * 4));
}

// One 128-thread block per tile: thread t copies cell-type bytes 4t..4t+3 (one 32-bit load; the
// byte offset is a multiple of 4 and tiles are 16-byte aligned) and compares them with the pool's.
__global__ void __launch_bounds__(128) k_compare_cell_types(const char* const* __restrict__ ptrs, size_t off,
                                                            const uint8_t* __restrict__ pool, uint8_t* dst, unsigned int* flag,
                                                            int n) {
    const int tile = blockIdx.x;
    if (tile >= n) return;
    const uint32_t v = *reinterpret_cast<const uint32_t*>(ptrs[tile] + off + threadIdx.x * 4);
    const size_t at = (size_t)tile * kTileCells + threadIdx.x * 4;
    *reinterpret_cast<uint32_t*>(dst + at) = v;
    const bool differs = v != *reinterpret_cast<const uint32_t*>(pool + at);
    if (__any_sync(0xffffffffu, differs) && (threadIdx.x & 31) == 0) atomicOr(flag, 1u);
}

// 512 bytes at ptrs[tile] + off into dst (tile-major), 4 per thread.
__global__ void __launch_bounds__(128) k_gather_bytes(const char* const* __restrict__ ptrs, size_t off, uint8_t* dst, int n) {
    const int tile = blockIdx.x;
    if (tile >= n) return;
    *reinterpret_cast<uint32_t*>(dst + (size_t)tile * kTileCells + threadIdx.x * 4) =
        *reinterpret_cast<const uint32_t*>(ptrs[tile] + off + threadIdx.x * 4);
}

}  // namespace

int gather_tile_bytes(const void* const* tile_ptrs, int n, size_t byte_offset, uint8_t* host_out, cudaStream_t s) {
    void** d_ptrs = nullptr;
    uint8_t* d_out = nullptr;
    int rc = 0;
    if (cudaMalloc(&d_ptrs, sizeof(void*) * n) != cudaSuccess || cudaMalloc(&d_out, (size_t)n * kTileCells) != cudaSuccess) rc = 3;
    if (!rc && cudaMemcpyAsync(d_ptrs, tile_ptrs, sizeof(void*) * n, cudaMemcpyHostToDevice, s) != cudaSuccess) rc = 2;
    if (!rc) {
        k_gather_bytes<<<n, 128, 0, s>>>(reinterpret_cast<const char* const*>(d_ptrs), byte_offset, d_out, n);
        if (cudaMemcpyAsync(host_out, d_out, (size_t)n * kTileCells, cudaMemcpyDeviceToHost, s) != cudaSuccess) rc = 2;
        if (cudaStreamSynchronize(s) != cudaSuccess) rc = 2;
    }
    cudaFree(d_ptrs);
    cudaFree(d_out);
    return rc;
}

namespace launch {

void compare_tile_cell_types(const DevGrid& g, size_t byte_offset, cudaStream_t s) {
    ++g.launch_count;
    cudaMemsetAsync(g.d_ct_flag, 0, sizeof(unsigned int), s);
    k_compare_cell_types<<<g.n, 128, 0, s>>>(reinterpret_cast<const char* const*>(g.d_tile_ptrs), byte_offset, g.topo.ctype,
                                             g.d_ct_gather, g.d_ct_flag, g.n);
}


void gather_tiles(const DevGrid& g, int channel, size_t byte_offset, cudaStream_t s) {
    ++g.launch_count;
    k_gather_tiles<<<g.n, 128, 0, s>>>(reinterpret_cast<const char* const*>(g.d_tile_ptrs), byte_offset, g.d_ch[channel], g.n);
}

void scatter_tiles(const DevGrid& g, int channel, size_t byte_offset, cudaStream_t s) {
    ++g.launch_count;
    k_scatter_tiles<<<g.n, 128, 0, s>>>(reinterpret_cast<char* const*>(g.d_tile_ptrs), byte_offset, g.d_ch[channel], g.n);
}

}  // namespace launch
}  // namespace cirrus
