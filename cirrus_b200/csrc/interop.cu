// Zero-copy interop with array-of-tiles storage (the reference keeps each tile as one
// allocation holding all channels, src/PoissonTile.h:51-56): gather one channel of every tile
// into the SoA pool and scatter it back, on the device, through a table of tile pointers.
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

}  // namespace

namespace launch {

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
