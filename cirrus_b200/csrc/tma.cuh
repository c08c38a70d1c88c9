// Bulk asynchronous copies (TMA) and transaction barriers for sm_100a, as inline PTX.
//
// A staged stencil kernel moves a tile and its halos from global to shared memory with a handful
// of bulk copies issued by one thread, each completing on an mbarrier of the destination stage
// with its byte count (complete_tx), instead of one 16-byte cp.async per thread and piece.
// Tensor copies address a channel as a 4-D tensor (k, j, i, tile) of FP32 through a tensor map
// made on the host (make_tile_maps); a box that lies wholly outside the tensor (tile coordinate
// -1: an absent neighbour) is filled with zeros and still counts its full byte size.
// No copy here uses cluster multicast: every source is this GPU's own memory.
#pragma once

#include <cuda.h>
#include <cstdint>

namespace cirrus {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
// Makes the initialised barriers visible to the async proxy (the copies' completions).
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// One bounded probe of the barrier's phase with the given parity (the hardware suspends the
// thread for a while inside try_wait before returning false).
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Waits for the phase with the given parity, giving up after `limit` probes (false).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int limit = 1 << 20) {
    for (int i = 0; i < limit; i++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// Orders this thread's generic-proxy shared-memory writes before later async-proxy (bulk copy)
// writes to the same bytes, once the stage is handed back through an mbarrier.
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Tiled 4-D tensor copy global -> shared, completing on `bar`.  The innermost coordinate c0 times
// the element size must be a multiple of 16 bytes (c0 in {0, 4} for FP32 here).
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(
            smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
        : "memory");
}
// Contiguous bulk copy global -> shared (both addresses 16-byte aligned, bytes a multiple of 16).
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void tma_prefetch_map(const CUtensorMap* map) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}
// Named barrier over `count` threads (id 1..15; 0 is __syncthreads).
__device__ __forceinline__ void named_bar(int id, int count) { asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory"); }

// The four tensor maps of one FP32 channel buffer viewed as (k 8, j 8, i 8, tile n): the whole
// tile, an x face (one i plane), a y face (one j row per i) and a z half-face (k 4..7 or 0..3 of
// every (i, j): the 4-byte z halo alone is below the 16-byte minimum box row).
struct TileMaps {
    CUtensorMap tile, xface, yface, zface;
};

}  // namespace cirrus
