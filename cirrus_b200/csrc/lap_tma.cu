// FullNegativeLaplacian over LEAF|GHOST tiles with the staged tiles moved by bulk asynchronous
// copies (TMA) through a ring of shared-memory stages (src/GMGSolver.cu:145-213 with
// PropagateValuesToGhostTiles and AccumulateToParents128, src/PoissonGrid.cu:585-605, 664-719,
// as k_laplacian_fused computes them; this kernel changes only how tiles reach shared memory).
//
// Persistent CTAs, warp-specialised:
//   * one producer warp walks the CTA's share of the staged-tile list (tiles q = cta + k*ncta),
//     loads each tile's metadata (its lanes prefetch 32 tiles' at a time, one batch ahead), and
//     for each tile waits until its stage is free, then issues 8 copies completing on the
//     stage's `full` barrier: the tile (2 KB box), its mask bytes (512 B), the x faces of its
//     x-/x+ neighbours (256 B boxes), their y faces (256 B) and z half-faces (1 KB boxes, k 4..7
//     or 0..3: a box row must span 16 bytes).  An absent neighbour is tile coordinate -1, which
//     the copy fills with zeros (the reference's empty-neighbour value, src/GMGSolver.cu:118-122).
//   * G consumer groups of 128 threads take the stages in turn (stage k: group k % G), compute
//     the stencil exactly as k_laplacian_fused does (same operations and order, so the same
//     bits), write A p, form the p.Ap tile parts or the GHOST rows, and hand the stage back
//     through its `empty` barrier.
// Every wait is bounded: a barrier that never completes sets a bit in `err` and the thread stops.
// The face-path GHOST tiles (k_laplacian_fused's item CTAs) are taken by all threads of the
// persistent CTAs once their staged tiles are done.
// Single-GPU code: all copies read this GPU's own memory; none uses cluster multicast.
#include "kernels.cuh"
#include "solver_internal.hpp"
#include "tma.cuh"

#include <map>
#include <mutex>

namespace cirrus {

namespace {

// Stage layout in bytes (every copy destination 128-byte aligned).
constexpr int kStXs = 0;       // the tile, 2048
constexpr int kStZm = 2048;    // z- neighbour, k 4..7 of every (i, j): [i][j][4], 1024
constexpr int kStZp = 3072;    // z+ neighbour, k 0..3, 1024
constexpr int kStXm = 4096;    // x- neighbour's i = 7 plane [j][k], 256
constexpr int kStXp = 4352;    // x+ neighbour's i = 0 plane, 256
constexpr int kStYm = 4608;    // y- neighbour's j = 7 rows [i][k], 256
constexpr int kStYp = 4864;    // y+ neighbour's j = 0 rows, 256
constexpr int kStMask = 5120;  // mask bytes, 512 (then the threads' p.Ap terms)
constexpr int kStHead = 5632;  // StageHead
constexpr int kStageBytes = 5760;
constexpr uint32_t kStageTx = 2048 + 2 * 1024 + 4 * 256 + 512;

struct __align__(16) StageHead {
    int tile, packed, slot;
    uint32_t fcls;
    float4 lc;
};

// Metadata of one tile, as a producer lane holds it.
struct PMeta {
    int tile, packed, slot;
    uint32_t fcls;
    int nb[6];
    float4 lc;
};

__device__ __forceinline__ void pmeta_load(const Topo& tp, const int* __restrict__ list, int q, bool with_slot, PMeta& m) {
    m.tile = list[q];
    const TileMeta tm = tp.meta[m.tile];
#pragma unroll
    for (int f = 0; f < 6; f++) m.nb[f] = tm.nb[f];
    m.packed = tm.packed;
    m.fcls = tp.fcls[m.tile];
    m.slot = with_slot ? tp.leafslot[m.tile] : -1;
    m.lc = tp.lconst[tp.inst[m.tile] * kLevelSlots + meta_level(tm.packed)];
}

__device__ __forceinline__ PMeta pmeta_shfl(const PMeta& m, int src) {
    PMeta o;
    o.tile = __shfl_sync(0xffffffffu, m.tile, src);
    o.packed = __shfl_sync(0xffffffffu, m.packed, src);
    o.slot = __shfl_sync(0xffffffffu, m.slot, src);
    o.fcls = __shfl_sync(0xffffffffu, m.fcls, src);
#pragma unroll
    for (int f = 0; f < 6; f++) o.nb[f] = __shfl_sync(0xffffffffu, m.nb[f], src);
    o.lc.x = __shfl_sync(0xffffffffu, m.lc.x, src);
    o.lc.y = __shfl_sync(0xffffffffu, m.lc.y, src);
    o.lc.z = __shfl_sync(0xffffffffu, m.lc.z, src);
    o.lc.w = __shfl_sync(0xffffffffu, m.lc.w, src);
    return o;
}

template <int G, int S>
__device__ __forceinline__ void consume(unsigned char* smem, uint64_t* full, uint64_t* empty, const Topo& tp, float* __restrict__ Y,
                                        float* __restrict__ GACC, const Scalars* __restrict__ Sc, double* __restrict__ WP,
                                        unsigned int* __restrict__ err, int count);

template <int G, int S>
__global__ void __launch_bounds__(128 * G + 32) k_laplacian_tma(const __grid_constant__ TileMaps maps, Topo tp,
                                                               const int* __restrict__ list, int n, const int4* __restrict__ items,
                                                               int nitems, const float* __restrict__ X,
                                                               float* __restrict__ Y, float* __restrict__ GACC,
                                                               const Scalars* __restrict__ Sc, double* __restrict__ WP,
                                                               unsigned int* __restrict__ err) {
    static_assert(G >= 1 && G <= 4 && S >= G && S % G == 0, "stage ring: S a multiple of the consumer groups");
    constexpr int kThreads = 128 * G + 32;
    pdl_entry();
    extern __shared__ unsigned char lt_smem_raw[];
    unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(lt_smem_raw) + 127) & ~uintptr_t(127));
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + S * kStageBytes);
    uint64_t* empty = full + S;
    const int cta = (int)blockIdx.x, ncta = (int)gridDim.x;
    const int count = n > cta ? (n - cta + ncta - 1) / ncta : 0;
    if (threadIdx.x == 0) {
        for (int i = 0; i < S; i++) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], 4);  // the four warps of the consuming group
        }
        mbar_init_fence();
    }
    __syncthreads();
    const int warp = (int)threadIdx.x >> 5, lane = (int)threadIdx.x & 31;
    if (warp == 4 * G) {
        // ---------------------------------------------------------------- producer warp
        if (lane == 0) {
            tma_prefetch_map(&maps.tile);
            tma_prefetch_map(&maps.xface);
            tma_prefetch_map(&maps.yface);
            tma_prefetch_map(&maps.zface);
        }
        PMeta cur = {}, nxt = {};
        if (lane < count) pmeta_load(tp, list, cta + lane * ncta, WP != nullptr, cur);
        for (int k0 = 0; k0 < count; k0 += 32) {
            if (k0 + 32 + lane < count) pmeta_load(tp, list, cta + (k0 + 32 + lane) * ncta, WP != nullptr, nxt);
            const int batch = min(32, count - k0);
            for (int j = 0; j < batch; j++) {
                const int k = k0 + j, s = k % S;
                if (k >= S && !mbar_wait(&empty[s], (uint32_t)((k / S - 1) & 1))) {
                    if (lane == 0) atomicOr(err, 1u);
                    return;
                }
                const PMeta m = pmeta_shfl(cur, j);
                unsigned char* st = smem + s * kStageBytes;
                if (lane == 0) {
                    StageHead h;
                    h.tile = m.tile;
                    h.packed = m.packed;
                    h.slot = m.slot;
                    h.fcls = m.fcls;
                    h.lc = m.lc;
                    *reinterpret_cast<StageHead*>(st + kStHead) = h;
                    mbar_arrive_expect_tx(&full[s], kStageTx);
                }
                __syncwarp();
                switch (lane) {
                case 0: tma_load_4d(st + kStXs, &maps.tile, 0, 0, 0, m.tile, &full[s]); break;
                case 1: bulk_load(st + kStMask, tp.mask_lap + (size_t)m.tile * kTileCells, kTileCells, &full[s]); break;
                case 2: tma_load_4d(st + kStXm, &maps.xface, 0, 0, 7, m.nb[0], &full[s]); break;
                case 3: tma_load_4d(st + kStXp, &maps.xface, 0, 0, 0, m.nb[1], &full[s]); break;
                case 4: tma_load_4d(st + kStYm, &maps.yface, 0, 7, 0, m.nb[2], &full[s]); break;
                case 5: tma_load_4d(st + kStYp, &maps.yface, 0, 0, 0, m.nb[3], &full[s]); break;
                case 6: tma_load_4d(st + kStZm, &maps.zface, 4, 0, 0, m.nb[4], &full[s]); break;
                case 7: tma_load_4d(st + kStZp, &maps.zface, 0, 0, 0, m.nb[5], &full[s]); break;
                default: break;
                }
            }
            cur = nxt;
        }
    } else {
        consume<G, S>(smem, full, empty, tp, Y, GACC, Sc, WP, err, count);
    }
    // ------------------------------------------------- the face path, after the CTA's staged tiles
    // every thread of the CTA takes items cta*kThreads + tid, then strides over the grid
    for (int q = cta * kThreads + (int)threadIdx.x; q < nitems; q += ncta * kThreads) {
        const int4 it = items[q];
        if (Sc != nullptr && Sc[it.w / kLevelSlots].done) continue;
        ghost_face_sum(tp, X, it, GACC);
    }
}

// The consumer groups of k_laplacian_tma: group grp takes stages k = grp, grp + G, ...
template <int G, int S>
__device__ __forceinline__ void consume(unsigned char* smem, uint64_t* full, uint64_t* empty, const Topo& tp, float* __restrict__ Y,
                                        float* __restrict__ GACC, const Scalars* __restrict__ Sc, double* __restrict__ WP,
                                        unsigned int* __restrict__ err, int count) {
    const int warp = (int)threadIdx.x >> 5, lane = (int)threadIdx.x & 31;
    const int grp = warp >> 2, t = (int)threadIdx.x & 127;
    for (int k = grp; k < count; k += G) {
        const int s = k % S;
        if (!mbar_wait(&full[s], (uint32_t)((k / S) & 1))) {
            if (t == 0) atomicOr(err, 2u);
            return;
        }
        unsigned char* st = smem + s * kStageBytes;
        const StageHead h = *reinterpret_cast<const StageHead*>(st + kStHead);
        float* xs = reinterpret_cast<float*>(st + kStXs);
        uint8_t* mask = st + kStMask;
        const bool act = !tile_done(tp, Sc, h.tile);
        const bool ghost = act && (meta_type(h.packed) & GHOST_T);
        float out[4] = {0.f, 0.f, 0.f, 0.f}, dg[4];
        if (act) {
            const LevelConst<float> L(h.lc);
            neg_lap4v<float, false, false>(xs, reinterpret_cast<const float*>(st + kStXm), reinterpret_cast<const float*>(st + kStXp),
                                           reinterpret_cast<const float*>(st + kStYm), reinterpret_cast<const float*>(st + kStYp),
                                           reinterpret_cast<const float*>(st + kStZm) + 3, reinterpret_cast<const float*>(st + kStZp), 4,
                                           t, *reinterpret_cast<const uint32_t*>(mask + t * 4), h.fcls & 0xfffu, L, out, dg);
            if (ghost) {
                const uint32_t ct4 = *reinterpret_cast<const uint32_t*>(tp.ctype + (size_t)h.tile * kTileCells + t * 4);
#pragma unroll
                for (int e = 0; e < 4; e++) out[e] = ((ct4 >> (8 * e)) & (INTERIOR_C | DIRICHLET_C | NEUMANN_C)) ? out[e] : 0.f;
            } else {
                V4<float> o;
                o.v[0] = out[0]; o.v[1] = out[1]; o.v[2] = out[2]; o.v[3] = out[3];
                st4(Y + (size_t)h.tile * kTileCells + t * 4, o);
                // the thread's p.Ap term, in its own (already read) mask bytes
                if (WP != nullptr && h.slot >= 0) reinterpret_cast<float*>(mask)[t] = dot4f32(ld4(xs + t * 4), o);
            }
        }
        named_bar(1 + grp, 128);  // every thread has read the tile and its halos
        if (ghost) {
#pragma unroll
            for (int e = 0; e < 4; e++) xs[t * 4 + e] = out[e];
        }
        named_bar(1 + grp, 128);
        if (act && !ghost && WP != nullptr && h.slot >= 0 && t < 32) {
            const double d = tile_part_sum(reinterpret_cast<const float*>(mask), t & 15);
            if (t == 0) WP[h.slot] = d;
        }
        if (ghost && t < 64) {
            // the GHOST tile's 2x2x2 child sums in AccumulateToParents128's (ii, jj, kk) order
            const int fi = t / 16 * 2, fj = (t / 4) % 4 * 2, fk = t % 4 * 2;
            float sum = 0.f;
#pragma unroll
            for (int ii = 0; ii < 2; ii++)
#pragma unroll
                for (int jj = 0; jj < 2; jj++)
#pragma unroll
                    for (int kk = 0; kk < 2; kk++) sum += xs[(fi + ii) * 64 + (fj + jj) * 8 + (fk + kk)];
            GACC[(size_t)tp.ghost_slot[h.tile] * 64 + t] = sum;
        }
        fence_proxy_async_smem();  // this thread's shared-memory writes before the stage's next copies
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
    }
}

// ------------------------------------------------------------------ host side
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*, const cuuint64_t*,
                                  const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<EncodeTiledFn>(p);
    }();
    return fn;
}

bool make_tile_maps(const float* base, int n, TileMaps* out) {
    EncodeTiledFn enc = encode_fn();
    if (!enc || n <= 0 || (reinterpret_cast<uintptr_t>(base) & 15u)) return false;
    const cuuint64_t dims[4] = {8, 8, 8, (cuuint64_t)n};
    const cuuint64_t strides[3] = {8 * sizeof(float), 64 * sizeof(float), kTileCells * sizeof(float)};
    const cuuint32_t elem[4] = {1, 1, 1, 1};
    auto mk = [&](CUtensorMap* m, cuuint32_t bk, cuuint32_t bj, cuuint32_t bi) {
        const cuuint32_t box[4] = {bk, bj, bi, 1};
        return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<float*>(base), dims, strides, box, elem,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
    };
    return mk(&out->tile, 8, 8, 8) && mk(&out->xface, 8, 8, 1) && mk(&out->yface, 8, 1, 8) && mk(&out->zface, 4, 8, 8);
}

// Tensor maps of a grid's channel buffers, made on first use per buffer.
struct MapCache {
    std::mutex mu;
    std::map<const float*, TileMaps> maps;
};

const TileMaps* tile_maps_for(const DevGrid& g, const float* X) {
    MapCache* c = static_cast<MapCache*>(g.tile_map_cache);
    if (!c) return nullptr;
    std::lock_guard<std::mutex> lk(c->mu);
    auto it = c->maps.find(X);
    if (it != c->maps.end()) return &it->second;
    TileMaps m;
    if (!make_tile_maps(X, g.n, &m)) return nullptr;
    return &c->maps.emplace(X, m).first->second;
}

template <int G, int S>
constexpr size_t tma_smem_bytes() {
    return (size_t)S * kStageBytes + 2 * S * sizeof(uint64_t) + 128;
}

template <int G, int S>
bool laplacian_tma_shape(const DevGrid& g, const float* X, float* Y, const Scalars* Sc, cudaStream_t s, double* WP) {
    const TileMaps* maps = tile_maps_for(g, X);
    if (!maps) return false;
    constexpr int threads = 128 * G + 32;
    constexpr size_t smem = tma_smem_bytes<G, S>();
    static int occ = [] {
        // all of the SM's unified L1/shared storage as shared memory, so the occupancy the grid is
        // sized for is the one the launch gets (the default carveout may hold fewer stage rings)
        cudaFuncSetAttribute(k_laplacian_tma<G, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaFuncSetAttribute(k_laplacian_tma<G, S>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        int o = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, k_laplacian_tma<G, S>, threads, smem) != cudaSuccess) o = 1;
        return o > 0 ? o : 1;
    }();
    // persistent: one wave of CTAs (fewer when there are few tiles and items)
    const int want = std::max((g.n_lapmain + G - 1) / G, (g.n_lapitems + threads - 1) / threads);
    const int ncta = std::max(1, std::min(g.sm_count * occ, want));
    launch::launch_kernel(k_laplacian_tma<G, S>, ncta, threads, smem, s, *maps, g.topo, g.d_lapmain, g.n_lapmain, g.d_lapitems,
                          g.n_lapitems, X, Y, g.d_gacc, Sc, WP, g.d_err);
    return true;
}

}  // namespace

void init_tile_map_cache(DevGrid& g) {
    if (!g.tile_map_cache) g.tile_map_cache = new MapCache();
}
void free_tile_map_cache(DevGrid& g) {
    delete static_cast<MapCache*>(g.tile_map_cache);
    g.tile_map_cache = nullptr;
}

namespace launch {

bool laplacian_tma(const DevGrid& g, int variant, const float* X, float* Y, const Scalars* S, cudaStream_t s, bool with_pap) {
    double* WP = with_pap ? g.d_wpart : nullptr;
    switch (variant) {
    case 0: return laplacian_tma_shape<2, 8>(g, X, Y, S, s, WP);
    case 1: return laplacian_tma_shape<4, 16>(g, X, Y, S, s, WP);
    case 2: return laplacian_tma_shape<2, 12>(g, X, Y, S, s, WP);
    default: return laplacian_tma_shape<1, 6>(g, X, Y, S, s, WP);
    }
}

}  // namespace launch
}  // namespace cirrus
