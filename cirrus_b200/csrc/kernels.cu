// Kernels of the GMG-PCG solve and their launchers.  Reference counterparts are cited per
// kernel (paths inside the reference project).
#include "kernels.cuh"
#include "solver_internal.hpp"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <mutex>

namespace cirrus {

// ------------------------------------------------------------------ ghost value propagation
// PropagateValuesToGhostTiles (src/PoissonGrid.cu:585-605): a GHOST cell takes its parent
// cell's value when both are INTERIOR, 0 otherwise.
template <class T>
__global__ void __launch_bounds__(128) k_propagate_ghosts(Topo tp, const int* __restrict__ list, int n, T* X,
                                                          const Scalars* __restrict__ S) {
    pdl_entry();
    const int q = blockIdx.x;
    if (q >= n) return;
    const int tile = list[q];
    if (tile_done(tp, S, tile)) return;
    const int t = threadIdx.x;
    const TileMeta m = tp.meta[tile];
    const TileIdx ix(t);
    const uint32_t ct4 = *reinterpret_cast<const uint32_t*>(tp.ctype + (size_t)tile * kTileCells + t * 4);
    V4<T> out = zero4<T>();
    if (m.parent >= 0) {
        const int oct = meta_octant(m.packed);
        const int pi = (oct & 1) * 4 + (ix.i >> 1), pj = ((oct >> 1) & 1) * 4 + (ix.j >> 1);
        const size_t pbase = (size_t)m.parent * kTileCells + pi * 64 + pj * 8 + ((oct >> 2) & 1) * 4 + (ix.k0 >> 1);
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const size_t pid = pbase + (e >> 1);
            const bool me = (ct4 >> (8 * e)) & INTERIOR_C;
            const bool pin = tp.ctype[pid] & INTERIOR_C;
            out.v[e] = (me && pin) ? X[pid] : T(0);
        }
    }
    st4(X + (size_t)tile * kTileCells + t * 4, out);
}

// ------------------------------------------------------------------ Laplacian apply
// NegativeLaplacianSameLevel128Kernel (src/GMGSolver.cu:145-194) on LEAF|GHOST tiles of all
// levels with the tile types as stored (subtree level -1).
// DIAG: the diagonal (the same sum over the face coefficients) instead of A x, as the
// reference's calc_diag argument selects.
template <class T, int TPB, bool DIAG = false>
__global__ void __launch_bounds__(128 * TPB) k_laplacian(Topo tp, const int* __restrict__ list, int n, const T* __restrict__ X,
                                                         T* __restrict__ Y, const Scalars* __restrict__ S) {
    pdl_entry();
    __shared__ TileShared<T> sh[TPB];
    const int g = threadIdx.x >> 7, t = threadIdx.x & 127;
    const int q = blockIdx.x * TPB + g;
    const int tile = q < n ? list[q] : 0;
    const bool active = q < n && !tile_done(tp, S, tile);
    TileMeta m;
    if (active) {
        m = tp.meta[tile];
        stage_tile<T>(X, tile, m, t, sh[g]);
    }
    __syncthreads();
    if (!active) return;
    const uint32_t mask4 = *reinterpret_cast<const uint32_t*>(tp.mask_lap + (size_t)tile * kTileCells + t * 4);
    const LevelConst<T> L((T)tile_h0(tp, tile), meta_level(m.packed));
    T out[4], dg[4];
    neg_lap4<T, DIAG, false>(sh[g].xs, sh[g].hx, t, mask4, tp.fcls[tile] & 0xfffu, L, out, dg);
    V4<T> o;
#pragma unroll
    for (int e = 0; e < 4; e++) o.v[e] = DIAG ? dg[e] : out[e];
    st4(Y + (size_t)tile * kTileCells + t * 4, o);
}

// NegativeLaplacianSameLevel128 (src/GMGSolver.cu:145-201) over the pool tiles [first,
// first + count): a tile whose subtreeType(subtree_level) -- NONLEAF counts as LEAF at its own
// level -- is in `types` gets A x (or the diagonal) on all 512 cells; other tiles are not
// written.  A tile at the subtree level sees its neighbours with the same rule (the multigrid
// level context, mask_mg); a tile at any other level sees their plain types (the full-tree
// context, mask_lap).  Products rounded before the add, as in the reference's kernel.
template <int TPB, bool DIAG>
__global__ void __launch_bounds__(128 * TPB) k_laplacian_same_level(Topo tp, int first, int count, int subtree_level,
                                                                      uint32_t types, const float* __restrict__ X,
                                                                      float* __restrict__ Y) {
    pdl_entry();
    __shared__ TileShared<float> sh[TPB];
    const int g = threadIdx.x >> 7, t = threadIdx.x & 127;
    const int q = blockIdx.x * TPB + g;
    const int tile = first + (q < count ? q : 0);
    bool active = false, own_level = false;
    TileMeta m;
    if (q < count) {
        m = tp.meta[tile];
        own_level = meta_level(m.packed) == subtree_level;
        const uint32_t type = (uint32_t)meta_type(m.packed);
        active = ((own_level && type == NONLEAF_T ? (uint32_t)LEAF_T : type) & types) != 0;
        if (active) stage_tile<float>(X, tile, m, t, sh[g]);
    }
    __syncthreads();
    if (!active) return;
    const uint8_t* masks = own_level ? tp.mask_mg : tp.mask_lap;
    const uint32_t mask4 = *reinterpret_cast<const uint32_t*>(masks + (size_t)tile * kTileCells + t * 4);
    const uint32_t cls = (own_level ? tp.fcls[tile] >> 12 : tp.fcls[tile]) & 0xfffu;
    const LevelConst<float> L((float)tile_h0(tp, tile), meta_level(m.packed));
    float out[4], dg[4];
    neg_lap4<float, DIAG, false>(sh[g].xs, sh[g].hx, t, mask4, cls, L, out, dg);
    V4<float> o;
#pragma unroll
    for (int e = 0; e < 4; e++) o.v[e] = DIAG ? dg[e] : out[e];
    st4(Y + (size_t)tile * kTileCells + t * 4, o);
}

// FullNegativeLaplacian in one launch over LEAF|GHOST tiles.  p on GHOST tiles is kept valid by
// the kernels that write p (push_to_ghost_child), so no propagation pass runs; LEAF tiles write
// A p; GHOST tiles write the 2x2x2 child sums of their A p (AccumulateToParents128's order) to a
// per-ghost row, added to the parent's A p by the p.Ap reduction that follows.  The first
// item_blocks CTAs take the face path, one thread per item of `items` (a coarse cell touching a
// coupled face of a face-path GHOST tile); the others take `list` (LEAF tiles and GHOST tiles
// coupled inside), staged with asynchronous copies, NT per 128-thread group.  Row entries in
// neither are constant zeros (set when the grid is created).
// With WP the launch also stores, for every LEAF tile without GHOST children (whose A p is final
// here), the tile's part of p.Ap (tile_part_sum of the threads' 4-cell FP32 products) at
// WP[LEAF slot]; k_pap_ghost forms those of the other LEAF tiles.
// tp.pf > 0: thread 0 of each group also prefetches into L2 the values and mask bytes of the
// tiles pf list entries ahead (the tiles a CTA about one resident wave later stages).
template <int TPB, int NT>
__device__ __forceinline__ void k_laplacian_fused_body(Topo tp, const int* __restrict__ list, int n, const int4* __restrict__ items,
                                                               int nitems, int item_blocks,
                                                               const float* __restrict__ X, float* __restrict__ Y,
                                                               float* __restrict__ GACC, const Scalars* __restrict__ S,
                                                               double* __restrict__ WP) {
    // the dot-part tail below gives tile u to 16-lane half (u & 1) of warp u >> 1: NT <= 8
    static_assert(NT >= 1 && NT <= 8, "k_laplacian_fused: the tile-part tail covers at most 8 tiles per group");
    pdl_trigger();
    if ((int)blockIdx.x < item_blocks) {
        pdl_wait();
        const int q = (int)blockIdx.x * (128 * TPB) + (int)threadIdx.x;
        if (q >= nitems) return;
        const int4 it = items[q];
        if (S != nullptr && S[it.w / kLevelSlots].done) return;
        ghost_face_sum(tp, X, it, GACC);
        return;
    }
    extern __shared__ __align__(16) unsigned char lap_smem[];
    LapStage* st = reinterpret_cast<LapStage*>(lap_smem);
    const int g = threadIdx.x >> 7, t = threadIdx.x & 127;
    int tile[NT], ptile[NT];
    bool act[NT];
#pragma unroll
    for (int u = 0; u < NT; u++) {
        const int q = (((int)blockIdx.x - item_blocks) * NT + u) * TPB + g;
        tile[u] = q < n ? list[q] : 0;
        act[u] = q < n;  // finished instances are dropped after the copies are issued (reading them is harmless)
        ptile[u] = (tp.pf > 0 && t == 0 && q + tp.pf < n) ? list[q + tp.pf] : -1;
    }
    TilePre pre[NT];
    tile_pre(tp, tile, t, pre);
    pdl_wait();
#pragma unroll
    for (int u = 0; u < NT; u++)
        if (act[u]) {
            stage_async(X, nullptr, tp.mask_lap, tile[u], pre[u].nb, t, st[u * TPB + g]);
            if (WP != nullptr && t == 0) cp_async4(st[u * TPB + g].aux, tp.leafslot + tile[u]);
        }
#pragma unroll
    for (int u = 0; u < NT; u++)
        if (ptile[u] >= 0) {
            prefetch_l2(X + (size_t)ptile[u] * kTileCells, kTileCells * sizeof(float));
            prefetch_l2(tp.mask_lap + (size_t)ptile[u] * kTileCells, kTileCells);
        }
#pragma unroll
    for (int u = 0; u < NT; u++) act[u] = act[u] && !tile_done(tp, S, tile[u]);
    cp_async_wait_all();
    __syncthreads();
    bool ghost[NT];
#pragma unroll
    for (int u = 0; u < NT; u++) {
        ghost[u] = false;
        if (!act[u]) continue;
        LapStage& ts = st[u * TPB + g];
        ghost[u] = meta_type(pre[u].packed) & GHOST_T;
        const LevelConst<float> L(pre[u].lc);
        float out[4], dg[4];
        neg_lap4<float, false, false>(ts.xs, ts.hx, t, *reinterpret_cast<const uint32_t*>(ts.mask + t * 4), pre[u].fcls & 0xfffu, L,
                                      out, dg);
        if (ghost[u]) {
            // the GHOST row: each coarse cell's 2x2x2 sum of the typed cells' A p, in
            // AccumulateToParents128's (ii, jj, kk) order.  The thread holds (ii, jj) = (0, 0) of
            // the coarse cells over its cells' pairs (kk = 0, 1); the threads t ^ 2 (jj = 1),
            // t ^ 16 (ii = 1) and t ^ 18 hold the others -- in the same warp.
            const uint32_t ct4 = *reinterpret_cast<const uint32_t*>(tp.ctype + (size_t)tile[u] * kTileCells + t * 4);
            float a[4], bj[4], bi[4], bij[4];
#pragma unroll
            for (int e = 0; e < 4; e++) a[e] = ((ct4 >> (8 * e)) & (INTERIOR_C | DIRICHLET_C | NEUMANN_C)) ? out[e] : 0.f;
#pragma unroll
            for (int e = 0; e < 4; e++) {
                bj[e] = __shfl_xor_sync(0xffffffffu, a[e], 2);
                bi[e] = __shfl_xor_sync(0xffffffffu, a[e], 16);
                bij[e] = __shfl_xor_sync(0xffffffffu, a[e], 18);
            }
            const TileIdx ix(t);
            if (((ix.i | ix.j) & 1) == 0) {
                const size_t row = (size_t)tp.ghost_slot[tile[u]] * 64;
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    float sum = 0.f;
                    sum += a[2 * h]; sum += a[2 * h + 1];
                    sum += bj[2 * h]; sum += bj[2 * h + 1];
                    sum += bi[2 * h]; sum += bi[2 * h + 1];
                    sum += bij[2 * h]; sum += bij[2 * h + 1];
                    GACC[row + (ix.i >> 1) * 16 + (ix.j >> 1) * 4 + ((ix.k0 + 2 * h) >> 1)] = sum;
                }
            }
        } else {
            V4<float> o;
            o.v[0] = out[0]; o.v[1] = out[1]; o.v[2] = out[2]; o.v[3] = out[3];
            st4(Y + (size_t)tile[u] * kTileCells + t * 4, o);
            // the thread's p.Ap term, in its own (already read) mask bytes
            if (WP != nullptr && ts.aux[0] >= 0) reinterpret_cast<float*>(ts.mask)[t] = dot4f32(ld4(ts.xs + t * 4), o);
        }
    }
    if (WP == nullptr) return;
    __syncthreads();
    // warp w of each group sums the LEAF tiles' terms of tiles u = 2w (lanes 0..15) and 2w + 1 (16..31)
    if (2 * (t >> 5) >= NT) return;  // whole warps
    const int u = 2 * (t >> 5) + ((t >> 4) & 1);
    bool ok = false;
#pragma unroll
    for (int k = 0; k < NT; k++)
        if (k == u) ok = act[k] && !ghost[k];
    const LapStage& ts = st[(u < NT ? u : 0) * TPB + g];
    const int sl = ts.aux[0];
    const double d = tile_part_sum(reinterpret_cast<const float*>(ts.mask), t & 15);
    if (ok && u < NT && sl >= 0 && (t & 15) == 0) WP[sl] = d;
}
template <int TPB, int NT>
__global__ void __launch_bounds__(128 * TPB) k_laplacian_fused(Topo tp, const int* __restrict__ list, int n, const int4* __restrict__ items,
                                                               int nitems, int item_blocks,
                                                               const float* __restrict__ X, float* __restrict__ Y,
                                                               float* __restrict__ GACC, const Scalars* __restrict__ S,
                                                               double* __restrict__ WP) {
    k_laplacian_fused_body<TPB, NT>(tp, list, n, items, nitems, item_blocks, X, Y, GACC, S, WP);
}
// the same kernel with at least MINB CTAs per SM (registers capped to fit)
template <int TPB, int NT, int MINB>
__global__ void __launch_bounds__(128 * TPB, MINB) k_laplacian_fused_occ(Topo tp, const int* __restrict__ list, int n, const int4* __restrict__ items,
                                                               int nitems, int item_blocks,
                                                               const float* __restrict__ X, float* __restrict__ Y,
                                                               float* __restrict__ GACC, const Scalars* __restrict__ S,
                                                               double* __restrict__ WP) {
    k_laplacian_fused_body<TPB, NT>(tp, list, n, items, nitems, item_blocks, X, Y, GACC, S, WP);
}
template <int TPB, int NT, int MINB>
constexpr auto k_laplacian_fused_shape() {
    if constexpr (MINB == 0) return &k_laplacian_fused<TPB, NT>;
    else return &k_laplacian_fused_occ<TPB, NT, MINB>;
}

// AccumulateToParents128Kernel on GHOST tiles, additive, coefficient 1, all cell types
// (src/PoissonGrid.cu:664-710).  2x2x2 sums in the reference's (ii,jj,kk) order.
template <class T>
__global__ void __launch_bounds__(64) k_accumulate_ghosts(Topo tp, const int* __restrict__ list, int n, T* Y,
                                                          const Scalars* __restrict__ S) {
    pdl_entry();
    const int q = blockIdx.x;
    if (q >= n) return;
    const int tile = list[q];
    if (tile_done(tp, S, tile)) return;
    const TileMeta m = tp.meta[tile];
    if (m.parent < 0) return;
    const int b = threadIdx.x;
    const int fi = b / 16 * 2, fj = (b / 4) % 4 * 2, fk = b % 4 * 2;
    const size_t base = (size_t)tile * kTileCells;
    T sum = T(0);
#pragma unroll
    for (int ii = 0; ii < 2; ii++)
#pragma unroll
        for (int jj = 0; jj < 2; jj++)
#pragma unroll
            for (int kk = 0; kk < 2; kk++) {
                const size_t id = base + (fi + ii) * 64 + (fj + jj) * 8 + (fk + kk);
                sum += (tp.ctype[id] & (INTERIOR_C | DIRICHLET_C | NEUMANN_C)) ? Y[id] : T(0);
            }
    const int oct = meta_octant(m.packed);
    const size_t pid = (size_t)m.parent * kTileCells + ((oct & 1) * 4 + fi / 2) * 64 + (((oct >> 1) & 1) * 4 + fj / 2) * 8 +
                       ((oct >> 2) & 1) * 4 + fk / 2;
    Y[pid] = Y[pid] + sum;
}

// ------------------------------------------------------------------ Gauss-Seidel colour sweep
// NegativeLaplacianAndGaussSeidelSameLevel128Kernel (src/GMGSolver.cu:216-269): on LEAF|NONLEAF
// tiles of one level (NONLEAF counted as LEAF), cells of one colour (i+j+k)%2:
// x += (b - A x) / D on INTERIOR cells.
// The tiles of a CTA are NT groups of TPB consecutive list entries, one 128-thread group per
// tile, all staged with asynchronous copies before any is computed (NT tiles per group in flight).
// With RD (the PCG residual r) the sweep also forms, for every LEAF tile it updates, the tile's
// part of the next r.z (DotAsync, src/GMGSolver.cu:636-640) and stores it at WP[LEAF slot]; the
// tile part is tile_part_sum of the threads' 4-cell FP32 products.  A LEAF tile's z is final
// after this sweep (finer levels only read it).  Its r is the staged right-hand side unless GHOST
// children added their residuals to that copy; then r is read.
template <int TPB, int NT>
__device__ __forceinline__ void k_gs_sweep_body(Topo tp, const int* __restrict__ list, int n, float* X,
                                                        const float* __restrict__ R, int color, const Scalars* __restrict__ S,
                                                        const float* __restrict__ RD, double* __restrict__ WP) {
    // the dot-part tail gives tile u to 16-lane half (u & 1) of warp 2 + (u >> 1): NT <= 4
    static_assert(NT >= 1 && NT <= 4, "k_gs_sweep: the tile-part tail covers at most 4 tiles per group");
    pdl_trigger();
    extern __shared__ __align__(16) unsigned char gs_smem[];
    TileStage* st = reinterpret_cast<TileStage*>(gs_smem);
    const int g = threadIdx.x >> 7, t = threadIdx.x & 127;
    int tile[NT], ptile[NT];
    bool act[NT];
#pragma unroll
    for (int u = 0; u < NT; u++) {
        const int q = (blockIdx.x * NT + u) * TPB + g;
        tile[u] = q < n ? list[q] : 0;
        act[u] = q < n;  // finished instances are dropped after the copies are issued (reading them is harmless)
        ptile[u] = (tp.pf > 0 && t == 0 && q + tp.pf < n) ? list[q + tp.pf] : -1;
    }
    TilePre pre[NT];
    tile_pre(tp, tile, t, pre);
    pdl_wait();
#pragma unroll
    for (int u = 0; u < NT; u++)
        if (act[u]) {
            stage_async(X, R, tp.mask_mg, tile[u], pre[u].nb, t, st[u * TPB + g]);
            if (RD != nullptr && t == 0) cp_async4(st[u * TPB + g].aux, tp.leafslot + tile[u]);
        }
#pragma unroll
    for (int u = 0; u < NT; u++)
        if (ptile[u] >= 0) {
            prefetch_l2(X + (size_t)ptile[u] * kTileCells, kTileCells * sizeof(float));
            prefetch_l2(R + (size_t)ptile[u] * kTileCells, kTileCells * sizeof(float));
            prefetch_l2(tp.mask_mg + (size_t)ptile[u] * kTileCells, kTileCells);
        }
#pragma unroll
    for (int u = 0; u < NT; u++) act[u] = act[u] && !tile_done(tp, S, tile[u]);
    cp_async_wait_all();
    __syncthreads();
#pragma unroll
    for (int u = 0; u < NT; u++) {
        if (!act[u]) continue;
        TileStage& ts = st[u * TPB + g];
        const LevelConst<float> L(pre[u].lc);
        const uint32_t mask4 = *reinterpret_cast<const uint32_t*>(ts.mask + t * 4);
        const size_t off = (size_t)tile[u] * kTileCells + t * 4;
        const V4<float> b = ld4(ts.b + t * 4);
        const V4<float> z = colour_update(ts.xs, ts.hx, t, mask4, (pre[u].fcls >> 12) & 0xfffu, L, b, color);
        st4(X + off, z);
        if (RD != nullptr) {  // the thread's term, in its own (already read) mask bytes
            const int sl = ts.aux[0];
            if (sl != -1) reinterpret_cast<float*>(ts.mask)[t] = dot4f32(sl >= 0 ? b : ld4(RD + off), z);
        }
    }
    if (RD == nullptr) return;
    __syncthreads();
    // warps 0 and 1 of each group sum the terms, each 16-lane half one tile: u = 2 * warp + half
    const int u = 2 * (t >> 5) + ((t >> 4) & 1);
    if (t >= 64 || 2 * (t >> 5) >= NT) return;  // whole warps
    bool ok = false;
#pragma unroll
    for (int k = 0; k < NT; k++)
        if (k == u) ok = act[k];
    const TileStage& ts = st[(u < NT ? u : 0) * TPB + g];
    const int sl = ts.aux[0];
    const double d = tile_part_sum(reinterpret_cast<const float*>(ts.mask), t & 15);
    if (ok && u < NT && sl != -1 && (t & 15) == 0) WP[sl >= 0 ? sl : -2 - sl] = d;
}
template <int TPB, int NT>
__global__ void __launch_bounds__(128 * TPB) k_gs_sweep(Topo tp, const int* __restrict__ list, int n, float* X,
                                                        const float* __restrict__ R, int color, const Scalars* __restrict__ S,
                                                        const float* __restrict__ RD, double* __restrict__ WP) {
    k_gs_sweep_body<TPB, NT>(tp, list, n, X, R, color, S, RD, WP);
}
// the same kernel with at least MINB CTAs per SM (registers capped to fit)
template <int TPB, int NT, int MINB>
__global__ void __launch_bounds__(128 * TPB, MINB) k_gs_sweep_occ(Topo tp, const int* __restrict__ list, int n, float* X,
                                                        const float* __restrict__ R, int color, const Scalars* __restrict__ S,
                                                        const float* __restrict__ RD, double* __restrict__ WP) {
    k_gs_sweep_body<TPB, NT>(tp, list, n, X, R, color, S, RD, WP);
}
template <int TPB, int NT, int MINB>
constexpr auto k_gs_sweep_shape() {
    if constexpr (MINB == 0) return &k_gs_sweep<TPB, NT>;
    else return &k_gs_sweep_occ<TPB, NT, MINB>;
}

// A whole sequence of colour sweeps over a small level inside one CTA (used for the coarsest
// level: GaussSeidelGMG(5, 0) + GaussSeidelGMG(5, 1), src/GMGSolver.cu:432-433).  Global-memory
// writes of one sweep are made visible to the next sweep's halo loads by __syncthreads.
__global__ void __launch_bounds__(1024) k_gs_sequence(Topo tp, const int* __restrict__ list, int n, float* X,
                                                      const float* __restrict__ R, uint32_t colors, int nsweeps,
                                                      const Scalars* __restrict__ S) {
    pdl_entry();
    __shared__ TileShared<float> sh[8];
    const int groups = blockDim.x >> 7;
    const int g = threadIdx.x >> 7, t = threadIdx.x & 127;
    for (int s = 0; s < nsweeps; s++) {
        const int color = (colors >> s) & 1;
        for (int base = 0; base < n; base += groups) {
            const int q = base + g;
            const int tile = q < n ? list[q] : 0;
            const bool active = q < n && !tile_done(tp, S, tile);
            TileMeta m;
            if (active) {
                m = tp.meta[tile];
                stage_tile<float>(X, tile, m, t, sh[g]);
            }
            __syncthreads();
            if (active) {
                const uint32_t mask4 = *reinterpret_cast<const uint32_t*>(tp.mask_mg + (size_t)tile * kTileCells + t * 4);
                const V4<float> b = ld4(R + (size_t)tile * kTileCells + t * 4);
                const LevelConst<float> L = tile_level_const(tp, tile, meta_level(m.packed));
                st4(X + (size_t)tile * kTileCells + t * 4,
                    colour_update(sh[g].xs, sh[g].hx, t, mask4, (tp.fcls[tile] >> 12) & 0xfffu, L, b, color));
            }
            __syncthreads();
        }
    }
}

// ------------------------------------------------------------------ residual + restriction
// Face path of the residual + restriction for one coarse cell of a GHOST tile whose x and
// right-hand side are 0 (the fused V-cycle keeps them so) and whose coupled cells all lie on its
// faces, coupled only outward.  Item: tile, coarse cell c | coupled faces << 6 | face classes <<
// 12 | octant << 24, parent tile, level-constant index.  r = 0 - A x on the block's cells (A x
// from the neighbours' values across coupled faces, fused as the full path rounds it; +0 on
// uncoupled cells), summed in (ii,jj,kk) order and added to the parent cell.
__device__ __forceinline__ void ghost_face_restrict(const Topo& tp, const float* __restrict__ X, int4 it, float* C) {
    const int tile = it.x, c = it.y & 63;
    const uint32_t faces = ((uint32_t)it.y >> 6) & 63u, cls = ((uint32_t)it.y >> 12) & 0xfffu;
    const int oct = ((uint32_t)it.y >> 24) & 7u;
    const int fi = c / 16 * 2, fj = (c / 4) % 4 * 2, fk = c % 4 * 2;
    const uint32_t touch = (fi == 0 ? 1u : 0u) | (fi == 6 ? 2u : 0u) | (fj == 0 ? 4u : 0u) | (fj == 6 ? 8u : 0u) | (fk == 0 ? 16u : 0u) |
                           (fk == 6 ? 32u : 0u);
    const uint32_t act = touch & faces;
    float sum = 0.f;
    if (act) {
        const size_t base = (size_t)tile * kTileCells;
        const int o0 = fi * 64 + fj * 8 + fk;
        uint32_t mk[4];
#pragma unroll
        for (int q = 0; q < 4; q++) mk[q] = *reinterpret_cast<const uint16_t*>(tp.mask_mg + base + o0 + (q >> 1) * 64 + (q & 1) * 8);
        const TileMeta& m = tp.meta[tile];
        float nv[6][4];
#pragma unroll
        for (int f = 0; f < 6; f++) {
            const int nb = ((act >> f) & 1u) ? m.nb[f] : -1;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int a = q >> 1, b = q & 1;
                int noff;
                if (f == 0) noff = 7 * 64 + (fj + a) * 8 + fk + b;
                else if (f == 1) noff = (fj + a) * 8 + fk + b;
                else if (f == 2) noff = (fi + a) * 64 + 7 * 8 + fk + b;
                else if (f == 3) noff = (fi + a) * 64 + fk + b;
                else if (f == 4) noff = (fi + a) * 64 + (fj + b) * 8 + 7;
                else noff = (fi + a) * 64 + (fj + b) * 8;
                nv[f][q] = nb >= 0 ? X[(size_t)nb * kTileCells + noff] : 0.f;
            }
        }
        const LevelConst<float> L(tp.lconst[it.w]);
#pragma unroll
        for (int ii = 0; ii < 2; ii++)
#pragma unroll
            for (int jj = 0; jj < 2; jj++)
#pragma unroll
                for (int kk = 0; kk < 2; kk++) {
                    const int i = fi + ii, j = fj + jj, k = fk + kk;
                    const uint32_t on = (i == 0 ? 1u : 0u) | (i == 7 ? 2u : 0u) | (j == 0 ? 4u : 0u) | (j == 7 ? 8u : 0u) |
                                        (k == 0 ? 16u : 0u) | (k == 7 ? 32u : 0u);
                    const uint32_t mm = (mk[ii * 2 + jj] >> (8 * kk)) & 0xffu;
                    float r = 0.f;
                    if ((on & act) && (mm & 0x3Fu)) {
                        float s = 0.f;
#pragma unroll
                        for (int f = 0; f < 6; f++) {
                            if (!(mm & (1u << f))) continue;
                            const float a = ((cls >> (2 * f)) & 3u) == 2u ? L.c2 : L.c1;
                            const float xf = nv[f][f < 2 ? jj * 2 + kk : (f < 4 ? ii * 2 + kk : ii * 2 + jj)];
                            s = fmaf(a, 0.f - xf, s);
                        }
                        const float ax = (mm & kMaskInterior) ? s * L.h * L.h * L.h : 0.f;
                        r = 0.f - ax;
                    }
                    sum += r;
                }
    } else {
#pragma unroll
        for (int e = 0; e < 8; e++) sum += 0.f;
    }
    C[(size_t)it.z * kTileCells + ((oct & 1) * 4 + fi / 2) * 64 + (((oct >> 1) & 1) * 4 + fj / 2) * 8 + ((oct >> 2) & 1) * 4 + fk / 2] += sum;
}

// ResidualAndRestrict128Kernel (src/GMGSolver.cu:284-339): r = rhs - A x on every cell of the
// level's tiles; 2x2x2 sums go to the parent cell: GHOST tiles add, others overwrite
// (times one_over_alpha).  The staged path takes tiles list[0..n) (or first..first+n when list is
// null); the first item_blocks CTAs take face-path GHOST cells (ghost_face_restrict), one per
// thread.
template <int TPB, int NT>
__device__ __forceinline__ void k_residual_restrict_body(Topo tp, int first, const int* __restrict__ list, int n,
                                                                 const int4* __restrict__ items, int nitems, int item_blocks,
                                                                 const float* __restrict__ X, const float* RHS, float* C,
                                                                 float one_over_alpha, const Scalars* __restrict__ S) {
    pdl_trigger();
    if ((int)blockIdx.x < item_blocks) {
        pdl_wait();
        const int q = (int)blockIdx.x * (128 * TPB) + (int)threadIdx.x;
        if (q >= nitems) return;
        const int4 it = items[q];
        if (S != nullptr && S[it.w / kLevelSlots].done) return;
        ghost_face_restrict(tp, X, it, C);
        return;
    }
    extern __shared__ __align__(16) unsigned char rr_smem[];
    TileStage* st = reinterpret_cast<TileStage*>(rr_smem);
    const int g = threadIdx.x >> 7, t = threadIdx.x & 127;
    int tile[NT], ptile[NT];
    bool act[NT];
#pragma unroll
    for (int u = 0; u < NT; u++) {
        const int q = (((int)blockIdx.x - item_blocks) * NT + u) * TPB + g;
        const int qq = q < n ? q : 0;
        tile[u] = list ? list[qq] : first + qq;
        act[u] = q < n;  // finished instances are dropped after the copies are issued (reading them is harmless)
        ptile[u] = (tp.pf > 0 && t == 0 && q + tp.pf < n) ? (list ? list[q + tp.pf] : first + q + tp.pf) : -1;
    }
    TilePre pre[NT];
    tile_pre(tp, tile, t, pre);
    pdl_wait();
#pragma unroll
    for (int u = 0; u < NT; u++)
        if (act[u]) stage_async(X, RHS, tp.mask_mg, tile[u], pre[u].nb, t, st[u * TPB + g]);
#pragma unroll
    for (int u = 0; u < NT; u++)
        if (ptile[u] >= 0) {
            prefetch_l2(X + (size_t)ptile[u] * kTileCells, kTileCells * sizeof(float));
            prefetch_l2(RHS + (size_t)ptile[u] * kTileCells, kTileCells * sizeof(float));
            prefetch_l2(tp.mask_mg + (size_t)ptile[u] * kTileCells, kTileCells);
        }
#pragma unroll
    for (int u = 0; u < NT; u++) act[u] = act[u] && !tile_done(tp, S, tile[u]);
    cp_async_wait_all();
    __syncthreads();
#pragma unroll
    for (int u = 0; u < NT; u++) {
        if (!act[u]) continue;
        TileStage& ts = st[u * TPB + g];
        const LevelConst<float> L(pre[u].lc);
        float ax[4], d[4];
        neg_lap4<float, false>(ts.xs, ts.hx, t, *reinterpret_cast<const uint32_t*>(ts.mask + t * 4), (pre[u].fcls >> 12) & 0xfffu, L,
                               ax, d);
        const V4<float> b = ld4(ts.b + t * 4);
        V4<float> r;
#pragma unroll
        for (int e = 0; e < 4; e++) r.v[e] = b.v[e] - ax[e];
        st4(ts.b + t * 4, r);  // the residual replaces the thread's own right-hand side values
    }
    __syncthreads();
    if (t >= 64) return;
    const int fi = t / 16 * 2, fj = (t / 4) % 4 * 2, fk = t % 4 * 2;
#pragma unroll
    for (int u = 0; u < NT; u++) {
        if (!act[u]) continue;
        const TileMeta m = tp.meta[tile[u]];
        if (m.parent < 0) continue;
        const float* res = st[u * TPB + g].b;
        float sum = 0.f;
#pragma unroll
        for (int ii = 0; ii < 2; ii++)
#pragma unroll
            for (int jj = 0; jj < 2; jj++)
#pragma unroll
                for (int kk = 0; kk < 2; kk++) sum += res[(fi + ii) * 64 + (fj + jj) * 8 + (fk + kk)];
        const int oct = meta_octant(m.packed);
        const size_t pid = (size_t)m.parent * kTileCells + ((oct & 1) * 4 + fi / 2) * 64 + (((oct >> 1) & 1) * 4 + fj / 2) * 8 +
                           ((oct >> 2) & 1) * 4 + fk / 2;
        if (meta_type(m.packed) & GHOST_T) C[pid] += sum;
        else C[pid] = sum * one_over_alpha;
    }}
template <int TPB, int NT>
__global__ void __launch_bounds__(128 * TPB) k_residual_restrict(Topo tp, int first, const int* __restrict__ list, int n,
                                                                 const int4* __restrict__ items, int nitems, int item_blocks,
                                                                 const float* __restrict__ X, const float* RHS, float* C,
                                                                 float one_over_alpha, const Scalars* __restrict__ S) {
    k_residual_restrict_body<TPB, NT>(tp, first, list, n, items, nitems, item_blocks, X, RHS, C, one_over_alpha, S);
}
// the same kernel with at least MINB CTAs per SM (registers capped to fit)
template <int TPB, int NT, int MINB>
__global__ void __launch_bounds__(128 * TPB, MINB) k_residual_restrict_occ(Topo tp, int first, const int* __restrict__ list, int n,
                                                                 const int4* __restrict__ items, int nitems, int item_blocks,
                                                                 const float* __restrict__ X, const float* RHS, float* C,
                                                                 float one_over_alpha, const Scalars* __restrict__ S) {
    k_residual_restrict_body<TPB, NT>(tp, first, list, n, items, nitems, item_blocks, X, RHS, C, one_over_alpha, S);
}
template <int TPB, int NT, int MINB>
constexpr auto k_residual_restrict_shape() {
    if constexpr (MINB == 0) return &k_residual_restrict<TPB, NT>;
    else return &k_residual_restrict_occ<TPB, NT, MINB>;
}

// ------------------------------------------------------------------ prolongation + update
// ProlongateAndUpdate128Kernel (src/GMGSolver.cu:345-376): injection of the parent value;
// GHOST: x = cx, others: x += prolong_coeff * cx; INTERIOR cells only (0 elsewhere).
__global__ void __launch_bounds__(128) k_prolongate(Topo tp, int first, int n, const float* __restrict__ CX, float* FX,
                                                    float prolong_coeff, const Scalars* __restrict__ S) {
    pdl_entry();
    const int q = blockIdx.x;
    if (q >= n) return;
    const int tile = first + q;
    if (tile_done(tp, S, tile)) return;
    const int t = threadIdx.x;
    const TileMeta m = tp.meta[tile];
    const TileIdx ix(t);
    const uint32_t ct4 = *reinterpret_cast<const uint32_t*>(tp.ctype + (size_t)tile * kTileCells + t * 4);
    float c[2] = {0.f, 0.f};
    if (m.parent >= 0) {
        const int oct = meta_octant(m.packed);
        const size_t pbase = (size_t)m.parent * kTileCells + ((oct & 1) * 4 + (ix.i >> 1)) * 64 +
                             (((oct >> 1) & 1) * 4 + (ix.j >> 1)) * 8 + ((oct >> 2) & 1) * 4 + (ix.k0 >> 1);
        c[0] = CX[pbase];
        c[1] = CX[pbase + 1];
    }
    const bool ghost = meta_type(m.packed) & GHOST_T;
    float* p = FX + (size_t)tile * kTileCells + t * 4;
    V4<float> fx = ld4(p);
#pragma unroll
    for (int e = 0; e < 4; e++) {
        const bool interior = (ct4 >> (8 * e)) & INTERIOR_C;
        const float cx = c[e >> 1];
        fx.v[e] = interior ? (ghost ? cx : fmaf(prolong_coeff, cx, fx.v[e])) : 0.f;
    }
    st4(p, fx);
}

// V-cycle initialisation (src/GMGSolver.cu:386-403): x = 0 everywhere; rhs = f on LEAF and
// NONLEAF tiles, 0 on GHOST tiles.
__global__ void __launch_bounds__(256) k_vcycle_init(Topo tp, int n, float* X, float* RHS, const float* __restrict__ F,
                                                     const Scalars* __restrict__ S) {
    pdl_entry();
    const size_t nv = (size_t)n * (kTileCells / 4);
    for (size_t v = (size_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += (size_t)gridDim.x * blockDim.x) {
        const int tile = (int)(v >> 7);
        if (tile_done(tp, S, tile)) continue;
        const bool ghost = meta_type(tp.meta[tile].packed) & GHOST_T;
        st4(X + v * 4, zero4<float>());
        st4(RHS + v * 4, ghost ? zero4<float>() : ld4(F + v * 4));
    }
}

// ------------------------------------------------------------------ reductions over LEAF tiles
// Deterministic two-level sum: fixed grid-stride assignment, warp-shuffle trees, partials per
// CTA, and the last CTA to finish (ticket counter) sums the partials in a fixed order and runs
// the epilogue on the scalar state.  Per 4-cell vector the FP32 products are formed as the
// reference's Dot128Kernel does (src/PoissonGrid.cu:177-181) and widened to FP64.
struct Double2 { double a, b; };

// Block-reduce (a, b), publish the partial, return true in thread 0 of the last CTA with the
// grand total in `tot`.
__device__ __forceinline__ bool reduce_and_elect(double a, double b, double* partials, unsigned int* counter, Double2& tot) {
    __shared__ double wa[32], wb[32];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    a = warp_sum(a);
    b = warp_sum(b);
    if (lane == 0) { wa[w] = a; wb[w] = b; }
    __syncthreads();
    if (w == 0) {
        a = lane < nw ? wa[lane] : 0.0;
        b = lane < nw ? wb[lane] : 0.0;
        a = warp_sum(a);
        b = warp_sum(b);
        if (lane == 0) {
            partials[2 * blockIdx.x] = a;
            partials[2 * blockIdx.x + 1] = b;
            __threadfence();
            const unsigned int ticket = atomicAdd(counter, 1u);
            last = (ticket == gridDim.x - 1);
        }
    }
    __syncthreads();
    if (!last) return false;
    if (w == 0) {
        __threadfence();
        double sa = 0.0, sb = 0.0;
        for (int i = lane; i < (int)gridDim.x; i += 32) {
            sa += __ldcg(partials + 2 * i);
            sb += __ldcg(partials + 2 * i + 1);
        }
        sa = warp_sum(sa);
        sb = warp_sum(sb);
        if (lane == 0) {
            tot.a = sa;
            tot.b = sb;
            *counter = 0u;
        }
    }
    return threadIdx.x == 0;
}

__device__ __forceinline__ void set_cond(const SolveCtl& c, unsigned int v) {
    if (c.use_cond) cudaGraphSetConditional(c.cond, v);
}

// Instance `inst` stops iterating: the last instance to stop ends the graph's while loop.
__device__ __forceinline__ void finish(Scalars* S, const SolveCtl& c) {
    S->done = 1;
    if (c.active && atomicSub(c.active, 1) == 1) set_cond(c, 0u);
}

// Scalar epilogues of the PCG (src/GMGSolver.cu:540-653) for one instance, executed by one thread.
__device__ void epilogue(int which, const Double2& tot, Scalars* S, const InstParams& P, const SolveCtl& c, int inst) {
    switch (which) {
    case EPI_INIT: {  // rhs_norm2, zero-RHS early exit, threshold
        S->rhs2 = tot.a;
        S->iter = 0;
        S->converged = 0;
        if (c.sync_stride > 0) {
            if (tot.a == 0.0) {
                S->converged = 1; S->iters = 0; S->rel = 0.0;
                finish(S, c);
                return;
            }
            const double thr = P.tol * P.tol * tot.a;
            S->thr2 = thr > 2.2250738585072014e-308 ? thr : 2.2250738585072014e-308;
        }
        if (P.max_iters <= 0) finish(S, c);
        break;
    }
    case EPI_GAMMA: S->gamma = tot.a; break;
    case EPI_ALPHA: S->fp = tot.a; S->alpha = S->gamma / tot.a; break;
    case EPI_CHECK: {
        const int i = S->iter;
        S->iter = i + 1;
        S->res2 = tot.a;
        if (c.sync_stride > 0 && (i + 1) % c.sync_stride == 0) {
            if (inst == 0 && c.history && i < c.history_cap) c.history[i] = sqrt(tot.a / S->rhs2);
            if (tot.a < S->thr2) {
                S->converged = 1; S->iters = i + 1; S->rel = sqrt(tot.a / S->rhs2);
                finish(S, c);
                return;
            }
            if (!(tot.a == tot.a) || isinf(tot.a)) {  // non-finite residual: stop, report
                S->nonfinite = 1; S->iters = i + 1; S->rel = tot.a;
                finish(S, c);
                return;
            }
        }
        if (i + 1 >= P.max_iters) {
            // the reference's loop runs its last iteration to the end: a pure-Neumann r is
            // recentred before the loop exits, so such an instance stops at EPI_BETA
            if (P.pure_neumann) S->capped = 1;
            else finish(S, c);
        }
        break;
    }
    case EPI_BETA:
        if (S->capped) {  // the iteration cap of a pure-Neumann instance (EPI_CHECK)
            finish(S, c);
            return;
        }
        S->gamma_old = S->gamma; S->gamma = tot.a; S->beta = tot.a / S->gamma_old;
        break;
    case EPI_MEAN: S->mean = tot.a / tot.b; break;
    case EPI_FINAL:
        if (!S->converged && !S->nonfinite) {
            S->iters = S->iter;
            S->res2 = tot.a;
            S->rel = c.sync_stride > 0 ? sqrt(tot.a / S->rhs2) : -1.0;
        }
        break;
    }
}

// Whole-grid dot over the 4-cell vectors of LEAF tiles (Dot, src/PoissonGrid.cu:199-228):
// grid-stride over the leaf list, per-vector FP32 products widened to FP64, the two-level
// deterministic sum of reduce_and_elect; the sum goes to S->gamma.
__global__ void __launch_bounds__(256) k_leaf_dot(const int* __restrict__ leaves, int nleaf, const float* __restrict__ A,
                                                  const float* __restrict__ B, Scalars* S, double* partials,
                                                  unsigned int* counter) {
    pdl_entry();
    double acc = 0.0;
    const size_t nv = (size_t)nleaf * 128;
    for (size_t v = (size_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += (size_t)gridDim.x * blockDim.x) {
        const size_t off = (size_t)leaves[v >> 7] * kTileCells + (v & 127) * 4;
        acc += dot4f(ld4(A + off), ld4(B + off));
    }
    Double2 tot{0.0, 0.0};
    if (reduce_and_elect(acc, 0.0, partials, counter, tot)) S->gamma = tot.a;
}

// Block-reduce (a, b) of one chunk, publish it as the chunk's partial, and in thread 0 of the
// instance's last chunk CTA return true with the instance's total, the chunk partials added in
// chunk order (fixed: the bits depend only on the instance's own data).
__device__ __forceinline__ bool chunk_reduce_and_elect(double a, double b, double* partials, unsigned int* counter, int2 ich,
                                                       Double2& tot) {
    __shared__ double wa[32], wb[32];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    a = warp_sum(a);
    b = warp_sum(b);
    if (lane == 0) { wa[w] = a; wb[w] = b; }
    __syncthreads();
    if (w == 0) {
        a = lane < nw ? wa[lane] : 0.0;
        b = lane < nw ? wb[lane] : 0.0;
        a = warp_sum(a);
        b = warp_sum(b);
        if (lane == 0) {
            partials[2 * blockIdx.x] = a;
            partials[2 * blockIdx.x + 1] = b;
            __threadfence();
            const unsigned int ticket = atomicAdd(counter, 1u);
            last = (ticket == (unsigned int)ich.y - 1u);
        }
    }
    __syncthreads();
    if (!last) return false;
    if (w == 0) {
        __threadfence();
        double sa = 0.0, sb = 0.0;
        for (int i = lane; i < ich.y; i += 32) {
            sa += __ldcg(partials + 2 * (ich.x + i));
            sb += __ldcg(partials + 2 * (ich.x + i) + 1);
        }
        sa = warp_sum(sa);
        sb = warp_sum(sb);
        if (lane == 0) {
            tot.a = sa;
            tot.b = sb;
            *counter = 0u;
        }
    }
    return threadIdx.x == 0;
}

// PropagateValuesToGhostTiles (src/PoissonGrid.cu:585-605) for the GHOST child, if any, of the
// octant holding the four cells (i, j, k0..k0+3) of vector qv of LEAF tile `tile`: the 2x2x2
// children of each cell take its new value p where child and parent cell are INTERIOR, 0
// elsewhere.  Every GHOST tile is the child of a LEAF tile, so the kernels that write p on LEAF
// tiles keep p valid on the GHOST tiles and the fused Laplacian reads it there directly.  Only
// the cells other tiles read are written: the faces towards non-GHOST neighbours (their halos and
// the Laplacian's face path), or every cell of a GHOST tile on the staged path (ghost_faces).
__device__ __forceinline__ void push_to_ghost_child(const Topo& tp, float* P, int tile, int qv, const V4<float>& p, uint32_t ct4) {
    const int i = qv >> 4, j = (qv >> 1) & 7, k0 = (qv & 1) * 4;
    const int gs = tp.ghost_child[(size_t)tile * 8 + ((i >> 2) | ((j >> 2) << 1) | ((k0 >> 2) << 2))];
    if (gs < 0) return;
    const uint32_t faces = tp.ghost_faces[gs];
    if (faces == 0) return;
    const int gt = tp.ghost_list[gs];
    float pv[4];
#pragma unroll
    for (int e = 0; e < 4; e++) pv[e] = ((ct4 >> (8 * e)) & INTERIOR_C) ? p.v[e] : 0.f;
#pragma unroll
    for (int di = 0; di < 2; di++)
#pragma unroll
        for (int dj = 0; dj < 2; dj++) {
            const int fi = 2 * (i & 3) + di, fj = 2 * (j & 3) + dj;
            const size_t row = (size_t)gt * kTileCells + fi * 64 + fj * 8;
            const bool whole = (faces & 0x40u) || ((faces & 1u) && fi == 0) || ((faces & 2u) && fi == 7) || ((faces & 4u) && fj == 0) ||
                               ((faces & 8u) && fj == 7);
            if (whole) {
                const uint2 cc = *reinterpret_cast<const uint2*>(tp.ctype + row);
                V4<float> lo, hi;
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    lo.v[k] = ((cc.x >> (8 * k)) & INTERIOR_C) ? pv[k >> 1] : 0.f;
                    hi.v[k] = ((cc.y >> (8 * k)) & INTERIOR_C) ? pv[2 + (k >> 1)] : 0.f;
                }
                st4(P + row, lo);
                st4(P + row + 4, hi);
            } else {
                // only the row's end cells can lie on a read face (z- at k = 0, z+ at k = 7)
                if (faces & 16u) P[row] = (tp.ctype[row] & INTERIOR_C) ? pv[0] : 0.f;
                if (faces & 32u) P[row + 7] = (tp.ctype[row + 7] & INTERIOR_C) ? pv[3] : 0.f;
            }
        }
}

// The multigrid right-hand side copy of r for vector qv of LEAF tile `tile`.  Under a GHOST child
// (a cell whose right-hand side the child's restriction adds to) -0 becomes +0: the reference
// adds the child's 2x2x2 sum to every such cell, which turns -0 into +0 even where the sum is
// +0, and the restriction's face path skips the cells whose sum is known to be +0.
__device__ __forceinline__ V4<float> mg_rhs_copy(const Topo& tp, int tile, int qv, const V4<float>& r) {
    const int i = qv >> 4, j = (qv >> 1) & 7, k0 = (qv & 1) * 4;
    if (tp.ghost_child[(size_t)tile * 8 + ((i >> 2) | ((j >> 2) << 1) | ((k0 >> 2) << 2))] < 0) return r;
    V4<float> c;
#pragma unroll
    for (int e = 0; e < 4; e++) c.v[e] = r.v[e] + 0.f;
    return c;
}

// Per-instance reduction over the 4-cell vectors of LEAF tiles, one CTA per chunk (the chunk table
// cuts every instance's leaf vectors into pieces of kChunkVecs).  OP selects the fused
// elementwise work done while reducing:
//   OP_DOT       a.b                                  (Dot)
//   OP_INIT      x = 0; D = r; r.r                    (Fill + Dot, src/GMGSolver.cu:537-542)
//   OP_COPY_DOT  p = z; z.r                           (Copy + DotAsync, :564-568)
//   OP_XR        r -= a Ap (INTERIOR); D = r; r.r      (:587-612; its x += a p is applied by k_update_p,
//                which reads p anyway, and after the loop by k_x_final)
//   OP_MEAN      (sum of 4 values, 2*#INTERIOR)       (MeanAsync, src/PoissonGrid.cu:231-325)
// skip: SKIP_DONE leaves out finished instances, SKIP_INACTIVE only those outside the solve;
// OP_MEAN also leaves out instances that are not pure Neumann.
template <int OP>
__global__ void __launch_bounds__(256) k_inst_reduce(Topo tp, const int* __restrict__ leaves, const int4* __restrict__ chunks,
                                                     const int2* __restrict__ inst_chunks, float* A, float* B, float* C, float* D,
                                                     Scalars* S, const InstParams* __restrict__ ip, SolveCtl ctl, int epi,
                                                     double* partials, unsigned int* counters, int skip) {
    pdl_trigger();
    const int4 ch = chunks[blockIdx.x];  // topology: read before pdl_wait
    pdl_wait();
    const int inst = ch.x;
    Scalars* Si = S + inst;
    const InstParams P = ip[inst];
    if (!P.active || (skip == SKIP_DONE && Si->done) || (OP == OP_MEAN && !P.pure_neumann)) return;
    double acc_a = 0.0, acc_b = 0.0;
    float alpha = 0.f;
    if (OP == OP_XR) alpha = (float)Si->alpha;
    for (int v = ch.y + threadIdx.x; v < ch.z; v += blockDim.x) {
        const int tile = leaves[v >> 7];
        const size_t off = (size_t)tile * kTileCells + (v & 127) * 4;
        if (OP == OP_DOT) {
            acc_a += dot4f(ld4(A + off), ld4(B + off));
        } else if (OP == OP_INIT) {  // A = x, B = r, D = multigrid right-hand side (copy of r)
            st4(A + off, zero4<float>());
            const V4<float> r = ld4(B + off);
            if (D) st4(D + off, mg_rhs_copy(tp, tile, v & 127, r));
            acc_a += dot4f(r, r);
        } else if (OP == OP_COPY_DOT) {  // A = z, B = r, C = p (also on the GHOST children)
            const V4<float> z = ld4(A + off);
            st4(C + off, z);
            push_to_ghost_child(tp, C, tile, v & 127, z, *reinterpret_cast<const uint32_t*>(tp.ctype + off));
            acc_a += dot4f(z, ld4(B + off));
        } else if (OP == OP_XR) {  // C = r, D = Ap
            const uint32_t ct4 = *reinterpret_cast<const uint32_t*>(tp.ctype + off);
            V4<float> r = ld4(C + off);
            const V4<float> ap = ld4(D + off);
#pragma unroll
            for (int e = 0; e < 4; e++)
                if ((ct4 >> (8 * e)) & INTERIOR_C) r.v[e] = fmaf(-alpha, ap.v[e], r.v[e]);
            st4(C + off, r);
            st4(D + off, mg_rhs_copy(tp, tile, v & 127, r));  // Ap is consumed; the channel now carries r as the multigrid right-hand side
            acc_a += dot4f(r, r);
        } else if (OP == OP_MEAN) {  // A = channel
            const V4<float> a = ld4(A + off);
            acc_a += (double)(a.v[0] + a.v[1] + a.v[2] + a.v[3]);
            const uint32_t ct4 = *reinterpret_cast<const uint32_t*>(tp.ctype + off);
            acc_b += (double)((ct4 & INTERIOR_C) + ((ct4 >> 8) & INTERIOR_C) + ((ct4 >> 16) & INTERIOR_C) + ((ct4 >> 24) & INTERIOR_C));
        }
    }
    Double2 tot{0.0, 0.0};
    if (chunk_reduce_and_elect(acc_a, acc_b, partials, counters + inst, inst_chunks[inst], tot)) epilogue(epi, tot, Si, P, ctl, inst);
}

// The r.z tile parts of LEAF tiles that no fused colour sweep updates (those at the levels of the
// shared-memory kernel), formed as the colour sweep forms them: 16 lanes per tile, lane j taking
// the 4-cell vectors j, j+16, ..., j+112.
__global__ void __launch_bounds__(256) k_leaf_wpart(Topo tp, const int* __restrict__ list, int n, const float* __restrict__ R,
                                                    const float* __restrict__ Z, double* __restrict__ WP, const Scalars* S) {
    pdl_trigger();
    const int w = (int)blockIdx.x * 8 + ((int)threadIdx.x >> 5);
    if (2 * w >= n) {  // whole warps
        pdl_wait();
        return;
    }
    const int j = threadIdx.x & 15;
    const int q = 2 * w + ((threadIdx.x >> 4) & 1);
    const int tile = list[q < n ? q : 2 * w];  // topology: read before pdl_wait
    pdl_wait();
    const bool ok = q < n && !tile_done(tp, S, tile);
    const size_t base = (size_t)tile * kTileCells + j * 4;
    float term[8];
#pragma unroll
    for (int k = 0; k < 8; k++) term[k] = dot4f32(ld4(R + base + 64 * k), ld4(Z + base + 64 * k));
    const double d = half_part_sum(term);
    const int slot = tp.leafslot[tile];
    if (ok && j == 0) WP[slot >= 0 ? slot : -2 - slot] = d;
}

// The p.Ap tile parts of the LEAF tiles with GHOST children: their A p first receives the
// children's 2x2x2 sums (the rows the fused Laplacian left in GACC, added in AccumulateToParents's
// way: Ap + sum), then the part is formed as the Laplacian forms it: 16 lanes per tile, lane j
// taking the 4-cell vectors j, j+16, ..., j+112.
__global__ void __launch_bounds__(256) k_pap_ghost(Topo tp, const int* __restrict__ list, int n, const float* __restrict__ P,
                                                   float* AP, const float* __restrict__ GACC, double* __restrict__ WP,
                                                   const Scalars* S) {
    pdl_trigger();
    const int w = (int)blockIdx.x * 8 + ((int)threadIdx.x >> 5);
    if (2 * w >= n) {  // whole warps
        pdl_wait();
        return;
    }
    const int j = threadIdx.x & 15;
    const int q = 2 * w + ((threadIdx.x >> 4) & 1);
    const int tile = list[q < n ? q : 2 * w];  // topology: read before pdl_wait
    pdl_wait();
    const bool ok = q < n && !tile_done(tp, S, tile);
    float term[8];
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const int qv = j + 16 * k;
        const size_t off = (size_t)tile * kTileCells + qv * 4;
        const V4<float> p = ld4(P + off);
        V4<float> ap = ld4(AP + off);
        const int i = qv >> 4, j = (qv >> 1) & 7, k0 = (qv & 1) * 4;
        const int gs = tp.ghost_child[(size_t)tile * 8 + ((i >> 2) | ((j >> 2) << 1) | ((k0 >> 2) << 2))];
        if (gs >= 0) {
            const float* row = GACC + (size_t)gs * 64 + (i & 3) * 16 + (j & 3) * 4 + (k0 & 3);
#pragma unroll
            for (int e = 0; e < 4; e++) ap.v[e] = ap.v[e] + row[e];
            if (ok) st4(AP + off, ap);
        }
        term[k] = dot4f32(p, ap);
    }
    const double d = half_part_sum(term);
    if (ok && j == 0) WP[-2 - tp.leafslot[tile]] = d;
}

// Per instance (one CTA each): the sum of its LEAF tiles' parts in LEAF-list order (thread-strided,
// warp trees, then the 8 warp sums in order), then the epilogue.  The order is fixed and involves
// only the instance's own tiles.
__global__ void __launch_bounds__(256) k_inst_wsum(const int2* __restrict__ ranges, const double* __restrict__ WP, Scalars* S,
                                                   const InstParams* __restrict__ ip, SolveCtl ctl, int epi, int skip) {
    pdl_trigger();
    __shared__ double ws[8];
    const int inst = blockIdx.x;
    const int2 r = ranges[inst];  // topology: read before pdl_wait
    pdl_wait();
    Scalars* Si = S + inst;
    const InstParams P = ip[inst];
    if (!P.active || (skip == SKIP_DONE && Si->done)) return;
    const double* w = WP + r.x;
    double acc = 0.0;
#pragma unroll 4
    for (int i = threadIdx.x; i < r.y; i += 256) acc += w[i];
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
#pragma unroll
        for (int k = 0; k < 8; k++) tot += ws[k];
        epilogue(epi, Double2{tot, 0.0}, Si, P, ctl, inst);
    }
}

// Start of a solve: per-instance scalars zeroed, instances outside the solve marked done, the
// count of iterating instances set (0 ends the graph's loop at once).
__global__ void __launch_bounds__(256) k_begin(Scalars* S, const InstParams* __restrict__ ip, int ninst, SolveCtl ctl) {
    pdl_entry();
    __shared__ int cnt;
    if (threadIdx.x == 0) cnt = 0;
    __syncthreads();
    int mine = 0;
    for (int i = threadIdx.x; i < ninst; i += blockDim.x) {
        Scalars z;
        memset(&z, 0, sizeof(z));
        z.done = ip[i].active ? 0 : 1;
        S[i] = z;
        mine += ip[i].active ? 1 : 0;
    }
    atomicAdd(&cnt, mine);
    __syncthreads();
    if (threadIdx.x == 0) {
        *ctl.active = cnt;
        if (cnt == 0) set_cond(ctl, 0u);
    }
}

// x += alpha p, then p = z + beta p on INTERIOR cells of LEAF tiles (src/GMGSolver.cu:587-600 and
// 642-653), per instance still iterating: the x update of this iteration, taken out of the x/r
// pass so that p is read once; the GHOST children receive the new p (push_to_ghost_child).  One
// 128-thread group per tile, one 4-cell vector per thread: the tile's values are loaded before
// its instance's state is read, so the loads do not wait on that lookup.
__global__ void __launch_bounds__(256) k_update_p(Topo tp, const int* __restrict__ leaves, int nleaf, float* P,
                                                  const float* __restrict__ Z, float* X, const Scalars* S) {
    pdl_trigger();
    const int q = (int)blockIdx.x * 2 + ((int)threadIdx.x >> 7);
    if (q >= nleaf) {
        pdl_wait();
        return;
    }
    const int t = threadIdx.x & 127;
    const int tile = leaves[q];  // topology: read before pdl_wait
    const size_t off = (size_t)tile * kTileCells + t * 4;
    const uint32_t ct4 = *reinterpret_cast<const uint32_t*>(tp.ctype + off);
    const int inst = tp.inst[tile];
    pdl_wait();
    V4<float> p = ld4(P + off), x = ld4(X + off);
    const V4<float> z = ld4(Z + off);
    const Scalars& Si = S[inst];
    if (Si.done) return;
    const float alpha = (float)Si.alpha, beta = (float)Si.beta;
#pragma unroll
    for (int e = 0; e < 4; e++)
        if ((ct4 >> (8 * e)) & INTERIOR_C) {
            x.v[e] = fmaf(alpha, p.v[e], x.v[e]);
            p.v[e] = fmaf(beta, p.v[e], z.v[e]);
        }
    st4(X + off, x);
    st4(P + off, p);
    push_to_ghost_child(tp, P, tile, t, p, ct4);
}

// After the loop: the last iteration's x += alpha p (its k_update_p did not run: the instance
// stopped in that iteration's x/r pass) for every instance that iterated at least once.
__global__ void __launch_bounds__(256) k_x_final(Topo tp, const int* __restrict__ leaves, int nleaf, float* X,
                                                 const float* __restrict__ P, const Scalars* S) {
    pdl_entry();
    const int q = (int)blockIdx.x * 2 + ((int)threadIdx.x >> 7);
    if (q >= nleaf) return;
    const int t = threadIdx.x & 127;
    const int tile = leaves[q];
    const Scalars& Si = S[tp.inst[tile]];
    if (Si.iter == 0) return;
    const size_t off = (size_t)tile * kTileCells + t * 4;
    const uint32_t ct4 = *reinterpret_cast<const uint32_t*>(tp.ctype + off);
    V4<float> x = ld4(X + off);
    const V4<float> p = ld4(P + off);
    const float alpha = (float)Si.alpha;
#pragma unroll
    for (int e = 0; e < 4; e++)
        if ((ct4 >> (8 * e)) & INTERIOR_C) x.v[e] = fmaf(alpha, p.v[e], x.v[e]);
    st4(X + off, x);
}

// r -= mean on INTERIOR cells of LEAF tiles (ReCenterLeafVoxels, src/PoissonSolver.cu:356-368)
// of the pure-Neumann instances still iterating; RC (optional) receives a copy of the recentred r
// (the multigrid right-hand side).
__global__ void __launch_bounds__(256) k_recenter(Topo tp, const int* __restrict__ leaves, int nleaf, float* R,
                                                  const Scalars* S, const InstParams* __restrict__ ip, float* RC) {
    pdl_entry();
    const size_t nv = (size_t)nleaf * 128;
    for (size_t v = (size_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += (size_t)gridDim.x * blockDim.x) {
        const int tile = leaves[v >> 7];
        const int inst = tp.inst[tile];
        if (S[inst].done || !ip[inst].pure_neumann) continue;
        const double mean = S[inst].mean;
        const size_t off = (size_t)tile * kTileCells + (v & 127) * 4;
        const uint32_t ct4 = *reinterpret_cast<const uint32_t*>(tp.ctype + off);
        V4<float> r = ld4(R + off);
#pragma unroll
        for (int e = 0; e < 4; e++)
            if ((ct4 >> (8 * e)) & INTERIOR_C) r.v[e] = (float)((double)r.v[e] - mean);
        st4(R + off, r);
        if (RC) st4(RC + off, mg_rhs_copy(tp, tile, (int)(v & 127), r));
    }
}

// ------------------------------------------------------------------ FP64 defect correction
// b - A x in FP64 for INTERIOR cells of LEAF tiles (0 elsewhere), with x held in FP64, for the
// active instances.  The FP64 operator is the same FullNegativeLaplacian with FP64 coefficients.
__global__ void __launch_bounds__(256) k_residual64(Topo tp, const int* __restrict__ leaves, int nleaf, const float* __restrict__ B,
                                                    const double* __restrict__ AX, double* R64, float* R32,
                                                    const InstParams* __restrict__ ip) {
    pdl_entry();
    const size_t nv = (size_t)nleaf * 128;
    for (size_t v = (size_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += (size_t)gridDim.x * blockDim.x) {
        const int tile = leaves[v >> 7];
        if (!ip[tp.inst[tile]].active) continue;
        const size_t off = (size_t)tile * kTileCells + (v & 127) * 4;
        const uint32_t ct4 = *reinterpret_cast<const uint32_t*>(tp.ctype + off);
        const V4<float> b = ld4(B + off);
        const V4<double> ax = AX ? ld4(AX + off) : zero4<double>();  // AX null: x = 0
        V4<double> r;
        V4<float> r32;
#pragma unroll
        for (int e = 0; e < 4; e++) {
            r.v[e] = ((ct4 >> (8 * e)) & INTERIOR_C) ? (double)b.v[e] - ax.v[e] : 0.0;
            r32.v[e] = (float)r.v[e];
        }
        st4(R64 + off, r);
        st4(R32 + off, r32);
    }
}

// Pure-Neumann instances of the FP64 defect correction: the residual's component along A's null
// space (the constant on INTERIOR cells of LEAF tiles) is removed -- r -= sum(r)/count on INTERIOR
// cells, sum over the instance's LEAF cells (r is 0 off INTERIOR), count its INTERIOR cells --
// and the FP32 copy refreshed.  Other instances are left alone.
__global__ void __launch_bounds__(256) k_sub_mean64(Topo tp, const int* __restrict__ leaves, int nleaf, double* R64, float* R32,
                                                    const double* __restrict__ sums, const double* __restrict__ counts,
                                                    const InstParams* __restrict__ ip) {
    pdl_entry();
    const size_t nv = (size_t)nleaf * 128;
    for (size_t v = (size_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += (size_t)gridDim.x * blockDim.x) {
        const int tile = leaves[v >> 7];
        const int inst = tp.inst[tile];
        if (!ip[inst].active || !ip[inst].pure_neumann || !(counts[inst] > 0.0)) continue;
        const double mean = sums[inst] / counts[inst];
        const size_t off = (size_t)tile * kTileCells + (v & 127) * 4;
        const uint32_t ct4 = *reinterpret_cast<const uint32_t*>(tp.ctype + off);
        V4<double> r = ld4(R64 + off);
        V4<float> r32;
#pragma unroll
        for (int e = 0; e < 4; e++) {
            if ((ct4 >> (8 * e)) & INTERIOR_C) r.v[e] -= mean;
            r32.v[e] = (float)r.v[e];
        }
        st4(R64 + off, r);
        st4(R32 + off, r32);
    }
}

// x64 += e (FP32 correction) on INTERIOR cells of LEAF tiles of the active instances.
__global__ void __launch_bounds__(256) k_accumulate_correction(Topo tp, const int* __restrict__ leaves, int nleaf, double* X64,
                                                               float* E, const InstParams* __restrict__ ip) {
    pdl_entry();
    const size_t nv = (size_t)nleaf * 128;
    for (size_t v = (size_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += (size_t)gridDim.x * blockDim.x) {
        const int tile = leaves[v >> 7];
        if (!ip[tp.inst[tile]].active) continue;
        const size_t off = (size_t)tile * kTileCells + (v & 127) * 4;
        const uint32_t ct4 = *reinterpret_cast<const uint32_t*>(tp.ctype + off);
        V4<double> x = ld4(X64 + off);
        const V4<float> e = ld4(E + off);
#pragma unroll
        for (int q = 0; q < 4; q++)
            if ((ct4 >> (8 * q)) & INTERIOR_C) x.v[q] += (double)e.v[q];
        st4(X64 + off, x);
    }
}

// Per-instance FP64 sum of squares of a leaf channel (FP64 A, or FP32 B32 widened) into
// out[instance], chunked like k_inst_reduce (every instance, active or not).  plain_sum: the sum of
// the FP64 values themselves instead (A only).
__global__ void __launch_bounds__(256) k_inst_norm64(const int* __restrict__ leaves, const int4* __restrict__ chunks,
                                                     const int2* __restrict__ inst_chunks, const double* __restrict__ A,
                                                     const float* __restrict__ B32, double* partials, unsigned int* counters,
                                                     double* out, int plain_sum) {
    pdl_entry();
    const int4 ch = chunks[blockIdx.x];
    double acc = 0.0;
    for (int v = ch.y + threadIdx.x; v < ch.z; v += blockDim.x) {
        const size_t off = (size_t)leaves[v >> 7] * kTileCells + (v & 127) * 4;
        if (A && plain_sum) {
            const V4<double> a = ld4(A + off);
            acc += a.v[0] + a.v[1] + a.v[2] + a.v[3];
        } else if (A) {
            const V4<double> a = ld4(A + off);
            acc += a.v[0] * a.v[0] + a.v[1] * a.v[1] + a.v[2] * a.v[2] + a.v[3] * a.v[3];
        } else {
            const V4<float> a = ld4(B32 + off);
            acc += (double)a.v[0] * a.v[0] + (double)a.v[1] * a.v[1] + (double)a.v[2] * a.v[2] + (double)a.v[3] * a.v[3];
        }
    }
    Double2 tot{0.0, 0.0};
    if (chunk_reduce_and_elect(acc, 0.0, partials, counters + ch.x, inst_chunks[ch.x], tot)) out[ch.x] = tot.a;
}

// float -> double and double -> float channel copies over all tiles
__global__ void k_widen(const float* __restrict__ a, double* b, size_t n) {
    pdl_entry();
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) b[i] = (double)a[i];
}
__global__ void k_narrow(const double* __restrict__ a, float* b, size_t n) {
    pdl_entry();
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) b[i] = (float)a[i];
}

// ================================================================== launchers
namespace launch {

constexpr int kTPB = 2;  // tiles per CTA of the stencil kernels

template <class T>
void propagate_ghosts(const DevGrid& g, T* X, const Scalars* S, cudaStream_t s) {
    if (g.n_ghost == 0) return;
    ++g.launch_count;
    launch_kernel(k_propagate_ghosts<T>, g.n_ghost, 128, 0, s, g.topo, g.d_ghost, g.n_ghost, X, S);
}
template <class T>
void laplacian_tiles(const DevGrid& g, const T* X, T* Y, const Scalars* S, cudaStream_t s, bool diag = false) {
    if (g.n_leafghost == 0) return;
    ++g.launch_count;
    if (diag)
        launch_kernel(k_laplacian<T, kTPB, true>, (g.n_leafghost + kTPB - 1) / kTPB, 128 * kTPB, 0, s, g.topo, g.d_leafghost,
                      g.n_leafghost, X, Y, S);
    else
        launch_kernel(k_laplacian<T, kTPB>, (g.n_leafghost + kTPB - 1) / kTPB, 128 * kTPB, 0, s, g.topo, g.d_leafghost,
                      g.n_leafghost, X, Y, S);
}
template <class T>
void accumulate_ghosts(const DevGrid& g, T* Y, const Scalars* S, cudaStream_t s) {
    if (g.n_ghost == 0) return;
    ++g.launch_count;
    launch_kernel(k_accumulate_ghosts<T>, g.n_ghost, 64, 0, s, g.topo, g.d_ghost, g.n_ghost, Y, S);
}
template <class T>
void full_laplacian(const DevGrid& g, T* X, T* Y, const Scalars* S, cudaStream_t s) {
    propagate_ghosts<T>(g, X, S, s);
    laplacian_tiles<T>(g, X, Y, S, s);
    accumulate_ghosts<T>(g, Y, S, s);
}
// FullNegativeLaplacian(grid, x, D, calc_diag = true): x propagated to the GHOST tiles, the
// diagonal of every LEAF|GHOST cell, the GHOST rows accumulated into their parents.
void full_laplacian_diag(const DevGrid& g, float* X, float* D, cudaStream_t s) {
    propagate_ghosts<float>(g, X, nullptr, s);
    laplacian_tiles<float>(g, X, D, nullptr, s, true);
    accumulate_ghosts<float>(g, D, nullptr, s);
}
template void propagate_ghosts<float>(const DevGrid&, float*, const Scalars*, cudaStream_t);
template void full_laplacian<float>(const DevGrid&, float*, float*, const Scalars*, cudaStream_t);
template void full_laplacian<double>(const DevGrid&, double*, double*, const Scalars*, cudaStream_t);

// prefetch: stage the tiles of a CTA about one resident wave later into L2 (pf > 0, see
// k_laplacian_fused_body): pf = the list entries the CTAs resident at once cover.
template <int TPB, int NT, int MINB = 0>
void laplacian_shape(const DevGrid& g, const float* X, float* Y, const Scalars* S, cudaStream_t s, double* WP, bool prefetch = false) {
    const int per = TPB * NT;
    const int item_blocks = (g.n_lapitems + 128 * TPB - 1) / (128 * TPB);
    const auto k = k_laplacian_fused_shape<TPB, NT, MINB>();
    launch_kernel(k, item_blocks + (g.n_lapmain + per - 1) / per, 128 * TPB, sizeof(LapStage) * per, s,
                  prefetch_topo(g, k, 128 * TPB, sizeof(LapStage) * per, per, prefetch), g.d_lapmain, g.n_lapmain, g.d_lapitems,
                  g.n_lapitems, item_blocks, X, Y, g.d_gacc, S, WP);
}

void laplacian_fused(const DevGrid& g, const float* X, float* Y, const Scalars* S, cudaStream_t s, bool with_pap) {
    if (g.n_lapmain + g.n_lapitems == 0) return;
    ++g.launch_count;
    double* WP = with_pap ? g.d_wpart : nullptr;
    const int shape = g.shape(KS_LAPLACIAN, 0);
    // shapes 12..15: eight cells per thread
    if (shape >= kFirstLap8Shape && shape < kFirstLap8Shape + 4) {
        laplacian8(g, shape - kFirstLap8Shape, X, Y, S, s, WP);
        return;
    }
    // shapes 8..11: the TMA-staged pipeline (the cp.async shape 1 if X's tensor maps cannot be made)
    if (shape >= kFirstTmaShape && shape < kFirstLap8Shape && laplacian_tma(g, shape - kFirstTmaShape, X, Y, S, s, with_pap)) return;
    switch (shape) {
    case 0: laplacian_shape<2, 1>(g, X, Y, S, s, WP); break;
    case 1: laplacian_shape<2, 2>(g, X, Y, S, s, WP); break;
    case 2: laplacian_shape<1, 4>(g, X, Y, S, s, WP); break;
    case 3: laplacian_shape<2, 4>(g, X, Y, S, s, WP); break;
    case 4: laplacian_shape<1, 1>(g, X, Y, S, s, WP); break;
    case 5: laplacian_shape<1, 2>(g, X, Y, S, s, WP); break;
    case 6: laplacian_shape<1, 1, 16>(g, X, Y, S, s, WP); break;
    case 7: laplacian_shape<1, 1, 12>(g, X, Y, S, s, WP); break;
    // 16..19: shapes 2, 3, 5, 1 with L2 prefetching one resident wave ahead
    case 16: laplacian_shape<1, 4>(g, X, Y, S, s, WP, true); break;
    case 17: laplacian_shape<2, 4>(g, X, Y, S, s, WP, true); break;
    case 18: laplacian_shape<1, 2>(g, X, Y, S, s, WP, true); break;
    case 19: laplacian_shape<2, 2>(g, X, Y, S, s, WP, true); break;
    default: laplacian_shape<2, 2>(g, X, Y, S, s, WP); break;  // shape 1 (the TMA shapes without tensor maps)
    }
}
void pap_ghost(const DevGrid& g, const float* P, float* AP, cudaStream_t s) {
    if (g.n_gpar_leaves == 0) return;
    ++g.launch_count;
    launch_kernel(k_pap_ghost, (g.n_gpar_leaves + 15) / 16, 256, 0, s, g.topo, g.d_gpar_leaves, g.n_gpar_leaves, P, AP,
                  (const float*)g.d_gacc, g.d_wpart, (const Scalars*)g.d_scalars);
}

// Launch shapes of the staged kernels: TPB tiles per CTA side by side, NT tiles per 128-thread
// group in flight.
template <int TPB, int NT, int MINB = 0>
void gs_sweep_shape(const DevGrid& g, int level, float* X, const float* R, int color, const Scalars* S, cudaStream_t s,
                    const float* RD, bool prefetch = false) {
    const int n = g.mg_count[level];
    const int per = TPB * NT;
    const auto k = k_gs_sweep_shape<TPB, NT, MINB>();
    launch_kernel(k, (n + per - 1) / per, 128 * TPB, sizeof(TileStage) * per, s,
                  prefetch_topo(g, k, 128 * TPB, sizeof(TileStage) * per, per, prefetch), g.d_mg + g.mg_offset[level], n, X, R, color,
                  S, RD, RD ? g.d_wpart : nullptr);
}

void gs_sweep(const DevGrid& g, int level, float* X, const float* R, int color, const Scalars* S, cudaStream_t s,
              const float* RD) {
    const int n = g.mg_count[level];
    if (n == 0) return;
    ++g.launch_count;
    switch (g.shape(KS_GS_SWEEP, level)) {
    case 0: gs_sweep_shape<2, 1>(g, level, X, R, color, S, s, RD); break;
    case 1: gs_sweep_shape<2, 2>(g, level, X, R, color, S, s, RD); break;
    case 2: gs_sweep_shape<1, 4>(g, level, X, R, color, S, s, RD); break;
    case 3: gs_sweep_shape<2, 4>(g, level, X, R, color, S, s, RD); break;
    case 4: gs_sweep_shape<1, 1>(g, level, X, R, color, S, s, RD); break;
    case 5: gs_sweep_shape<1, 2>(g, level, X, R, color, S, s, RD); break;
    case 6: gs_sweep_shape<1, 1, 16>(g, level, X, R, color, S, s, RD); break;
    case 7: gs_sweep_shape<1, 1, 12>(g, level, X, R, color, S, s, RD); break;
    // 8..11: shapes 2, 5, 6, 1 prefetching later CTAs' tiles into L2
    case 8: gs_sweep_shape<1, 4>(g, level, X, R, color, S, s, RD, true); break;
    case 9: gs_sweep_shape<1, 2>(g, level, X, R, color, S, s, RD, true); break;
    case 10: gs_sweep_shape<1, 1, 16>(g, level, X, R, color, S, s, RD, true); break;
    default: gs_sweep_shape<2, 2>(g, level, X, R, color, S, s, RD, true); break;
    }
}

void gs_sequence(const DevGrid& g, int level, float* X, const float* R, uint32_t colors, int nsweeps, const Scalars* S,
                 cudaStream_t s) {
    const int n = g.mg_count[level];
    if (n == 0 || nsweeps == 0) return;
    if (n <= 8) {
        ++g.launch_count;
        launch_kernel(k_gs_sequence, 1, 128 * n, 0, s, g.topo, g.d_mg + g.mg_offset[level], n, X, R, colors, nsweeps, S);
        return;
    }
    for (int k = 0; k < nsweeps; k++) gs_sweep(g, level, X, R, (colors >> k) & 1, S, s);
}

template <int TPB, int NT, int MINB = 0>
void residual_shape(const DevGrid& g, int level, const float* X, const float* RHS, float* C, float one_over_alpha, const Scalars* S,
                    cudaStream_t s, bool ghosts_zero, bool prefetch = false) {
    const int per = TPB * NT;
    const int* list = ghosts_zero ? g.d_rrmain + g.rr_off[level] : nullptr;
    const int n = ghosts_zero ? g.rr_cnt[level] : g.level_count[level];
    const int nitems = ghosts_zero ? g.rri_cnt[level] : 0;
    const int4* items = ghosts_zero ? g.d_rritems + g.rri_off[level] : nullptr;
    const int item_blocks = (nitems + 128 * TPB - 1) / (128 * TPB);
    const auto k = k_residual_restrict_shape<TPB, NT, MINB>();
    launch_kernel(k, item_blocks + (n + per - 1) / per, 128 * TPB, sizeof(TileStage) * per, s,
                  prefetch_topo(g, k, 128 * TPB, sizeof(TileStage) * per, per, prefetch), g.level_first[level], list, n, items, nitems,
                  item_blocks, X, RHS, C, one_over_alpha, S);
}

void residual_restrict(const DevGrid& g, int level, const float* X, const float* RHS, float* C, float one_over_alpha,
                       const Scalars* S, cudaStream_t s, bool ghosts_zero) {
    if (g.level_count[level] == 0) return;
    ++g.launch_count;
    switch (g.shape(KS_RESIDUAL, level)) {
    case 0: residual_shape<2, 1>(g, level, X, RHS, C, one_over_alpha, S, s, ghosts_zero); break;
    case 1: residual_shape<2, 2>(g, level, X, RHS, C, one_over_alpha, S, s, ghosts_zero); break;
    case 2: residual_shape<1, 4>(g, level, X, RHS, C, one_over_alpha, S, s, ghosts_zero); break;
    case 3: residual_shape<2, 4>(g, level, X, RHS, C, one_over_alpha, S, s, ghosts_zero); break;
    case 4: residual_shape<1, 1>(g, level, X, RHS, C, one_over_alpha, S, s, ghosts_zero); break;
    case 5: residual_shape<1, 2>(g, level, X, RHS, C, one_over_alpha, S, s, ghosts_zero); break;
    case 6: residual_shape<1, 1, 16>(g, level, X, RHS, C, one_over_alpha, S, s, ghosts_zero); break;
    case 7: residual_shape<1, 1, 12>(g, level, X, RHS, C, one_over_alpha, S, s, ghosts_zero); break;
    // 8..11: shapes 2, 5, 6, 1 prefetching later CTAs' tiles into L2
    case 8: residual_shape<1, 4>(g, level, X, RHS, C, one_over_alpha, S, s, ghosts_zero, true); break;
    case 9: residual_shape<1, 2>(g, level, X, RHS, C, one_over_alpha, S, s, ghosts_zero, true); break;
    case 10: residual_shape<1, 1, 16>(g, level, X, RHS, C, one_over_alpha, S, s, ghosts_zero, true); break;
    default: residual_shape<2, 2>(g, level, X, RHS, C, one_over_alpha, S, s, ghosts_zero, true); break;
    }
}

void prolongate(const DevGrid& g, int level, const float* CX, float* FX, float prolong_coeff, const Scalars* S, cudaStream_t s) {
    const int n = g.level_count[level];
    if (n == 0) return;
    ++g.launch_count;
    launch_kernel(k_prolongate, n, 128, 0, s, g.topo, g.level_first[level], n, CX, FX, prolong_coeff, S);
}

void vcycle_init(const DevGrid& g, float* X, float* RHS, const float* F, const Scalars* S, cudaStream_t s) {
    const size_t nv = (size_t)g.n * 128;
    int blocks = (int)std::min<size_t>((nv + 255) / 256, (size_t)g.sm_count * 8);
    if (blocks < 1) blocks = 1;
    ++g.launch_count;
    launch_kernel(k_vcycle_init, blocks, 256, 0, s, g.topo, g.n, X, RHS, F, S);
}

void laplacian_same_level(const DevGrid& g, int level, int subtree_level, uint32_t types, const float* X, float* Y, bool diag,
                          cudaStream_t s) {
    const int first = level < 0 ? 0 : g.level_first[level], count = level < 0 ? g.n : g.level_count[level];
    if (count == 0) return;
    ++g.launch_count;
    const int blocks = (count + kTPB - 1) / kTPB;
    if (diag)
        launch_kernel(k_laplacian_same_level<kTPB, true>, blocks, 128 * kTPB, 0, s, g.topo, first, count, subtree_level, types, X, Y);
    else
        launch_kernel(k_laplacian_same_level<kTPB, false>, blocks, 128 * kTPB, 0, s, g.topo, first, count, subtree_level, types, X, Y);
}

// dampedJacobiSolve's residual step (src/GMGSolver.cu:479-490): Ax = b - Ax on INTERIOR cells
// of LEAF tiles (other cells keep A x).
__global__ void __launch_bounds__(128) k_jacobi_residual(Topo tp, const int* __restrict__ leaves, int nleaf, const float* __restrict__ B,
                                                         float* AX) {
    pdl_entry();
    const int q = blockIdx.x;
    if (q >= nleaf) return;
    const size_t off = (size_t)leaves[q] * kTileCells + threadIdx.x * 4;
    const uint32_t ct4 = *reinterpret_cast<const uint32_t*>(tp.ctype + off);
    const V4<float> b = ld4(B + off);
    V4<float> ax = ld4(AX + off);
#pragma unroll
    for (int e = 0; e < 4; e++)
        if ((ct4 >> (8 * e)) & INTERIOR_C) ax.v[e] = b.v[e] - ax.v[e];
    st4(AX + off, ax);
}
// dampedJacobiSolve's update (src/GMGSolver.cu:508-525): on INTERIOR cells of LEAF tiles
// x += omega * r / D, or x = 0 where D is 0.
__global__ void __launch_bounds__(128) k_jacobi_update(Topo tp, const int* __restrict__ leaves, int nleaf, float* X,
                                                       const float* __restrict__ R, const float* __restrict__ D, float omega) {
    pdl_entry();
    const int q = blockIdx.x;
    if (q >= nleaf) return;
    const size_t off = (size_t)leaves[q] * kTileCells + threadIdx.x * 4;
    const uint32_t ct4 = *reinterpret_cast<const uint32_t*>(tp.ctype + off);
    const V4<float> r = ld4(R + off), d = ld4(D + off);
    V4<float> x = ld4(X + off);
#pragma unroll
    for (int e = 0; e < 4; e++)
        if ((ct4 >> (8 * e)) & INTERIOR_C) x.v[e] = d.v[e] == 0.f ? 0.f : x.v[e] + __fdiv_rn(__fmul_rn(omega, r.v[e]), d.v[e]);
    st4(X + off, x);
}
void jacobi_residual(const DevGrid& g, const float* B, float* AX, cudaStream_t s) {
    if (g.n_leaf == 0) return;
    ++g.launch_count;
    launch_kernel(k_jacobi_residual, g.n_leaf, 128, 0, s, g.topo, g.d_leaf, g.n_leaf, B, AX);
}
void jacobi_update(const DevGrid& g, float* X, const float* R, const float* D, float omega, cudaStream_t s) {
    if (g.n_leaf == 0) return;
    ++g.launch_count;
    launch_kernel(k_jacobi_update, g.n_leaf, 128, 0, s, g.topo, g.d_leaf, g.n_leaf, X, R, D, omega);
}
// a dot over an arbitrary tile list (the whole-grid reduction of cirrus_dot), result on the host
double list_dot(const DevGrid& g, const float* A, const float* B, const int* list, int n, cudaStream_t s) {
    if (n == 0) return 0.0;
    ++g.launch_count;
    k_leaf_dot<<<g.red_blocks, 256, 0, s>>>(list, n, A, B, g.d_dot, g.d_partials, g.d_counter);
    double v = 0.0;
    cudaMemcpyAsync(&v, &g.d_dot->gamma, sizeof(double), cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    return v;
}

void init_stencil_attributes() {
    static std::once_flag once;
    std::call_once(once, [] {
    cudaFuncSetAttribute(k_gs_sweep<2, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(TileStage) * 8);
    cudaFuncSetAttribute(k_laplacian_fused<2, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(LapStage) * 8);
    cudaFuncSetAttribute(k_residual_restrict<2, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(TileStage) * 8);
    });
}

bool pdl_enabled() {
    static const bool on = [] {
        const char* e = std::getenv("CIRRUS_NO_PDL");
        return !(e && e[0] == '1');
    }();
    return on;
}

int leaf_blocks(const DevGrid& g) { return g.red_blocks; }

void inst_reduce(int op, const DevGrid& g, float* A, float* B, float* C, float* D, const SolveCtl& ctl, int epi, int skip,
                 cudaStream_t s) {
    ++g.launch_count;
#define CIRRUS_INST_REDUCE(OPV)                                                                                         \
    launch_kernel(k_inst_reduce<OPV>, g.n_chunks, 256, 0, s, g.topo, g.d_leaf, g.d_chunks, g.d_inst_chunks, A, B, C, D, \
                  g.d_scalars, g.d_iparams, ctl, epi, g.d_partials, g.d_counters, skip)
    switch (op) {
    case OP_DOT: CIRRUS_INST_REDUCE(OP_DOT); break;
    case OP_INIT: CIRRUS_INST_REDUCE(OP_INIT); break;
    case OP_COPY_DOT: CIRRUS_INST_REDUCE(OP_COPY_DOT); break;
    case OP_XR: CIRRUS_INST_REDUCE(OP_XR); break;
    case OP_MEAN: CIRRUS_INST_REDUCE(OP_MEAN); break;
    }
#undef CIRRUS_INST_REDUCE
}

void leaf_wpart(const DevGrid& g, const float* R, const float* Z, cudaStream_t s) {
    if (g.n_bottom_leaves == 0) return;
    ++g.launch_count;
    launch_kernel(k_leaf_wpart, (g.n_bottom_leaves + 15) / 16, 256, 0, s, g.topo, g.d_bottom_leaves, g.n_bottom_leaves, R, Z, g.d_wpart,
                  (const Scalars*)g.d_scalars);
}
void inst_wsum(const DevGrid& g, const SolveCtl& ctl, int epi, int skip, cudaStream_t s) {
    ++g.launch_count;
    launch_kernel(k_inst_wsum, g.num_inst, 256, 0, s, g.d_inst_leafrange, (const double*)g.d_wpart, g.d_scalars,
                  (const InstParams*)g.d_iparams, ctl, epi, skip);
}

void grid_dot(const DevGrid& g, const float* A, const float* B, cudaStream_t s) {
    ++g.launch_count;
    k_leaf_dot<<<leaf_blocks(g), 256, 0, s>>>(g.d_leaf, g.n_leaf, A, B, g.d_dot, g.d_partials, g.d_counter);
}

void leaf_dot_raw(const float* A, const float* B, const int* leaves, int nleaf, int blocks, double* partials,
                  unsigned int* counter, Scalars* S, cudaStream_t s) {
    k_leaf_dot<<<blocks, 256, 0, s>>>(leaves, nleaf, A, B, S, partials, counter);
}

void begin_solve(const DevGrid& g, const SolveCtl& ctl, cudaStream_t s) {
    ++g.launch_count;
    launch_kernel(k_begin, 1, 256, 0, s, g.d_scalars, g.d_iparams, g.num_inst, ctl);
}

void update_p(const DevGrid& g, float* P, const float* Z, float* X, cudaStream_t s) {
    if (g.n_leaf == 0) return;
    ++g.launch_count;
    launch_kernel(k_update_p, (g.n_leaf + 1) / 2, 256, 0, s, g.topo, g.d_leaf, g.n_leaf, P, Z, X, (const Scalars*)g.d_scalars);
}
void x_final(const DevGrid& g, float* X, const float* P, cudaStream_t s) {
    if (g.n_leaf == 0) return;
    ++g.launch_count;
    launch_kernel(k_x_final, (g.n_leaf + 1) / 2, 256, 0, s, g.topo, g.d_leaf, g.n_leaf, X, P, (const Scalars*)g.d_scalars);
}

void recenter(const DevGrid& g, float* R, float* RC, cudaStream_t s) {
    ++g.launch_count;
    launch_kernel(k_recenter, leaf_blocks(g), 256, 0, s, g.topo, g.d_leaf, g.n_leaf, R, (const Scalars*)g.d_scalars,
                  (const InstParams*)g.d_iparams, RC);
}

void residual64(const DevGrid& g, const float* B, const double* AX, double* R64, float* R32, cudaStream_t s) {
    ++g.launch_count;
    launch_kernel(k_residual64, leaf_blocks(g), 256, 0, s, g.topo, g.d_leaf, g.n_leaf, B, AX, R64, R32, (const InstParams*)g.d_iparams);
}
void accumulate_correction(const DevGrid& g, double* X64, float* E, cudaStream_t s) {
    ++g.launch_count;
    launch_kernel(k_accumulate_correction, leaf_blocks(g), 256, 0, s, g.topo, g.d_leaf, g.n_leaf, X64, E,
                  (const InstParams*)g.d_iparams);
}
void norm64(const DevGrid& g, const double* A, const float* B32, double* out, cudaStream_t s, bool plain_sum) {
    ++g.launch_count;
    launch_kernel(k_inst_norm64, g.n_chunks, 256, 0, s, (const int*)g.d_leaf, (const int4*)g.d_chunks, (const int2*)g.d_inst_chunks, A,
                  B32, g.d_partials, g.d_counters, out, plain_sum ? 1 : 0);
}
void sub_mean64(const DevGrid& g, double* R64, float* R32, const double* sums, const double* counts, cudaStream_t s) {
    ++g.launch_count;
    launch_kernel(k_sub_mean64, leaf_blocks(g), 256, 0, s, g.topo, g.d_leaf, g.n_leaf, R64, R32, sums, counts,
                  (const InstParams*)g.d_iparams);
}
void widen(const DevGrid& g, const float* a, double* b, size_t n, cudaStream_t s) {
    ++g.launch_count;
    launch_kernel(k_widen, (int)std::min<size_t>((n + 255) / 256, 4096), 256, 0, s, a, b, n);
}
void narrow(const DevGrid& g, const double* a, float* b, size_t n, cudaStream_t s) {
    ++g.launch_count;
    launch_kernel(k_narrow, (int)std::min<size_t>((n + 255) / 256, 4096), 256, 0, s, a, b, n);
}

}  // namespace launch
}  // namespace cirrus
