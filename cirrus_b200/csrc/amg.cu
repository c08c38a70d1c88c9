// The AMG variant of the preconditioner (AMGSolver, src/AMGSolver.h, src/AMGSolver.cu): explicit
// per-cell face coefficients, coarse-level coefficients and cell types formed from the children
// (Galerkin-style), Gauss-Seidel smoothing and residuals on those coefficients, and the same PCG
// as GMGSolver::solve around the V-cycle.  In the reference the class is dead code at its only
// call site (src/FluidEuler.h:592-593, commented out) and its file does not build in this
// environment (VTK and Eigen includes), so the arithmetic here is the CPU restatement's
// (oracle/cirrus_oracle.cpp, AMG section), checked bit for bit on the GPU, with no reference
// output to pin it.
//
// Storage: four FP32 planes of n*512 (off-diagonal coefficient of each cell's x-, y-, z- face,
// then the diagonal) and a byte plane of AMG cell types (the grid's cell types with GHOST cells
// re-derived from their parents and NONLEAF cells rewritten by the coarsening), allocated on the
// first prepare.  The kernels take one 128-thread CTA per tile, thread t owning the cells
// 4t..4t+3 (column (t >> 4, (t >> 1) & 7), k = 4 (t & 1) .. +3); the coarsest level's sweeps run
// as one CTA per instance looping over its tiles (k_amg_gs_sequence).  Tiles of finished
// instances are skipped (per-instance scalars S), so the V-cycle runs inside batched solves too.
#include "kernels.cuh"
#include "solver_internal.hpp"

#include <algorithm>
#include <vector>

namespace cirrus {

namespace {

constexpr uint8_t kTypedCell = INTERIOR_C | DIRICHLET_C | NEUMANN_C;

__device__ __forceinline__ int cell_of(int i, int j, int k) { return (i << 6) | (j << 3) | k; }

// GHOST cells take their parent cell's type, DIRICHLET without a parent (src/AMGSolver.cu:118-133);
// every other cell keeps the grid's type.
__global__ void __launch_bounds__(128) k_amg_types(Topo tp, int n, uint8_t* __restrict__ act) {
    const int tile = blockIdx.x;
    if (tile >= n) return;
    const TileMeta m = tp.meta[tile];
    const bool ghost = meta_type(m.packed) & GHOST_T;
    const int oct = meta_octant(m.packed);
    for (int c = threadIdx.x; c < kTileCells; c += blockDim.x) {
        uint8_t v = tp.ctype[(size_t)tile * kTileCells + c];
        if (ghost) {
            const int i = c >> 6, j = (c >> 3) & 7, k = c & 7;
            v = m.parent < 0 ? DIRICHLET_C
                             : tp.ctype[(size_t)m.parent * kTileCells +
                                        cell_of((oct & 1) * 4 + (i >> 1), ((oct >> 1) & 1) * 4 + (j >> 1), ((oct >> 2) & 1) * 4 + (k >> 1))];
        }
        act[(size_t)tile * kTileCells + c] = v;
    }
}

// CalculateAMGCoefficients on LEAF|GHOST tiles (src/AMGSolver.cu:16-108): per cell and face in
// (axis, -/+) order the coefficient 1/h^2 (LEAF-LEAF) or (1/(1.5h))/h (LEAF-GHOST), 0 for other
// pairs or next to a NEUMANN cell, times h^3; an absent neighbour tile counts as a DIRICHLET cell
// of the cell's own tile type.  The diagonal sums the six; the off-diagonal of a lower face is
// minus its coefficient when the neighbour is INTERIOR.  Non-INTERIOR cells store zeros.
// Products and sums rounded one by one (no fused multiply-adds).
__global__ void __launch_bounds__(128) k_amg_coeffs(Topo tp, const int* __restrict__ list, int n, const uint8_t* __restrict__ act,
                                                    float* __restrict__ C, size_t plane) {
    const int q = blockIdx.x;
    if (q >= n) return;
    const int tile = list[q];
    const TileMeta m = tp.meta[tile];
    const int tt0 = meta_type(m.packed);
    int ntt[6];
#pragma unroll
    for (int f = 0; f < 6; f++) ntt[f] = m.nb[f] >= 0 ? meta_type(tp.meta[m.nb[f]].packed) : tt0;
    const float h = tile_level_const(tp, tile, meta_level(m.packed)).h;
    const float oh = __fdiv_rn(1.f, h), ogh = __fdiv_rn(1.f, __fmul_rn(1.5f, h));
    const size_t base = (size_t)tile * kTileCells;
    for (int c = threadIdx.x; c < kTileCells; c += blockDim.x) {
        const int ijk[3] = {c >> 6, (c >> 3) & 7, c & 7};
        const uint8_t ct0 = act[base + c];
        float diag = 0.f, off[3] = {0.f, 0.f, 0.f};
#pragma unroll
        for (int axis = 0; axis < 3; axis++)
#pragma unroll
            for (int s = 0; s < 2; s++) {
                const int stride = axis == 0 ? 64 : axis == 1 ? 8 : 1;
                const bool inside = s == 0 ? ijk[axis] > 0 : ijk[axis] < 7;
                const int f = 2 * axis + s;
                int tt1 = tt0;
                uint8_t ct1 = DIRICHLET_C;
                if (inside) {
                    ct1 = act[base + c + (s == 0 ? -stride : stride)];
                } else if (m.nb[f] >= 0) {
                    tt1 = ntt[f];
                    ct1 = act[(size_t)m.nb[f] * kTileCells + c + (s == 0 ? 7 * stride : -7 * stride)];
                }
                const bool both = (tt0 & LEAF_T) && (tt1 & LEAF_T);
                const bool olog = ((tt0 & LEAF_T) && (tt1 & GHOST_T)) || ((tt0 & GHOST_T) && (tt1 & LEAF_T));
                const float odh = both ? oh : olog ? ogh : 0.f;
                const bool nm = (ct0 & NEUMANN_C) || (ct1 & NEUMANN_C);
                float cf = nm ? 0.f : __fdiv_rn(odh, h);
                cf = __fmul_rn(__fmul_rn(__fmul_rn(cf, h), h), h);
                if (s == 0 && ct1 == INTERIOR_C) off[axis] = -cf;
                diag = __fadd_rn(diag, cf);
            }
        const bool interior = ct0 == INTERIOR_C;
#pragma unroll
        for (int a = 0; a < 3; a++) C[a * plane + base + c] = interior ? off[a] : 0.f;
        C[3 * plane + base + c] = interior ? diag : 0.f;
    }
}

// CoarsenTypesAndAMGCoeffs step 3 on the LEAF and NONLEAF tiles of one level, after the finer
// level (src/AMGSolver.cu:138-203): per cell over its 2x2x2 children in (ci, cj, ck) order the
// sum of their diagonals and INTERIOR count, then the lower-face off-diagonals of the children on
// the cell's lower faces summed per axis and twice those of the interior faces added to the
// diagonal.  NONLEAF: type INTERIOR if any child is, else DIRICHLET; coefficients = sums times
// one_over_alpha.  LEAF with a GHOST child tile: sums added to its own coefficients.
__global__ void __launch_bounds__(128) k_amg_coarsen(Topo tp, const int* __restrict__ child, int first, int count, uint8_t* __restrict__ act,
                                                     float* __restrict__ C, size_t plane, float one_over_alpha) {
    const int q = blockIdx.x;
    if (q >= count) return;
    const int tile = first + q;
    const int tt = meta_type(tp.meta[tile].packed);
    if (tt != LEAF_T && tt != NONLEAF_T) return;
    const size_t base = (size_t)tile * kTileCells;
    for (int c = threadIdx.x; c < kTileCells; c += blockDim.x) {
        const int i = c >> 6, j = (c >> 3) & 7, k = c & 7;
        const int ch = child[(size_t)tile * 8 + ((i >> 2) | ((j >> 2) << 1) | ((k >> 2) << 2))];
        bool ghost_child = false;
        float cod[3][8];
        float diag_sum = 0.f;
        int interior_cnt = 0;
        if (ch >= 0) {
            ghost_child = meta_type(tp.meta[ch].packed) == GHOST_T;
            const size_t cb = (size_t)ch * kTileCells;
#pragma unroll
            for (int b = 0; b < 8; b++) {
                const int cid = cell_of(2 * (i & 3) + (b >> 2), 2 * (j & 3) + ((b >> 1) & 1), 2 * (k & 3) + (b & 1));
                diag_sum = __fadd_rn(diag_sum, C[3 * plane + cb + cid]);
                interior_cnt += act[cb + cid] == INTERIOR_C ? 1 : 0;
#pragma unroll
                for (int a = 0; a < 3; a++) cod[a][b] = C[a * plane + cb + cid];
            }
        } else {
#pragma unroll
            for (int b = 0; b < 8; b++)
#pragma unroll
                for (int a = 0; a < 3; a++) cod[a][b] = 0.f;
        }
        float offs[3] = {0.f, 0.f, 0.f};
#pragma unroll
        for (int b = 0; b < 8; b++) {
            const int ci = b >> 2, cj = (b >> 1) & 1, ck = b & 1;
            if (ci == 0) offs[0] = __fadd_rn(offs[0], cod[0][b]);
            else diag_sum = __fadd_rn(diag_sum, __fmul_rn(2.f, cod[0][b]));
            if (cj == 0) offs[1] = __fadd_rn(offs[1], cod[1][b]);
            else diag_sum = __fadd_rn(diag_sum, __fmul_rn(2.f, cod[1][b]));
            if (ck == 0) offs[2] = __fadd_rn(offs[2], cod[2][b]);
            else diag_sum = __fadd_rn(diag_sum, __fmul_rn(2.f, cod[2][b]));
        }
        if (tt == NONLEAF_T) {
            act[base + c] = interior_cnt > 0 ? INTERIOR_C : DIRICHLET_C;
#pragma unroll
            for (int a = 0; a < 3; a++) C[a * plane + base + c] = __fmul_rn(offs[a], one_over_alpha);
            C[3 * plane + base + c] = __fmul_rn(diag_sum, one_over_alpha);
        } else if (ghost_child) {
#pragma unroll
            for (int a = 0; a < 3; a++) C[a * plane + base + c] = __fadd_rn(C[a * plane + base + c], offs[a]);
            C[3 * plane + base + c] = __fadd_rn(C[3 * plane + base + c], diag_sum);
        }
    }
}

// AMGLaplacianTileData::negativeLapSameLevel (src/AMGSolver.cu:231-250) of cell (i, j, k) of a
// staged tile: x0 * diag, then per face in (axis, -/+) order the off-diagonal stored at the face's
// upper cell times the neighbour's x, fused into the sum.  A lower face's coefficient is the
// cell's own; an upper face's is the next cell's, across the tile face the neighbour tile's first
// cell (0 when that tile is absent, as is its x in the staged halo).
__device__ __forceinline__ float amg_lap(const TileShared<float>& sh, const float* __restrict__ C, size_t plane, size_t base,
                                         const TileMeta& m, int i, int j, int k) {
    const int c = cell_of(i, j, k);
    float sum = __fmul_rn(sh.xs[c], C[3 * plane + base + c]);
    const int ijk[3] = {i, j, k};
#pragma unroll
    for (int axis = 0; axis < 3; axis++) {
        const int stride = axis == 0 ? 64 : axis == 1 ? 8 : 1;
        // halo slot of the cell's column on an axis face: x faces [j*8 + k], y faces [i*8 + k], z faces [i*8 + j]
        const int hs = axis == 0 ? j * 8 + k : axis == 1 ? i * 8 + k : i * 8 + j;
        const float xm = ijk[axis] > 0 ? sh.xs[c - stride] : sh.hx[(2 * axis) * 64 + hs];
        sum = fmaf(C[axis * plane + base + c], xm, sum);
        float xp, cp;
        if (ijk[axis] < 7) {
            xp = sh.xs[c + stride];
            cp = C[axis * plane + base + c + stride];
        } else {
            xp = sh.hx[(2 * axis + 1) * 64 + hs];
            const int nb = m.nb[2 * axis + 1];
            cp = nb >= 0 ? C[axis * plane + (size_t)nb * kTileCells + c - 7 * stride] : 0.f;
        }
        sum = fmaf(cp, xp, sum);
    }
    return sum;
}

// NegativeLaplacianAndGaussSeidelSameLevel128Kernel (src/AMGSolver.cu:540-578) on the LEAF|NONLEAF
// tiles of one level: cells of colour (i+j+k)%2 == color get x + (b - A x)/D where INTERIOR, x + 0
// elsewhere.
// The colour update of thread t's four cells of a staged tile (see k_amg_gs).
__device__ __forceinline__ void amg_gs_cells(const TileShared<float>& sh, const float* __restrict__ C, size_t plane, int tile, const TileMeta& m,
                                             int t, float* X, const float* __restrict__ RHS, const uint8_t* __restrict__ act, int color) {
    const TileIdx ix(t);
    const size_t base = (size_t)tile * kTileCells;
#pragma unroll
    for (int e = 0; e < 4; e++) {
        const int k = ix.k0 + e;
        if (((ix.i + ix.j + k) & 1) != color) continue;
        const int c = cell_of(ix.i, ix.j, k);
        float delta = 0.f;
        if (act[base + c] & INTERIOR_C) {
            const float ax = amg_lap(sh, C, plane, base, m, ix.i, ix.j, k);
            delta = __fdiv_rn(RHS[base + c] - ax, C[3 * plane + base + c]);
        }
        X[base + c] = sh.xs[c] + delta;
    }
}

__global__ void __launch_bounds__(128) k_amg_gs(Topo tp, const int* __restrict__ list, int n, float* X, const float* __restrict__ RHS,
                                                const uint8_t* __restrict__ act, const float* __restrict__ C, size_t plane, int color,
                                                const Scalars* __restrict__ S) {
    pdl_entry();
    __shared__ TileShared<float> sh;
    const int q = blockIdx.x, t = threadIdx.x;
    const int tile = q < n ? list[q] : 0;
    const bool active = q < n && !tile_done(tp, S, tile);
    TileMeta m;
    if (active) {
        m = tp.meta[tile];
        stage_tile<float>(X, tile, m, t, sh);
    }
    __syncthreads();
    if (!active) return;
    amg_gs_cells(sh, C, plane, tile, m, t, X, RHS, act, color);
}

// A sequence of colour sweeps (bit s of `colors` = the colour of sweep s) over one level's
// LEAF|NONLEAF tiles, one CTA per instance: CTA i takes the list entries ranges[i] = (first, count)
// -- one instance's tiles, coupled to no other instance's -- in rounds of blockDim/128 tiles, and
// a __syncthreads makes each round's global writes visible to the next round's halo loads.  A
// colour's cells never neighbour each other, so updating a sweep's tiles round by round gives
// the bits of one launch per sweep.
__global__ void __launch_bounds__(1024) k_amg_gs_sequence(Topo tp, const int* __restrict__ list, const int2* __restrict__ ranges,
                                                          float* X, const float* __restrict__ RHS, const uint8_t* __restrict__ act,
                                                          const float* __restrict__ C, size_t plane, uint32_t colors, int nsweeps,
                                                          const Scalars* __restrict__ S) {
    pdl_entry();
    __shared__ TileShared<float> sh[8];
    const int2 r = ranges[blockIdx.x];
    const int groups = blockDim.x >> 7;
    const int g = threadIdx.x >> 7, t = threadIdx.x & 127;
    for (int s = 0; s < nsweeps; s++) {
        const int color = (colors >> s) & 1;
        for (int base = 0; base < r.y; base += groups) {
            const int q = base + g;
            const int tile = q < r.y ? list[r.x + q] : 0;
            const bool active = q < r.y && !tile_done(tp, S, tile);
            TileMeta m;
            if (active) {
                m = tp.meta[tile];
                stage_tile<float>(X, tile, m, t, sh[g]);
            }
            __syncthreads();
            if (active) amg_gs_cells(sh[g], C, plane, tile, m, t, X, RHS, act, color);
            __syncthreads();
        }
    }
}

// The downstroke's residual (src/AMGSolver.cu:640-643): on every tile of the level,
// TMP = RHS - A x on INTERIOR cells, 0 elsewhere.
__global__ void __launch_bounds__(128) k_amg_residual(Topo tp, int first, int n, const float* __restrict__ X, const float* __restrict__ RHS,
                                                      float* __restrict__ TMP, const uint8_t* __restrict__ act, const float* __restrict__ C,
                                                      size_t plane, const Scalars* __restrict__ S) {
    pdl_entry();
    __shared__ TileShared<float> sh;
    const int q = blockIdx.x, t = threadIdx.x;
    const int tile = first + (q < n ? q : 0);
    const bool active = q < n && !tile_done(tp, S, tile);
    TileMeta m;
    if (active) {
        m = tp.meta[tile];
        stage_tile<float>(X, tile, m, t, sh);
    }
    __syncthreads();
    if (!active) return;
    const TileIdx ix(t);
    const size_t base = (size_t)tile * kTileCells;
#pragma unroll
    for (int e = 0; e < 4; e++) {
        const int c = cell_of(ix.i, ix.j, ix.k0 + e);
        TMP[base + c] = act[base + c] == INTERIOR_C ? RHS[base + c] - amg_lap(sh, C, plane, base, m, ix.i, ix.j, ix.k0 + e) : 0.f;
    }
}

// Restriction to the coarser level (src/AMGSolver.cu:646-652) on every tile of that level:
// NONLEAF: Restrict (src/PoissonSolver.cu:292-319) -- 0 on non-INTERIOR cells, then, if the
// tile's first child tile exists, the children's INTERIOR residuals summed in child-index order
// (x fastest) times one_over_alpha; LEAF: Copy of F + AccumulateToParents of the GHOST children's
// residuals (src/PoissonGrid.cu:721-755, typed cells, added with coefficient 1); GHOST: Fill 0.
__global__ void __launch_bounds__(128) k_amg_restrict(Topo tp, const int* __restrict__ child, int first, int n, const float* __restrict__ F,
                                                      const float* __restrict__ TMP, float* __restrict__ RHS, const uint8_t* __restrict__ act,
                                                      float one_over_alpha, const Scalars* __restrict__ S) {
    pdl_entry();
    const int q = blockIdx.x;
    if (q >= n) return;
    const int tile = first + q;
    if (tile_done(tp, S, tile)) return;
    const int tt = meta_type(tp.meta[tile].packed);
    const size_t base = (size_t)tile * kTileCells;
    const bool has_child0 = child[(size_t)tile * 8] >= 0;
    for (int c = threadIdx.x; c < kTileCells; c += blockDim.x) {
        const int i = c >> 6, j = (c >> 3) & 7, k = c & 7;
        const uint8_t ct = act[base + c];
        const int ch = child[(size_t)tile * 8 + ((i >> 2) | ((j >> 2) << 1) | ((k >> 2) << 2))];
        auto child_sum = [&](uint8_t types) {
            float sum = 0.f;
            if (ch < 0) return sum;
            const size_t cb = (size_t)ch * kTileCells;
#pragma unroll
            for (int s = 0; s < 8; s++) {
                const int cid = cell_of(2 * (i & 3) + (s & 1), 2 * (j & 3) + ((s >> 1) & 1), 2 * (k & 3) + ((s >> 2) & 1));
                if (act[cb + cid] & types) sum = __fadd_rn(sum, TMP[cb + cid]);
            }
            return sum;
        };
        if (tt == NONLEAF_T) {
            if (!(ct & INTERIOR_C)) RHS[base + c] = 0.f;
            if (has_child0) RHS[base + c] = __fmul_rn(child_sum(INTERIOR_C), one_over_alpha);
        } else if (tt == LEAF_T) {
            if (ct & kTypedCell) RHS[base + c] = __fadd_rn(F[base + c], child_sum(kTypedCell));
        } else if (tt == GHOST_T) {
            if (ct & kTypedCell) RHS[base + c] = 0.f;
        }
    }
}

// ProlongateAndUpdate128 (src/GMGSolver.cu:345-380) with the AMG cell types, on every tile of
// the level: GHOST cells take the parent cell's x where INTERIOR, other tiles add prolong_coeff
// times it (fused); non-INTERIOR cells 0.
__global__ void __launch_bounds__(128) k_amg_prolong(Topo tp, int first, int n, float* X, const uint8_t* __restrict__ act, float pc,
                                                     const Scalars* __restrict__ S) {
    pdl_entry();
    const int q = blockIdx.x;
    if (q >= n) return;
    const int tile = first + q;
    if (tile_done(tp, S, tile)) return;
    const TileMeta m = tp.meta[tile];
    const bool ghost = meta_type(m.packed) & GHOST_T;
    const int oct = meta_octant(m.packed);
    const size_t base = (size_t)tile * kTileCells;
    for (int c = threadIdx.x; c < kTileCells; c += blockDim.x) {
        const int i = c >> 6, j = (c >> 3) & 7, k = c & 7;
        const float cx = m.parent < 0 ? 0.f
                                      : X[(size_t)m.parent * kTileCells +
                                          cell_of((oct & 1) * 4 + (i >> 1), ((oct >> 1) & 1) * 4 + (j >> 1), ((oct >> 2) & 1) * 4 + (k >> 1))];
        const bool interior = act[base + c] & INTERIOR_C;
        X[base + c] = !interior ? 0.f : ghost ? cx : fmaf(pc, cx, X[base + c]);
    }
}

size_t amg_plane(const DevGrid& g) { return (size_t)g.n * kTileCells; }

void amg_gauss_seidel(const DevGrid& g, int iters, int order, int level, float* X, const float* RHS, const Scalars* S, cudaStream_t s) {
    const int n = g.mg_count[level];
    if (n == 0) return;
    for (int it = 0; it < iters; it++)
        for (int color : {order, 1 - order}) {
            ++g.launch_count;
            launch::launch_kernel(k_amg_gs, n, 128, 0, s, g.topo, g.d_mg + g.mg_offset[level], n, X, RHS, (const uint8_t*)g.d_amg_ct,
                                  (const float*)g.d_amg, amg_plane(g), color, S);
        }
}

}  // namespace

int amg_prepare(DevGrid& g, float one_over_alpha, cudaStream_t s) {
    const size_t cells = amg_plane(g);
    if (!g.d_amg) {
        if (cudaMalloc(&g.d_amg, 4 * cells * sizeof(float)) != cudaSuccess) return 3;
        if (cudaMalloc(&g.d_amg_ct, cells) != cudaSuccess) {
            cudaFree(g.d_amg);
            g.d_amg = nullptr;
            return 3;
        }
        g.bytes += 4 * cells * sizeof(float) + cells;
    }
    cudaMemsetAsync(g.d_amg, 0, 4 * cells * sizeof(float), s);
    k_amg_types<<<g.n, 128, 0, s>>>(g.topo, g.n, g.d_amg_ct);
    if (g.n_leafghost > 0) k_amg_coeffs<<<g.n_leafghost, 128, 0, s>>>(g.topo, g.d_leafghost, g.n_leafghost, g.d_amg_ct, g.d_amg, cells);
    for (int l = g.max_level; l >= 0; l--)
        if (g.level_count[l] > 0)
            k_amg_coarsen<<<g.level_count[l], 128, 0, s>>>(g.topo, g.d_child, g.level_first[l], g.level_count[l], g.d_amg_ct, g.d_amg, cells,
                                                           one_over_alpha);
    g.launch_count += 2 + g.max_level + 1;
    if (cudaGetLastError() != cudaSuccess) return 2;
    // per instance, its entries of the level-0 LEAF|NONLEAF list (the list is instance by
    // instance): the coarsest level's sweeps run as one CTA per instance
    if (!g.d_amg_l0 && g.mg_count[0] > 0) {
        // from the host tables: the level-0 list holds the level's LEAF|NONLEAF tiles in pool
        // order, and each instance's tiles of a level are one run of the pool
        std::vector<int> inst(g.n, -1);
        for (int i = 0; i < g.num_inst; i++)
            for (const TileRun& r : g.inst_runs[i])
                for (int t = r.global; t < r.global + r.count; t++) inst[t] = i;
        std::vector<int2> ranges(g.num_inst, int2{0, 0});
        bool contiguous = true;
        int q = 0;
        for (int t = g.level_first[0]; t < g.level_first[0] + g.level_count[0]; t++) {
            if (!(g.h_tile_type[t] & (LEAF_T | NONLEAF_T))) continue;
            int2& r = ranges[inst[t]];
            if (r.y == 0) r.x = q;
            else if (r.x + r.y != q) contiguous = false;
            r.y++;
            q++;
        }
        if (q != g.mg_count[0]) contiguous = false;
        g.amg_l0_max = 0;
        if (contiguous)  // (else the sweeps take one launch each)
            for (const int2& r : ranges) g.amg_l0_max = std::max(g.amg_l0_max, (int)r.y);
        if (cudaMalloc(&g.d_amg_l0, sizeof(int2) * g.num_inst) != cudaSuccess) return 3;
        if (cudaMemcpy(g.d_amg_l0, ranges.data(), sizeof(int2) * g.num_inst, cudaMemcpyHostToDevice) != cudaSuccess) return 2;
    }
    g.amg_ready = true;
    return 0;
}

int amg_download(const DevGrid& g, float* coeffs, uint8_t* types, cudaStream_t s) {
    if (!g.amg_ready) return 1;
    const size_t cells = amg_plane(g);
    if (coeffs && cudaMemcpyAsync(coeffs, g.d_amg, 4 * cells * sizeof(float), cudaMemcpyDeviceToHost, s) != cudaSuccess) return 2;
    if (types && cudaMemcpyAsync(types, g.d_amg_ct, cells, cudaMemcpyDeviceToHost, s) != cudaSuccess) return 2;
    return cudaStreamSynchronize(s) == cudaSuccess ? 0 : 2;
}

// VCycleAMG (src/AMGSolver.cu:610-715): x = 0, rhs = f (0 on GHOST tiles); downstroke per level
// GaussSeidelAMG(level_iters, order 0), residual, restriction; level 0 GaussSeidelAMG(ci/2, 0) +
// GaussSeidelAMG(ci/2, 1); upstroke ProlongateAndUpdate128 + GaussSeidelAMG(level_iters, 1).
void vcycle_amg(const DevGrid& g, float* X, const float* F, float* TMP, float* RHS, int level_iters, int coarsest_iters,
                float one_over_alpha, float prolong_coeff, const Scalars* S, cudaStream_t s) {
    const size_t plane = amg_plane(g);
    launch::vcycle_init(g, X, RHS, F, S, s);
    for (int l = g.max_level; l > 0; l--) {
        amg_gauss_seidel(g, level_iters, 0, l, X, RHS, S, s);
        if (g.level_count[l] > 0) {
            ++g.launch_count;
            launch::launch_kernel(k_amg_residual, g.level_count[l], 128, 0, s, g.topo, g.level_first[l], g.level_count[l], (const float*)X,
                                  (const float*)RHS, TMP, (const uint8_t*)g.d_amg_ct, (const float*)g.d_amg, plane, S);
        }
        if (g.level_count[l - 1] > 0) {
            ++g.launch_count;
            launch::launch_kernel(k_amg_restrict, g.level_count[l - 1], 128, 0, s, g.topo, (const int*)g.d_child, g.level_first[l - 1],
                                  g.level_count[l - 1], F, (const float*)TMP, RHS, (const uint8_t*)g.d_amg_ct, one_over_alpha, S);
        }
    }
    // level 0: GaussSeidelAMG(ci/2, 0) + GaussSeidelAMG(ci/2, 1), as one sequence per instance
    // where every instance's level-0 tiles fit one CTA's rounds, else one launch per sweep
    if (g.d_amg_l0 && g.amg_l0_max > 0 && g.mg_count[0] > 0) {
        std::vector<int> cols;
        for (int it = 0; it < coarsest_iters / 2; it++) { cols.push_back(0); cols.push_back(1); }
        for (int it = 0; it < coarsest_iters / 2; it++) { cols.push_back(1); cols.push_back(0); }
        const int threads = 128 * std::min(8, g.amg_l0_max);
        for (size_t c0 = 0; c0 < cols.size(); c0 += 32) {
            uint32_t colors = 0;
            const int ns = (int)std::min<size_t>(32, cols.size() - c0);
            for (int k = 0; k < ns; k++) colors |= (uint32_t)cols[c0 + k] << k;
            ++g.launch_count;
            launch::launch_kernel(k_amg_gs_sequence, g.num_inst, threads, 0, s, g.topo, (const int*)(g.d_mg + g.mg_offset[0]),
                                  (const int2*)g.d_amg_l0, X, (const float*)RHS, (const uint8_t*)g.d_amg_ct, (const float*)g.d_amg, plane,
                                  colors, ns, S);
        }
    } else {
        amg_gauss_seidel(g, coarsest_iters / 2, 0, 0, X, RHS, S, s);
        amg_gauss_seidel(g, coarsest_iters / 2, 1, 0, X, RHS, S, s);
    }
    for (int l = 1; l <= g.max_level; l++) {
        if (g.level_count[l] > 0) {
            ++g.launch_count;
            launch::launch_kernel(k_amg_prolong, g.level_count[l], 128, 0, s, g.topo, g.level_first[l], g.level_count[l], X,
                                  (const uint8_t*)g.d_amg_ct, prolong_coeff, S);
        }
        amg_gauss_seidel(g, level_iters, 1, l, X, RHS, S, s);
    }
}

}  // namespace cirrus
