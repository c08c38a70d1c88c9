// V-cycle with fewer, lean launches -- the reference's V-cycle schedule (src/GMGSolver.cu:383-447
// with level_iters = 1) and arithmetic, bit for bit:
//
//   down, level l:  k_presmooth      GaussSeidelGMG(1, order 0) from x = 0 in one launch: the
//                                    first colour is pointwise (x = b/D), so the second colour
//                                    only needs first-colour values of the tile's own cells and
//                                    of the first cell layer of each face neighbour, recomputed
//                                    in place;
//                   k_residual_restrict (GHOST x and right-hand sides are 0)
//   levels 0..lb:   k_bottom         the whole V-cycle of the small coarse levels in one CTA with
//                                    x, right-hand side, masks and metadata in shared memory
//   up, level l:    k_prolong_sweep  ProlongateAndUpdate128 applied while staging the tile and
//                                    its face halos, then the first colour (1) of
//                                    GaussSeidelGMG(1, 1);
//                   k_gs_sweep       the second colour (0)
//
// The pre-smoothed x goes to a separate buffer (xpre, zero on GHOST tiles) so that no kernel
// reads values that another CTA of the same launch writes.  The multigrid right-hand side of
// LEAF tiles is r, written by the PCG kernels that write r, so no V-cycle initialisation pass
// runs; the right-hand side of GHOST tiles must hold 0 (zero_ghost_tiles once per solve).
#include "kernels.cuh"
#include "solver_internal.hpp"

namespace cirrus {

namespace {

// Diagonal h^3 * sum_f c_f of cell (i, j, k) with stencil mask mm in a tile whose multigrid
// cross-face classes are `cls`: the summation order of neg_lap4's diagonal.
__device__ __forceinline__ float cell_diag(int i, int j, int k, uint32_t mm, uint32_t cls, const LevelConst<float>& L) {
    auto cross = [&](int f) -> float { return ((cls >> (2 * f)) & 3u) == 2u ? L.c2 : L.c1; };
    const float a0 = (mm & 1u) ? (i == 0 ? cross(0) : L.c1) : 0.f;
    const float a1 = (mm & 2u) ? (i == 7 ? cross(1) : L.c1) : 0.f;
    const float a2 = (mm & 4u) ? (j == 0 ? cross(2) : L.c1) : 0.f;
    const float a3 = (mm & 8u) ? (j == 7 ? cross(3) : L.c1) : 0.f;
    const float a4 = (mm & 16u) ? (k == 0 ? cross(4) : L.c1) : 0.f;
    const float a5 = (mm & 32u) ? (k == 7 ? cross(5) : L.c1) : 0.f;
    float d = 0.f;
    d = d + a0; d = d + a1; d = d + a2; d = d + a3; d = d + a4; d = d + a5;
    return (mm & kMaskInterior) ? d * L.h * L.h * L.h : 0.f;
}

// Cell of face neighbour f's first layer stored in halo slot h (the hx[f][64] order of
// load_halo: x faces [j][k], y faces [i][k], z faces [i][j]).
__device__ __forceinline__ void halo_cell_ijk(int face, int h, int& i, int& j, int& k) {
    const int a = h >> 3, b = h & 7;
    switch (face) {
        case 0: i = 7; j = a; k = b; break;
        case 1: i = 0; j = a; k = b; break;
        case 2: i = a; j = 7; k = b; break;
        case 3: i = a; j = 0; k = b; break;
        case 4: i = a; j = b; k = 7; break;
        default: i = a; j = b; k = 0; break;
    }
}

// First-colour (0) value of cell (i, j, k) of mg tile `tile` after one sweep from x = 0:
// 0 + (b - 0) / D on INTERIOR cells of colour 0, else 0.
__device__ __forceinline__ float first_colour(const Topo& tp, const float* __restrict__ RHS, int tile, int i, int j, int k,
                                              const LevelConst<float>& L) {
    if (((i + j + k) & 1) != 0) return 0.f;
    const int off = (i << 6) | (j << 3) | k;
    const uint32_t mm = tp.mask_mg[(size_t)tile * kTileCells + off];
    if (!(mm & kMaskInterior)) return 0.f;
    const float D = cell_diag(i, j, k, mm, (tp.fcls[tile] >> 12) & 0xfffu, L);
    return 0.f + (RHS[(size_t)tile * kTileCells + off] - 0.f) / D;
}

}  // namespace

// ---------------------------------------------------------------------------- down: pre-smoother
// GaussSeidelGMG(1, 0) on the mg tiles (LEAF|NONLEAF) of one level, x starting from 0; the
// result goes to XP.  GHOST neighbours hold x = 0 on the way down (they are not smoothed).
template <int TPB>
__global__ void __launch_bounds__(128 * TPB) k_presmooth(Topo tp, const int* __restrict__ list, int n, float* XP,
                                                         const float* __restrict__ RHS, const int* __restrict__ done) {
    __shared__ TileShared<float> sh[TPB];
    if (done && *done) return;
    const int g = threadIdx.x >> 7, t = threadIdx.x & 127;
    const int q = blockIdx.x * TPB + g;
    const bool active = q < n;
    const int tile = active ? list[q] : 0;
    const TileIdx ix(t);
    TileMeta m;
    V4<float> b;
    uint32_t mask4 = 0, cls = 0;
    LevelConst<float> L(tp.h0, 0);
    if (active) {
        m = tp.meta[tile];
        L = LevelConst<float>(tp.h0, meta_level(m.packed));
        b = ld4(RHS + (size_t)tile * kTileCells + t * 4);
        mask4 = *reinterpret_cast<const uint32_t*>(tp.mask_mg + (size_t)tile * kTileCells + t * 4);
        cls = (tp.fcls[tile] >> 12) & 0xfffu;
        // first colour of the own cells
        V4<float> x1;
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const int k = ix.k0 + e;
            const uint32_t mm = (mask4 >> (8 * e)) & 0xffu;
            float v = 0.f;
            if (((ix.i + ix.j + k) & 1) == 0 && (mm & kMaskInterior))
                v = 0.f + (b.v[e] - 0.f) / cell_diag(ix.i, ix.j, k, mm, cls, L);
            x1.v[e] = v;
        }
        st4(sh[g].xs + t * 4, x1);
        // first colour of the face neighbours' first cell layer
        if (t < 64) {
            const int face = t >> 4, qq = t & 15;
            const int nb = m.nb[face];
            const bool live = nb >= 0 && !meta_nb_ghost(m.packed, face);
            V4<float> v;
#pragma unroll
            for (int e = 0; e < 4; e++) {
                int i, j, k;
                halo_cell_ijk(face, qq * 4 + e, i, j, k);
                v.v[e] = live ? first_colour(tp, RHS, nb, i, j, k, L) : 0.f;
            }
            st4(sh[g].hx + face * 64 + qq * 4, v);
        }
        {
            const int face = 4 + (t >> 6), c = t & 63;
            const int nb = m.nb[face];
            int i, j, k;
            halo_cell_ijk(face, c, i, j, k);
            sh[g].hx[face * 64 + c] = (nb >= 0 && !meta_nb_ghost(m.packed, face)) ? first_colour(tp, RHS, nb, i, j, k, L) : 0.f;
        }
    }
    __syncthreads();
    if (!active) return;
    // second colour (1), from the first-colour values
    float ax[4], d[4];
    neg_lap4<float, true>(sh[g].xs, sh[g].hx, t, mask4, cls, L, ax, d);
    V4<float> o = ld4(sh[g].xs + t * 4);
#pragma unroll
    for (int e = 0; e < 4; e++) {
        if (((ix.i + ix.j + ix.k0 + e) & 1) != 1) continue;
        const bool interior = (mask4 >> (8 * e)) & kMaskInterior;
        o.v[e] = o.v[e] + (interior ? (b.v[e] - ax[e]) / d[e] : 0.f);
    }
    st4(XP + (size_t)tile * kTileCells + t * 4, o);
}

// ---------------------------------------------------------------------------- up: prolongation + first colour
// Value of cell `off` of `tile` after ProlongateAndUpdate128 (src/GMGSolver.cu:345-376): parent
// value by injection; GHOST: x = cx, others x = fma(prolong_coeff, cx, xpre); 0 off INTERIOR.
__device__ __forceinline__ float prolongated(const Topo& tp, const float* __restrict__ Z, const float* __restrict__ XP, int tile,
                                             const TileMeta& tm, int off, float prolong_coeff) {
    if (!(tp.mask_mg[(size_t)tile * kTileCells + off] & kMaskInterior)) return 0.f;
    float cx = 0.f;
    if (tm.parent >= 0) {
        const int oct = meta_octant(tm.packed);
        cx = Z[(size_t)tm.parent * kTileCells + ((oct & 1) * 4 + (off >> 7)) * 64 + (((oct >> 1) & 1) * 4 + ((off >> 4) & 3)) * 8 +
               ((oct >> 2) & 1) * 4 + ((off & 7) >> 1)];
    }
    return (meta_type(tm.packed) & GHOST_T) ? cx : fmaf(prolong_coeff, cx, XP[(size_t)tile * kTileCells + off]);
}

// Prolongation into every tile of one level; on mg tiles also the first colour (1) of
// GaussSeidelGMG(1, 1).  Reads Z of the coarser level and XP of this level, writes Z of this level.
template <int TPB>
__global__ void __launch_bounds__(128 * TPB) k_prolong_sweep(Topo tp, int first, int n, float* Z, const float* __restrict__ XP,
                                                             const float* __restrict__ RHS, float prolong_coeff,
                                                             const int* __restrict__ done) {
    __shared__ TileShared<float> sh[TPB];
    if (done && *done) return;
    const int g = threadIdx.x >> 7, t = threadIdx.x & 127;
    const int q = blockIdx.x * TPB + g;
    const bool active = q < n;
    const int tile = first + (active ? q : 0);
    TileMeta m;
    bool ghost = false;
    if (active) {
        m = tp.meta[tile];
        ghost = meta_type(m.packed) & GHOST_T;
        V4<float> own;
#pragma unroll
        for (int e = 0; e < 4; e++) own.v[e] = prolongated(tp, Z, XP, tile, m, t * 4 + e, prolong_coeff);
        st4(sh[g].xs + t * 4, own);
        if (!ghost) {
            if (t < 64) {
                const int face = t >> 4, qq = t & 15;
                const int nb = m.nb[face];
                int off;
                if (face == 0) off = 448 + qq * 4;
                else if (face == 1) off = qq * 4;
                else if (face == 2) off = (qq >> 1) * 64 + 56 + (qq & 1) * 4;
                else off = (qq >> 1) * 64 + (qq & 1) * 4;
                V4<float> v = zero4<float>();
                if (nb >= 0) {
                    const TileMeta nm = tp.meta[nb];
#pragma unroll
                    for (int e = 0; e < 4; e++) v.v[e] = prolongated(tp, Z, XP, nb, nm, off + e, prolong_coeff);
                }
                st4(sh[g].hx + face * 64 + qq * 4, v);
            }
            {
                const int face = 4 + (t >> 6), c = t & 63;
                const int nb = m.nb[face];
                sh[g].hx[face * 64 + c] =
                    nb >= 0 ? prolongated(tp, Z, XP, nb, tp.meta[nb], (c >> 3) * 64 + (c & 7) * 8 + (face == 4 ? 7 : 0), prolong_coeff)
                            : 0.f;
            }
        }
    }
    __syncthreads();
    if (!active) return;
    V4<float> o = ld4(sh[g].xs + t * 4);
    if (!ghost) {
        const uint32_t mask4 = *reinterpret_cast<const uint32_t*>(tp.mask_mg + (size_t)tile * kTileCells + t * 4);
        const V4<float> b = ld4(RHS + (size_t)tile * kTileCells + t * 4);
        const LevelConst<float> L(tp.h0, meta_level(m.packed));
        float ax[4], d[4];
        neg_lap4<float, true>(sh[g].xs, sh[g].hx, t, mask4, (tp.fcls[tile] >> 12) & 0xfffu, L, ax, d);
        const TileIdx ix(t);
#pragma unroll
        for (int e = 0; e < 4; e++) {
            if (((ix.i + ix.j + ix.k0 + e) & 1) != 1) continue;
            const bool interior = (mask4 >> (8 * e)) & kMaskInterior;
            o.v[e] = o.v[e] + (interior ? (b.v[e] - ax[e]) / d[e] : 0.f);
        }
    }
    st4(Z + (size_t)tile * kTileCells + t * 4, o);
}

// Right-hand sides of GHOST tiles to 0 (the V-cycle's initialisation of them, src/GMGSolver.cu:393-396).
__global__ void __launch_bounds__(128) k_zero_tiles(const int* __restrict__ list, int n, float* X) {
    const int q = blockIdx.x;
    if (q < n) st4(X + (size_t)list[q] * kTileCells + threadIdx.x * 4, zero4<float>());
}

// ---------------------------------------------------------------------------- small levels
// Levels 0..lb (the first nb tiles of the all-tiles order) in one CTA: x, right-hand side, masks,
// metadata and the mg list in shared memory; a phase program of colour sweeps, residual +
// restrictions and prolongations (the reference's schedule) separated by __syncthreads.
constexpr int kBottomMaxPhases = 256;
constexpr int kBottomMaxLevels = 16;
struct BottomProgram {
    int nphase;
    uint8_t op[kBottomMaxPhases];  // 1 sweep, 2 residual+restrict, 3 prolongate
    uint8_t level[kBottomMaxPhases];
    uint8_t color[kBottomMaxPhases];
};
struct BottomLevels {
    int mg_off[kBottomMaxLevels], mg_cnt[kBottomMaxLevels], first[kBottomMaxLevels], cnt[kBottomMaxLevels];
};

struct BottomView {
    const float* X;
    const uint8_t* MK;
    const TileMeta* M;
    const uint32_t* CL;
};

// negativeLap (times h^3, INTERIOR cells) of cell (i, j, k) of shared tile `tile`, and its
// diagonal: the operation order of neg_lap4.
template <bool DIAG>
__device__ __forceinline__ float smem_neglap(const BottomView& v, int tile, int i, int j, int k, const LevelConst<float>& L,
                                             float* diag) {
    const float* xs = v.X + tile * kTileCells;
    const TileMeta& m = v.M[tile];
    auto nbv = [&](int f, int off) -> float { return m.nb[f] >= 0 ? v.X[m.nb[f] * kTileCells + off] : 0.f; };
    const int c = (i << 6) | (j << 3) | k;
    const uint32_t mm = v.MK[tile * kTileCells + c];
    const uint32_t cls = v.CL[tile];
    auto cross = [&](int f) -> float { return ((cls >> (2 * f)) & 3u) == 2u ? L.c2 : L.c1; };
    const float x0 = xs[c];
    const float xm = i > 0 ? xs[c - 64] : nbv(0, 448 + (c & 63));
    const float xp = i < 7 ? xs[c + 64] : nbv(1, c & 63);
    const float ym = j > 0 ? xs[c - 8] : nbv(2, (i << 6) | 56 | k);
    const float yp = j < 7 ? xs[c + 8] : nbv(3, (i << 6) | k);
    const float zm = k > 0 ? xs[c - 1] : nbv(4, c | 7);
    const float zp = k < 7 ? xs[c + 1] : nbv(5, c & ~7);
    const float a0 = (mm & 1u) ? (i == 0 ? cross(0) : L.c1) : 0.f;
    const float a1 = (mm & 2u) ? (i == 7 ? cross(1) : L.c1) : 0.f;
    const float a2 = (mm & 4u) ? (j == 0 ? cross(2) : L.c1) : 0.f;
    const float a3 = (mm & 8u) ? (j == 7 ? cross(3) : L.c1) : 0.f;
    const float a4 = (mm & 16u) ? (k == 0 ? cross(4) : L.c1) : 0.f;
    const float a5 = (mm & 32u) ? (k == 7 ? cross(5) : L.c1) : 0.f;
    float s = 0.f;
    s = fmaf(a0, x0 - xm, s);
    s = fmaf(a1, x0 - xp, s);
    s = fmaf(a2, x0 - ym, s);
    s = fmaf(a3, x0 - yp, s);
    s = fmaf(a4, x0 - zm, s);
    s = fmaf(a5, x0 - zp, s);
    const bool interior = mm & kMaskInterior;
    if (DIAG) {
        float d = 0.f;
        d = d + a0; d = d + a1; d = d + a2; d = d + a3; d = d + a4; d = d + a5;
        *diag = interior ? d * L.h * L.h * L.h : 0.f;
    }
    return interior ? s * L.h * L.h * L.h : 0.f;
}

size_t bottom_smem_bytes(int nb) {
    return (size_t)nb * (2 * kTileCells * sizeof(float) + kTileCells + sizeof(TileMeta) + sizeof(uint32_t) + sizeof(int)) + 64;
}

__global__ void __launch_bounds__(1024) k_bottom(Topo tp, int nb, int nmg, const int* __restrict__ mg, float* Z,
                                                 const float* __restrict__ RHS, float one_over_alpha, float prolong_coeff,
                                                 BottomProgram prog, BottomLevels lv, const int* __restrict__ done) {
    extern __shared__ __align__(16) unsigned char bsm[];
    float* X = reinterpret_cast<float*>(bsm);
    float* B = X + nb * kTileCells;
    TileMeta* M = reinterpret_cast<TileMeta*>(B + nb * kTileCells);
    uint8_t* MK = reinterpret_cast<uint8_t*>(M + nb);
    uint32_t* CL = reinterpret_cast<uint32_t*>(MK + nb * kTileCells);
    int* MG = reinterpret_cast<int*>(CL + nb);
    if (done && *done) return;
    for (int t = threadIdx.x; t < nb; t += blockDim.x) {
        M[t] = tp.meta[t];
        CL[t] = (tp.fcls[t] >> 12) & 0xfffu;
    }
    for (int i = threadIdx.x; i < nmg; i += blockDim.x) MG[i] = mg[i];
    for (int u = threadIdx.x; u < nb * 128; u += blockDim.x) {
        const bool ghost = meta_type(tp.meta[u >> 7].packed) & GHOST_T;
        st4(X + u * 4, zero4<float>());
        st4(B + u * 4, ghost ? zero4<float>() : ld4(RHS + (size_t)u * 4));
        *reinterpret_cast<uint32_t*>(MK + u * 4) = *reinterpret_cast<const uint32_t*>(tp.mask_mg + (size_t)u * 4);
    }
    __syncthreads();
    const BottomView v{X, MK, M, CL};
    for (int ph = 0; ph < prog.nphase; ph++) {
        const int op = prog.op[ph], level = prog.level[ph];
        const LevelConst<float> L(tp.h0, level);
        if (op == 1) {
            // one colour of GaussSeidelGMG on the level's mg tiles; items are the 256 cells of the
            // colour, whose neighbours all have the other colour
            const int color = prog.color[ph];
            const int n = lv.mg_cnt[level] * 256, base = lv.mg_off[level];
            for (int it = threadIdx.x; it < n; it += blockDim.x) {
                const int tile = MG[base + (it >> 8)], u = it & 255;
                const int i = u >> 5, j = (u >> 2) & 7, k = ((u & 3) << 1) | ((i + j + color) & 1);
                float d;
                const float ax = smem_neglap<true>(v, tile, i, j, k, L, &d);
                const int c = tile * kTileCells + ((i << 6) | (j << 3) | k);
                const bool interior = MK[c] & kMaskInterior;
                X[c] = X[c] + (interior ? (B[c] - ax) / d : 0.f);
            }
        } else if (op == 2) {
            // residual and restriction; items are the 64 2x2x2 blocks of the level's tiles
            const int n = lv.cnt[level] * 64, first = lv.first[level];
            for (int it = threadIdx.x; it < n; it += blockDim.x) {
                const int tile = first + (it >> 6), blk = it & 63;
                const TileMeta& m = M[tile];
                if (m.parent < 0) continue;
                const int fi = blk / 16 * 2, fj = (blk / 4) % 4 * 2, fk = blk % 4 * 2;
                float sum = 0.f;
#pragma unroll
                for (int ii = 0; ii < 2; ii++)
#pragma unroll
                    for (int jj = 0; jj < 2; jj++)
#pragma unroll
                        for (int kk = 0; kk < 2; kk++) {
                            const int i = fi + ii, j = fj + jj, k = fk + kk;
                            const float ax = smem_neglap<false>(v, tile, i, j, k, L, nullptr);
                            sum += B[tile * kTileCells + ((i << 6) | (j << 3) | k)] - ax;
                        }
                const int oct = meta_octant(m.packed);
                const int pid = m.parent * kTileCells + ((oct & 1) * 4 + fi / 2) * 64 + (((oct >> 1) & 1) * 4 + fj / 2) * 8 +
                                ((oct >> 2) & 1) * 4 + fk / 2;
                // parents are one level coarser: no cell written here is read in this phase, and
                // each parent cell has exactly one child block
                if (meta_type(m.packed) & GHOST_T) B[pid] += sum;
                else B[pid] = sum * one_over_alpha;
            }
        } else {
            // prolongation and update of the level's tiles (parents one level coarser)
            const int n = lv.cnt[level] * kTileCells, first = lv.first[level];
            for (int it = threadIdx.x; it < n; it += blockDim.x) {
                const int tile = first + (it >> 9), c = it & (kTileCells - 1);
                const TileMeta& m = M[tile];
                float cx = 0.f;
                if (m.parent >= 0) {
                    const int oct = meta_octant(m.packed);
                    cx = X[m.parent * kTileCells + ((oct & 1) * 4 + (c >> 7)) * 64 + (((oct >> 1) & 1) * 4 + ((c >> 4) & 3)) * 8 +
                           ((oct >> 2) & 1) * 4 + ((c & 7) >> 1)];
                }
                float& x = X[tile * kTileCells + c];
                x = (MK[tile * kTileCells + c] & kMaskInterior) ? ((meta_type(m.packed) & GHOST_T) ? cx : fmaf(prolong_coeff, cx, x)) : 0.f;
            }
        }
        __syncthreads();
    }
    for (int u = threadIdx.x; u < nb * 128; u += blockDim.x) st4(Z + (size_t)u * 4, ld4(X + u * 4));
}

namespace launch {

constexpr int kTPB2 = 2;

void presmooth(const DevGrid& g, int level, float* XP, const float* RHS, const int* done, cudaStream_t s) {
    const int n = g.mg_count[level];
    if (n == 0) return;
    ++g.launch_count;
    k_presmooth<kTPB2><<<(n + kTPB2 - 1) / kTPB2, 128 * kTPB2, 0, s>>>(g.topo, g.d_mg + g.mg_offset[level], n, XP, RHS, done);
}

void prolong_sweep(const DevGrid& g, int level, float* Z, const float* XP, const float* RHS, float prolong_coeff, const int* done,
                   cudaStream_t s) {
    const int n = g.level_count[level];
    if (n == 0) return;
    ++g.launch_count;
    k_prolong_sweep<kTPB2><<<(n + kTPB2 - 1) / kTPB2, 128 * kTPB2, 0, s>>>(g.topo, g.level_first[level], n, Z, XP, RHS,
                                                                           prolong_coeff, done);
}

void zero_ghost_tiles(const DevGrid& g, float* X, cudaStream_t s) {
    if (g.n_ghost == 0) return;
    ++g.launch_count;
    k_zero_tiles<<<g.n_ghost, 128, 0, s>>>(g.d_ghost, g.n_ghost, X);
}

bool bottom(const DevGrid& g, int lb, int coarsest_iters, float* Z, const float* RHS, float one_over_alpha, float prolong_coeff,
            const int* done, cudaStream_t s) {
    BottomProgram p{};
    auto push = [&](int op, int level, int color) {
        if (p.nphase >= kBottomMaxPhases) return false;
        p.op[p.nphase] = (uint8_t)op;
        p.level[p.nphase] = (uint8_t)level;
        p.color[p.nphase] = (uint8_t)color;
        p.nphase++;
        return true;
    };
    bool ok = lb < kBottomMaxLevels;
    for (int l = lb; ok && l > 0; l--) ok = push(1, l, 0) && push(1, l, 1) && push(2, l, 0);
    for (int it = 0; ok && it < coarsest_iters / 2; it++) ok = push(1, 0, 0) && push(1, 0, 1);
    for (int it = 0; ok && it < coarsest_iters / 2; it++) ok = push(1, 0, 1) && push(1, 0, 0);
    for (int l = 1; ok && l <= lb; l++) ok = push(3, l, 0) && push(1, l, 1) && push(1, l, 0);
    if (!ok) return false;
    BottomLevels lv{};
    for (int l = 0; l <= lb; l++) {
        lv.mg_off[l] = g.mg_offset[l];
        lv.mg_cnt[l] = g.mg_count[l];
        lv.first[l] = g.level_first[l];
        lv.cnt[l] = g.level_count[l];
    }
    const int nb = g.level_first[lb] + g.level_count[lb];
    const int nmg = g.mg_offset[lb] + g.mg_count[lb];
    if (nb > kBottomTiles) return false;
    ++g.launch_count;
    k_bottom<<<1, 1024, bottom_smem_bytes(nb), s>>>(g.topo, nb, nmg, g.d_mg, Z, RHS, one_over_alpha, prolong_coeff, p, lv, done);
    return true;
}

bool bottom_supported(int coarsest_iters, int lb) {
    return lb < kBottomMaxLevels && 2 * coarsest_iters + 6 * lb <= kBottomMaxPhases;
}

void init_kernel_attributes() {
    cudaFuncSetAttribute(k_bottom, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bottom_smem_bytes(kBottomTiles));
}

}  // namespace launch
}  // namespace cirrus
