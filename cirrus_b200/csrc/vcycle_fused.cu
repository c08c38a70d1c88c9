// V-cycle with fewer, lean launches -- the reference's V-cycle schedule (src/GMGSolver.cu:383-447
// with level_iters = 1) and arithmetic, bit for bit:
//
//   down, level l:  k_presmooth      GaussSeidelGMG(1, order 0) from x = 0 in one launch: the
//                                    first colour is pointwise (x = b/D), so the second colour
//                                    only needs first-colour values of the tile's own cells and
//                                    of the first cell layer of each face neighbour, recomputed
//                                    in place;
//                   k_residual_restrict (GHOST x and right-hand sides are 0)
//   levels 0..lb:   k_bottom         the whole V-cycle of the small coarse levels in one CTA, each
//                                    level a dense box of x, right-hand side and stencil codes in
//                                    shared memory
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
    if (mm == (uint32_t)kMaskFull) return L.dfast;
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

}  // namespace

// ---------------------------------------------------------------------------- down: pre-smoother
// Staging area of the pre-smoother: first-colour values of the tile (xs) and of the face
// neighbours' first layer (hx) are computed in place from the staged right-hand sides (b, hx)
// and masks (mask, hmask).
struct __align__(16) PreStage {
    float xs[kTileCells];
    float hx[6 * 64];
    float b[kTileCells];
    uint8_t mask[kTileCells];
    uint8_t hmask[6 * 64];
};

// GaussSeidelGMG(1, 0) on the mg tiles (LEAF|NONLEAF) of one level, x starting from 0; the
// result goes to XP.  GHOST neighbours hold x = 0 on the way down (they are not smoothed).
// NT tiles per 128-thread group are staged with asynchronous copies before any is computed.
template <int TPB, int NT>
__device__ __forceinline__ void k_presmooth_body(Topo tp, const int* __restrict__ list, int n, float* XP,
                                                         const float* __restrict__ RHS, const Scalars* __restrict__ S) {
    pdl_trigger();
    extern __shared__ __align__(16) unsigned char pre_smem[];
    PreStage* st = reinterpret_cast<PreStage*>(pre_smem);
    const int g = threadIdx.x >> 7, t = threadIdx.x & 127;
    const TileIdx ix(t);
    int tile[NT], ptile[NT];
    bool act[NT];
#pragma unroll
    for (int u = 0; u < NT; u++) {
        const int q = (blockIdx.x * NT + u) * TPB + g;
        tile[u] = q < n ? list[q] : 0;
        act[u] = q < n;  // finished instances are dropped after the copies are issued (reading them is harmless)
        ptile[u] = (tp.pf > 0 && t == 0 && q + tp.pf < n) ? list[q + tp.pf] : -1;
    }
    // neighbour of this thread's x/y-face piece (t < 64) and z-face cell; GHOST neighbours count
    // as absent (their x is 0 on the way down).  Metadata of all NT tiles is loaded before any
    // copy is issued (see TilePre).
    const int fface = t >> 4, qq = t & 15;
    int foff;
    if (fface == 0) foff = 448 + qq * 4;
    else if (fface == 1) foff = qq * 4;
    else if (fface == 2) foff = (qq >> 1) * 64 + 56 + (qq & 1) * 4;
    else foff = (qq >> 1) * 64 + (qq & 1) * 4;
    const int zface = 4 + (t >> 6), zc = t & 63;
    const int zoff = (zc >> 3) * 64 + (zc & 7) * 8 + (zface == 4 ? 7 : 0);
    int nbf[NT], nbz[NT], inst[NT];
    int packed[NT];
    uint32_t fc[NT], nfc_f[NT], nfc_z[NT], zmb[NT];
    float4 lc[NT];
#pragma unroll
    for (int u = 0; u < NT; u++) {
        const TileMeta& m = tp.meta[tile[u]];
        packed[u] = m.packed;
        const int nf = t < 64 ? m.nb[fface] : -1, nz = m.nb[zface];
        nbf[u] = (act[u] && nf >= 0 && !meta_nb_ghost(m.packed, fface)) ? nf : -1;
        nbz[u] = (act[u] && nz >= 0 && !meta_nb_ghost(m.packed, zface)) ? nz : -1;
        fc[u] = tp.fcls[tile[u]];
        inst[u] = tp.inst[tile[u]];
    }
#pragma unroll
    for (int u = 0; u < NT; u++) {
        lc[u] = tp.lconst[inst[u] * kLevelSlots + meta_level(packed[u])];
        nfc_f[u] = nbf[u] >= 0 ? tp.fcls[nbf[u]] : 0u;
        nfc_z[u] = nbz[u] >= 0 ? tp.fcls[nbz[u]] : 0u;
        zmb[u] = nbz[u] >= 0 ? tp.mask_mg[(size_t)nbz[u] * kTileCells + zoff] : 0u;
    }
    pdl_wait();
#pragma unroll
    for (int u = 0; u < NT; u++) {
        if (!act[u]) continue;
        PreStage& ps = st[u * TPB + g];
        const size_t base = (size_t)tile[u] * kTileCells;
        if (t < 32) cp_async16(ps.mask + t * 16, tp.mask_mg + base + t * 16);
        if (nbf[u] >= 0) cp_async4(ps.hmask + fface * 64 + qq * 4, tp.mask_mg + (size_t)nbf[u] * kTileCells + foff);
        cp_async16(ps.b + t * 4, RHS + base + t * 4);
        if (nbf[u] >= 0) cp_async16(ps.hx + fface * 64 + qq * 4, RHS + (size_t)nbf[u] * kTileCells + foff);
        if (nbz[u] >= 0) cp_async4(ps.hx + zface * 64 + zc, RHS + (size_t)nbz[u] * kTileCells + zoff);
    }
#pragma unroll
    for (int u = 0; u < NT; u++)
        if (ptile[u] >= 0) {
            prefetch_l2(RHS + (size_t)ptile[u] * kTileCells, kTileCells * sizeof(float));
            prefetch_l2(tp.mask_mg + (size_t)ptile[u] * kTileCells, kTileCells);
        }
#pragma unroll
    for (int u = 0; u < NT; u++)
        if (nbz[u] >= 0) st[u * TPB + g].hmask[zface * 64 + zc] = (uint8_t)zmb[u];
#pragma unroll
    for (int u = 0; u < NT; u++) act[u] = act[u] && !tile_done(tp, S, tile[u]);
    cp_async_wait_all();
    __syncthreads();
    // first colour (0) of the own cells and of the live neighbours' first layer, in place
#pragma unroll
    for (int u = 0; u < NT; u++) {
        if (!act[u]) continue;
        PreStage& ps = st[u * TPB + g];
        const LevelConst<float> L(lc[u]);
        const uint32_t cls = (fc[u] >> 12) & 0xfffu;
        const uint32_t mask4 = *reinterpret_cast<const uint32_t*>(ps.mask + t * 4);
        st4(ps.xs + t * 4, first_colour_run(ix.i, ix.j, ix.k0, mask4, ld4(ps.b + t * 4), cls, L));
        if (t < 64) {
            const int face = fface;
            V4<float> v = zero4<float>();
            if (nbf[u] >= 0) {
                const int ni = foff >> 6, nj = (foff >> 3) & 7, nk0 = foff & 7;
                v = first_colour_run(ni, nj, nk0, *reinterpret_cast<const uint32_t*>(ps.hmask + face * 64 + qq * 4),
                                     ld4(ps.hx + face * 64 + qq * 4), (nfc_f[u] >> 12) & 0xfffu, L);
            }
            st4(ps.hx + face * 64 + qq * 4, v);
        }
        {
            const int face = zface, c = zc;
            float v = 0.f;
            if (nbz[u] >= 0) {
                int i, j, k;
                halo_cell_ijk(face, c, i, j, k);
                const uint32_t mm = ps.hmask[face * 64 + c];
                if (((i + j + k) & 1) == 0 && (mm & kMaskInterior))
                    v = 0.f + (ps.hx[face * 64 + c] - 0.f) / cell_diag(i, j, k, mm, (nfc_z[u] >> 12) & 0xfffu, L);
            }
            ps.hx[face * 64 + c] = v;
        }
    }
    __syncthreads();
    // second colour (1), from the first-colour values
#pragma unroll
    for (int u = 0; u < NT; u++) {
        if (!act[u]) continue;
        PreStage& ps = st[u * TPB + g];
        st4(XP + (size_t)tile[u] * kTileCells + t * 4,
            colour_update(ps.xs, ps.hx, t, *reinterpret_cast<const uint32_t*>(ps.mask + t * 4), (fc[u] >> 12) & 0xfffu,
                          LevelConst<float>(lc[u]), ld4(ps.b + t * 4), 1));
    }}
template <int TPB, int NT>
__global__ void __launch_bounds__(128 * TPB) k_presmooth(Topo tp, const int* __restrict__ list, int n, float* XP,
                                                         const float* __restrict__ RHS, const Scalars* __restrict__ S) {
    k_presmooth_body<TPB, NT>(tp, list, n, XP, RHS, S);
}
// the same kernel with at least MINB CTAs per SM (registers capped to fit)
template <int TPB, int NT, int MINB>
__global__ void __launch_bounds__(128 * TPB, MINB) k_presmooth_occ(Topo tp, const int* __restrict__ list, int n, float* XP,
                                                         const float* __restrict__ RHS, const Scalars* __restrict__ S) {
    k_presmooth_body<TPB, NT>(tp, list, n, XP, RHS, S);
}
template <int TPB, int NT, int MINB>
constexpr auto k_presmooth_shape() {
    if constexpr (MINB == 0) return &k_presmooth<TPB, NT>;
    else return &k_presmooth_occ<TPB, NT, MINB>;
}

// ---------------------------------------------------------------------------- up: prolongation + first colour
// Staging area of the prolongation kernel: the tile's pre-smoothed x, right-hand side, mask and
// its parent's octant block (4x4x4 coarse values); per face neighbour the pre-smoothed x and mask
// of its first layer and the coarse values over it.  xs/hx receive the prolongated values.
struct __align__(16) ProStage {
    float xs[kTileCells];
    float hx[6 * 64];
    float xp[kTileCells];
    float b[kTileCells];
    float hxp[6 * 64];
    float pblk[64];
    float hpar[4 * 16 * 2 + 2 * 64];  // x/y faces: 2 coarse values per 4-cell run; z faces: 1 per cell
    uint8_t mask[kTileCells];
    uint8_t hmask[6 * 64];
};

// The coarse cell under fine cell `off` of a tile in octant `oct` of its parent.
__device__ __forceinline__ int parent_cell(int oct, int off) {
    return ((oct & 1) * 4 + (off >> 7)) * 64 + (((oct >> 1) & 1) * 4 + ((off >> 4) & 3)) * 8 + ((oct >> 2) & 1) * 4 + ((off & 7) >> 1);
}

// prolongated() from staged values: mask byte mm, coarse value cx (0 without a parent), x.
__device__ __forceinline__ float prolong_value(uint32_t mm, bool ghost, float cx, float x, float prolong_coeff) {
    return (mm & kMaskInterior) ? (ghost ? cx : fmaf(prolong_coeff, cx, x)) : 0.f;
}

// Prolongation into one face layer of a GHOST tile (item: tile, face, parent tile, octant in the
// parent), one thread per cell: x = the parent value on INTERIOR cells, 0 elsewhere.  A GHOST
// tile's x is read only as the face halo of its non-GHOST neighbours at the same level (the
// second colour sweep), so only the faces towards those are written.
__device__ __forceinline__ void ghost_face_prolong(const Topo& tp, float* Z, int4 it, int c) {
    const int a = c >> 3, b = c & 7;
    int i, j, k;
    switch (it.y) {
        case 0: i = 0; j = a; k = b; break;
        case 1: i = 7; j = a; k = b; break;
        case 2: i = a; j = 0; k = b; break;
        case 3: i = a; j = 7; k = b; break;
        case 4: i = a; j = b; k = 0; break;
        default: i = a; j = b; k = 7; break;
    }
    const int off = i * 64 + j * 8 + k;
    const size_t base = (size_t)it.x * kTileCells;
    const float cx = it.z >= 0 ? Z[(size_t)it.z * kTileCells + parent_cell(it.w, off)] : 0.f;
    Z[base + off] = prolong_value(tp.mask_mg[base + off], true, cx, 0.f, 0.f);
}

// Prolongation into the tiles of one level; on non-GHOST tiles (list[0..n)) also the first
// colour (1) of GaussSeidelGMG(1, 1), NT tiles per 128-thread group staged with asynchronous
// copies; the first item_blocks CTAs prolongate GHOST face layers (ghost_face_prolong), two per
// 128 threads.  Reads Z of the coarser level and XP of this level, writes Z of this level.
template <int TPB, int NT>
__device__ __forceinline__ void k_prolong_sweep_body(Topo tp, const int* __restrict__ list, int n,
                                                             const int4* __restrict__ items, int nitems, int item_blocks, float* Z,
                                                             const float* __restrict__ XP, const float* __restrict__ RHS,
                                                             float prolong_coeff, const Scalars* __restrict__ S) {
    pdl_trigger();
    if ((int)blockIdx.x < item_blocks) {
        pdl_wait();
        const int q = (int)blockIdx.x * (2 * TPB) + ((int)threadIdx.x >> 6);
        if (q >= nitems) return;
        const int4 it = items[q];
        if (tile_done(tp, S, it.x)) return;
        ghost_face_prolong(tp, Z, it, threadIdx.x & 63);
        return;
    }
    extern __shared__ __align__(16) unsigned char pro_smem[];
    ProStage* st = reinterpret_cast<ProStage*>(pro_smem);
    const int g = threadIdx.x >> 7, t = threadIdx.x & 127;
    // this thread's halo pieces: x/y-face run (t < 64) and z-face cell
    const int fface = t >> 4, qq = t & 15;
    int foff;
    if (fface == 0) foff = 448 + qq * 4;
    else if (fface == 1) foff = qq * 4;
    else if (fface == 2) foff = (qq >> 1) * 64 + 56 + (qq & 1) * 4;
    else foff = (qq >> 1) * 64 + (qq & 1) * 4;
    const int zface = 4 + (t >> 6), zc = t & 63;
    const int zoff = (zc >> 3) * 64 + (zc & 7) * 8 + (zface == 4 ? 7 : 0);
    int tile[NT];
    bool act[NT], ghost[NT];
    // hf bits: 0 f-neighbour, 1 f ghost, 2 f has parent, 3 z-neighbour, 4 z ghost, 5 z has parent,
    // 6 own parent, 8-10 / 11-13 the f / z neighbour's octant
    uint32_t hf[NT];
    // metadata of all NT tiles and of their neighbours first, then the copies (see TilePre)
    int packed[NT], parent[NT], nbf[NT], nbz[NT], inst[NT], fpar[NT], zpar[NT];
    uint32_t fc[NT], zmb[NT];
    float4 lc[NT];
    int ptile[NT];
#pragma unroll
    for (int u = 0; u < NT; u++) {
        const int q = (((int)blockIdx.x - item_blocks) * NT + u) * TPB + g;
        tile[u] = list[q < n ? q : 0];
        act[u] = q < n;  // finished instances are dropped after the copies are issued
        ptile[u] = (tp.pf > 0 && t == 0 && q + tp.pf < n) ? list[q + tp.pf] : -1;
        const TileMeta& m = tp.meta[tile[u]];
        packed[u] = m.packed;
        parent[u] = m.parent;
        nbf[u] = t < 64 ? m.nb[fface] : -1;
        nbz[u] = m.nb[zface];
        fc[u] = tp.fcls[tile[u]];
        inst[u] = tp.inst[tile[u]];
    }
#pragma unroll
    for (int u = 0; u < NT; u++) {
        ghost[u] = meta_type(packed[u]) & GHOST_T;
        lc[u] = tp.lconst[inst[u] * kLevelSlots + meta_level(packed[u])];
        hf[u] = parent[u] >= 0 ? 64u : 0u;
        if (!act[u] || ghost[u]) nbf[u] = nbz[u] = -1;  // a GHOST tile only takes the prolongation
        fpar[u] = zpar[u] = -1;
        zmb[u] = 0;
        if (nbf[u] >= 0) {
            const TileMeta& nm = tp.meta[nbf[u]];
            const int np = nm.packed;
            hf[u] |= 1u | ((meta_type(np) & GHOST_T) ? 2u : 0u);
            if (nm.parent >= 0) {
                hf[u] |= 4u | ((uint32_t)meta_octant(np) << 8);
                fpar[u] = nm.parent;
            }
        }
        if (nbz[u] >= 0) {
            const TileMeta& nm = tp.meta[nbz[u]];
            const int np = nm.packed;
            hf[u] |= 8u | ((meta_type(np) & GHOST_T) ? 16u : 0u);
            if (nm.parent >= 0) {
                hf[u] |= 32u | ((uint32_t)meta_octant(np) << 11);
                zpar[u] = nm.parent;
            }
            zmb[u] = tp.mask_mg[(size_t)nbz[u] * kTileCells + zoff];
        }
    }
    pdl_wait();
#pragma unroll
    for (int u = 0; u < NT; u++) {
        if (!act[u]) continue;
        ProStage& ps = st[u * TPB + g];
        const size_t base = (size_t)tile[u] * kTileCells;
        if (t < 32) cp_async16(ps.mask + t * 16, tp.mask_mg + base + t * 16);
        if (nbf[u] >= 0) cp_async4(ps.hmask + fface * 64 + qq * 4, tp.mask_mg + (size_t)nbf[u] * kTileCells + foff);
        if (!ghost[u]) {
            cp_async16(ps.xp + t * 4, XP + base + t * 4);
            cp_async16(ps.b + t * 4, RHS + base + t * 4);
        }
        if (parent[u] >= 0 && t < 16) {
            const int oct = meta_octant(packed[u]);
            cp_async16(ps.pblk + t * 4, Z + (size_t)parent[u] * kTileCells + ((oct & 1) * 4 + (t >> 2)) * 64 +
                                            (((oct >> 1) & 1) * 4 + (t & 3)) * 8 + ((oct >> 2) & 1) * 4);
        }
        if (nbf[u] >= 0) {
            const size_t nbase = (size_t)nbf[u] * kTileCells;
            if (!(hf[u] & 2u)) cp_async16(ps.hxp + fface * 64 + qq * 4, XP + nbase + foff);
            if (fpar[u] >= 0)
                cp_async8(ps.hpar + (fface * 16 + qq) * 2, Z + (size_t)fpar[u] * kTileCells + parent_cell((hf[u] >> 8) & 7u, foff));
        }
        if (nbz[u] >= 0) {
            if (!(hf[u] & 16u)) cp_async4(ps.hxp + zface * 64 + zc, XP + (size_t)nbz[u] * kTileCells + zoff);
            if (zpar[u] >= 0)
                cp_async4(ps.hpar + 128 + (zface - 4) * 64 + zc, Z + (size_t)zpar[u] * kTileCells + parent_cell((hf[u] >> 11) & 7u, zoff));
        }
    }
#pragma unroll
    for (int u = 0; u < NT; u++)
        if (ptile[u] >= 0) {
            prefetch_l2(XP + (size_t)ptile[u] * kTileCells, kTileCells * sizeof(float));
            prefetch_l2(RHS + (size_t)ptile[u] * kTileCells, kTileCells * sizeof(float));
            prefetch_l2(tp.mask_mg + (size_t)ptile[u] * kTileCells, kTileCells);
        }
#pragma unroll
    for (int u = 0; u < NT; u++)
        if (nbz[u] >= 0) st[u * TPB + g].hmask[zface * 64 + zc] = (uint8_t)zmb[u];
#pragma unroll
    for (int u = 0; u < NT; u++) act[u] = act[u] && !tile_done(tp, S, tile[u]);
    cp_async_wait_all();
    __syncthreads();
    // prolongated values of the tile and of its neighbours' first layer
    const TileIdx ix(t);
#pragma unroll
    for (int u = 0; u < NT; u++) {
        if (!act[u]) continue;
        ProStage& ps = st[u * TPB + g];
        const uint32_t mask4 = *reinterpret_cast<const uint32_t*>(ps.mask + t * 4);
        const bool par = hf[u] & 64u;
        const float* pb = ps.pblk + (ix.i >> 1) * 16 + (ix.j >> 1) * 4 + (ix.k0 >> 1);
        const float c0 = par ? pb[0] : 0.f, c1 = par ? pb[1] : 0.f;
        const V4<float> xp = ghost[u] ? zero4<float>() : ld4(ps.xp + t * 4);
        V4<float> o;
#pragma unroll
        for (int e = 0; e < 4; e++) o.v[e] = prolong_value((mask4 >> (8 * e)) & 0xffu, ghost[u], e < 2 ? c0 : c1, xp.v[e], prolong_coeff);
        st4(ps.xs + t * 4, o);
        if (ghost[u]) continue;
        if (t < 64) {
            V4<float> v = zero4<float>();
            if (hf[u] & 1u) {
                const bool ng = hf[u] & 2u;
                const uint32_t nm4 = *reinterpret_cast<const uint32_t*>(ps.hmask + fface * 64 + qq * 4);
                const float h0 = (hf[u] & 4u) ? ps.hpar[(fface * 16 + qq) * 2] : 0.f;
                const float h1 = (hf[u] & 4u) ? ps.hpar[(fface * 16 + qq) * 2 + 1] : 0.f;
                const V4<float> nxp = ng ? zero4<float>() : ld4(ps.hxp + fface * 64 + qq * 4);
#pragma unroll
                for (int e = 0; e < 4; e++) v.v[e] = prolong_value((nm4 >> (8 * e)) & 0xffu, ng, e < 2 ? h0 : h1, nxp.v[e], prolong_coeff);
            }
            st4(ps.hx + fface * 64 + qq * 4, v);
        }
        {
            float v = 0.f;
            if (hf[u] & 8u) {
                const bool ng = hf[u] & 16u;
                const float cx = (hf[u] & 32u) ? ps.hpar[128 + (zface - 4) * 64 + zc] : 0.f;
                v = prolong_value(ps.hmask[zface * 64 + zc], ng, cx, ng ? 0.f : ps.hxp[zface * 64 + zc], prolong_coeff);
            }
            ps.hx[zface * 64 + zc] = v;
        }
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < NT; u++) {
        if (!act[u]) continue;
        ProStage& ps = st[u * TPB + g];
        V4<float> o = ld4(ps.xs + t * 4);
        if (!ghost[u])
            o = colour_update(ps.xs, ps.hx, t, *reinterpret_cast<const uint32_t*>(ps.mask + t * 4), (fc[u] >> 12) & 0xfffu,
                              LevelConst<float>(lc[u]), ld4(ps.b + t * 4), 1);
        st4(Z + (size_t)tile[u] * kTileCells + t * 4, o);
    }}
template <int TPB, int NT>
__global__ void __launch_bounds__(128 * TPB) k_prolong_sweep(Topo tp, const int* __restrict__ list, int n,
                                                             const int4* __restrict__ items, int nitems, int item_blocks, float* Z,
                                                             const float* __restrict__ XP, const float* __restrict__ RHS,
                                                             float prolong_coeff, const Scalars* __restrict__ S) {
    k_prolong_sweep_body<TPB, NT>(tp, list, n, items, nitems, item_blocks, Z, XP, RHS, prolong_coeff, S);
}
// the same kernel with at least MINB CTAs per SM (registers capped to fit)
template <int TPB, int NT, int MINB>
__global__ void __launch_bounds__(128 * TPB, MINB) k_prolong_sweep_occ(Topo tp, const int* __restrict__ list, int n,
                                                             const int4* __restrict__ items, int nitems, int item_blocks, float* Z,
                                                             const float* __restrict__ XP, const float* __restrict__ RHS,
                                                             float prolong_coeff, const Scalars* __restrict__ S) {
    k_prolong_sweep_body<TPB, NT>(tp, list, n, items, nitems, item_blocks, Z, XP, RHS, prolong_coeff, S);
}
template <int TPB, int NT, int MINB>
constexpr auto k_prolong_sweep_shape() {
    if constexpr (MINB == 0) return &k_prolong_sweep<TPB, NT>;
    else return &k_prolong_sweep_occ<TPB, NT, MINB>;
}

// Right-hand sides of GHOST tiles to 0 (the V-cycle's initialisation of them, src/GMGSolver.cu:393-396).
__global__ void __launch_bounds__(128) k_zero_tiles(const int* __restrict__ list, int n, float* X) {
    pdl_entry();
    const int q = blockIdx.x;
    if (q < n) st4(X + (size_t)list[q] * kTileCells + threadIdx.x * 4, zero4<float>());
}

// ---------------------------------------------------------------------------- coarse levels
// Levels 0..lb of each instance in one CTA per instance.  Each level lives in
// shared memory as a dense box over its tiles' bounding box plus a one-cell halo, so a stencil
// reads x at q +- 1 (z), q +- sz (y), q +- sy (x); cells of absent tiles and of the halo hold 0,
// the value the reference gives a missing neighbour.  A per-cell 16-bit code carries the stencil
// mask (bits 0-5 faces x-,x+,y-,y+,z-,z+, bit 6 INTERIOR) and, on tile faces, the cross-level
// coefficient flag (bits 7-12: (2/3)/h^2 instead of 1/h^2).  A phase program of colour sweeps,
// residual + restrictions and prolongations (the reference's schedule) runs with __syncthreads
// between phases.
constexpr int kBottomMaxPhases = 256;
struct BottomProgram {
    int nphase;
    uint8_t op[kBottomMaxPhases];  // 1 sweep, 2 residual+restrict, 3 prolongate
    uint8_t level[kBottomMaxPhases];
    uint8_t color[kBottomMaxPhases];
};
// negativeLap (times h^3, INTERIOR cells) of box cell q, and its diagonal: the operation order of
// neg_lap4 (coefficients a_f, fused multiply-adds in face order, diagonal summed in face order).
template <bool DIAG>
__device__ __forceinline__ float box_neglap(const float* X, int q, uint32_t code, int sy, int sz, const LevelConst<float>& L,
                                            float* diag) {
    const float x0 = X[q];
    const float xm = X[q - sy], xp = X[q + sy], ym = X[q - sz], yp = X[q + sz], zm = X[q - 1], zp = X[q + 1];
    if ((code & 0x1FFFu) == (uint32_t)kMaskFull) {  // INTERIOR, six 1/h^2 faces
        float s = 0.f;
        s = fmaf(L.c1, x0 - xm, s);
        s = fmaf(L.c1, x0 - xp, s);
        s = fmaf(L.c1, x0 - ym, s);
        s = fmaf(L.c1, x0 - yp, s);
        s = fmaf(L.c1, x0 - zm, s);
        s = fmaf(L.c1, x0 - zp, s);
        if (DIAG) *diag = L.dfast;
        return mul_h3(s, L.h);
    }
    auto coef = [&](int f) -> float { return ((code >> f) & 1u) ? (((code >> (7 + f)) & 1u) ? L.c2 : L.c1) : 0.f; };
    const float a0 = coef(0), a1 = coef(1), a2 = coef(2), a3 = coef(3), a4 = coef(4), a5 = coef(5);
    float s = 0.f;
    s = fmaf(a0, x0 - xm, s);
    s = fmaf(a1, x0 - xp, s);
    s = fmaf(a2, x0 - ym, s);
    s = fmaf(a3, x0 - yp, s);
    s = fmaf(a4, x0 - zm, s);
    s = fmaf(a5, x0 - zp, s);
    const bool interior = code & kMaskInterior;
    if (DIAG) {
        float d = 0.f;
        d = d + a0; d = d + a1; d = d + a2; d = d + a3; d = d + a4; d = d + a5;
        *diag = interior ? d * L.h * L.h * L.h : 0.f;
    }
    return interior ? s * L.h * L.h * L.h : 0.f;
}

// One cell of a sweep colour with its stencil coefficients, diagonal and right-hand side held in
// registers over a run of sweeps on one level (the level's right-hand side and codes do not change
// during the run): what box_neglap<true> and the sweep update derive from the codes every sweep.
struct SweepCell {
    int q;  // box index; -1: no cell (GHOST tile or beyond the colour's items)
    float a[6], d, b;
    bool interior;
};
__device__ __forceinline__ void sweep_cell_load(SweepCell& c, const int4* T, const float* B, const uint16_t* CODE, int first, int it,
                                                int n, int color, int sy, int sz, const LevelConst<float>& L) {
    c.q = -1;
    if (it >= n) return;
    const int4 r = T[first + (it >> 8)];
    if (r.z & GHOST_T) return;
    const int u = it & 255;
    const int i = u >> 5, j = (u >> 2) & 7, k = ((u & 3) << 1) | ((i + j + color) & 1);
    c.q = r.x + i * sy + j * sz + k;
    const uint32_t code = CODE[c.q];
    c.b = B[c.q];
    c.interior = code & kMaskInterior;
    if ((code & 0x1FFFu) == (uint32_t)kMaskFull) {
#pragma unroll
        for (int f = 0; f < 6; f++) c.a[f] = L.c1;
        c.d = L.dfast;
        return;
    }
    float d = 0.f;
#pragma unroll
    for (int f = 0; f < 6; f++) {
        c.a[f] = ((code >> f) & 1u) ? (((code >> (7 + f)) & 1u) ? L.c2 : L.c1) : 0.f;
        d = d + c.a[f];
    }
    c.d = c.interior ? mul_h3(d, L.h) : 0.f;
}
// the sweep update of box_neglap<true> + X += (B - Ax) / D with the cached terms: the same
// operations in the same order
__device__ __forceinline__ void sweep_cell_update(const SweepCell& c, float* X, int sy, int sz, const LevelConst<float>& L) {
    if (c.q < 0) return;
    const int q = c.q;
    const float x0 = X[q];
    const float xm = X[q - sy], xp = X[q + sy], ym = X[q - sz], yp = X[q + sz], zm = X[q - 1], zp = X[q + 1];
    float s = 0.f;
    s = fmaf(c.a[0], x0 - xm, s);
    s = fmaf(c.a[1], x0 - xp, s);
    s = fmaf(c.a[2], x0 - ym, s);
    s = fmaf(c.a[3], x0 - yp, s);
    s = fmaf(c.a[4], x0 - zm, s);
    s = fmaf(c.a[5], x0 - zp, s);
    const float ax = c.interior ? mul_h3(s, L.h) : 0.f;
    X[q] = x0 + (c.interior ? (c.b - ax) / c.d : 0.f);
}

namespace launch {
size_t bottom_smem_bytes(long long cells, int tiles) {
    return (size_t)tiles * sizeof(int4) + (size_t)cells * (2 * sizeof(float) + sizeof(uint16_t)) + 16;
}
}  // namespace launch

__global__ void __launch_bounds__(1024) k_bottom(Topo tp, const BottomInst* __restrict__ insts, const int4* __restrict__ tiles,
                                                 const uint16_t* __restrict__ codes, float* Z, const float* __restrict__ RHS,
                                                 float one_over_alpha, float prolong_coeff, BottomProgram prog,
                                                 const Scalars* __restrict__ S) {
    pdl_trigger();
    extern __shared__ __align__(16) unsigned char bsm[];
    __shared__ BottomInst bi;
    __shared__ float4 lcs[kBottomMaxLevels];  // the instance's level constants, read once
    const int inst = blockIdx.x;
    // the boxes' records, codes and zeroed x / right-hand sides come from the topology: set up
    // before pdl_wait
    if (threadIdx.x == 0) bi = insts[inst];
    if (threadIdx.x < kBottomMaxLevels) lcs[threadIdx.x] = tp.lconst[inst * kLevelSlots + threadIdx.x];
    __syncthreads();
    const int nb = bi.nrec, cells = bi.cells;
    int4* T = reinterpret_cast<int4*>(bsm);  // base, parent-cell base, type | level << 8, tile
    float* X = reinterpret_cast<float*>(T + nb);
    float* B = X + cells;
    uint16_t* CODE = reinterpret_cast<uint16_t*>(B + cells);
    // cells is a multiple of 8: every region is 16-byte aligned and copied in 16-byte vectors
    for (int t = threadIdx.x; t < nb; t += blockDim.x) T[t] = tiles[bi.rec_off + t];
    for (int v = threadIdx.x; v < cells / 4; v += blockDim.x) {
        st4(X + 4 * v, zero4<float>());
        st4(B + 4 * v, zero4<float>());
    }
    for (int v = threadIdx.x; v < cells / 8; v += blockDim.x)
        reinterpret_cast<uint4*>(CODE)[v] = reinterpret_cast<const uint4*>(codes + bi.code_off)[v];
    __syncthreads();
    pdl_wait();
    if (S && S[inst].done) return;
    // right-hand sides of the non-GHOST tiles (GHOST right-hand sides are 0); a tile row of 8
    // cells is contiguous in its box
    for (int v = threadIdx.x; v < nb * 128; v += blockDim.x) {
        const int4 r = T[v >> 7];
        if (r.z & GHOST_T) continue;
        const int lvl = r.z >> 8;
        const int c = (v & 127) * 4;
        const V4<float> b = ld4(RHS + (size_t)r.w * kTileCells + c);
        float* dst = B + r.x + (c >> 6) * bi.sy[lvl] + ((c >> 3) & 7) * bi.sz[lvl] + (c & 7);
        dst[0] = b.v[0]; dst[1] = b.v[1]; dst[2] = b.v[2]; dst[3] = b.v[3];
    }
    __syncthreads();
    for (int ph = 0; ph < prog.nphase; ph++) {
        const int op = prog.op[ph], level = prog.level[ph];
        const LevelConst<float> L(lcs[level]);
        const int sy = bi.sy[level], sz = bi.sz[level], first = bi.first[level];
        if (op == 1 && bi.cnt[level] * 256 <= (int)blockDim.x && ph + 1 < prog.nphase && prog.op[ph + 1] == 1 &&
            prog.level[ph + 1] == level) {
            // a run of sweeps on a level whose colours have at most one cell per thread (the
            // coarsest level's coarsest_iters sweeps): each thread keeps its cell of either colour
            SweepCell cell[2];
            const int n = bi.cnt[level] * 256;
            sweep_cell_load(cell[0], T, B, CODE, first, threadIdx.x, n, 0, sy, sz, L);
            sweep_cell_load(cell[1], T, B, CODE, first, threadIdx.x, n, 1, sy, sz, L);
            for (; ph < prog.nphase && prog.op[ph] == 1 && prog.level[ph] == level; ph++) {
                if (prog.color[ph] & 1) sweep_cell_update(cell[1], X, sy, sz, L);
                else sweep_cell_update(cell[0], X, sy, sz, L);
                __syncthreads();
            }
            ph--;
            continue;
        }
        if (op == 1) {
            // one colour of GaussSeidelGMG on the level's LEAF|NONLEAF tiles; items are the 256 cells
            // of the colour (a warp covers one (tile, i) plane), whose neighbours all have the other colour
            const int color = prog.color[ph];
            const int n = bi.cnt[level] * 256;
            for (int it = threadIdx.x; it < n; it += blockDim.x) {
                const int4 r = T[first + (it >> 8)];
                if (r.z & GHOST_T) continue;
                const int u = it & 255;
                const int i = u >> 5, j = (u >> 2) & 7, k = ((u & 3) << 1) | ((i + j + color) & 1);
                const int q = r.x + i * sy + j * sz + k;
                const uint32_t code = CODE[q];
                float d;
                const float ax = box_neglap<true>(X, q, code, sy, sz, L, &d);
                X[q] = X[q] + ((code & kMaskInterior) ? (B[q] - ax) / d : 0.f);
            }
        } else if (op == 2) {
            // residual and restriction into level - 1; items are the 64 2x2x2 blocks of each tile
            const int syp = bi.sy[level - 1], szp = bi.sz[level - 1];
            const int n = bi.cnt[level] * 64;
            for (int it = threadIdx.x; it < n; it += blockDim.x) {
                const int4 r = T[first + (it >> 6)];
                if (r.y < 0) continue;
                const int blk = it & 63;
                const int fi = blk / 16 * 2, fj = (blk / 4) % 4 * 2, fk = blk % 4 * 2;
                float sum = 0.f;
#pragma unroll
                for (int ii = 0; ii < 2; ii++)
#pragma unroll
                    for (int jj = 0; jj < 2; jj++)
#pragma unroll
                        for (int kk = 0; kk < 2; kk++) {
                            const int q = r.x + (fi + ii) * sy + (fj + jj) * sz + fk + kk;
                            const float ax = box_neglap<false>(X, q, CODE[q], sy, sz, L, nullptr);
                            sum += B[q] - ax;
                        }
                // parents are one level coarser: no cell written here is read in this phase, and
                // each parent cell has exactly one child block
                const int p = r.y + (fi / 2) * syp + (fj / 2) * szp + fk / 2;
                if (r.z & GHOST_T) B[p] += sum;
                else B[p] = sum * one_over_alpha;
            }
        } else {
            // prolongation and update of the level's tiles from level - 1
            const int syp = bi.sy[level - 1], szp = bi.sz[level - 1];
            const int n = bi.cnt[level] * kTileCells;
            for (int it = threadIdx.x; it < n; it += blockDim.x) {
                const int4 r = T[first + (it >> 9)];
                const int c = it & (kTileCells - 1);
                const int i = c >> 6, j = (c >> 3) & 7, k = c & 7;
                const int q = r.x + i * sy + j * sz + k;
                const float cx = r.y >= 0 ? X[r.y + (i >> 1) * syp + (j >> 1) * szp + (k >> 1)] : 0.f;
                X[q] = (CODE[q] & kMaskInterior) ? ((r.z & GHOST_T) ? cx : fmaf(prolong_coeff, cx, X[q])) : 0.f;
            }
        }
        __syncthreads();
    }
    for (int v = threadIdx.x; v < nb * 128; v += blockDim.x) {
        const int4 r = T[v >> 7];
        const int lvl = r.z >> 8;
        const int c = (v & 127) * 4;
        const float* src = X + r.x + (c >> 6) * bi.sy[lvl] + ((c >> 3) & 7) * bi.sz[lvl] + (c & 7);
        V4<float> o;
        o.v[0] = src[0]; o.v[1] = src[1]; o.v[2] = src[2]; o.v[3] = src[3];
        st4(Z + (size_t)r.w * kTileCells + c, o);
    }
}

namespace launch {

constexpr int kTPB2 = 2;

template <int TPB, int NT, int MINB = 0>
void presmooth_shape(const DevGrid& g, int level, float* XP, const float* RHS, const Scalars* S, cudaStream_t s, bool prefetch = false) {
    const int n = g.mg_count[level];
    const int per = TPB * NT;
    const auto k = k_presmooth_shape<TPB, NT, MINB>();
    launch_kernel(k, (n + per - 1) / per, 128 * TPB, sizeof(PreStage) * per, s,
                  prefetch_topo(g, k, 128 * TPB, sizeof(PreStage) * per, per, prefetch), g.d_mg + g.mg_offset[level], n, XP, RHS, S);
}

void presmooth(const DevGrid& g, int level, float* XP, const float* RHS, const Scalars* S, cudaStream_t s) {
    const int n = g.mg_count[level];
    if (n == 0) return;
    ++g.launch_count;
    switch (g.shape(KS_PRESMOOTH, level)) {
    case 0: presmooth_shape<2, 1>(g, level, XP, RHS, S, s); break;
    case 1: presmooth_shape<2, 2>(g, level, XP, RHS, S, s); break;
    case 2: presmooth_shape<1, 4>(g, level, XP, RHS, S, s); break;
    case 3: presmooth_shape<2, 4>(g, level, XP, RHS, S, s); break;
    case 4: presmooth_shape<1, 1>(g, level, XP, RHS, S, s); break;
    case 5: presmooth_shape<1, 2>(g, level, XP, RHS, S, s); break;
    case 6: presmooth_shape<1, 1, 16>(g, level, XP, RHS, S, s); break;
    case 7: presmooth_shape<1, 1, 12>(g, level, XP, RHS, S, s); break;
    // 8..11: shapes 2, 5, 6, 1 prefetching later CTAs' tiles into L2
    case 8: presmooth_shape<1, 4>(g, level, XP, RHS, S, s, true); break;
    case 9: presmooth_shape<1, 2>(g, level, XP, RHS, S, s, true); break;
    case 10: presmooth_shape<1, 1, 16>(g, level, XP, RHS, S, s, true); break;
    default: presmooth_shape<2, 2>(g, level, XP, RHS, S, s, true); break;
    }
}

template <int TPB, int NT, int MINB = 0>
void prolong_shape(const DevGrid& g, int level, float* Z, const float* XP, const float* RHS, float prolong_coeff, const Scalars* S,
                   cudaStream_t s, bool prefetch = false) {
    const int n = g.pr_cnt[level], nitems = g.pri_cnt[level];
    const int per = TPB * NT;
    const int item_blocks = (nitems + 2 * TPB - 1) / (2 * TPB);
    const auto k = k_prolong_sweep_shape<TPB, NT, MINB>();
    launch_kernel(k, item_blocks + (n + per - 1) / per, 128 * TPB, sizeof(ProStage) * per, s,
                  prefetch_topo(g, k, 128 * TPB, sizeof(ProStage) * per, per, prefetch), g.d_prmain + g.pr_off[level], n,
                  g.d_pritems + g.pri_off[level], nitems, item_blocks, Z, XP, RHS, prolong_coeff, S);
}

void prolong_sweep(const DevGrid& g, int level, float* Z, const float* XP, const float* RHS, float prolong_coeff, const Scalars* S,
                   cudaStream_t s) {
    const int n = g.level_count[level];
    if (n == 0) return;
    ++g.launch_count;
    switch (g.shape(KS_PROLONG, level)) {
    case 0: prolong_shape<2, 1>(g, level, Z, XP, RHS, prolong_coeff, S, s); break;
    case 1: prolong_shape<2, 2>(g, level, Z, XP, RHS, prolong_coeff, S, s); break;
    case 2: prolong_shape<1, 4>(g, level, Z, XP, RHS, prolong_coeff, S, s); break;
    case 3: prolong_shape<1, 2>(g, level, Z, XP, RHS, prolong_coeff, S, s); break;
    case 4: prolong_shape<1, 1>(g, level, Z, XP, RHS, prolong_coeff, S, s); break;
    case 5: prolong_shape<4, 1>(g, level, Z, XP, RHS, prolong_coeff, S, s); break;
    case 6: prolong_shape<1, 1, 16>(g, level, Z, XP, RHS, prolong_coeff, S, s); break;
    case 7: prolong_shape<1, 1, 12>(g, level, Z, XP, RHS, prolong_coeff, S, s); break;
    // 8..11: shapes 2, 3, 6, 1 prefetching later CTAs' tiles into L2
    case 8: prolong_shape<1, 4>(g, level, Z, XP, RHS, prolong_coeff, S, s, true); break;
    case 9: prolong_shape<1, 2>(g, level, Z, XP, RHS, prolong_coeff, S, s, true); break;
    case 10: prolong_shape<1, 1, 16>(g, level, Z, XP, RHS, prolong_coeff, S, s, true); break;
    default: prolong_shape<2, 2>(g, level, Z, XP, RHS, prolong_coeff, S, s, true); break;
    }
}

void zero_ghost_tiles(const DevGrid& g, float* X, cudaStream_t s) {
    if (g.n_ghost == 0) return;
    ++g.launch_count;
    launch_kernel(k_zero_tiles, g.n_ghost, 128, 0, s, g.d_ghost, g.n_ghost, X);
}

bool bottom(const DevGrid& g, int lb, int coarsest_iters, float* Z, const float* RHS, float one_over_alpha, float prolong_coeff,
            const Scalars* S, cudaStream_t s) {
    if (lb < 0 || lb != g.bottom_level) return false;
    BottomProgram p{};
    auto push = [&](int op, int level, int color) {
        if (p.nphase >= kBottomMaxPhases) return false;
        p.op[p.nphase] = (uint8_t)op;
        p.level[p.nphase] = (uint8_t)level;
        p.color[p.nphase] = (uint8_t)color;
        p.nphase++;
        return true;
    };
    bool ok = true;
    for (int l = lb; ok && l > 0; l--) ok = push(1, l, 0) && push(1, l, 1) && push(2, l, 0);
    for (int it = 0; ok && it < coarsest_iters / 2; it++) ok = push(1, 0, 0) && push(1, 0, 1);
    for (int it = 0; ok && it < coarsest_iters / 2; it++) ok = push(1, 0, 1) && push(1, 0, 0);
    for (int l = 1; ok && l <= lb; l++) ok = push(3, l, 0) && push(1, l, 1) && push(1, l, 0);
    if (!ok) return false;
    ++g.launch_count;
    launch_kernel(k_bottom, g.num_inst, 1024, g.bottom_smem, s, g.topo, (const BottomInst*)g.d_bottom_inst,
                  (const int4*)g.d_bottom_tiles, (const uint16_t*)g.d_bottom_code, Z, RHS, one_over_alpha, prolong_coeff, p, S);
    return true;
}

bool bottom_supported(int coarsest_iters, int lb) {
    return lb >= 0 && lb < kBottomMaxLevels && 2 * coarsest_iters + 6 * lb <= kBottomMaxPhases;
}

void init_kernel_attributes() {
    cudaFuncSetAttribute(k_bottom, cudaFuncAttributeMaxDynamicSharedMemorySize, kBottomSmemBudget);
    cudaFuncSetAttribute(k_presmooth<2, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(PreStage) * 8);
    cudaFuncSetAttribute(k_prolong_sweep<2, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(ProStage) * 4);
    cudaFuncSetAttribute(k_prolong_sweep<1, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(ProStage) * 4);
}

}  // namespace launch
}  // namespace cirrus
