// One red-black colour sweep (NegativeLaplacianAndGaussSeidelSameLevel128Kernel,
// src/GMGSolver.cu:216-269, the launch k_gs_sweep performs) with a column of eight cells per
// thread: a tile is one group of 64 threads, thread t owning the cells (i, j, 0..7) of column
// (i, j) (column_of: the warps split the columns by the parity of i + j).  The four cells of the
// sweep's colour in a column are k = P, P + 2, P + 4, P + 6 with P = (color + i + j) & 1; each
// gets gs_cell's (or, on uniform warps, gs_cell_fast's) operations, as in the 4-cell kernel, so
// the bits are the same, and so is every r.z term (4-cell vectors 2 col and 2 col + 1 of the
// 4-cell layout).  Launch shapes 8..11 of the sweep.
#include "kernels.cuh"
#include "solver_internal.hpp"

namespace cirrus {

namespace {

// Thread t of a 64-thread tile group owns column (i, j) with (i + j) & 1 = t >> 5: warp 0 of the
// group takes the 32 columns of even parity, warp 1 the odd ones, so the cells of a sweep's
// colour sit at the same places k = P, P + 2, P + 4, P + 6 (P = (color + i + j) & 1) in every
// column of a warp -- a warp-uniform choice instead of per-cell selects.
__device__ __forceinline__ int column_of(int t) {
    const int w = t >> 5, r = t & 31, i = r >> 2;
    return i * 8 + 2 * (r & 3) + ((i + w) & 1);
}

// The colour update of column col = (i, j) whose colour cells start at P: staged tile values xs,
// halos hx (x faces [j*8 + k], y faces [i*8 + k], z faces [i*8 + j]), right-hand sides b, mask
// bytes m8; x[] holds the column's values on entry and after the sweep.
template <int P>
__device__ __forceinline__ void colour_cells8(const float* xs, const float* hx, int col, uint2 m8, uint32_t cls, const LevelConst<float>& L,
                                              const float (&b)[8], float (&x)[8]) {
    const int i = col >> 3, j = col & 7;
    const float* c = xs + col * 8;
    const float* pm = i > 0 ? c - 64 : hx + 0 * 64 + j * 8;
    const float* pp = i < 7 ? c + 64 : hx + 1 * 64 + j * 8;
    const float* qm = j > 0 ? c - 8 : hx + 2 * 64 + i * 8;
    const float* qp = j < 7 ? c + 8 : hx + 3 * 64 + i * 8;
    const V4<float> xm0 = ld4(pm), xm1 = ld4(pm + 4);
    const V4<float> xp0 = ld4(pp), xp1 = ld4(pp + 4);
    const V4<float> ym0 = ld4(qm), ym1 = ld4(qm + 4);
    const V4<float> yp0 = ld4(qp), yp1 = ld4(qp + 4);
    const float zlo = hx[4 * 64 + col], zhi = hx[5 * 64 + col];
    float xm[8], xp[8], ym[8], yp[8];
#pragma unroll
    for (int e = 0; e < 4; e++) {
        xm[e] = xm0.v[e]; xm[e + 4] = xm1.v[e];
        xp[e] = xp0.v[e]; xp[e + 4] = xp1.v[e];
        ym[e] = ym0.v[e]; ym[e + 4] = ym1.v[e];
        yp[e] = yp0.v[e]; yp[e + 4] = yp1.v[e];
    }
    // the other colour's values, read before any cell of this colour changes (they do not change)
    if (__all_sync(__activemask(), m8.x == 0x7F7F7F7Fu && m8.y == 0x7F7F7F7Fu)) {
#pragma unroll
        for (int e = P; e < 8; e += 2)
            x[e] = gs_cell_fast(x[e], xm[e], xp[e], ym[e], yp[e], e > 0 ? x[e - 1] : zlo, e < 7 ? x[e + 1] : zhi, b[e], L);
    } else {
        auto cross = [&](int f) -> float { return ((cls >> (2 * f)) & 3u) == 2u ? L.c2 : L.c1; };
        FaceCoef<float> C;
        C.xm = i == 0 ? cross(0) : L.c1;
        C.xp = i == 7 ? cross(1) : L.c1;
        C.ym = j == 0 ? cross(2) : L.c1;
        C.yp = j == 7 ? cross(3) : L.c1;
        C.zlo = cross(4);
        C.zhi = cross(5);
#pragma unroll
        for (int e = P; e < 8; e += 2) {
            const uint32_t m = ((e < 4 ? m8.x : m8.y) >> (8 * (e & 3))) & 0xffu;
            x[e] = gs_cell(x[e], xm[e], xp[e], ym[e], yp[e], e > 0 ? x[e - 1] : zlo, e < 7 ? x[e + 1] : zhi, b[e], m, C,
                           e == 0 ? C.zlo : L.c1, e == 7 ? C.zhi : L.c1, L);
        }
    }
}

// k_gs_sweep_body's launch with 64-thread tile groups: NT tiles per group in flight, TPB groups
// per CTA; with RD the r.z parts of the LEAF tiles (see k_gs_sweep_body).
template <int TPB, int NT, int MINB>
__global__ void __launch_bounds__(64 * TPB, MINB > 0 ? MINB : 1) k_gs_sweep8(Topo tp, const int* __restrict__ list, int n, float* X,
                                                                        const float* __restrict__ R, int color, const Scalars* __restrict__ S,
                                                                        const float* __restrict__ RD, double* __restrict__ WP) {
    static_assert(NT >= 1 && NT <= 4, "k_gs_sweep8: the tile-part tail covers at most 4 tiles per group");
    pdl_entry();
    extern __shared__ __align__(16) unsigned char gs8_smem[];
    TileStage* st = reinterpret_cast<TileStage*>(gs8_smem);
    const int g = threadIdx.x >> 6, t = threadIdx.x & 63;
    int tile[NT];
    bool act[NT];
#pragma unroll
    for (int u = 0; u < NT; u++) {
        const int q = ((int)blockIdx.x * NT + u) * TPB + g;
        tile[u] = q < n ? list[q] : 0;
        act[u] = q < n;
    }
    int4 ma[NT], mb[NT];
    uint32_t fcls[NT];
    int inst[NT];
#pragma unroll
    for (int u = 0; u < NT; u++) {
        const int4* mp = reinterpret_cast<const int4*>(tp.meta + tile[u]);
        ma[u] = mp[0];
        mb[u] = mp[1];
        fcls[u] = tp.fcls[tile[u]];
        inst[u] = tp.inst[tile[u]];
    }
    float4 lc[NT];
#pragma unroll
    for (int u = 0; u < NT; u++) lc[u] = tp.lconst[inst[u] * kLevelSlots + meta_level(mb[u].w)];
    const int face = t >> 4, q = t & 15;
    const int hoff = face == 0 ? 448 + q * 4 : face == 1 ? q * 4 : face == 2 ? (q >> 1) * 64 + 56 + (q & 1) * 4 : (q >> 1) * 64 + (q & 1) * 4;
    const int col = column_of(t);
    const int zo = (col >> 3) * 64 + (col & 7) * 8;
#pragma unroll
    for (int u = 0; u < NT; u++)
        if (act[u]) {
            TileStage& ts = st[u * TPB + g];
            const size_t base = (size_t)tile[u] * kTileCells;
            cp_async16(ts.xs + col * 8, X + base + col * 8);
            cp_async16(ts.xs + col * 8 + 4, X + base + col * 8 + 4);
            cp_async16(ts.b + col * 8, R + base + col * 8);
            cp_async16(ts.b + col * 8 + 4, R + base + col * 8 + 4);
            if (t < 32) cp_async16(ts.mask + t * 16, tp.mask_mg + base + t * 16);
            const int nbf = face == 0 ? ma[u].x : face == 1 ? ma[u].y : face == 2 ? ma[u].z : ma[u].w;
            if (nbf >= 0) cp_async16(ts.hx + face * 64 + q * 4, X + (size_t)nbf * kTileCells + hoff);
            else st4(ts.hx + face * 64 + q * 4, zero4<float>());
            if (mb[u].x >= 0) cp_async4(ts.hx + 4 * 64 + col, X + (size_t)mb[u].x * kTileCells + zo + 7);
            else ts.hx[4 * 64 + col] = 0.f;
            if (mb[u].y >= 0) cp_async4(ts.hx + 5 * 64 + col, X + (size_t)mb[u].y * kTileCells + zo);
            else ts.hx[5 * 64 + col] = 0.f;
            if (RD != nullptr && t == 0) cp_async4(ts.aux, tp.leafslot + tile[u]);
        }
#pragma unroll
    for (int u = 0; u < NT; u++) act[u] = act[u] && !(S != nullptr && S[inst[u]].done != 0);
    cp_async_wait_all();
    __syncthreads();
    const int P = (color + (t >> 5)) & 1;  // warp-uniform: every column of the warp has parity t >> 5
#pragma unroll
    for (int u = 0; u < NT; u++) {
        if (!act[u]) continue;
        TileStage& ts = st[u * TPB + g];
        const LevelConst<float> L(lc[u]);
        const uint2 m8 = *reinterpret_cast<const uint2*>(ts.mask + col * 8);
        const size_t off = (size_t)tile[u] * kTileCells + col * 8;
        const V4<float> b0 = ld4(ts.b + col * 8), b1 = ld4(ts.b + col * 8 + 4);
        const V4<float> xc0 = ld4(ts.xs + col * 8), xc1 = ld4(ts.xs + col * 8 + 4);
        float x[8], b[8];
#pragma unroll
        for (int e = 0; e < 4; e++) {
            x[e] = xc0.v[e]; x[e + 4] = xc1.v[e];
            b[e] = b0.v[e]; b[e + 4] = b1.v[e];
        }
        if (P) colour_cells8<1>(ts.xs, ts.hx, col, m8, (fcls[u] >> 12) & 0xfffu, L, b, x);
        else colour_cells8<0>(ts.xs, ts.hx, col, m8, (fcls[u] >> 12) & 0xfffu, L, b, x);
        V4<float> z0, z1;
#pragma unroll
        for (int e = 0; e < 4; e++) {
            z0.v[e] = x[e];
            z1.v[e] = x[e + 4];
        }
        st4(X + off, z0);
        st4(X + off + 4, z1);
        if (RD != nullptr) {  // the column's two terms (4-cell vectors 2 col, 2 col + 1), in its own (already read) mask bytes
            const int sl = ts.aux[0];
            if (sl != -1) {
                float* terms = reinterpret_cast<float*>(ts.mask);
                terms[2 * col] = dot4f32(sl >= 0 ? b0 : ld4(RD + off), z0);
                terms[2 * col + 1] = dot4f32(sl >= 0 ? b1 : ld4(RD + off + 4), z1);
            }
        }
    }
    if (RD == nullptr) return;
    __syncthreads();
    if (2 * (t >> 5) >= NT) return;  // whole warps
    // warp w of the group sums the terms of tiles u = 2w (lanes 0..15) and 2w + 1 (16..31)
    const int u = 2 * (t >> 5) + ((t >> 4) & 1);
    bool ok = false;
#pragma unroll
    for (int k = 0; k < NT; k++)
        if (k == u) ok = act[k];
    const TileStage& ts = st[(u < NT ? u : 0) * TPB + g];
    const int sl = ts.aux[0];
    const double d = tile_part_sum(reinterpret_cast<const float*>(ts.mask), t & 15);
    if (ok && u < NT && sl != -1 && (t & 15) == 0) WP[sl >= 0 ? sl : -2 - sl] = d;
}

template <int TPB, int NT, int MINB = 0>
void gs8_shape(const DevGrid& g, int level, float* X, const float* R, int color, const Scalars* S, cudaStream_t s, const float* RD) {
    const int n = g.mg_count[level];
    const int per = TPB * NT;
    launch::launch_kernel(k_gs_sweep8<TPB, NT, MINB>, (n + per - 1) / per, 64 * TPB, sizeof(TileStage) * per, s, g.topo,
                          g.d_mg + g.mg_offset[level], n, X, R, color, S, RD, RD ? g.d_wpart : nullptr);
}

}  // namespace

namespace launch {
void gs_sweep8(const DevGrid& g, int variant, int level, float* X, const float* R, int color, const Scalars* S, cudaStream_t s,
               const float* RD) {
    switch (variant) {
    case 0: gs8_shape<2, 2>(g, level, X, R, color, S, s, RD); break;
    case 1: gs8_shape<4, 1>(g, level, X, R, color, S, s, RD); break;
    case 2: gs8_shape<1, 4>(g, level, X, R, color, S, s, RD); break;
    default: gs8_shape<2, 1>(g, level, X, R, color, S, s, RD); break;
    }
}
}  // namespace launch

}  // namespace cirrus
