// The fused Laplacian (FullNegativeLaplacian over LEAF|GHOST tiles with the p.Ap tile parts, the
// launch k_laplacian_fused performs; src/GMGSolver.cu:145-201, src/PoissonGrid.cu:664-710) with
// a column of eight cells per thread: a tile is one group of 64 threads, thread t owning the
// cells (i, j, 0..7) of column (i, j) = (t >> 3, t & 7), i.e. the cells t*8 .. t*8+7.  Twice the
// cells of the 4-cell layout per thread, so the per-thread work that does not grow with the
// cells -- tile metadata, address arithmetic, copy issue, path votes -- is spread over twice as
// many cells, and the z neighbours inside the column come from registers.  Every cell is
// computed with the 4-cell kernel's operations in the same order (the same bits), and every dot
// term is the same 4-cell FP32 product (vector v = 2t, 2t + 1 of the 4-cell layout).
// Launch shapes 12..15 of the Laplacian.
#include "kernels.cuh"
#include "solver_internal.hpp"

namespace cirrus {

namespace {

// Negative Laplacian of the column of thread t (64-thread layout), times h^3, on INTERIOR cells
// (0 elsewhere): neg_lap4v's operations per cell.  xs: tile values (512), hx: the six face halos
// (x-, x+: [j*8 + k]; y-, y+: [i*8 + k]; z-, z+: [i*8 + j]); m8: the column's eight mask bytes.
__device__ __forceinline__ void neg_lap8(const float* xs, const float* hx, int t, uint2 m8, uint32_t cls, const LevelConst<float>& L,
                                         float out[8], V4<float>& xc0, V4<float>& xc1) {
    const int i = t >> 3, j = t & 7;
    const float* c = xs + t * 8;
    const float* pm = i > 0 ? c - 64 : hx + 0 * 64 + j * 8;
    const float* pp = i < 7 ? c + 64 : hx + 1 * 64 + j * 8;
    const float* qm = j > 0 ? c - 8 : hx + 2 * 64 + i * 8;
    const float* qp = j < 7 ? c + 8 : hx + 3 * 64 + i * 8;
    xc0 = ld4(c);
    xc1 = ld4(c + 4);
    const V4<float> xm0 = ld4(pm), xm1 = ld4(pm + 4);
    const V4<float> xp0 = ld4(pp), xp1 = ld4(pp + 4);
    const V4<float> ym0 = ld4(qm), ym1 = ld4(qm + 4);
    const V4<float> yp0 = ld4(qp), yp1 = ld4(qp + 4);
    const float zlo = hx[4 * 64 + t], zhi = hx[5 * 64 + t];
    float x[8], xm[8], xp[8], ym[8], yp[8];
#pragma unroll
    for (int e = 0; e < 4; e++) {
        x[e] = xc0.v[e]; x[e + 4] = xc1.v[e];
        xm[e] = xm0.v[e]; xm[e + 4] = xm1.v[e];
        xp[e] = xp0.v[e]; xp[e + 4] = xp1.v[e];
        ym[e] = ym0.v[e]; ym[e + 4] = ym1.v[e];
        yp[e] = yp0.v[e]; yp[e + 4] = yp1.v[e];
    }
    const unsigned lanes = __activemask();
    if (__all_sync(lanes, m8.x == 0x7F7F7F7Fu && m8.y == 0x7F7F7F7Fu)) {
#pragma unroll
        for (int e = 0; e < 8; e++) {
            const float x0 = x[e];
            const float zl = e > 0 ? x[e - 1] : zlo;
            const float zr = e < 7 ? x[e + 1] : zhi;
            float s = 0.f;
            s = fmadd<false>(L.c1, x0 - xm[e], s);
            s = fmadd<false>(L.c1, x0 - xp[e], s);
            s = fmadd<false>(L.c1, x0 - ym[e], s);
            s = fmadd<false>(L.c1, x0 - yp[e], s);
            s = fmadd<false>(L.c1, x0 - zl, s);
            s = fmadd<false>(L.c1, x0 - zr, s);
            out[e] = mul_h3(s, L.h);
        }
        return;
    }
    if (__all_sync(lanes, ((m8.x | m8.y) & 0x3F3F3F3Fu) == 0u)) {
#pragma unroll
        for (int e = 0; e < 8; e++) out[e] = 0.f;
        return;
    }
    auto cross = [&](int f) -> float { return ((cls >> (2 * f)) & 3u) == 2u ? L.c2 : L.c1; };
    const float cxm = i == 0 ? cross(0) : L.c1;
    const float cxp = i == 7 ? cross(1) : L.c1;
    const float cym = j == 0 ? cross(2) : L.c1;
    const float cyp = j == 7 ? cross(3) : L.c1;
    const float czlo = cross(4), czhi = cross(5);
#pragma unroll
    for (int e = 0; e < 8; e++) {
        const uint32_t m = ((e < 4 ? m8.x : m8.y) >> (8 * (e & 3))) & 0xffu;
        const float x0 = x[e];
        const float zl = e > 0 ? x[e - 1] : zlo;
        const float zr = e < 7 ? x[e + 1] : zhi;
        const float a0 = (m & 1u) ? cxm : 0.f;
        const float a1 = (m & 2u) ? cxp : 0.f;
        const float a2 = (m & 4u) ? cym : 0.f;
        const float a3 = (m & 8u) ? cyp : 0.f;
        const float a4 = (m & 16u) ? (e == 0 ? czlo : L.c1) : 0.f;
        const float a5 = (m & 32u) ? (e == 7 ? czhi : L.c1) : 0.f;
        float s = 0.f;
        s = fmadd<false>(a0, x0 - xm[e], s);
        s = fmadd<false>(a1, x0 - xp[e], s);
        s = fmadd<false>(a2, x0 - ym[e], s);
        s = fmadd<false>(a3, x0 - yp[e], s);
        s = fmadd<false>(a4, x0 - zl, s);
        s = fmadd<false>(a5, x0 - zr, s);
        out[e] = (m & kMaskInterior) ? s * L.h * L.h * L.h : 0.f;
    }
}

// The launch: the first item_blocks CTAs take the face path (one thread per item), the others
// NT tiles per 64-thread group, TPB groups per CTA, staged with asynchronous copies before any is
// computed.  Thread t copies its column (two 16-byte pieces), a 16-byte piece of the mask bytes
// (t < 32), a 16-byte piece of an x/y face halo (face t >> 4) and the z-halo values of its own
// column from both z neighbours.
// MINB > 0: at least MINB CTAs per SM (registers capped to fit).
template <int TPB, int NT, int MINB>
__global__ void __launch_bounds__(64 * TPB, MINB > 0 ? MINB : 1) k_laplacian8(Topo tp, const int* __restrict__ list, int n, const int4* __restrict__ items,
                                                         int nitems, int item_blocks, const float* __restrict__ X, float* __restrict__ Y,
                                                         float* __restrict__ GACC, const Scalars* __restrict__ S, double* __restrict__ WP) {
    // the tile-part tail gives tile u to 16-lane half (u & 1) of warp u >> 1 of the group
    static_assert(NT >= 1 && NT <= 4, "k_laplacian8: the tile-part tail covers at most 4 tiles per group");
    pdl_entry();
    if ((int)blockIdx.x < item_blocks) {
        const int q = (int)blockIdx.x * (64 * TPB) + (int)threadIdx.x;
        if (q >= nitems) return;
        const int4 it = items[q];
        if (S != nullptr && S[it.w / kLevelSlots].done) return;
        ghost_face_sum(tp, X, it, GACC);
        return;
    }
    extern __shared__ __align__(16) unsigned char lap8_smem[];
    TileStage* st = reinterpret_cast<TileStage*>(lap8_smem);
    const int g = threadIdx.x >> 6, t = threadIdx.x & 63;
    int tile[NT];
    bool act[NT];
#pragma unroll
    for (int u = 0; u < NT; u++) {
        const int q = (((int)blockIdx.x - item_blocks) * NT + u) * TPB + g;
        tile[u] = q < n ? list[q] : 0;
        act[u] = q < n;  // finished instances are dropped after the copies are issued (reading them is harmless)
    }
    // metadata of all NT tiles before any copy (the copies are asm statements with a memory clobber)
    int4 ma[NT], mb[NT];
    uint32_t fcls[NT];
    int inst[NT];
#pragma unroll
    for (int u = 0; u < NT; u++) {
        const int4* mp = reinterpret_cast<const int4*>(tp.meta + tile[u]);
        ma[u] = mp[0];  // nb x-, x+, y-, y+
        mb[u] = mp[1];  // nb z-, z+, parent, packed
        fcls[u] = tp.fcls[tile[u]];
        inst[u] = tp.inst[tile[u]];
    }
    float4 lc[NT];
#pragma unroll
    for (int u = 0; u < NT; u++) lc[u] = tp.lconst[inst[u] * kLevelSlots + meta_level(mb[u].w)];
    const int face = t >> 4, q = t & 15;
    const int hoff = face == 0 ? 448 + q * 4 : face == 1 ? q * 4 : face == 2 ? (q >> 1) * 64 + 56 + (q & 1) * 4 : (q >> 1) * 64 + (q & 1) * 4;
    const int zo = (t >> 3) * 64 + (t & 7) * 8;
#pragma unroll
    for (int u = 0; u < NT; u++)
        if (act[u]) {
            TileStage& ts = st[u * TPB + g];
            const size_t base = (size_t)tile[u] * kTileCells;
            cp_async16(ts.xs + t * 8, X + base + t * 8);
            cp_async16(ts.xs + t * 8 + 4, X + base + t * 8 + 4);
            if (t < 32) cp_async16(ts.mask + t * 16, tp.mask_lap + base + t * 16);
            const int nbf = face == 0 ? ma[u].x : face == 1 ? ma[u].y : face == 2 ? ma[u].z : ma[u].w;
            if (nbf >= 0) cp_async16(ts.hx + face * 64 + q * 4, X + (size_t)nbf * kTileCells + hoff);
            else st4(ts.hx + face * 64 + q * 4, zero4<float>());
            if (mb[u].x >= 0) cp_async4(ts.hx + 4 * 64 + t, X + (size_t)mb[u].x * kTileCells + zo + 7);
            else ts.hx[4 * 64 + t] = 0.f;
            if (mb[u].y >= 0) cp_async4(ts.hx + 5 * 64 + t, X + (size_t)mb[u].y * kTileCells + zo);
            else ts.hx[5 * 64 + t] = 0.f;
            if (WP != nullptr && t == 0) cp_async4(ts.aux, tp.leafslot + tile[u]);
        }
#pragma unroll
    for (int u = 0; u < NT; u++) act[u] = act[u] && !(S != nullptr && S[inst[u]].done != 0);
    cp_async_wait_all();
    __syncthreads();
    bool ghost[NT];
#pragma unroll
    for (int u = 0; u < NT; u++) {
        ghost[u] = false;
        if (!act[u]) continue;
        TileStage& ts = st[u * TPB + g];
        ghost[u] = meta_type(mb[u].w) & GHOST_T;
        const LevelConst<float> L(lc[u]);
        const uint2 m8 = *reinterpret_cast<const uint2*>(ts.mask + t * 8);
        float out[8];
        V4<float> xc0, xc1;
        neg_lap8(ts.xs, ts.hx, t, m8, fcls[u] & 0xfffu, L, out, xc0, xc1);
        if (ghost[u]) {
            const uint2 ct8 = *reinterpret_cast<const uint2*>(tp.ctype + (size_t)tile[u] * kTileCells + t * 8);
#pragma unroll
            for (int e = 0; e < 8; e++)
                ts.b[t * 8 + e] = ((((e < 4 ? ct8.x : ct8.y) >> (8 * (e & 3))) & (INTERIOR_C | DIRICHLET_C | NEUMANN_C)) != 0) ? out[e] : 0.f;
        } else {
            V4<float> o0, o1;
#pragma unroll
            for (int e = 0; e < 4; e++) {
                o0.v[e] = out[e];
                o1.v[e] = out[e + 4];
            }
            float* y = Y + (size_t)tile[u] * kTileCells + t * 8;
            st4(y, o0);
            st4(y + 4, o1);
            // the thread's two p.Ap terms (4-cell vectors 2t, 2t + 1), in its own (already read) mask bytes
            if (WP != nullptr && ts.aux[0] >= 0) {
                float* terms = reinterpret_cast<float*>(ts.mask);
                terms[2 * t] = dot4f32(xc0, o0);
                terms[2 * t + 1] = dot4f32(xc1, o1);
            }
        }
    }
    __syncthreads();
    if (WP != nullptr && 2 * (t >> 5) < NT) {  // whole warps
        // warp w of the group sums the terms of tiles u = 2w (lanes 0..15) and 2w + 1 (16..31)
        const int u = 2 * (t >> 5) + ((t >> 4) & 1);
        bool ok = false;
#pragma unroll
        for (int k = 0; k < NT; k++)
            if (k == u) ok = act[k] && !ghost[k];
        const TileStage& ts = st[(u < NT ? u : 0) * TPB + g];
        const int sl = ts.aux[0];
        const double d = tile_part_sum(reinterpret_cast<const float*>(ts.mask), t & 15);
        if (ok && u < NT && sl >= 0 && (t & 15) == 0) WP[sl] = d;
    }
    // GHOST tiles staged here: thread t forms coarse cell t's 2x2x2 sum in (ii, jj, kk) order
    const int fi = t / 16 * 2, fj = (t / 4) % 4 * 2, fk = t % 4 * 2;
#pragma unroll
    for (int u = 0; u < NT; u++) {
        if (!act[u] || !ghost[u]) continue;
        const float* gsum = st[u * TPB + g].b;
        float sum = 0.f;
#pragma unroll
        for (int ii = 0; ii < 2; ii++)
#pragma unroll
            for (int jj = 0; jj < 2; jj++)
#pragma unroll
                for (int kk = 0; kk < 2; kk++) sum += gsum[(fi + ii) * 64 + (fj + jj) * 8 + (fk + kk)];
        GACC[(size_t)tp.ghost_slot[tile[u]] * 64 + t] = sum;
    }
}

template <int TPB, int NT, int MINB = 0>
void lap8_shape(const DevGrid& g, const float* X, float* Y, const Scalars* S, cudaStream_t s, double* WP) {
    const int per = TPB * NT;
    const int item_blocks = (g.n_lapitems + 64 * TPB - 1) / (64 * TPB);
    launch::launch_kernel(k_laplacian8<TPB, NT, MINB>, item_blocks + (g.n_lapmain + per - 1) / per, 64 * TPB, sizeof(TileStage) * per, s,
                          g.topo, g.d_lapmain, g.n_lapmain, g.d_lapitems, g.n_lapitems, item_blocks, X, Y, g.d_gacc, S, WP);
}

}  // namespace

namespace launch {
void laplacian8(const DevGrid& g, int variant, const float* X, float* Y, const Scalars* S, cudaStream_t s, double* WP) {
    switch (variant) {
    case 0: lap8_shape<2, 2>(g, X, Y, S, s, WP); break;
    case 1: lap8_shape<4, 1>(g, X, Y, S, s, WP); break;
    case 2: lap8_shape<1, 4>(g, X, Y, S, s, WP); break;
    default: lap8_shape<2, 2, 7>(g, X, Y, S, s, WP); break;
    }
}
}  // namespace launch

}  // namespace cirrus
