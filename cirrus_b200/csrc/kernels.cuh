// Device kernels of the GMG-PCG solve.  Layout: structure-of-arrays tile pool, 512 cells per
// tile, cell c = i*64 + j*8 + k.  A tile is processed by a 128-thread group; thread t owns the
// four consecutive cells (i, j, k0..k0+3) with i = t>>4, j = (t>>1)&7, k0 = 4*(t&1), so every
// channel access of a tile is one coalesced 2 KB sweep of 16-byte vectors.  The six face halos
// are staged in shared memory: the x and y faces of a neighbour tile are runs of 16-byte
// vectors, the z faces are 64 strided scalars.
//
// Arithmetic mirrors the reference operation by operation so results agree bit for bit:
//   coefficient  NegativeLaplacianCoeff          src/GMGSolver.cu:12-40
//   stencil sum  GMGLaplacianTileData::negativeLap src/GMGSolver.cu:56-76 (face order x-,x+,
//                y-,y+,z-,z+; fused multiply-add in the smoother and residual kernels,
//                product-then-sum in the Laplacian apply, as the reference's build rounds them)
#pragma once

#include "common.cuh"

namespace cirrus {

// Programmatic dependent launch.  Solve kernels are launched with programmatic stream
// serialisation (launch_kernel), so a kernel's CTAs may be scheduled while its predecessor is
// still running.  Every kernel first allows its own successor to be scheduled, then waits until
// its predecessor grid has completed and that grid's memory operations are visible, before it
// reads or writes anything; so results are those of plain stream order.  Without the launch
// attribute both instructions return at once.
__device__ __forceinline__ void pdl_entry() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

template <class T> struct alignas(4 * sizeof(T)) V4 { T v[4]; };

template <class T> __device__ __forceinline__ V4<T> ld4(const T* p) { return *reinterpret_cast<const V4<T>*>(p); }
template <class T> __device__ __forceinline__ void st4(T* p, const V4<T>& v) { *reinterpret_cast<V4<T>*>(p) = v; }
template <class T> __device__ __forceinline__ V4<T> zero4() { V4<T> r; r.v[0] = r.v[1] = r.v[2] = r.v[3] = T(0); return r; }

// sum + a*b.  FUSED: one rounding (fused multiply-add); otherwise the product is rounded, then
// the sum, with intrinsics the compiler may not contract.  The reference's build fuses the
// stencil sum in its Gauss-Seidel and residual kernels (negativeLap inlined with a literal
// `diag`) but not in NegativeLaplacianSameLevel128Kernel, whose calc_diag is a runtime value.
template <bool FUSED> __device__ __forceinline__ float fmadd(float a, float b, float c) {
    return FUSED ? fmaf(a, b, c) : __fadd_rn(c, __fmul_rn(a, b));
}
template <bool FUSED> __device__ __forceinline__ double fmadd(double a, double b, double c) {
    return FUSED ? fma(a, b, c) : __dadd_rn(c, __dmul_rn(a, b));
}

// Per-level constants of the stencil.  h = h0 / 2^level (src/HAAccessor.h:72-74); c1 = 1/h^2;
// c2 = (2*(1/h)/3)*(1/h) exactly as the reference rounds it.
template <class T> struct LevelConst {
    T h, c1, c2;
    __device__ __forceinline__ LevelConst(T h0, int level) {
        h = h0 / T(1 << level);
        const T ooh = T(1) / h;
        c1 = ooh * ooh;                  // (ooh*1 + x*0) * ooh
        c2 = (T(2) * ooh / T(3)) * ooh;  // (ooh*0 + (2*ooh/3)*1) * ooh
    }
};

struct TileIdx {
    int i, j, k0;
    __device__ __forceinline__ explicit TileIdx(int t) : i(t >> 4), j((t >> 1) & 7), k0((t & 1) << 2) {}
};

// Stage the face halos of tile `m` from channel X into hx[6][64] (face order x-,x+,y-,y+,z-,z+).
// An empty neighbour contributes 0 (src/GMGSolver.cu:118-122, 136-140).
template <class T>
__device__ __forceinline__ void load_halo(const T* __restrict__ X, const TileMeta& m, int t, T* hx) {
    if (t < 64) {
        int face = t >> 4, q = t & 15;
        int nb = m.nb[face];
        V4<T> v = zero4<T>();
        if (nb >= 0) {
            int off;
            if (face == 0) off = 448 + q * 4;
            else if (face == 1) off = q * 4;
            else if (face == 2) off = (q >> 1) * 64 + 56 + (q & 1) * 4;
            else off = (q >> 1) * 64 + (q & 1) * 4;
            v = ld4(X + (size_t)nb * kTileCells + off);
        }
        st4(hx + face * 64 + q * 4, v);
    }
    {
        int face = 4 + (t >> 6), c = t & 63;
        int nb = m.nb[face];
        T v = T(0);
        if (nb >= 0) v = X[(size_t)nb * kTileCells + (c >> 3) * 64 + (c & 7) * 8 + (face == 4 ? 7 : 0)];
        hx[face * 64 + c] = v;
    }
}

// Negative Laplacian of the four cells of thread t, times h^3, for INTERIOR cells (0 elsewhere).
// xs = tile values in shared memory (512), hx = halos, mask4 = the four mask bytes, cls = the
// 12-bit cross-face class field of the context.  DIAG additionally returns the diagonal;
// FUSED selects the rounding of the stencil sum (see fmadd).
template <class T, bool DIAG, bool FUSED = true>
__device__ __forceinline__ void neg_lap4(const T* xs, const T* hx, int t, uint32_t mask4, uint32_t cls,
                                         const LevelConst<T>& L, T out[4], T diag[4]) {
    const TileIdx ix(t);
    const V4<T> xc = ld4(xs + t * 4);
    const V4<T> xm = ix.i > 0 ? ld4(xs + (t - 16) * 4) : ld4(hx + 0 * 64 + ix.j * 8 + ix.k0);
    const V4<T> xp = ix.i < 7 ? ld4(xs + (t + 16) * 4) : ld4(hx + 1 * 64 + ix.j * 8 + ix.k0);
    const V4<T> ym = ix.j > 0 ? ld4(xs + (t - 2) * 4) : ld4(hx + 2 * 64 + ix.i * 8 + ix.k0);
    const V4<T> yp = ix.j < 7 ? ld4(xs + (t + 2) * 4) : ld4(hx + 3 * 64 + ix.i * 8 + ix.k0);
    const T zlo = ix.k0 > 0 ? xs[t * 4 - 1] : hx[4 * 64 + ix.i * 8 + ix.j];
    const T zhi = ix.k0 < 4 ? xs[t * 4 + 4] : hx[5 * 64 + ix.i * 8 + ix.j];
    auto cross = [&](int f) -> T { return ((cls >> (2 * f)) & 3u) == 2u ? L.c2 : L.c1; };
    const T cxm = ix.i == 0 ? cross(0) : L.c1;
    const T cxp = ix.i == 7 ? cross(1) : L.c1;
    const T cym = ix.j == 0 ? cross(2) : L.c1;
    const T cyp = ix.j == 7 ? cross(3) : L.c1;
    const T czlo = cross(4), czhi = cross(5);
#pragma unroll
    for (int e = 0; e < 4; e++) {
        const uint32_t m = (mask4 >> (8 * e)) & 0xffu;
        const T x0 = xc.v[e];
        const T zl = e > 0 ? xc.v[e - 1] : zlo;
        const T zr = e < 3 ? xc.v[e + 1] : zhi;
        const int k = ix.k0 + e;
        const T a0 = (m & 1u) ? cxm : T(0);
        const T a1 = (m & 2u) ? cxp : T(0);
        const T a2 = (m & 4u) ? cym : T(0);
        const T a3 = (m & 8u) ? cyp : T(0);
        const T a4 = (m & 16u) ? (k == 0 ? czlo : L.c1) : T(0);
        const T a5 = (m & 32u) ? (k == 7 ? czhi : L.c1) : T(0);
        T s = T(0);
        s = fmadd<FUSED>(a0, x0 - xm.v[e], s);
        s = fmadd<FUSED>(a1, x0 - xp.v[e], s);
        s = fmadd<FUSED>(a2, x0 - ym.v[e], s);
        s = fmadd<FUSED>(a3, x0 - yp.v[e], s);
        s = fmadd<FUSED>(a4, x0 - zl, s);
        s = fmadd<FUSED>(a5, x0 - zr, s);
        const bool interior = m & kMaskInterior;
        out[e] = interior ? s * L.h * L.h * L.h : T(0);
        if (DIAG) {
            T d = T(0);
            d = d + a0; d = d + a1; d = d + a2; d = d + a3; d = d + a4; d = d + a5;
            diag[e] = interior ? d * L.h * L.h * L.h : T(0);
        }
    }
}

// Shared memory of one 128-thread tile group.
template <class T> struct TileShared {
    T xs[kTileCells];
    T hx[6 * 64];
};

// Load the own tile (channel X) and its halos; returns this thread's own four values.
template <class T>
__device__ __forceinline__ V4<T> stage_tile(const T* __restrict__ X, int tile, const TileMeta& m, int t, TileShared<T>& sh) {
    V4<T> own = ld4(X + (size_t)tile * kTileCells + t * 4);
    st4(sh.xs + t * 4, own);
    load_halo<T>(X, m, t, sh.hx);
    return own;
}

}  // namespace cirrus
