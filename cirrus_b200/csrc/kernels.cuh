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
// reads or writes any data a kernel writes; so results are those of plain stream order.
// Without the launch attribute both instructions return at once.
__device__ __forceinline__ void pdl_entry() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
}
// The same two steps apart, for the stencil, coarse-level and vector kernels: between them a
// kernel reads only the grid's topology (tile lists, metadata, coefficient classes, level
// constants, chunk and range tables, coarse-level boxes), which is written once when the grid is
// created and never by a kernel, and writes only its own shared memory -- so that part overlaps
// the predecessor's tail without changing any result.  The staged copies (mask bytes included)
// follow the wait: issued before it, they cost the batched solve more than they saved.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

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
// dfast: the diagonal of a cell with six 1/h^2 faces, summed and scaled as neg_lap4 does.
template <class T> struct LevelConst {
    T h, c1, c2, dfast;
    __device__ __forceinline__ explicit LevelConst(float4 v) : h(v.x), c1(v.y), c2(v.z), dfast(v.w) {}
    __host__ __device__ __forceinline__ LevelConst(T h0, int level) {
        h = h0 / T(1 << level);
        const T ooh = T(1) / h;
        c1 = ooh * ooh;                  // (ooh*1 + x*0) * ooh
        c2 = (T(2) * ooh / T(3)) * ooh;  // (ooh*0 + (2*ooh/3)*1) * ooh
        T d = T(0);
        d = d + c1; d = d + c1; d = d + c1; d = d + c1; d = d + c1; d = d + c1;
        dfast = d * h * h * h;
    }
};

// s * h * h * h rounded after each product, as three separate multiplies (intrinsics, so the
// compiler never fuses the last product into a following addition).
__device__ __forceinline__ float mul_h3(float s, float h) { return __fmul_rn(__fmul_rn(__fmul_rn(s, h), h), h); }
__device__ __forceinline__ double mul_h3(double s, double h) { return __dmul_rn(__dmul_rn(__dmul_rn(s, h), h), h); }

// The level constants of a tile from the per-instance table (the same values LevelConst's
// constructor computes, precomputed once per grid).
__device__ __forceinline__ LevelConst<float> tile_level_const(const Topo& tp, int tile, int level) {
    const float4 v = tp.lconst[tp.inst[tile] * kLevelSlots + level];
    return LevelConst<float>(v);
}

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
// xs = tile values in shared memory (512); the six face halos: hxm/hxp (x-/x+, [j*8 + k]),
// hym/hyp (y-/y+, [i*8 + k]), hzm/hzp (z-/z+: the value of column (i, j) at [(i*8 + j)*zs]);
// mask4 = the four mask bytes, cls = the 12-bit cross-face class field of the context.  DIAG
// additionally returns the diagonal; FUSED selects the rounding of the stencil sum (see fmadd).
template <class T, bool DIAG, bool FUSED = true>
__device__ __forceinline__ void neg_lap4v(const T* xs, const T* hxm, const T* hxp, const T* hym, const T* hyp, const T* hzm,
                                          const T* hzp, int zs, int t, uint32_t mask4, uint32_t cls, const LevelConst<T>& L,
                                          T out[4], T diag[4]) {
    const TileIdx ix(t);
    // each neighbour vector comes from the tile or from its halo: the address is selected, then
    // one load issued
    const V4<T> xc = ld4(xs + t * 4);
    const V4<T> xm = ld4(ix.i > 0 ? xs + (t - 16) * 4 : hxm + ix.j * 8 + ix.k0);
    const V4<T> xp = ld4(ix.i < 7 ? xs + (t + 16) * 4 : hxp + ix.j * 8 + ix.k0);
    const V4<T> ym = ld4(ix.j > 0 ? xs + (t - 2) * 4 : hym + ix.i * 8 + ix.k0);
    const V4<T> yp = ld4(ix.j < 7 ? xs + (t + 2) * 4 : hyp + ix.i * 8 + ix.k0);
    const T zlo = *(ix.k0 > 0 ? xs + t * 4 - 1 : hzm + (ix.i * 8 + ix.j) * zs);
    const T zhi = *(ix.k0 < 4 ? xs + t * 4 + 4 : hzp + (ix.i * 8 + ix.j) * zs);
    // The path is chosen per warp (a vote over the converged lanes), so a warp never runs two
    // paths one after the other: each path gives a lane's cells the same bits (the general one
    // with a_f = c1 on uniform cells, +0 on cells without coupled faces), so the choice only
    // affects speed.
    const unsigned lanes = __activemask();
    if (__all_sync(lanes, mask4 == 0x7F7F7F7Fu)) {
        // the four cells are INTERIOR with six 1/h^2 faces: every coefficient is c1 (the same
        // operations as the general path below with a_f = c1)
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const T x0 = xc.v[e];
            const T zl = e > 0 ? xc.v[e - 1] : zlo;
            const T zr = e < 3 ? xc.v[e + 1] : zhi;
            T s = T(0);
            s = fmadd<FUSED>(L.c1, x0 - xm.v[e], s);
            s = fmadd<FUSED>(L.c1, x0 - xp.v[e], s);
            s = fmadd<FUSED>(L.c1, x0 - ym.v[e], s);
            s = fmadd<FUSED>(L.c1, x0 - yp.v[e], s);
            s = fmadd<FUSED>(L.c1, x0 - zl, s);
            s = fmadd<FUSED>(L.c1, x0 - zr, s);
            out[e] = mul_h3(s, L.h);
            if (DIAG) diag[e] = L.dfast;
        }
        return;
    }
    if (__all_sync(lanes, (mask4 & 0x3F3F3F3Fu) == 0u)) {
        // no coupled face on any of the four cells (e.g. inside a GHOST tile, whose ghost-ghost
        // faces carry no coefficient): every product is 0, the sum stays +0, and so do the
        // result and the diagonal (for finite values, the general path's bits)
#pragma unroll
        for (int e = 0; e < 4; e++) {
            out[e] = T(0);
            if (DIAG) diag[e] = T(0);
        }
        return;
    }
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

// neg_lap4v with the halos of hx[6][64] (face order x-, x+, y-, y+, z-, z+).
template <class T, bool DIAG, bool FUSED = true>
__device__ __forceinline__ void neg_lap4(const T* xs, const T* hx, int t, uint32_t mask4, uint32_t cls, const LevelConst<T>& L,
                                         T out[4], T diag[4]) {
    neg_lap4v<T, DIAG, FUSED>(xs, hx, hx + 64, hx + 128, hx + 192, hx + 256, hx + 320, 1, t, mask4, cls, L, out, diag);
}

// Coefficients of the general stencil path for thread t's column of four cells: the x and y
// faces of its (i, j) column and the outer z faces of its first and last cell (1/h^2 inside the
// tile, the cross-face class's coefficient on a tile face).
template <class T> struct FaceCoef {
    T xm, xp, ym, yp, zlo, zhi;
};
template <class T>
__device__ __forceinline__ FaceCoef<T> face_coef(int i, int j, int k0, uint32_t cls, const LevelConst<T>& L) {
    auto cross = [&](int f) -> T { return ((cls >> (2 * f)) & 3u) == 2u ? L.c2 : L.c1; };
    FaceCoef<T> c;
    c.xm = i == 0 ? cross(0) : L.c1;
    c.xp = i == 7 ? cross(1) : L.c1;
    c.ym = j == 0 ? cross(2) : L.c1;
    c.yp = j == 7 ? cross(3) : L.c1;
    c.zlo = k0 == 0 ? cross(4) : L.c1;
    c.zhi = k0 == 4 ? cross(5) : L.c1;
    return c;
}
template <class T>
__device__ __forceinline__ FaceCoef<T> face_coef(const TileIdx& ix, uint32_t cls, const LevelConst<T>& L) {
    return face_coef(ix.i, ix.j, ix.k0, cls, L);
}

// Diagonal h^3 * sum_f a_f of a cell with mask byte m (the sum in face order, as neg_lap4 forms
// it; 0 off INTERIOR), x/y-face coefficients C and z-face coefficients azl, azr.  On a uniform
// cell it equals the level's dfast bit for bit.
__device__ __forceinline__ float diag_cell(uint32_t m, const FaceCoef<float>& C, float azl, float azr, const LevelConst<float>& L) {
    const float a0 = (m & 1u) ? C.xm : 0.f;
    const float a1 = (m & 2u) ? C.xp : 0.f;
    const float a2 = (m & 4u) ? C.ym : 0.f;
    const float a3 = (m & 8u) ? C.yp : 0.f;
    const float a4 = (m & 16u) ? azl : 0.f;
    const float a5 = (m & 32u) ? azr : 0.f;
    float d = 0.f;
    d = d + a0; d = d + a1; d = d + a2; d = d + a3; d = d + a4; d = d + a5;
    return (m & kMaskInterior) ? mul_h3(d, L.h) : 0.f;
}

// First colour (0) of a red-black sweep from x = 0 on a 4-cell column run (i, j, k0..k0+3):
// x = b/D on its two colour-0 cells (e = q, q + 2 with q = (i + j) & 1, k0 even), 0 elsewhere and
// off INTERIOR.  The warp takes D = dfast when every lane's four cells are uniform (by vote),
// else the general diagonal on every lane: the same bits either way.
__device__ __forceinline__ V4<float> first_colour_run(int i, int j, int k0, uint32_t mask4, const V4<float>& b, uint32_t cls,
                                                      const LevelConst<float>& L) {
    const int q = (i + j) & 1;
    const uint32_t mA = (mask4 >> (q ? 8 : 0)) & 0xffu, mB = (mask4 >> (q ? 24 : 16)) & 0xffu;
    const float bA = q ? b.v[1] : b.v[0], bB = q ? b.v[3] : b.v[2];
    float dA, dB;
    if (__all_sync(__activemask(), mask4 == 0x7F7F7F7Fu)) {
        dA = L.dfast;
        dB = L.dfast;
    } else {
        const FaceCoef<float> C = face_coef(i, j, k0, cls, L);
        dA = diag_cell(mA, C, q ? L.c1 : C.zlo, L.c1, L);
        dB = diag_cell(mB, C, L.c1, q ? C.zhi : L.c1, L);
    }
    const float vA = (mA & kMaskInterior) ? 0.f + (bA - 0.f) / dA : 0.f;
    const float vB = (mB & kMaskInterior) ? 0.f + (bB - 0.f) / dB : 0.f;
    V4<float> o = zero4<float>();
    if (q) { o.v[1] = vA; o.v[3] = vB; } else { o.v[0] = vA; o.v[2] = vB; }
    return o;
}

// One Gauss-Seidel update x0 + (b - A x)/D of a single cell with mask byte m, given its six
// neighbour values in face order and the coefficients of its x/y faces (C) and z faces (azl,
// azr): the operations of neg_lap4 + the sweep update.  On a uniform cell (m = 0x7F, every
// coefficient 1/h^2) it gives gs_cell_fast's bits.
__device__ __forceinline__ float gs_cell(float x0, float xm, float xp, float ym, float yp, float zl, float zr, float b, uint32_t m,
                                         const FaceCoef<float>& C, float azl, float azr, const LevelConst<float>& L) {
    const float a0 = (m & 1u) ? C.xm : 0.f;
    const float a1 = (m & 2u) ? C.xp : 0.f;
    const float a2 = (m & 4u) ? C.ym : 0.f;
    const float a3 = (m & 8u) ? C.yp : 0.f;
    const float a4 = (m & 16u) ? azl : 0.f;
    const float a5 = (m & 32u) ? azr : 0.f;
    float s = 0.f;
    s = fmaf(a0, x0 - xm, s);
    s = fmaf(a1, x0 - xp, s);
    s = fmaf(a2, x0 - ym, s);
    s = fmaf(a3, x0 - yp, s);
    s = fmaf(a4, x0 - zl, s);
    s = fmaf(a5, x0 - zr, s);
    float d = 0.f;
    d = d + a0; d = d + a1; d = d + a2; d = d + a3; d = d + a4; d = d + a5;
    return x0 + ((m & kMaskInterior) ? (b - mul_h3(s, L.h)) / mul_h3(d, L.h) : 0.f);
}
// gs_cell on a uniform cell: every coefficient 1/h^2, the diagonal the level's constant.
__device__ __forceinline__ float gs_cell_fast(float x0, float xm, float xp, float ym, float yp, float zl, float zr, float b,
                                              const LevelConst<float>& L) {
    float s = 0.f;
    s = fmaf(L.c1, x0 - xm, s);
    s = fmaf(L.c1, x0 - xp, s);
    s = fmaf(L.c1, x0 - ym, s);
    s = fmaf(L.c1, x0 - yp, s);
    s = fmaf(L.c1, x0 - zl, s);
    s = fmaf(L.c1, x0 - zr, s);
    return x0 + (b - mul_h3(s, L.h)) / L.dfast;
}

// One colour of a red-black sweep on thread t's four cells: the two cells of colour `color`
// (k0 is even, so they are e = p and p + 2 with p = (color + i + j) & 1) get the update, the
// other two keep their values.  xs/hx: the tile and its halos in shared memory.  Uniform warps
// (every lane's four cells uniform, by vote) take the fast form, the others the general one for
// every lane: the same bits either way.
__device__ __forceinline__ V4<float> colour_update(const float* xs, const float* hx, int t, uint32_t mask4, uint32_t cls,
                                                   const LevelConst<float>& L, const V4<float>& b, int color) {
    const TileIdx ix(t);
    const V4<float> xc = ld4(xs + t * 4);
    const V4<float> xm = ld4(ix.i > 0 ? xs + (t - 16) * 4 : hx + 0 * 64 + ix.j * 8 + ix.k0);
    const V4<float> xp = ld4(ix.i < 7 ? xs + (t + 16) * 4 : hx + 1 * 64 + ix.j * 8 + ix.k0);
    const V4<float> ym = ld4(ix.j > 0 ? xs + (t - 2) * 4 : hx + 2 * 64 + ix.i * 8 + ix.k0);
    const V4<float> yp = ld4(ix.j < 7 ? xs + (t + 2) * 4 : hx + 3 * 64 + ix.i * 8 + ix.k0);
    const float zlo = *(ix.k0 > 0 ? xs + t * 4 - 1 : hx + 4 * 64 + ix.i * 8 + ix.j);
    const float zhi = *(ix.k0 < 4 ? xs + t * 4 + 4 : hx + 5 * 64 + ix.i * 8 + ix.j);
    const bool p = (color + ix.i + ix.j) & 1;
    // cell A = e p, cell B = e p + 2
    const float x0A = p ? xc.v[1] : xc.v[0], x0B = p ? xc.v[3] : xc.v[2];
    const float xmA = p ? xm.v[1] : xm.v[0], xmB = p ? xm.v[3] : xm.v[2];
    const float xpA = p ? xp.v[1] : xp.v[0], xpB = p ? xp.v[3] : xp.v[2];
    const float ymA = p ? ym.v[1] : ym.v[0], ymB = p ? ym.v[3] : ym.v[2];
    const float ypA = p ? yp.v[1] : yp.v[0], ypB = p ? yp.v[3] : yp.v[2];
    const float zlA = p ? xc.v[0] : zlo, zrA = p ? xc.v[2] : xc.v[1];
    const float zlB = p ? xc.v[2] : xc.v[1], zrB = p ? zhi : xc.v[3];
    const float bA = p ? b.v[1] : b.v[0], bB = p ? b.v[3] : b.v[2];
    float A, B;
    if (__all_sync(__activemask(), mask4 == 0x7F7F7F7Fu)) {
        A = gs_cell_fast(x0A, xmA, xpA, ymA, ypA, zlA, zrA, bA, L);
        B = gs_cell_fast(x0B, xmB, xpB, ymB, ypB, zlB, zrB, bB, L);
    } else {
        const FaceCoef<float> C = face_coef(ix, cls, L);
        const uint32_t mA = (mask4 >> (p ? 8 : 0)) & 0xffu, mB = (mask4 >> (p ? 24 : 16)) & 0xffu;
        // cell A is the column's first cell (outer z- face) when p = 0; B its last (z+) when p = 1
        A = gs_cell(x0A, xmA, xpA, ymA, ypA, zlA, zrA, bA, mA, C, p ? L.c1 : C.zlo, L.c1, L);
        B = gs_cell(x0B, xmB, xpB, ymB, ypB, zlB, zrB, bB, mB, C, L.c1, p ? C.zhi : L.c1, L);
    }
    V4<float> o = xc;
    if (p) { o.v[1] = A; o.v[3] = B; } else { o.v[0] = A; o.v[2] = B; }
    return o;
}

// Asynchronous global -> shared copies (cp.async): the data goes straight to shared memory
// without passing through registers, so a CTA can keep several tiles' loads in flight at once.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
// Bulk prefetch of `bytes` (a multiple of 16, 16-byte aligned) at `p` into L2, without waiting
// and without a destination: a hint that raises the number of bytes in flight for tiles a later
// CTA of the same launch will stage.
__device__ __forceinline__ void prefetch_l2(const void* p, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Staging area of one tile: its values, face halos, a second channel (right-hand side) and the
// stencil mask bytes.
struct __align__(16) TileStage {
    static constexpr bool kHasB = true;
    float xs[kTileCells];
    float hx[6 * 64];
    float b[kTileCells];
    uint8_t mask[kTileCells];
    int aux[4];  // per-tile word copied with the tile (the LEAF slot, for the kernels that form dot partials)
};
// The same without the second channel: the fused Laplacian's staging area (4 KB per tile).
struct __align__(16) LapStage {
    static constexpr bool kHasB = false;
    float xs[kTileCells];
    float hx[6 * 64];
    uint8_t mask[kTileCells];
    int aux[4];
};

// Neighbour tiles whose halo cells thread t copies: face t>>4 (threads 0..63, 16-byte pieces of
// an x or y face) and z face 4 + (t>>6) (one scalar).
struct HaloNb {
    int f, z;
};
__device__ __forceinline__ HaloNb halo_nb(const TileMeta* __restrict__ meta, int tile, int t) {
    HaloNb h;
    h.f = t < 64 ? meta[tile].nb[t >> 4] : -1;
    h.z = meta[tile].nb[4 + (t >> 6)];
    return h;
}

// Per-tile values a staged kernel needs besides the copied data: halo neighbours, packed
// metadata, face classes and level constants.  Loaded for all of a group's tiles before any copy
// is issued -- the copies are asm statements with a memory clobber, so loads written after one
// are not moved ahead of it, and a load per tile between the copies would cost one memory round
// trip per tile.
struct TilePre {
    HaloNb nb;
    int packed;
    uint32_t fcls;
    float4 lc;
};
template <int NT>
__device__ __forceinline__ void tile_pre(const Topo& tp, const int (&tile)[NT], int t, TilePre (&pre)[NT]) {
    int inst[NT];
#pragma unroll
    for (int u = 0; u < NT; u++) {
        pre[u].nb = halo_nb(tp.meta, tile[u], t);
        pre[u].packed = tp.meta[tile[u]].packed;
        pre[u].fcls = tp.fcls[tile[u]];
        inst[u] = tp.inst[tile[u]];
    }
#pragma unroll
    for (int u = 0; u < NT; u++) pre[u].lc = tp.lconst[inst[u] * kLevelSlots + meta_level(pre[u].packed)];
}

// Issue the copies of `tile` into st: channel X's values and face halos (0 for absent
// neighbours), channel B (if given) and the mask bytes (if given).  Completed by
// cp_async_wait_all + __syncthreads.
template <class Stage>
__device__ __forceinline__ void stage_async(const float* __restrict__ X, const float* __restrict__ B, const uint8_t* __restrict__ mask,
                                            int tile, HaloNb nb, int t, Stage& st) {
    const size_t base = (size_t)tile * kTileCells;
    cp_async16(st.xs + t * 4, X + base + t * 4);
    if constexpr (Stage::kHasB) {
        if (B) cp_async16(st.b + t * 4, B + base + t * 4);
    }
    if (mask && t < 32) cp_async16(st.mask + t * 16, mask + base + t * 16);
    if (t < 64) {
        const int face = t >> 4, q = t & 15;
        int off;
        if (face == 0) off = 448 + q * 4;
        else if (face == 1) off = q * 4;
        else if (face == 2) off = (q >> 1) * 64 + 56 + (q & 1) * 4;
        else off = (q >> 1) * 64 + (q & 1) * 4;
        if (nb.f >= 0) cp_async16(st.hx + face * 64 + q * 4, X + (size_t)nb.f * kTileCells + off);
        else st4(st.hx + face * 64 + q * 4, zero4<float>());
    }
    {
        const int face = 4 + (t >> 6), c = t & 63;
        if (nb.z >= 0) cp_async4(st.hx + face * 64 + c, X + (size_t)nb.z * kTileCells + (c >> 3) * 64 + (c & 7) * 8 + (face == 4 ? 7 : 0));
        else st.hx[face * 64 + c] = 0.f;
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

// 4-cell dot product as the reference's Dot128Kernel forms it (src/PoissonGrid.cu:177-181): FP32
// products and sums, widened to FP64.
__device__ __forceinline__ float dot4f32(const V4<float>& a, const V4<float>& b) {
    float s = fmaf(a.v[0], b.v[0], a.v[1] * b.v[1]);
    s = fmaf(a.v[2], b.v[2], s);
    return fmaf(a.v[3], b.v[3], s);
}
__device__ __forceinline__ double dot4f(const V4<float>& a, const V4<float>& b) { return (double)dot4f32(a, b); }
// shuffle-down tree over a full warp; lane 0 holds the sum
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}
// A tile's part of a dot product from its 128 per-vector FP32 terms, formed by 16 lanes: lane j
// (0..15) adds the terms of vectors j, j+16, ..., j+112 in FP64 in that order (term[k] = vector
// j + 16k), then a 4-level shuffle tree over the 16 lanes.  Both 16-lane halves of the warp take
// part (each its own tile, or a discarded one); lane 0 of each half holds its tile's part.  The
// order is the same in every kernel and launch shape.
__device__ __forceinline__ double half_part_sum(const float term[8]) {
    double d = (double)term[0];
#pragma unroll
    for (int k = 1; k < 8; k++) d += (double)term[k];
#pragma unroll
    for (int o = 8; o > 0; o >>= 1) d += __shfl_down_sync(0xffffffffu, d, o, 16);
    return d;
}
// the same from terms laid out by vector in shared memory (terms[v], v = 0..127), lane j = 0..15
__device__ __forceinline__ double tile_part_sum(const float* terms, int j) {
    float term[8];
#pragma unroll
    for (int k = 0; k < 8; k++) term[k] = terms[j + 16 * k];
    return half_part_sum(term);
}

// Face path of the fused Laplacian: one coarse cell of a GHOST tile whose coupled cells all lie
// on its faces and couple only outward.  Item: tile, ghost slot << 6 | coarse cell c, coupled
// faces | face classes << 6, level-constant index.  Forms the cell's partial sum -- its 2x2x2
// block of A p values in AccumulateToParents128's (ii,jj,kk) order -- computing A p only on
// cells with coupled faces, each term from the neighbour's value across the face.  Every other
// cell's A p is +0 in the full path, which also adds the zero-coefficient terms skipped here (as
// +-0, which leaves finite sums unchanged).  All loads are issued before the arithmetic: the
// block's own values, mask and type bytes (four 2-cell runs along k), then the neighbour values
// across each coupled face it touches.
__device__ __forceinline__ void ghost_face_sum(const Topo& tp, const float* __restrict__ X, int4 it, float* __restrict__ GACC) {
    const int tile = it.x, c = it.y & 63;
    const uint32_t faces = (uint32_t)it.z & 63u, cls = (uint32_t)it.z >> 6;
    const int fi = c / 16 * 2, fj = (c / 4) % 4 * 2, fk = c % 4 * 2;
    const size_t base = (size_t)tile * kTileCells;
    const int o0 = fi * 64 + fj * 8 + fk;
    float2 xo[4];
    uint32_t mk[4], ck[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int o = o0 + (q >> 1) * 64 + (q & 1) * 8;
        xo[q] = *reinterpret_cast<const float2*>(X + base + o);
        mk[q] = *reinterpret_cast<const uint16_t*>(tp.mask_lap + base + o);
        ck[q] = *reinterpret_cast<const uint16_t*>(tp.ctype + base + o);
    }
    const uint32_t touch = (fi == 0 ? 1u : 0u) | (fi == 6 ? 2u : 0u) | (fj == 0 ? 4u : 0u) | (fj == 6 ? 8u : 0u) | (fk == 0 ? 16u : 0u) |
                           (fk == 6 ? 32u : 0u);
    const uint32_t act = touch & faces;
    const TileMeta& m = tp.meta[tile];
    // nv[f][a*2+b]: the neighbour's value across face f for the block's cell (a, b) on that face,
    // (a, b) = (jj, kk) on x faces, (ii, kk) on y faces, (ii, jj) on z faces
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
    float sum = 0.f;
#pragma unroll
    for (int ii = 0; ii < 2; ii++)
#pragma unroll
        for (int jj = 0; jj < 2; jj++)
#pragma unroll
            for (int kk = 0; kk < 2; kk++) {
                const int i = fi + ii, j = fj + jj, k = fk + kk;
                const uint32_t on = (i == 0 ? 1u : 0u) | (i == 7 ? 2u : 0u) | (j == 0 ? 4u : 0u) | (j == 7 ? 8u : 0u) |
                                    (k == 0 ? 16u : 0u) | (k == 7 ? 32u : 0u);
                const int q = ii * 2 + jj;
                const uint32_t mm = (mk[q] >> (8 * kk)) & 0xffu;
                float v = 0.f;
                if ((on & act) && (mm & 0x3Fu)) {
                    const float x0 = kk ? xo[q].y : xo[q].x;
                    float s = 0.f;
#pragma unroll
                    for (int f = 0; f < 6; f++) {
                        if (!(mm & (1u << f))) continue;
                        const float a = ((cls >> (2 * f)) & 3u) == 2u ? L.c2 : L.c1;
                        const float xf = nv[f][f < 2 ? jj * 2 + kk : (f < 4 ? ii * 2 + kk : ii * 2 + jj)];
                        s = __fadd_rn(s, __fmul_rn(a, x0 - xf));
                    }
                    const float out = (mm & kMaskInterior) ? mul_h3(s, L.h) : 0.f;
                    v = (((ck[q] >> (8 * kk)) & 0xffu) & (INTERIOR_C | DIRICHLET_C | NEUMANN_C)) ? out : 0.f;
                }
                sum += v;
            }
    GACC[(size_t)(it.y >> 6) * 64 + c] = sum;
}

}  // namespace cirrus
