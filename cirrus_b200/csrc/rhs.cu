// Right-hand side of the pressure projection, built on the device as FluidEuler::project does
// (src/FluidEuler.h:583-586) after the velocity boundary step's face clearing
// (src/FluidEuler.cu:43-60).  Velocities live on the three lower faces of each cell
// (channels u, u+1, u+2); all arithmetic is FP32 as in the reference.
#include "kernels.cuh"
#include "solver_internal.hpp"

namespace cirrus {

namespace {

// ClearAllNeumannNeighborFaces on LEAF tiles: the lower face of axis a is zeroed when the cell
// or a cell across it is NEUMANN, or both are DIRICHLET.  Across a NONLEAF or GHOST neighbour
// the four finer cells behind the face are tested (IterateFaceNeighborCellTypes,
// src/PoissonGrid.h:451-489).
__global__ void __launch_bounds__(128) k_clear_faces(Topo tp, const int* __restrict__ child, const int* __restrict__ list, int n,
                                                     float* U0, float* U1, float* U2) {
    const int q = blockIdx.x;
    if (q >= n) return;
    const int tile = list[q];
    const TileMeta m = tp.meta[tile];
    const int t = threadIdx.x;
    float* U[3] = {U0, U1, U2};
    for (int e = 0; e < 4; e++) {
        const int o = t * 4 + e;
        const int l[3] = {o >> 6, (o >> 3) & 7, o & 7};
        const uint8_t t0 = tp.ctype[(size_t)tile * kTileCells + o];
        for (int a = 0; a < 3; a++) {
            bool to_set = false;
            auto test = [&](uint8_t t1) {
                if ((t0 & NEUMANN_C) || (t1 & NEUMANN_C) || ((t0 & DIRICHLET_C) && (t1 & DIRICHLET_C))) to_set = true;
            };
            int nl[3] = {l[0], l[1], l[2]};
            nl[a] -= 1;
            if (nl[a] >= 0) {
                test(tp.ctype[(size_t)tile * kTileCells + (nl[0] << 6 | nl[1] << 3 | nl[2])]);
            } else {
                const int nb = m.nb[2 * a];
                nl[a] = 7;
                if (nb >= 0) {
                    if (meta_type(tp.meta[nb].packed) & LEAF_T) {
                        test(tp.ctype[(size_t)nb * kTileCells + (nl[0] << 6 | nl[1] << 3 | nl[2])]);
                    } else {
                        for (int oj = 0; oj < 2; oj++)
                            for (int ok = 0; ok < 2; ok++) {
                                int off[3];
                                off[a] = 1; off[(a + 1) % 3] = oj; off[(a + 2) % 3] = ok;
                                int c[3], oct = 0;
                                for (int d = 0; d < 3; d++) {
                                    c[d] = nl[d] * 2 + off[d];
                                    oct |= (c[d] >> 3) << d;
                                }
                                const int ct = child[(size_t)nb * 8 + oct];
                                if (ct >= 0) test(tp.ctype[(size_t)ct * kTileCells + ((c[0] & 7) << 6 | (c[1] & 7) << 3 | (c[2] & 7))]);
                            }
                    }
                }
            }
            if (to_set) U[a][(size_t)tile * kTileCells + o] = 0.f;
        }
    }
}

// PropagateToChildren(c, c, -1, GHOST, LAUNCH_SUBTREE, I|D|N) (src/PoissonGrid.cu:635-661):
// typed GHOST cells copy their parent cell's value (0 if the parent cell is untyped or absent).
__global__ void __launch_bounds__(128) k_propagate_children(Topo tp, const int* __restrict__ list, int n, float* X) {
    const int q = blockIdx.x;
    if (q >= n) return;
    const int tile = list[q];
    const TileMeta m = tp.meta[tile];
    const int t = threadIdx.x;
    const TileIdx ix(t);
    const int oct = meta_octant(m.packed);
    for (int e = 0; e < 4; e++) {
        const size_t id = (size_t)tile * kTileCells + t * 4 + e;
        if (!(tp.ctype[id] & 7)) continue;
        float val = 0.f;
        if (m.parent >= 0) {
            const size_t pid = (size_t)m.parent * kTileCells + ((oct & 1) * 4 + (ix.i >> 1)) * 64 +
                               (((oct >> 1) & 1) * 4 + (ix.j >> 1)) * 8 + ((oct >> 2) & 1) * 4 + ((ix.k0 + e) >> 1);
            val = X[pid];
            if (!(tp.ctype[pid] & 7)) val = 0.f;
        }
        X[id] = val;
    }
}

// VelocityVolumeDivergenceOnLeafs (src/PoissonSolver.cu:66-137) on LEAF|GHOST tiles: the sum of
// outgoing face fluxes u*h*h over LEAF-LEAF, LEAF-GHOST and GHOST-LEAF faces on INTERIOR cells.
__global__ void __launch_bounds__(128) k_divergence(Topo tp, const int* __restrict__ list, int n, const float* __restrict__ U0,
                                                    const float* __restrict__ U1, const float* __restrict__ U2, float* B) {
    const int q = blockIdx.x;
    if (q >= n) return;
    const int tile = list[q];
    const TileMeta m = tp.meta[tile];
    const int t = threadIdx.x;
    const uint8_t tt = (uint8_t)meta_type(m.packed);
    const float h = tile_h0(tp, tile) / float(1 << meta_level(m.packed));
    const float* U[3] = {U0, U1, U2};
    for (int e = 0; e < 4; e++) {
        const int o = t * 4 + e;
        const size_t id = (size_t)tile * kTileCells + o;
        if (!(tp.ctype[id] & INTERIOR_C)) {
            B[id] = 0.f;
            continue;
        }
        const int l[3] = {o >> 6, (o >> 3) & 7, o & 7};
        float sum = 0.f;
        for (int a = 0; a < 3; a++) {
            for (int sg = 0; sg < 2; sg++) {
                const int sgn = sg ? 1 : -1;
                int nl[3] = {l[0], l[1], l[2]};
                nl[a] += sgn;
                int nt = tile;
                if (nl[a] < 0 || nl[a] > 7) {
                    nt = m.nb[2 * a + sg];
                    nl[a] &= 7;
                }
                const float u0 = U[a][id];
                float u1;
                uint8_t ntt;
                if (nt < 0) {
                    ntt = tt;
                    u1 = 0.f;
                } else {
                    ntt = (uint8_t)meta_type(tp.meta[nt].packed);
                    u1 = U[a][(size_t)nt * kTileCells + (nl[0] << 6 | nl[1] << 3 | nl[2])];
                }
                const bool ok = (tt == LEAF_T && ntt == LEAF_T) || (tt == LEAF_T && ntt == GHOST_T) || (tt == GHOST_T && ntt == LEAF_T);
                if (!ok) continue;
                const float u = (sgn == -1) ? -u0 : u1;
                sum += u * h * h;
            }
        }
        B[id] = sum;
    }
}

// AccumulateToParents(b, b, -1, LEAF, LAUNCH_SUBTREE, INTERIOR, 1, additive)
// (src/PoissonGrid.cu:721-755): cells of LEAF tiles whose type is in cell_types add coeff times
// the sum of their children's values over children of those types (childCoord order, x fastest).
__global__ void __launch_bounds__(128) k_accumulate_children(Topo tp, const int* __restrict__ child, const int* __restrict__ list,
                                                             int n, float* B, uint8_t cell_types, float coeff) {
    const int q = blockIdx.x;
    if (q >= n) return;
    const int tile = list[q];
    const int t = threadIdx.x;
    const TileIdx ix(t);
    for (int e = 0; e < 4; e++) {
        const size_t id = (size_t)tile * kTileCells + t * 4 + e;
        if (!(tp.ctype[id] & cell_types)) continue;
        const int l[3] = {ix.i, ix.j, ix.k0 + e};
        const int oct = (l[0] >> 2) | ((l[1] >> 2) << 1) | ((l[2] >> 2) << 2);
        const int ct = child[(size_t)tile * 8 + oct];
        if (ct < 0) continue;
        float sum = 0.f;
        for (int cid = 0; cid < 8; cid++) {
            const int c0 = (l[0] * 2 + (cid & 1)) & 7, c1 = (l[1] * 2 + ((cid >> 1) & 1)) & 7, c2 = (l[2] * 2 + ((cid >> 2) & 1)) & 7;
            const size_t cidx = (size_t)ct * kTileCells + (c0 << 6 | c1 << 3 | c2);
            if (tp.ctype[cidx] & cell_types) sum += B[cidx];
        }
        B[id] = fmaf(sum, coeff, B[id]);
    }
}

// The face terms of AddGradientToFaceCenters (src/PoissonSolver.cu:144-200) on LEAF|GHOST tiles:
// on each lower face (x-, y-, z-) u += (p1 - p0) / dh with dh = h between LEAF cells and 1.5 h
// across a LEAF-GHOST face (no term otherwise, nor across a NEUMANN cell); p1, p0 the INTERIOR
// values (0 elsewhere); an absent neighbour counts as the cell's own tile and cell type with
// p0 = 0.  GHOST tiles start from u = 0.
__global__ void __launch_bounds__(128) k_gradient(Topo tp, const int* __restrict__ list, int n, const float* __restrict__ P, float* U0,
                                                  float* U1, float* U2) {
    const int q = blockIdx.x;
    if (q >= n) return;
    const int tile = list[q];
    const TileMeta m = tp.meta[tile];
    const int t = threadIdx.x;
    const uint8_t tt = (uint8_t)meta_type(m.packed);
    const float h = tile_h0(tp, tile) / float(1 << meta_level(m.packed));
    const float h15 = (float)(1.5 * (double)h);
    float* U[3] = {U0, U1, U2};
    for (int e = 0; e < 4; e++) {
        const int o = t * 4 + e;
        const size_t id = (size_t)tile * kTileCells + o;
        const uint8_t ct = tp.ctype[id];
        const float p1 = (ct & INTERIOR_C) ? P[id] : 0.f;
        const int l[3] = {o >> 6, (o >> 3) & 7, o & 7};
        for (int a = 0; a < 3; a++) {
            float u = tt == GHOST_T ? 0.f : U[a][id];
            int nl[3] = {l[0], l[1], l[2]};
            nl[a] -= 1;
            uint8_t ntt, nct;
            float p0;
            if (nl[a] >= 0) {
                const size_t nid = (size_t)tile * kTileCells + (nl[0] << 6 | nl[1] << 3 | nl[2]);
                ntt = tt;
                nct = tp.ctype[nid];
                p0 = (nct & INTERIOR_C) ? P[nid] : 0.f;
            } else {
                const int nb = m.nb[2 * a];
                nl[a] = 7;
                if (nb < 0) {
                    ntt = tt;
                    nct = ct;
                    p0 = 0.f;
                } else {
                    const size_t nid = (size_t)nb * kTileCells + (nl[0] << 6 | nl[1] << 3 | nl[2]);
                    ntt = (uint8_t)meta_type(tp.meta[nb].packed);
                    nct = tp.ctype[nid];
                    p0 = (nct & INTERIOR_C) ? P[nid] : 0.f;
                }
            }
            float dh;
            bool term = true;
            if ((tt & LEAF_T) && (ntt & LEAF_T)) dh = h;
            else if (((tt & LEAF_T) && (ntt & GHOST_T)) || ((tt & GHOST_T) && (ntt & LEAF_T))) dh = h15;
            else term = false;
            if ((ct & NEUMANN_C) || (nct & NEUMANN_C)) term = false;
            if (term) u = u + (p1 - p0) / dh;
            if (term || tt == GHOST_T) U[a][id] = u;
        }
    }
}

}  // namespace

namespace launch {

void clear_neumann_faces(const DevGrid& g, int u_channel, cudaStream_t s) {
    if (g.n_leaf == 0) return;
    ++g.launch_count;
    k_clear_faces<<<g.n_leaf, 128, 0, s>>>(g.topo, g.d_child, g.d_leaf, g.n_leaf, g.d_ch[u_channel], g.d_ch[u_channel + 1],
                                          g.d_ch[u_channel + 2]);
}

void propagate_to_children(const DevGrid& g, int channel, cudaStream_t s) {
    if (g.n_ghost == 0) return;
    ++g.launch_count;
    k_propagate_children<<<g.n_ghost, 128, 0, s>>>(g.topo, g.d_ghost, g.n_ghost, g.d_ch[channel]);
}

void velocity_divergence(const DevGrid& g, int u_channel, int b_channel, cudaStream_t s) {
    if (g.n_leafghost == 0) return;
    ++g.launch_count;
    k_divergence<<<g.n_leafghost, 128, 0, s>>>(g.topo, g.d_leafghost, g.n_leafghost, g.d_ch[u_channel], g.d_ch[u_channel + 1],
                                              g.d_ch[u_channel + 2], g.d_ch[b_channel]);
    ++g.launch_count;
    k_accumulate_children<<<g.n_leaf, 128, 0, s>>>(g.topo, g.d_child, g.d_leaf, g.n_leaf, g.d_ch[b_channel], (uint8_t)INTERIOR_C,
                                                   1.0f);
}

void add_gradient(const DevGrid& g, int p_channel, int u_channel, cudaStream_t s) {
    propagate_ghosts<float>(g, g.d_ch[p_channel], nullptr, s);
    if (g.n_leafghost > 0) {
        ++g.launch_count;
        k_gradient<<<g.n_leafghost, 128, 0, s>>>(g.topo, g.d_leafghost, g.n_leafghost, g.d_ch[p_channel], g.d_ch[u_channel],
                                                 g.d_ch[u_channel + 1], g.d_ch[u_channel + 2]);
    }
    if (g.n_leaf == 0) return;
    for (int a = 0; a < 3; a++) {
        ++g.launch_count;
        k_accumulate_children<<<g.n_leaf, 128, 0, s>>>(g.topo, g.d_child, g.d_leaf, g.n_leaf, g.d_ch[u_channel + a],
                                                       (uint8_t)(INTERIOR_C | DIRICHLET_C), 0.25f);
    }
}

}  // namespace launch
}  // namespace cirrus
