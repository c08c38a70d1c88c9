// Device grid construction: turns a finalised host topology into the HBM-resident tile pool.
//
// Layout (all-tiles order, level-major as the reference's dAllTiles):
//   channels   9 x n x 512 FP32, one contiguous buffer (channel-major SoA)
//   u8         ctype | mask_lap | mask_mg, 3 x n x 512 bytes
//   meta       n x TileMeta (32 B): neighbours in stencil face order, parent, level/type/octant
//   fcls       n x uint32 cross-face coefficient classes (Laplacian and multigrid contexts)
//   lists      LEAF, GHOST, LEAF|GHOST tiles; LEAF|NONLEAF tiles per level
// The per-cell stencil masks fold NegativeLaplacianCoeff's tile-type and Neumann tests
// (src/GMGSolver.cu:26-39) into one byte so the kernels never load neighbour cell types.
#include "solver_internal.hpp"
#include "topology.hpp"

#include <algorithm>
#include <cstring>

namespace cirrus {

namespace {

inline uint8_t subtree_type(uint8_t type, int level, int sl) {
    return (level == sl && type == NONLEAF_T) ? LEAF_T : type;  // src/HATileInfo.h:82-87
}
inline uint32_t coeff_class(uint8_t a, uint8_t b) {
    if ((a & LEAF_T) && (b & LEAF_T)) return 1u;
    if (((a & LEAF_T) && (b & GHOST_T)) || ((a & GHOST_T) && (b & LEAF_T))) return 2u;
    return 0u;
}

#define CK(x)                                                        \
    do {                                                             \
        cudaError_t e_ = (x);                                        \
        if (e_ != cudaSuccess) {                                     \
            if (err) *err = std::string(#x ": ") + cudaGetErrorString(e_); \
            grid_destroy(g);                                         \
            return e_ == cudaErrorMemoryAllocation ? 3 : 2;          \
        }                                                            \
    } while (0)

}  // namespace

int grid_create(const Topology& topo, DevGrid** out, std::string* err) {
    const int n = topo.num_tiles();
    if (n <= 0) {
        if (err) *err = "empty topology";
        return 1;
    }
    std::vector<int32_t> t5((size_t)n * 5), nb6((size_t)n * 6), par(n), ch8((size_t)n * 8), e12((size_t)n * 12);
    std::vector<uint8_t> ct((size_t)n * kTileCells);
    topo.tiles(t5.data());
    topo.neighbor_tiles(nb6.data());
    topo.parent_tiles(par.data());
    topo.child_tiles(ch8.data());
    topo.edge_tiles(e12.data());
    topo.cell_types(ct.data());

    std::vector<TileMeta> meta(n);
    std::vector<uint32_t> fcls(n);
    std::vector<uint8_t> mlap((size_t)n * kTileCells), mmg((size_t)n * kTileCells);
    std::vector<int> level(n), type(n);
    for (int t = 0; t < n; t++) {
        level[t] = t5[5 * t];
        type[t] = t5[5 * t + 4];
    }
#pragma omp parallel for schedule(dynamic, 64)
    for (int t = 0; t < n; t++) {
        TileMeta& m = meta[t];
        for (int f = 0; f < 6; f++) {
            const int axis = f >> 1, plus = f & 1;
            m.nb[f] = nb6[6 * t + axis + (plus ? 3 : 0)];
        }
        m.parent = par[t];
        const int oct = (t5[5 * t + 1] & 1) | ((t5[5 * t + 2] & 1) << 1) | ((t5[5 * t + 3] & 1) << 2);
        m.packed = level[t] | (type[t] << 8) | (oct << 16);
        for (int f = 0; f < 6; f++)
            if (m.nb[f] >= 0 && (type[m.nb[f]] & GHOST_T)) m.packed |= 1 << (24 + f);
        uint32_t cls_all = 0;
        for (int ctx = 0; ctx < 2; ctx++) {
            const int sl = ctx == 0 ? -1 : level[t];
            const uint8_t tt0 = subtree_type((uint8_t)type[t], level[t], sl);
            uint32_t cross[6];
            for (int f = 0; f < 6; f++) {
                const int nb = m.nb[f];
                cross[f] = nb < 0 ? coeff_class(tt0, tt0) : coeff_class(tt0, subtree_type((uint8_t)type[nb], level[nb], sl));
                cls_all |= cross[f] << (2 * f + 12 * ctx);
            }
            const uint32_t inner = coeff_class(tt0, tt0);
            uint8_t* mask = (ctx == 0 ? mlap.data() : mmg.data()) + (size_t)t * kTileCells;
            const uint8_t* c0 = ct.data() + (size_t)t * kTileCells;
            for (int o = 0; o < kTileCells; o++) {
                const int ijk[3] = {o >> 6, (o >> 3) & 7, o & 7};
                const uint8_t ct0 = c0[o];
                uint8_t bits = (ct0 & INTERIOR_C) ? kMaskInterior : 0;
                for (int f = 0; f < 6; f++) {
                    const int axis = f >> 1, sgn = (f & 1) ? 1 : -1;
                    int nn[3] = {ijk[0], ijk[1], ijk[2]};
                    nn[axis] += sgn;
                    uint32_t cls;
                    uint8_t ct1;
                    if (nn[axis] >= 0 && nn[axis] < 8) {
                        cls = inner;
                        ct1 = c0[(nn[0] << 6) | (nn[1] << 3) | nn[2]];
                    } else {
                        const int nb = m.nb[f];
                        cls = cross[f];
                        nn[axis] &= 7;
                        ct1 = nb < 0 ? DIRICHLET_C : ct[(size_t)nb * kTileCells + ((nn[0] << 6) | (nn[1] << 3) | nn[2])];
                    }
                    const bool neumann = (ct0 & NEUMANN_C) || (ct1 & NEUMANN_C);
                    if (cls != 0 && !neumann) bits |= (uint8_t)(1u << f);
                }
                mask[o] = bits;
            }
        }
        fcls[t] = cls_all;
    }

    // lists
    std::vector<int> leaf, ghost, leafghost, mg;
    const int num_layers = topo.num_layers();
    std::vector<int> mg_off(num_layers, 0), mg_cnt(num_layers, 0), lfirst(num_layers, 0), lcnt(num_layers, 0);
    int64_t dof = 0;
    for (int t = 0; t < n; t++) {
        if (type[t] & LEAF_T) {
            leaf.push_back(t);
            for (int o = 0; o < kTileCells; o++) dof += (ct[(size_t)t * kTileCells + o] & INTERIOR_C) ? 1 : 0;
        }
        if (type[t] & GHOST_T) ghost.push_back(t);
        if (type[t] & (LEAF_T | GHOST_T)) leafghost.push_back(t);
    }
    for (int l = 0; l < num_layers; l++) {
        mg_off[l] = (int)mg.size();
        bool first = true;
        for (int t = 0; t < n; t++) {
            if (level[t] != l) continue;
            if (first) { lfirst[l] = t; first = false; }
            lcnt[l]++;
            if (subtree_type((uint8_t)type[t], l, l) & (LEAF_T | NONLEAF_T)) mg.push_back(t);
        }
        mg_cnt[l] = (int)mg.size() - mg_off[l];
    }

    DevGrid* g = new DevGrid();
    cudaGetDevice(&g->device);
    cudaDeviceGetAttribute(&g->sm_count, cudaDevAttrMultiProcessorCount, g->device);
    g->n = n;
    g->num_layers = num_layers;
    g->max_level = topo.max_level();
    g->h0 = (float)topo.h0();
    g->dof = dof;
    g->n_leaf = (int)leaf.size();
    g->n_ghost = (int)ghost.size();
    g->n_leafghost = (int)leafghost.size();
    g->mg_offset = mg_off;
    g->mg_count = mg_cnt;
    g->level_first = lfirst;
    g->level_count = lcnt;
    g->h_tile_type.assign(type.begin(), type.end());
    {
        long long vecs = (long long)g->n_leaf * 128;
        long long want = (vecs + 255) / 256;
        long long cap = (long long)g->sm_count * 4;
        g->red_blocks = (int)std::max(1LL, std::min(want, cap));
    }

    const size_t cells = (size_t)n * kTileCells;
    CK(cudaMalloc(&g->d_chbuf, cells * kNumChannels * sizeof(float)));
    CK(cudaMemset(g->d_chbuf, 0, cells * kNumChannels * sizeof(float)));
    for (int c = 0; c < kNumChannels; c++) g->d_ch[c] = g->d_chbuf + cells * c;
    CK(cudaMalloc(&g->d_u8, cells * 3));
    CK(cudaMemcpy(g->d_u8, ct.data(), cells, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(g->d_u8 + cells, mlap.data(), cells, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(g->d_u8 + 2 * cells, mmg.data(), cells, cudaMemcpyHostToDevice));
    CK(cudaMalloc(&g->d_meta, sizeof(TileMeta) * n));
    CK(cudaMemcpy(g->d_meta, meta.data(), sizeof(TileMeta) * n, cudaMemcpyHostToDevice));
    CK(cudaMalloc(&g->d_fcls, sizeof(uint32_t) * n));
    CK(cudaMemcpy(g->d_fcls, fcls.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice));
    CK(cudaMalloc(&g->d_child, sizeof(int) * 8 * n));
    CK(cudaMemcpy(g->d_child, ch8.data(), sizeof(int) * 8 * n, cudaMemcpyHostToDevice));
    CK(cudaMalloc(&g->d_edge, sizeof(int) * 12 * n));
    CK(cudaMemcpy(g->d_edge, e12.data(), sizeof(int) * 12 * n, cudaMemcpyHostToDevice));
    {
        // ghost bookkeeping of the fused Laplacian: slot of each GHOST tile, the ghost slot of the
        // GHOST child in each octant, and a 64-float partial-sum row per ghost
        std::vector<int> gslot(n, -1), gchild((size_t)n * 8, -1);
        for (size_t i = 0; i < ghost.size(); i++) gslot[ghost[i]] = (int)i;
        for (int t = 0; t < n; t++)
            for (int o = 0; o < 8; o++) {
                const int c = ch8[(size_t)t * 8 + o];
                if (c >= 0 && (type[c] & GHOST_T)) gchild[(size_t)t * 8 + o] = gslot[c];
            }
        CK(cudaMalloc(&g->d_ghost_tables, sizeof(int) * 9 * (size_t)n));
        CK(cudaMemcpy(g->d_ghost_tables, gslot.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(g->d_ghost_tables + n, gchild.data(), sizeof(int) * 8 * (size_t)n, cudaMemcpyHostToDevice));
        CK(cudaMalloc(&g->d_gacc, sizeof(float) * 64 * std::max<size_t>(ghost.size(), 1)));
        CK(cudaMalloc(&g->d_xpre, sizeof(float) * kTileCells * (size_t)n));
        CK(cudaMemset(g->d_xpre, 0, sizeof(float) * kTileCells * (size_t)n));  // GHOST tiles stay 0
    }
    const size_t nl = leaf.size() + ghost.size() + leafghost.size() + mg.size() + 1;
    CK(cudaMalloc(&g->d_lists, sizeof(int) * nl));
    std::vector<int> lists;
    lists.reserve(nl);
    lists.insert(lists.end(), leaf.begin(), leaf.end());
    lists.insert(lists.end(), ghost.begin(), ghost.end());
    lists.insert(lists.end(), leafghost.begin(), leafghost.end());
    lists.insert(lists.end(), mg.begin(), mg.end());
    lists.push_back(0);
    CK(cudaMemcpy(g->d_lists, lists.data(), sizeof(int) * lists.size(), cudaMemcpyHostToDevice));
    g->d_leaf = g->d_lists;
    g->d_ghost = g->d_leaf + leaf.size();
    g->d_leafghost = g->d_ghost + ghost.size();
    g->d_mg = g->d_leafghost + leafghost.size();
    {
        std::vector<int> lt(4 * num_layers);
        for (int l = 0; l < num_layers; l++) {
            lt[l] = mg_off[l];
            lt[num_layers + l] = mg_cnt[l];
            lt[2 * num_layers + l] = lfirst[l];
            lt[3 * num_layers + l] = lcnt[l];
        }
        CK(cudaMalloc(&g->d_level_tables, sizeof(int) * lt.size()));
        CK(cudaMemcpy(g->d_level_tables, lt.data(), sizeof(int) * lt.size(), cudaMemcpyHostToDevice));
        // levels handled by the shared-memory small-level kernel: the longest prefix of levels
        // holding at most launch::kBottomTiles tiles in total
        g->bottom_level = -1;
        int cum = 0;
        for (int l = 0; l <= g->max_level && cum + lcnt[l] <= launch::kBottomTiles; l++) {
            cum += lcnt[l];
            g->bottom_level = l;
        }
        launch::init_kernel_attributes();
    }
    CK(cudaMalloc(&g->d_partials, sizeof(double) * 2 * std::max(g->red_blocks, 1)));
    CK(cudaMalloc(&g->d_counter, sizeof(unsigned int) * 4));
    CK(cudaMemset(g->d_counter, 0, sizeof(unsigned int) * 4));
    CK(cudaMalloc(&g->d_scalars, sizeof(Scalars)));
    CK(cudaMemset(g->d_scalars, 0, sizeof(Scalars)));
    CK(cudaMallocHost(&g->h_scalars, sizeof(Scalars)));
    g->history_cap = 4096;
    CK(cudaMalloc(&g->d_history, sizeof(double) * g->history_cap));
    CK(cudaMalloc(&g->d_norm, sizeof(double) * 4));

    g->topo.ctype = g->d_u8;
    g->topo.mask_lap = g->d_u8 + cells;
    g->topo.mask_mg = g->d_u8 + 2 * cells;
    g->topo.meta = g->d_meta;
    g->topo.fcls = g->d_fcls;
    g->topo.edge = g->d_edge;
    g->topo.ghost_slot = g->d_ghost_tables;
    g->topo.ghost_child = g->d_ghost_tables + n;
    g->topo.h0 = g->h0;
    g->bytes = cells * kNumChannels * sizeof(float) + cells * 3 + sizeof(TileMeta) * n + sizeof(uint32_t) * n + sizeof(int) * nl +
               sizeof(int) * 8 * n;
    *out = g;
    return 0;
}

void grid_destroy(DevGrid* g) {
    if (!g) return;
    for (auto& kv : g->graphs) cudaGraphExecDestroy(kv.second.exec);
    cudaFree(g->d_chbuf);
    cudaFree(g->d_u8);
    cudaFree(g->d_meta);
    cudaFree(g->d_fcls);
    cudaFree(g->d_child);
    cudaFree(g->d_edge);
    cudaFree(g->d_ghost_tables);
    cudaFree(g->d_gacc);
    cudaFree(g->d_xpre);
    cudaFree(g->d_level_tables);
    cudaFree(g->d_tile_ptrs);
    cudaFree(g->d_lists);
    cudaFree(g->d_partials);
    cudaFree(g->d_counter);
    cudaFree(g->d_scalars);
    if (g->h_scalars) cudaFreeHost(g->h_scalars);
    cudaFree(g->d_history);
    cudaFree(g->d_x64);
    cudaFree(g->d_ax64);
    cudaFree(g->d_r64);
    cudaFree(g->d_norm);
    cudaFree(g->d_bsave);
    delete g;
}

}  // namespace cirrus
