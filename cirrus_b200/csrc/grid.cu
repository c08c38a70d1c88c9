// Device grid construction: turns one or more finalised host topologies (the instances of a
// batch) into one HBM-resident tile pool.
//
// Layout (level-major across the batch: all instances' level-0 tiles, then level 1, ...; inside a
// level, instance by instance in each instance's all-tiles order, so a single instance keeps the
// reference's dAllTiles order):
//   channels   9 x n x 512 FP32, one contiguous buffer (channel-major SoA)
//   u8         ctype | mask_lap | mask_mg, 3 x n x 512 bytes
//   meta       n x TileMeta (32 B): neighbours in stencil face order, parent, level/type/octant
//   fcls       n x uint32 cross-face coefficient classes (Laplacian and multigrid contexts)
//   inst       n x int32 instance of each tile
//   lists      LEAF (instance by instance), GHOST, LEAF|GHOST tiles; LEAF|NONLEAF tiles per level
// The per-cell stencil masks fold NegativeLaplacianCoeff's tile-type and Neumann tests
// (src/GMGSolver.cu:26-39) into one byte so the kernels never load neighbour cell types.
#include "kernels.cuh"
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

template <class T> int upload(T** dst, const std::vector<T>& src) {
    if (cudaMalloc(dst, sizeof(T) * std::max<size_t>(src.size(), 1)) != cudaSuccess) return 3;
    if (!src.empty() && cudaMemcpy(*dst, src.data(), sizeof(T) * src.size(), cudaMemcpyHostToDevice) != cudaSuccess) return 2;
    return 0;
}

}  // namespace

int grid_create(const std::vector<const Topology*>& topos, DevGrid** out, std::string* err) {
    const int K = (int)topos.size();
    if (K <= 0) {
        if (err) *err = "no instances";
        return 1;
    }
    // ------------------------------------------------------------------ merge the instances
    int num_layers = 0;
    std::vector<int> ni(K);
    for (int i = 0; i < K; i++) {
        ni[i] = topos[i]->num_tiles();
        if (ni[i] <= 0) {
            if (err) *err = "empty topology (instance " + std::to_string(i) + ")";
            return 1;
        }
        num_layers = std::max(num_layers, topos[i]->num_layers());
    }
    // local tables, then the global order
    std::vector<std::vector<int32_t>> lt5(K), lnb6(K), lpar(K), lch8(K), le12(K);
    std::vector<std::vector<uint8_t>> lct(K);
    for (int i = 0; i < K; i++) {
        const Topology& tp = *topos[i];
        const size_t m = (size_t)ni[i];
        lt5[i].resize(m * 5); lnb6[i].resize(m * 6); lpar[i].resize(m); lch8[i].resize(m * 8); le12[i].resize(m * 12);
        lct[i].resize(m * kTileCells);
        tp.tiles(lt5[i].data());
        tp.neighbor_tiles(lnb6[i].data());
        tp.parent_tiles(lpar[i].data());
        tp.child_tiles(lch8[i].data());
        tp.edge_tiles(le12[i].data());
        tp.cell_types(lct[i].data());
    }
    std::vector<std::vector<int>> l2g(K);
    std::vector<std::vector<TileRun>> runs(K);
    std::vector<int> g_inst, g_local;
    for (int i = 0; i < K; i++) l2g[i].assign(ni[i], -1);
    for (int l = 0; l < num_layers; l++)
        for (int i = 0; i < K; i++) {
            int first = -1, cnt = 0;
            for (int t = 0; t < ni[i]; t++)
                if (lt5[i][5 * t] == l) {
                    if (first < 0) first = t;
                    cnt++;
                }
            if (cnt == 0) continue;
            runs[i].push_back({(int)g_inst.size(), first, cnt});
            for (int t = first; t < first + cnt; t++) {
                if (lt5[i][5 * t] != l) {
                    if (err) *err = "instance tiles are not level-major";
                    return 1;
                }
                l2g[i][t] = (int)g_inst.size();
                g_inst.push_back(i);
                g_local.push_back(t);
            }
        }
    const int n = (int)g_inst.size();
    std::vector<int32_t> t5((size_t)n * 5), nb6((size_t)n * 6), par(n), ch8((size_t)n * 8), e12((size_t)n * 12);
    std::vector<uint8_t> ct((size_t)n * kTileCells);
    auto remap = [&](int i, int v) { return v >= 0 ? l2g[i][v] : -1; };
    for (int t = 0; t < n; t++) {
        const int i = g_inst[t], lt = g_local[t];
        for (int a = 0; a < 5; a++) t5[5 * (size_t)t + a] = lt5[i][5 * (size_t)lt + a];
        for (int a = 0; a < 6; a++) nb6[6 * (size_t)t + a] = remap(i, lnb6[i][6 * (size_t)lt + a]);
        par[t] = remap(i, lpar[i][lt]);
        for (int a = 0; a < 8; a++) ch8[8 * (size_t)t + a] = remap(i, lch8[i][8 * (size_t)lt + a]);
        for (int a = 0; a < 12; a++) e12[12 * (size_t)t + a] = remap(i, le12[i][12 * (size_t)lt + a]);
        std::memcpy(&ct[(size_t)t * kTileCells], &lct[i][(size_t)lt * kTileCells], kTileCells);
    }
    lt5.clear(); lnb6.clear(); lpar.clear(); lch8.clear(); le12.clear(); lct.clear();

    // ------------------------------------------------------------------ per-tile metadata and masks
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
                    if (cls != 0 && !neumann) {
                        bits |= (uint8_t)(1u << f);
                        if (cls == 2u) bits |= kMaskC2;  // a face with the (2/3)/h^2 coefficient
                    }
                }
                mask[o] = bits;
            }
        }
        fcls[t] = cls_all;
    }

    // ------------------------------------------------------------------ lists
    std::vector<int> leaf, ghost, leafghost, mg, lapmain;
    std::vector<int> mg_off(num_layers, 0), mg_cnt(num_layers, 0), lfirst(num_layers, 0), lcnt(num_layers, 0);
    std::vector<int> inst_leaves(K, 0);
    std::vector<int64_t> inst_dof(K, 0);
    for (int i = 0; i < K; i++)  // LEAF tiles instance by instance (each instance's reductions see its own order)
        for (const TileRun& r : runs[i])
            for (int t = r.global; t < r.global + r.count; t++)
                if (type[t] & LEAF_T) {
                    leaf.push_back(t);
                    inst_leaves[i]++;
                    for (int o = 0; o < kTileCells; o++) inst_dof[i] += (ct[(size_t)t * kTileCells + o] & INTERIOR_C) ? 1 : 0;
                }
    for (int t = 0; t < n; t++) {
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
    g->num_inst = K;
    g->num_layers = num_layers;
    for (int i = 0; i < K; i++) {
        g->max_level = std::max(g->max_level, topos[i]->max_level());
        g->inst_h0.push_back((float)topos[i]->h0());
        g->inst_tiles.push_back(ni[i]);
        g->inst_max_level.push_back(topos[i]->max_level());
        g->dof += inst_dof[i];
    }
    g->inst_leaves = inst_leaves;
    g->inst_dof = inst_dof;
    g->inst_runs = runs;
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
    CK((cudaError_t)(upload(&g->d_inst, g_inst) ? cudaErrorMemoryAllocation : cudaSuccess));
    CK((cudaError_t)(upload(&g->d_inst_h0, g->inst_h0) ? cudaErrorMemoryAllocation : cudaSuccess));
    {
        // level constants per instance and level, computed here with the device's IEEE float
        // operations (the kernels would otherwise recompute them in every thread)
        std::vector<float4> lc((size_t)K * kLevelSlots);
        for (int i = 0; i < K; i++)
            for (int l = 0; l < kLevelSlots; l++) {
                const LevelConst<float> L(g->inst_h0[i], l);
                lc[(size_t)i * kLevelSlots + l] = make_float4(L.h, L.c1, L.c2, L.dfast);
            }
        CK((cudaError_t)(upload(&g->d_lconst, lc) ? cudaErrorMemoryAllocation : cudaSuccess));
    }
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
        CK(cudaMemset(g->d_gacc, 0, sizeof(float) * 64 * std::max<size_t>(ghost.size(), 1)));
        // split of the fused Laplacian's GHOST tiles: a tile whose coupled cells (mask face bits)
        // all lie on its faces, each coupled only across the tile faces it lies on, takes the
        // face path with the set of those faces (none: its row stays 0); any other goes through
        // the staged path with the LEAF tiles
        std::vector<int4> lapitems;
        int n_face = 0;
        for (int t : leafghost) {
            if (!(type[t] & GHOST_T)) {
                lapmain.push_back(t);
                continue;
            }
            uint32_t faces = 0;
            bool outward = true;
            for (int o = 0; o < kTileCells && outward; o++) {
                const uint32_t bits = mlap[(size_t)t * kTileCells + o] & 0x3Fu;
                const int i = o >> 6, j = (o >> 3) & 7, k = o & 7;
                const uint32_t on = (i == 0 ? 1u : 0u) | (i == 7 ? 2u : 0u) | (j == 0 ? 4u : 0u) | (j == 7 ? 8u : 0u) |
                                    (k == 0 ? 16u : 0u) | (k == 7 ? 32u : 0u);
                if (bits & ~on) outward = false;
                faces |= bits;
            }
            if (!outward) {
                lapmain.push_back(t);
            } else if (faces) {
                n_face++;
                const int cf = (int)(faces | ((fcls[t] & 0xfffu) << 6)), lc = g_inst[t] * kLevelSlots + level[t];
                for (int c = 0; c < 64; c++) {
                    // coarse cell c covers fine cells 2*(c/16).., 2*((c/4)%4).., 2*(c%4)..
                    const int ci = c / 16, cj = (c / 4) % 4, ck = c % 4;
                    const uint32_t touch = (ci == 0 ? 1u : 0u) | (ci == 3 ? 2u : 0u) | (cj == 0 ? 4u : 0u) | (cj == 3 ? 8u : 0u) |
                                           (ck == 0 ? 16u : 0u) | (ck == 3 ? 32u : 0u);
                    if (touch & faces) lapitems.push_back(make_int4(t, (gslot[t] << 6) | c, cf, lc));
                }
            }
        }
        g->n_lapface = n_face;
        {
            // faces of each GHOST tile whose p other tiles read: those toward a non-GHOST
            // neighbour (its halo, and the face path's own values); a GHOST tile on the staged
            // Laplacian path is read whole
            std::vector<uint8_t> gf(std::max<size_t>(ghost.size(), 1), 0);
            for (size_t q = 0; q < ghost.size(); q++) {
                const int t = ghost[q];
                uint8_t f6 = 0;
                for (int f = 0; f < 6; f++) {
                    const int nb = meta[t].nb[f];
                    if (nb >= 0 && !(type[nb] & GHOST_T)) f6 |= (uint8_t)(1u << f);
                }
                gf[q] = f6;
            }
            for (int t : lapmain)
                if (type[t] & GHOST_T) gf[gslot[t]] = 0x40;
            CK(cudaMalloc(&g->d_ghost_faces, gf.size()));
            CK(cudaMemcpy(g->d_ghost_faces, gf.data(), gf.size(), cudaMemcpyHostToDevice));
        }
        g->n_lapitems = (int)lapitems.size();
        if (!lapitems.empty()) {
            if (ghost.size() >= (1u << 25)) {
                if (err) *err = "too many GHOST tiles";
                grid_destroy(g);
                return 1;
            }
            CK(cudaMalloc(&g->d_lapitems, sizeof(int4) * lapitems.size()));
            CK(cudaMemcpy(g->d_lapitems, lapitems.data(), sizeof(int4) * lapitems.size(), cudaMemcpyHostToDevice));
        }
        // the same split for the residual + restriction of the fused V-cycle, per level, from the
        // multigrid masks: face-path GHOST tiles give one item per coarse cell touching a coupled
        // face
        std::vector<int> rrmain;
        std::vector<int4> rritems;
        g->rr_off.assign(num_layers, 0);
        g->rr_cnt.assign(num_layers, 0);
        g->rri_off.assign(num_layers, 0);
        g->rri_cnt.assign(num_layers, 0);
        for (int l = 0; l < num_layers; l++) {
            g->rr_off[l] = (int)rrmain.size();
            g->rri_off[l] = (int)rritems.size();
            for (int t = lfirst[l]; t < lfirst[l] + lcnt[l]; t++) {
                bool face = (type[t] & GHOST_T) && par[t] >= 0;
                uint32_t faces = 0;
                for (int o = 0; o < kTileCells && face; o++) {
                    const uint32_t bits = mmg[(size_t)t * kTileCells + o] & 0x3Fu;
                    const int i = o >> 6, j = (o >> 3) & 7, k = o & 7;
                    const uint32_t on = (i == 0 ? 1u : 0u) | (i == 7 ? 2u : 0u) | (j == 0 ? 4u : 0u) | (j == 7 ? 8u : 0u) |
                                        (k == 0 ? 16u : 0u) | (k == 7 ? 32u : 0u);
                    if (bits & ~on) face = false;
                    faces |= bits;
                }
                if (!face) {
                    rrmain.push_back(t);
                    continue;
                }
                // only the coarse cells touching a coupled face: the others' sums are +0, and the
                // multigrid right-hand side copies of r are written without -0 under GHOST children
                const int oct = (meta[t].packed >> 16) & 7;
                for (int c = 0; c < 64; c++) {
                    const int ci = c / 16, cj = (c / 4) % 4, ck = c % 4;
                    const uint32_t touch = (ci == 0 ? 1u : 0u) | (ci == 3 ? 2u : 0u) | (cj == 0 ? 4u : 0u) | (cj == 3 ? 8u : 0u) |
                                           (ck == 0 ? 16u : 0u) | (ck == 3 ? 32u : 0u);
                    if (!(touch & faces)) continue;
                    rritems.push_back(make_int4(t, c | (int)(faces << 6) | (int)(((fcls[t] >> 12) & 0xfffu) << 12) | (oct << 24), par[t],
                                                g_inst[t] * kLevelSlots + level[t]));
                }
            }
            g->rr_cnt[l] = (int)rrmain.size() - g->rr_off[l];
            g->rri_cnt[l] = (int)rritems.size() - g->rri_off[l];
        }
        CK(cudaMalloc(&g->d_rrmain, sizeof(int) * std::max<size_t>(rrmain.size(), 1)));
        if (!rrmain.empty()) CK(cudaMemcpy(g->d_rrmain, rrmain.data(), sizeof(int) * rrmain.size(), cudaMemcpyHostToDevice));
        CK(cudaMalloc(&g->d_rritems, sizeof(int4) * std::max<size_t>(rritems.size(), 1)));
        if (!rritems.empty()) CK(cudaMemcpy(g->d_rritems, rritems.data(), sizeof(int4) * rritems.size(), cudaMemcpyHostToDevice));
        // prolongation split: non-GHOST tiles per level, and the GHOST faces that a non-GHOST
        // neighbour at the same level reads as its halo
        std::vector<int> prmain;
        std::vector<int4> pritems;
        g->pr_off.assign(num_layers, 0);
        g->pr_cnt.assign(num_layers, 0);
        g->pri_off.assign(num_layers, 0);
        g->pri_cnt.assign(num_layers, 0);
        for (int l = 0; l < num_layers; l++) {
            g->pr_off[l] = (int)prmain.size();
            g->pri_off[l] = (int)pritems.size();
            for (int t = lfirst[l]; t < lfirst[l] + lcnt[l]; t++) {
                if (!(type[t] & GHOST_T)) {
                    prmain.push_back(t);
                    continue;
                }
                for (int f = 0; f < 6; f++) {
                    const int nb = meta[t].nb[f];
                    if (nb >= 0 && !(type[nb] & GHOST_T)) pritems.push_back(make_int4(t, f, par[t], (meta[t].packed >> 16) & 7));
                }
            }
            g->pr_cnt[l] = (int)prmain.size() - g->pr_off[l];
            g->pri_cnt[l] = (int)pritems.size() - g->pri_off[l];
        }
        CK(cudaMalloc(&g->d_prmain, sizeof(int) * std::max<size_t>(prmain.size(), 1)));
        if (!prmain.empty()) CK(cudaMemcpy(g->d_prmain, prmain.data(), sizeof(int) * prmain.size(), cudaMemcpyHostToDevice));
        CK(cudaMalloc(&g->d_pritems, sizeof(int4) * std::max<size_t>(pritems.size(), 1)));
        if (!pritems.empty()) CK(cudaMemcpy(g->d_pritems, pritems.data(), sizeof(int4) * pritems.size(), cudaMemcpyHostToDevice));
        CK(cudaMalloc(&g->d_xpre, sizeof(float) * kTileCells * (size_t)n));
        CK(cudaMemset(g->d_xpre, 0, sizeof(float) * kTileCells * (size_t)n));  // GHOST tiles stay 0
    }
    const size_t nl = leaf.size() + ghost.size() + leafghost.size() + mg.size() + lapmain.size() + 1;
    CK(cudaMalloc(&g->d_lists, sizeof(int) * nl));
    std::vector<int> lists;
    lists.reserve(nl);
    lists.insert(lists.end(), leaf.begin(), leaf.end());
    lists.insert(lists.end(), ghost.begin(), ghost.end());
    lists.insert(lists.end(), leafghost.begin(), leafghost.end());
    lists.insert(lists.end(), mg.begin(), mg.end());
    lists.insert(lists.end(), lapmain.begin(), lapmain.end());
    lists.push_back(0);
    CK(cudaMemcpy(g->d_lists, lists.data(), sizeof(int) * lists.size(), cudaMemcpyHostToDevice));
    g->d_leaf = g->d_lists;
    g->d_ghost = g->d_leaf + leaf.size();
    g->d_leafghost = g->d_ghost + ghost.size();
    g->d_mg = g->d_leafghost + leafghost.size();
    g->d_lapmain = g->d_mg + mg.size();
    g->n_lapmain = (int)lapmain.size();

    // ------------------------------------------------------------------ coarse-level boxes
    // Levels handled by the shared-memory kernel, one CTA per instance: the longest prefix of
    // levels (common to all instances, at most each instance's finest level) whose padded dense
    // boxes (a level's tile bounding box in cells plus a one-cell halo) fit the kernel's
    // shared-memory budget in every instance.  Absent tiles and the halo hold x = 0, the value the
    // reference gives a missing neighbour.
    {
        struct Box { int off, sy, sz, cells; int lo[3]; };
        int lb = *std::min_element(g->inst_max_level.begin(), g->inst_max_level.end());
        lb = std::min(lb, kBottomMaxLevels - 1);
        std::vector<std::vector<Box>> boxes(K);
        std::vector<std::vector<int>> ifirst(K, std::vector<int>(num_layers, 0)), icnt(K, std::vector<int>(num_layers, 0));
        for (int i = 0; i < K; i++)
            for (const TileRun& r : runs[i]) {
                ifirst[i][level[r.global]] = r.global;
                icnt[i][level[r.global]] = r.count;
            }
        for (int i = 0; i < K && lb >= 0; i++) {
            long long acc = 0;
            int tiles = 0, fit = -1;
            for (int l = 0; l <= lb && icnt[i][l] > 0; l++) {
                int lo[3] = {INT32_MAX, INT32_MAX, INT32_MAX}, hi[3] = {INT32_MIN, INT32_MIN, INT32_MIN};
                for (int t = ifirst[i][l]; t < ifirst[i][l] + icnt[i][l]; t++)
                    for (int a = 0; a < 3; a++) {
                        lo[a] = std::min(lo[a], t5[5 * t + 1 + a]);
                        hi[a] = std::max(hi[a], t5[5 * t + 1 + a]);
                    }
                // z rows carry two unused cells after the halo: a row stride of 4 mod 8 floats puts
                // the 32 cells of one colour that a warp sweeps (8 rows x 4) in 32 different banks
                const long long ex = 8LL * (hi[0] - lo[0] + 1) + 2, ey = 8LL * (hi[1] - lo[1] + 1) + 2, ez = 8LL * (hi[2] - lo[2] + 1) + 4;
                if (ex > (1 << 15) || ey > (1 << 15) || ez > (1 << 15)) break;
                const long long c = ex * ey * ez;
                if (launch::bottom_smem_bytes(acc + c + 8, tiles + icnt[i][l]) > (size_t)launch::kBottomSmemBudget) break;
                boxes[i].push_back({(int)acc, (int)(ey * ez), (int)ez, (int)c, {lo[0], lo[1], lo[2]}});
                acc += c;
                tiles += icnt[i][l];
                fit = l;
            }
            lb = std::min(lb, fit);
        }
        g->bottom_level = lb;
        if (lb >= 0) {
            std::vector<int4> rec;
            std::vector<uint16_t> code;
            std::vector<BottomInst> bi(K);
            std::vector<int> base(n, -1);
            for (int i = 0; i < K; i++) {
                BottomInst& b = bi[i];
                std::memset(&b, 0, sizeof(b));
                b.rec_off = (int)rec.size();
                b.code_off = (int)code.size();
                // cells of levels 0..lb, padded to whole 16-byte vectors of codes
                const long long cells_i = (long long)boxes[i][lb].off + boxes[i][lb].cells;
                b.cells = (int)((cells_i + 7) & ~7LL);
                code.resize(code.size() + b.cells, 0);
                for (int l = 0; l <= lb; l++) {
                    b.first[l] = (int)rec.size() - b.rec_off;
                    b.cnt[l] = icnt[i][l];
                    b.sy[l] = boxes[i][l].sy;
                    b.sz[l] = boxes[i][l].sz;
                    for (int t = ifirst[i][l]; t < ifirst[i][l] + icnt[i][l]; t++) {
                        const Box& bx = boxes[i][l];
                        base[t] = bx.off + (8 * (t5[5 * t + 1] - bx.lo[0]) + 1) * bx.sy + (8 * (t5[5 * t + 2] - bx.lo[1]) + 1) * bx.sz +
                                  8 * (t5[5 * t + 3] - bx.lo[2]) + 1;
                        int pbase = -1;
                        if (par[t] >= 0) {
                            const int lp = level[par[t]];
                            const int oct = meta_octant(meta[t].packed);
                            pbase = base[par[t]] + (oct & 1) * 4 * boxes[i][lp].sy + ((oct >> 1) & 1) * 4 * boxes[i][lp].sz +
                                    ((oct >> 2) & 1) * 4;
                        }
                        rec.push_back(make_int4(base[t], pbase, type[t] | (level[t] << 8), t));
                        const uint32_t mgcls = fcls[t] >> 12;
                        for (int o = 0; o < kTileCells; o++) {
                            const int ijk[3] = {o >> 6, (o >> 3) & 7, o & 7};
                            uint16_t c = mmg[(size_t)t * kTileCells + o] & (kMaskFull);
                            for (int f = 0; f < 6; f++) {
                                const bool edge = (f & 1) ? ijk[f >> 1] == 7 : ijk[f >> 1] == 0;
                                if (edge && ((mgcls >> (2 * f)) & 3u) == 2u) c |= (uint16_t)(1u << (7 + f));
                            }
                            code[(size_t)b.code_off + base[t] + ijk[0] * bx.sy + ijk[1] * bx.sz + ijk[2]] = c;
                        }
                    }
                }
                b.nrec = (int)rec.size() - b.rec_off;
                g->bottom_smem = std::max(g->bottom_smem, launch::bottom_smem_bytes(b.cells, b.nrec));
            }
            CK((cudaError_t)(upload(&g->d_bottom_tiles, rec) ? cudaErrorMemoryAllocation : cudaSuccess));
            CK((cudaError_t)(upload(&g->d_bottom_code, code) ? cudaErrorMemoryAllocation : cudaSuccess));
            CK((cudaError_t)(upload(&g->d_bottom_inst, bi) ? cudaErrorMemoryAllocation : cudaSuccess));
        }
        launch::init_kernel_attributes();
        launch::init_stencil_attributes();
        g->shapes.assign((size_t)KS_COUNT * num_layers, kDefaultShape);
        init_tile_map_cache(*g);
        CK(cudaMalloc(&g->d_err, sizeof(unsigned int)));
        CK(cudaMemset(g->d_err, 0, sizeof(unsigned int)));
        CK(cudaMallocHost(&g->h_err, sizeof(unsigned int)));
        *g->h_err = 0;
    }

    // ------------------------------------------------------------------ per-instance reductions
    {
        std::vector<int4> chunks;
        std::vector<int2> ich(K);
        long long vbeg = 0;
        for (int i = 0; i < K; i++) {
            const long long nv = (long long)inst_leaves[i] * 128;
            const int nch = (int)std::max(1LL, (nv + kChunkVecs - 1) / kChunkVecs);
            ich[i] = make_int2((int)chunks.size(), nch);
            for (int c = 0; c < nch; c++) {
                const long long b = vbeg + (long long)c * kChunkVecs;
                chunks.push_back(make_int4(i, (int)b, (int)std::min(vbeg + nv, b + kChunkVecs), 0));
            }
            vbeg += nv;
        }
        g->n_chunks = (int)chunks.size();
        CK((cudaError_t)(upload(&g->d_chunks, chunks) ? cudaErrorMemoryAllocation : cudaSuccess));
        CK((cudaError_t)(upload(&g->d_inst_chunks, ich) ? cudaErrorMemoryAllocation : cudaSuccess));
    }
    // LEAF slots (with the GHOST-children mark), per-instance LEAF ranges, bottom-level LEAF tiles
    {
        std::vector<int> slot(n, -1), bl, gp;
        for (size_t q = 0; q < leaf.size(); q++) {
            const int t = leaf[q];
            bool kids = false;
            for (int o = 0; o < 8; o++) {
                const int c = ch8[(size_t)t * 8 + o];
                kids = kids || (c >= 0 && (type[c] & GHOST_T));
            }
            slot[t] = kids ? -2 - (int)q : (int)q;
            if (kids) gp.push_back(t);
            if (level[t] <= g->bottom_level) bl.push_back(t);
        }
        std::vector<int2> lr(K);
        int first = 0;
        for (int i = 0; i < K; i++) {
            lr[i] = make_int2(first, inst_leaves[i]);
            first += inst_leaves[i];
        }
        CK((cudaError_t)(upload(&g->d_leafslot, slot) ? cudaErrorMemoryAllocation : cudaSuccess));
        CK((cudaError_t)(upload(&g->d_inst_leafrange, lr) ? cudaErrorMemoryAllocation : cudaSuccess));
        g->n_bottom_leaves = (int)bl.size();
        bl.push_back(0);
        CK((cudaError_t)(upload(&g->d_bottom_leaves, bl) ? cudaErrorMemoryAllocation : cudaSuccess));
        g->n_gpar_leaves = (int)gp.size();
        gp.push_back(0);
        CK((cudaError_t)(upload(&g->d_gpar_leaves, gp) ? cudaErrorMemoryAllocation : cudaSuccess));
        CK(cudaMalloc(&g->d_wpart, sizeof(double) * std::max<size_t>(leaf.size(), 1)));
    }
    CK(cudaMalloc(&g->d_partials, sizeof(double) * 2 * std::max(g->red_blocks, g->n_chunks)));
    CK(cudaMalloc(&g->d_counter, sizeof(unsigned int) * 4));
    CK(cudaMemset(g->d_counter, 0, sizeof(unsigned int) * 4));
    CK(cudaMalloc(&g->d_counters, sizeof(unsigned int) * K));
    CK(cudaMemset(g->d_counters, 0, sizeof(unsigned int) * K));
    CK(cudaMalloc(&g->d_scalars, sizeof(Scalars) * K));
    CK(cudaMemset(g->d_scalars, 0, sizeof(Scalars) * K));
    CK(cudaMallocHost(&g->h_scalars, sizeof(Scalars) * K));
    std::memset(g->h_scalars, 0, sizeof(Scalars) * K);
    CK(cudaMalloc(&g->d_dot, sizeof(Scalars)));
    CK(cudaMemset(g->d_dot, 0, sizeof(Scalars)));
    CK(cudaMalloc(&g->d_iparams, sizeof(InstParams) * K));
    CK(cudaMemset(g->d_iparams, 0, sizeof(InstParams) * K));
    CK(cudaMallocHost(&g->h_iparams, sizeof(InstParams) * K));
    std::memset(g->h_iparams, 0, sizeof(InstParams) * K);
    CK(cudaMalloc(&g->d_active, sizeof(int)));
    CK(cudaMemset(g->d_active, 0, sizeof(int)));
    g->history_cap = 4096;
    CK(cudaMalloc(&g->d_history, sizeof(double) * g->history_cap));
    CK(cudaMalloc(&g->d_norm, sizeof(double) * (K + 4)));

    g->topo.ctype = g->d_u8;
    g->topo.mask_lap = g->d_u8 + cells;
    g->topo.mask_mg = g->d_u8 + 2 * cells;
    g->topo.meta = g->d_meta;
    g->topo.fcls = g->d_fcls;
    g->topo.edge = g->d_edge;
    g->topo.ghost_slot = g->d_ghost_tables;
    g->topo.ghost_faces = g->d_ghost_faces;
    g->topo.ghost_child = g->d_ghost_tables + n;
    g->topo.ghost_list = g->d_ghost;
    g->topo.inst = g->d_inst;
    g->topo.inst_h0 = g->d_inst_h0;
    g->topo.lconst = g->d_lconst;
    g->topo.leafslot = g->d_leafslot;
    g->bytes = cells * kNumChannels * sizeof(float) + cells * 3 + sizeof(TileMeta) * n + sizeof(uint32_t) * n + sizeof(int) * nl +
               sizeof(int) * 22 * (size_t)n + cells * sizeof(float) +
               sizeof(int) * ((size_t)n + g->n_bottom_leaves + g->n_gpar_leaves) + sizeof(double) * leaf.size();
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
    cudaFree(g->d_inst);
    cudaFree(g->d_inst_h0);
    cudaFree(g->d_lconst);
    cudaFree(g->d_ghost_tables);
    cudaFree(g->d_gacc);
    cudaFree(g->d_lapitems);
    cudaFree(g->d_ghost_faces);
    cudaFree(g->d_rrmain);
    cudaFree(g->d_rritems);
    cudaFree(g->d_prmain);
    cudaFree(g->d_pritems);
    cudaFree(g->d_xpre);
    cudaFree(g->d_bottom_tiles);
    cudaFree(g->d_bottom_code);
    cudaFree(g->d_bottom_inst);
    cudaFree(g->d_tile_ptrs);
    cudaFree(g->d_ct_gather);
    cudaFree(g->d_err);
    if (g->h_err) cudaFreeHost(g->h_err);
    if (g->side_stream) cudaStreamDestroy(g->side_stream);
    if (g->side_join) cudaEventDestroy(g->side_join);
    free_tile_map_cache(*g);
    cudaFree(g->d_ct_flag);
    cudaFree(g->d_lists);
    cudaFree(g->d_leafslot);
    cudaFree(g->d_wpart);
    cudaFree(g->d_inst_leafrange);
    cudaFree(g->d_bottom_leaves);
    cudaFree(g->d_gpar_leaves);
    cudaFree(g->d_chunks);
    cudaFree(g->d_inst_chunks);
    cudaFree(g->d_partials);
    cudaFree(g->d_counter);
    cudaFree(g->d_counters);
    cudaFree(g->d_scalars);
    if (g->h_scalars) cudaFreeHost(g->h_scalars);
    cudaFree(g->d_dot);
    cudaFree(g->d_iparams);
    if (g->h_iparams) cudaFreeHost(g->h_iparams);
    cudaFree(g->d_active);
    cudaFree(g->d_history);
    cudaFree(g->d_x64);
    cudaFree(g->d_ax64);
    cudaFree(g->d_r64);
    cudaFree(g->d_norm);
    cudaFree(g->d_msum);
    cudaFree(g->d_dofd);
    cudaFree(g->d_bsave);
    cudaFree(g->d_amg);
    cudaFree(g->d_amg_ct);
    cudaFree(g->d_amg_l0);
    delete g;
}

}  // namespace cirrus
