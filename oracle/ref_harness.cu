// Harness around the reference's own CUDA implementation of the Poisson path.
// TEST INFRASTRUCTURE ONLY: it is compiled together with the reference's unmodified sources
// (src/GMGSolver.cu, src/PoissonSolver.cu, src/PoissonGrid.cu, src/HAGrid.cu,
// common/Common.cpp) by oracle/build_ref.sh into oracle/_ref/libcirrus_ref.so, and is loaded
// only by tests/, the fixture generator in tests/golden/ and bench.py's reference arm.  The
// library contains nothing of this project's solver and links none of its libraries; the
// product's drop-in header is exercised on these grids by oracle/ref_dropin_harness.cu, a
// separate library that only tests load.
//
// It drives the reference through its public functions exactly as FluidEuler does
// (src/FluidEuler.h:413-447 grid construction, :464 IterativeRefine, :581-612 project), with
// a level-target lambda that reads dense per-level refinement masks.  The one piece restated
// here is ClearAllNeumannNeighborFaces (src/FluidEuler.cu:43-60), because FluidEuler.cu needs
// libraries absent from this image; it calls the reference's IterateFaceNeighborCellTypes.

#include "GMGSolver.h"
#include "PoissonSolver.h"

#include <chrono>
#include <cstddef>
#include <cstdio>
#include <map>
#include <memory>

// Non-static free functions of src/GMGSolver.cu that its header does not declare.
void GaussSeidelGMG(int iters, int order, HADeviceGrid<Tile>& grid, int level, int x_channel, int rhs_channel);
void ResidualAndRestrict(HADeviceGrid<Tile>& grid, int fine_x_channel, int fine_rhs_channel, int coarse_residual_channel,
                         int level, uint8_t launch_tile_types, T one_over_alpha);
void NegativeLaplacianAndGaussSeidelSameLevel128(HADeviceGrid<Tile>& grid, thrust::device_vector<HATileInfo<Tile>>& tiles,
                                                 int launch_tile_num, int subtree_level, uint8_t launch_tile_types,
                                                 int x_channel, int rhs_channel, int color);

namespace {

struct RefGrid {
    std::unique_ptr<HADeviceGrid<Tile>> g;
    std::unique_ptr<GMGSolver> solver;
};

__global__ void GatherChannelKernel(HATileInfo<Tile>* tiles, int c, float* out) {
    const HATileInfo<Tile>& info = tiles[blockIdx.x];
    for (int v = threadIdx.x; v < 512; v += blockDim.x) out[(size_t)blockIdx.x * 512 + v] = info.tile().mData[c][v];
}
__global__ void ScatterChannelKernel(HATileInfo<Tile>* tiles, int c, const float* in) {
    const HATileInfo<Tile>& info = tiles[blockIdx.x];
    for (int v = threadIdx.x; v < 512; v += blockDim.x) info.tile().mData[c][v] = in[(size_t)blockIdx.x * 512 + v];
}
__global__ void GatherTypesKernel(HATileInfo<Tile>* tiles, uint8_t* out) {
    const HATileInfo<Tile>& info = tiles[blockIdx.x];
    for (int v = threadIdx.x; v < 512; v += blockDim.x) out[(size_t)blockIdx.x * 512 + v] = info.tile().mCellType[v];
}
__global__ void ScatterTypesKernel(HATileInfo<Tile>* tiles, const uint8_t* in) {
    const HATileInfo<Tile>& info = tiles[blockIdx.x];
    for (int v = threadIdx.x; v < 512; v += blockDim.x) info.tile().mCellType[v] = in[(size_t)blockIdx.x * 512 + v];
}

}  // namespace

extern "C" {

int ref_device_ok() {
    int n = 0;
    return cudaGetDeviceCount(&n) == cudaSuccess && n > 0 ? 1 : 0;
}

void* ref_create(int num_layers, const uint32_t* log2hash, double h0) {
    thrust::host_vector<uint32_t> l2(log2hash, log2hash + num_layers);
    RefGrid* r = new RefGrid();
    r->g = std::make_unique<HADeviceGrid<Tile>>((T)h0, l2);
    return r;
}
void ref_destroy(void* h) {
    RefGrid* r = (RefGrid*)h;
    r->solver.reset();
    r->g.reset();
    delete r;
}
void ref_set_tile(void* h, int level, int x, int y, int z, int type) {
    ((RefGrid*)h)->g->setTileHost(level, nanovdb::Coord(x, y, z), Tile(), (uint8_t)type);
}
// src/FluidEuler.h:445-447
void ref_compress_sync_spawn(void* h) {
    auto& grid = *((RefGrid*)h)->g;
    grid.compressHost(false);
    grid.syncHostAndDevice();
    SpawnGhostTiles(grid, false);
}
// Dense per-level masks on the device, for level-target lambdas.
struct DeviceMasks {
    std::vector<thrust::device_vector<uint8_t>> dm;
    thrust::device_vector<const uint8_t*> dptr;
    thrust::device_vector<int> ddims;
    DeviceMasks(const uint8_t* const* masks, const int* dims, int num_levels) : dm(num_levels) {
        thrust::host_vector<const uint8_t*> hp(num_levels, nullptr);
        thrust::host_vector<int> hd(3 * num_levels, 0);
        for (int l = 0; l < num_levels; l++) {
            hd[3 * l] = dims[3 * l]; hd[3 * l + 1] = dims[3 * l + 1]; hd[3 * l + 2] = dims[3 * l + 2];
            size_t n = (size_t)dims[3 * l] * dims[3 * l + 1] * dims[3 * l + 2];
            if (masks[l] && n > 0) {
                dm[l] = thrust::device_vector<uint8_t>(masks[l], masks[l] + n);
                hp[l] = thrust::raw_pointer_cast(dm[l].data());
            }
        }
        dptr = hp;
        ddims = hd;
    }
    const uint8_t* const* ptrs() const { return thrust::raw_pointer_cast(dptr.data()); }
    const int* dims() const { return thrust::raw_pointer_cast(ddims.data()); }
};
__host__ __device__ inline bool mask_hit(const uint8_t* const* mp, const int* dp, int nl, int l, int x, int y, int z) {
    if (l >= nl || mp[l] == nullptr) return false;
    if (x < 0 || y < 0 || z < 0 || x >= dp[3 * l] || y >= dp[3 * l + 1] || z >= dp[3 * l + 2]) return false;
    return mp[l][((size_t)x * dp[3 * l + 1] + y) * dp[3 * l + 2] + z] != 0;
}

// IterativeRefine with level_target(tile) = level + mask[level][tile], masks dense per level.
void ref_iterative_refine(void* h, const uint8_t* const* masks, const int* dims, int num_levels) {
    auto& grid = *((RefGrid*)h)->g;
    DeviceMasks m(masks, dims, num_levels);
    const uint8_t* const* mp = m.ptrs();
    const int* dp = m.dims();
    int nl = num_levels;
    auto level_target = [mp, dp, nl] __device__(const HATileAccessor<Tile>& acc, HATileInfo<Tile>& info) -> int {
        int l = info.mLevel;
        return mask_hit(mp, dp, nl, l, info.mTileCoord[0], info.mTileCoord[1], info.mTileCoord[2]) ? l + 1 : l;
    };
    IterativeRefine(grid, level_target, false);
    cudaDeviceSynchronize();
}
// RefineLeafsOneStep alone (no ghost spawning), the same level targets; refined tiles per level.
void ref_refine_one_step(void* h, const uint8_t* const* masks, const int* dims, int num_levels, int* counts) {
    auto& grid = *((RefGrid*)h)->g;
    DeviceMasks m(masks, dims, num_levels);
    const uint8_t* const* mp = m.ptrs();
    const int* dp = m.dims();
    int nl = num_levels;
    auto level_target = [mp, dp, nl] __device__(const HATileAccessor<Tile>& acc, HATileInfo<Tile>& info) -> int {
        int l = info.mLevel;
        return mask_hit(mp, dp, nl, l, info.mTileCoord[0], info.mTileCoord[1], info.mTileCoord[2]) ? l + 1 : l;
    };
    auto c = RefineLeafsOneStep(grid, level_target, false);
    cudaDeviceSynchronize();
    for (size_t i = 0; i < c.size(); i++) counts[i] = c[i];
}
void ref_spawn_ghosts(void* h) {
    SpawnGhostTiles(*((RefGrid*)h)->g, false);
    cudaDeviceSynchronize();
}
// CoarsenStep (src/PoissonGrid.h:164-314) with level_target(tile) = level - mask[level][tile];
// deleted tiles per level.
void ref_coarsen_step(void* h, const uint8_t* const* masks, const int* dims, int num_levels, int* deleted) {
    auto& grid = *((RefGrid*)h)->g;
    DeviceMasks m(masks, dims, num_levels);
    const uint8_t* const* mp = m.ptrs();
    const int* dp = m.dims();
    int nl = num_levels;
    auto level_target = [mp, dp, nl] __device__(const HATileAccessor<Tile>& acc, HATileInfo<Tile>& info) -> int {
        int l = info.mLevel;
        return mask_hit(mp, dp, nl, l, info.mTileCoord[0], info.mTileCoord[1], info.mTileCoord[2]) ? l - 1 : l;
    };
    auto c = CoarsenStep(grid, level_target, false);
    cudaDeviceSynchronize();
    for (size_t i = 0; i < c.size(); i++) deleted[i] = c[i];
}
// mStatus of every tile, all-tiles order
void ref_statuses(void* h, int* out) {
    auto& grid = *((RefGrid*)h)->g;
    for (size_t i = 0; i < grid.hAllTiles.size(); i++) {
        int st = 0;
        cudaMemcpy(&st, (const char*)grid.hAllTiles[i].mTilePtr + offsetof(Tile, mStatus), sizeof(int), cudaMemcpyDeviceToHost);
        out[i] = st;
    }
}
// The reference grid object itself (HADeviceGrid<Tile>*), for harnesses that run other code on it.
void* ref_grid(void* h) { return ((RefGrid*)h)->g.get(); }
int ref_num_tiles(void* h) { return (int)((RefGrid*)h)->g->hAllTiles.size(); }
int ref_max_level(void* h) { return ((RefGrid*)h)->g->mMaxLevel; }
void ref_tiles(void* h, int* out) {
    auto& grid = *((RefGrid*)h)->g;
    for (size_t i = 0; i < grid.hAllTiles.size(); i++) {
        const auto& o = grid.hAllTiles[i];
        out[5 * i] = o.mLevel; out[5 * i + 1] = o.mTileCoord[0]; out[5 * i + 2] = o.mTileCoord[1];
        out[5 * i + 3] = o.mTileCoord[2]; out[5 * i + 4] = o.mType;
    }
}
void ref_slots(void* h, int* out) {
    auto& grid = *((RefGrid*)h)->g;
    auto acc = grid.hostAccessor();
    for (size_t i = 0; i < grid.hAllTiles.size(); i++) {
        const auto& o = grid.hAllTiles[i];
        out[i] = (int)acc.tileIdx(o.mLevel, o.mTileCoord);
    }
}
void ref_set_ctypes(void* h, const uint8_t* ct) {
    auto& grid = *((RefGrid*)h)->g;
    size_t n = grid.dAllTiles.size();
    thrust::device_vector<uint8_t> d(ct, ct + n * 512);
    ScatterTypesKernel<<<n, 128>>>(thrust::raw_pointer_cast(grid.dAllTiles.data()), thrust::raw_pointer_cast(d.data()));
    cudaDeviceSynchronize();
}
void ref_get_ctypes(void* h, uint8_t* ct) {
    auto& grid = *((RefGrid*)h)->g;
    size_t n = grid.dAllTiles.size();
    thrust::device_vector<uint8_t> d(n * 512);
    GatherTypesKernel<<<n, 128>>>(thrust::raw_pointer_cast(grid.dAllTiles.data()), thrust::raw_pointer_cast(d.data()));
    thrust::copy(d.begin(), d.end(), ct);
}
void ref_calc_cell_types(void* h) { CalcCellTypesFromLeafs(*((RefGrid*)h)->g); cudaDeviceSynchronize(); }
void ref_calc_neighbors(void* h) { CalculateNeighborTiles(*((RefGrid*)h)->g); cudaDeviceSynchronize(); }
// neighbour table read back from each tile's mNeighbors, as indices into the all-tiles order
void ref_neighbors(void* h, int* out) {
    auto& grid = *((RefGrid*)h)->g;
    std::map<const Tile*, int> idx;
    for (size_t i = 0; i < grid.hAllTiles.size(); i++) idx[grid.hAllTiles[i].mTilePtr] = (int)i;
    for (size_t i = 0; i < grid.hAllTiles.size(); i++) {
        HATileInfo<Tile> nb[6];
        cudaMemcpy(nb, (const char*)grid.hAllTiles[i].mTilePtr + offsetof(Tile, mNeighbors), sizeof(nb), cudaMemcpyDeviceToHost);
        for (int f = 0; f < 6; f++) {
            auto it = idx.find(nb[f].mTilePtr);
            out[6 * i + f] = (nb[f].mTilePtr == nullptr || it == idx.end()) ? -1 : it->second;
        }
    }
}
void ref_set_channel(void* h, int c, const float* data) {
    auto& grid = *((RefGrid*)h)->g;
    size_t n = grid.dAllTiles.size();
    thrust::device_vector<float> d(data, data + n * 512);
    ScatterChannelKernel<<<n, 128>>>(thrust::raw_pointer_cast(grid.dAllTiles.data()), c, thrust::raw_pointer_cast(d.data()));
    cudaDeviceSynchronize();
}
void ref_get_channel(void* h, int c, float* data) {
    auto& grid = *((RefGrid*)h)->g;
    size_t n = grid.dAllTiles.size();
    thrust::device_vector<float> d(n * 512);
    GatherChannelKernel<<<n, 128>>>(thrust::raw_pointer_cast(grid.dAllTiles.data()), c, thrust::raw_pointer_cast(d.data()));
    thrust::copy(d.begin(), d.end(), data);
}
// RHS exactly as FluidEuler::project builds it (src/FluidEuler.h:583-586), after the
// velocity boundary step's face clearing (src/FluidEuler.cu:43-60).
void ref_rhs(void* h) {
    auto& grid = *((RefGrid*)h)->g;
    grid.launchVoxelFunc(
        [=] __device__(HATileAccessor<Tile>& acc, HATileInfo<Tile>& info, const Coord& l_ijk) {
            for (int axis : {0, 1, 2}) {
                bool to_set = false;
                IterateFaceNeighborCellTypes(acc, info, l_ijk, axis, [&](const uint8_t type0, const uint8_t type1) {
                    if ((type0 & NEUMANN) || (type1 & NEUMANN) || ((type0 & DIRICHLET) && (type1 & DIRICHLET))) to_set = true;
                });
                if (to_set) info.tile()(Tile::u_channel + axis, l_ijk) = 0;
            }
        },
        -1, LEAF, LAUNCH_SUBTREE);
    for (int axis : {0, 1, 2})
        PropagateToChildren(grid, Tile::u_channel + axis, Tile::u_channel + axis, -1, GHOST, LAUNCH_SUBTREE, INTERIOR | DIRICHLET | NEUMANN);
    VelocityVolumeDivergenceOnLeafs(grid, Tile::u_channel, Tile::b_channel);
    cudaDeviceSynchronize();
}
void ref_add_gradient(void* h, int pc, int uc) {
    AddGradientToFaceCenters(*((RefGrid*)h)->g, pc, uc);
    cudaDeviceSynchronize();
}
void ref_full_lap(void* h, int xc, int yc) {
    FullNegativeLaplacian(*((RefGrid*)h)->g, xc, yc, false);
    cudaDeviceSynchronize();
}
void ref_full_lap_ex(void* h, int xc, int yc, int calc_diag) {
    FullNegativeLaplacian(*((RefGrid*)h)->g, xc, yc, calc_diag != 0);
    cudaDeviceSynchronize();
}
// NegativeLaplacianSameLevel128 on grid.dAllTiles (tile_level -1) or grid.dTileArrays[tile_level]
void ref_lap_same_level(void* h, int tile_level, int subtree_level, int types, int xc, int yc, int calc_diag) {
    auto& grid = *((RefGrid*)h)->g;
    if (tile_level < 0)
        NegativeLaplacianSameLevel128(grid, grid.dAllTiles, grid.dAllTiles.size(), subtree_level, (uint8_t)types, xc, yc, calc_diag != 0);
    else
        NegativeLaplacianSameLevel128(grid, grid.dTileArrays[tile_level], grid.hNumTiles[tile_level], subtree_level, (uint8_t)types, xc,
                                      yc, calc_diag != 0);
    cudaDeviceSynchronize();
}
void ref_gs_sweep(void* h, int level, int xc, int rc, int color) {
    auto& grid = *((RefGrid*)h)->g;
    NegativeLaplacianAndGaussSeidelSameLevel128(grid, grid.dTileArrays[level], grid.hNumTiles[level], level, LEAF | NONLEAF, xc, rc, color);
    cudaDeviceSynchronize();
}
void ref_residual_restrict(void* h, int level, int xc, int rhsc, int coarsec) {
    ResidualAndRestrict(*((RefGrid*)h)->g, xc, rhsc, coarsec, level, LEAF | NONLEAF | GHOST, (T)1);
    cudaDeviceSynchronize();
}
void ref_prolongate(void* h, int level, int cxc, int fxc) {
    ProlongateAndUpdate128(*((RefGrid*)h)->g, cxc, fxc, level, (T)1);
    cudaDeviceSynchronize();
}
void ref_vcycle(void* h, int xc, int fc, int rhsc, int level_iters, int coarsest_iters) {
    RefGrid* r = (RefGrid*)h;
    if (!r->solver) r->solver = std::make_unique<GMGSolver>(1., 1.);
    r->solver->VCycle(*r->g, xc, fc, rhsc, level_iters, coarsest_iters);
    cudaDeviceSynchronize();
}
double ref_dot(void* h, int a, int b) { return Dot(*((RefGrid*)h)->g, a, b, LEAF); }
// GMGSolver::solve as FluidEuler::project calls it; returns iterations, writes the relative
// residual and the wall time of the call bracketed by device synchronisation (ms).
int ref_solve(void* h, int max_iters, double tol, int level_iters, int coarsest_iters, int sync_stride, int pure_neumann,
              double* rel, double* ms) {
    RefGrid* r = (RefGrid*)h;
    if (!r->solver) r->solver = std::make_unique<GMGSolver>(1., 1.);
    cudaDeviceSynchronize();
    auto t0 = std::chrono::high_resolution_clock::now();
    auto [iters, err] = r->solver->solve(*r->g, false, max_iters, tol, level_iters, coarsest_iters, sync_stride, pure_neumann != 0);
    cudaDeviceSynchronize();
    auto t1 = std::chrono::high_resolution_clock::now();
    if (rel) *rel = err;
    if (ms) *ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    return iters;
}
// GMGSolver::dampedJacobiSolve (src/GMGSolver.cu:449-531)
int ref_damped_jacobi(void* h, int max_iters, double tol, float omega, double* rel) {
    RefGrid* r = (RefGrid*)h;
    if (!r->solver) r->solver = std::make_unique<GMGSolver>(1., 1.);
    auto [iters, err] = r->solver->dampedJacobiSolve(*r->g, false, max_iters, tol, omega);
    cudaDeviceSynchronize();
    if (rel) *rel = err;
    return iters;
}
int ref_last_error() { return (int)cudaGetLastError(); }

// Layout of the reference's PoissonTile<float> and HATileInfo as this compiler lays them out --
// what a tile-holder file's records are: sizeof(Tile), offsets of mData, mNeighbors, mCellType,
// mIsInterestArea, mIsLockedRefine, mStatus, mSerialIdx, sizeof(HATileInfo), sizeof(T), CHNLSIZE.
void ref_tile_layout(long long* out) {
    out[0] = (long long)sizeof(Tile);
    out[1] = (long long)offsetof(Tile, mData);
    out[2] = (long long)offsetof(Tile, mNeighbors);
    out[3] = (long long)offsetof(Tile, mCellType);
    out[4] = (long long)offsetof(Tile, mIsInterestArea);
    out[5] = (long long)offsetof(Tile, mIsLockedRefine);
    out[6] = (long long)offsetof(Tile, mStatus);
    out[7] = (long long)offsetof(Tile, mSerialIdx);
    out[8] = (long long)sizeof(HATileInfo<Tile>);
    out[9] = (long long)sizeof(T);
    out[10] = (long long)Tile::CHNLSIZE;
}

// The tile-holder writer and reader (IOFunc::WriteHAHostTileHolderToFile /
// ReadHAHostTileHolderFromFile, src/PoissonIOFunc.cu:38-121), restated here because
// PoissonIOFunc.cu needs libraries absent from this image.  They run on the reference's own
// HAHostTileHolder, filled by getHostTileHolder (src/HAGrid.h:433-462) and consumed by
// setTilesFromHolder (src/HAGrid.h:316-331): header fields, the raw tile records, then per level
// the infos with each tile's record index.
int ref_write_holder(void* h, int tile_types, const char* path) {
    auto& grid = *((RefGrid*)h)->g;
    auto holder = grid.getHostTileHolder((uint8_t)tile_types);
    std::FILE* f = std::fopen(path, "wb");
    if (!f) return 1;
    std::fwrite(&holder->mH0, sizeof(holder->mH0), 1, f);
    std::fwrite(&holder->mNumLayers, sizeof(holder->mNumLayers), 1, f);
    std::fwrite(&holder->mMaxLevel, sizeof(holder->mMaxLevel), 1, f);
    const size_t ntiles = holder->mHostTiles.size();
    std::fwrite(&ntiles, sizeof(ntiles), 1, f);
    if (ntiles) std::fwrite(holder->mHostTiles.data(), sizeof(Tile), ntiles, f);
    const size_t nlev = holder->mHostLevels.size();
    std::fwrite(&nlev, sizeof(nlev), 1, f);
    for (const auto& lv : holder->mHostLevels) {
        const size_t cnt = lv.size();
        std::fwrite(&cnt, sizeof(cnt), 1, f);
        for (const auto& info : lv) {
            std::fwrite(&info.mTileCoord, sizeof(info.mTileCoord), 1, f);
            std::fwrite(&info.mLevel, sizeof(info.mLevel), 1, f);
            std::fwrite(&info.mType, sizeof(info.mType), 1, f);
            const intptr_t idx = info.mTilePtr ? (intptr_t)(info.mTilePtr - holder->mHostTiles.data()) : (intptr_t)-1;
            std::fwrite(&idx, sizeof(idx), 1, f);
        }
    }
    return std::fclose(f) == 0 ? 0 : 1;
}
// A new reference grid (hash sizes log2hash) filled from a holder file: read, setTilesFromHolder,
// compressHost, syncHostAndDevice.  NULL if the file cannot be read.
void* ref_read_holder(const char* path, int num_layers, const uint32_t* log2hash) {
    std::FILE* f = std::fopen(path, "rb");
    if (!f) return nullptr;
    HAHostTileHolder<Tile> holder;
    bool ok = std::fread(&holder.mH0, sizeof(holder.mH0), 1, f) == 1 && std::fread(&holder.mNumLayers, sizeof(holder.mNumLayers), 1, f) == 1 &&
              std::fread(&holder.mMaxLevel, sizeof(holder.mMaxLevel), 1, f) == 1;
    size_t ntiles = 0, nlev = 0;
    ok = ok && std::fread(&ntiles, sizeof(ntiles), 1, f) == 1;
    if (ok) {
        holder.mHostTiles.resize(ntiles);
        ok = ntiles == 0 || std::fread(holder.mHostTiles.data(), sizeof(Tile), ntiles, f) == ntiles;
    }
    ok = ok && std::fread(&nlev, sizeof(nlev), 1, f) == 1;
    if (ok) holder.mHostLevels.resize(nlev);
    for (size_t l = 0; ok && l < nlev; l++) {
        size_t cnt = 0;
        ok = std::fread(&cnt, sizeof(cnt), 1, f) == 1;
        if (ok) holder.mHostLevels[l].resize(cnt);
        for (size_t i = 0; ok && i < cnt; i++) {
            auto& info = holder.mHostLevels[l][i];
            intptr_t idx = -1;
            ok = std::fread(&info.mTileCoord, sizeof(info.mTileCoord), 1, f) == 1 && std::fread(&info.mLevel, sizeof(info.mLevel), 1, f) == 1 &&
                 std::fread(&info.mType, sizeof(info.mType), 1, f) == 1 && std::fread(&idx, sizeof(idx), 1, f) == 1;
            info.mTilePtr = (ok && idx >= 0 && (size_t)idx < ntiles) ? &holder.mHostTiles[idx] : nullptr;
        }
    }
    std::fclose(f);
    if (!ok || holder.mNumLayers != num_layers) return nullptr;
    thrust::host_vector<uint32_t> l2(log2hash, log2hash + num_layers);
    RefGrid* r = new RefGrid();
    r->g = std::make_unique<HADeviceGrid<Tile>>(holder.mH0, l2);
    r->g->setTilesFromHolder(holder);
    r->g->compressHost(false);
    r->g->syncHostAndDevice();
    return r;
}

}  // extern "C"
