/*
 * cirrus_gmg_dropin.hpp -- header-only drop-in for the reference's GMGSolver
 * (src/GMGSolver.h:17-52), for C++ callers that keep their grid in the reference's
 * HADeviceGrid<PoissonTile<float>> (array-of-tiles storage, one allocation per tile).
 *
 *   // FluidEuler::project (src/FluidEuler.h:591-598), unchanged except for the type:
 *   cirrus_dropin::GMGSolver<HADeviceGrid<Tile>> solver(1., 1.);
 *   auto [iters, err] = solver.solve(grid, false, 1000, 1e-6, 1, 10, 1, mIsPureNeumann);
 *
 * Same preconditions and results as the reference: b in channel 1 of LEAF tiles, x written to
 * channel 0, channel 1 left holding the final residual.  The first solve on a grid (and the first
 * after its tiles change) imports the tile list and cell types and builds the device tile pool;
 * every solve then moves channels between the reference's tiles and the pool with device
 * gather/scatter kernels (no host copies) and runs the whole PCG as one CUDA graph.
 * Template parameter Grid needs: hAllTiles (host array of infos with mTileCoord, mTilePtr,
 * mLevel, mType), hLog2Hashes, mNumLayers, mH0; its Tile needs mData[c][...] and mCellType[512].
 */
#ifndef CIRRUS_GMG_DROPIN_HPP
#define CIRRUS_GMG_DROPIN_HPP

#include "cirrus_b200.h"

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <tuple>
#include <type_traits>
#include <utility>
#include <vector>

namespace cirrus_dropin {

inline void check(cirrus_status s, const char* what) {
    if (s != CIRRUS_OK) throw std::runtime_error(std::string(what) + ": " + cirrus_status_string(s));
}

template <class Grid>
class GMGSolver {
public:
    explicit GMGSolver(float one_over_alpha = 1.f, float prolong_coeff = 1.f)
        : one_over_alpha_(one_over_alpha), prolong_coeff_(prolong_coeff) {}
    ~GMGSolver() { release(); }
    GMGSolver(const GMGSolver&) = delete;
    GMGSolver& operator=(const GMGSolver&) = delete;

    /* GMGSolver::solve (src/GMGSolver.cu:531-666): returns (iterations, relative residual). */
    std::tuple<int, double> solve(Grid& grid, bool verbose, int max_iters, double relative_tolerance, int level_iters,
                                  int coarsest_iters, int sync_stride, bool is_pure_neumann) {
        bind(grid);
        check(cirrus_grid_gather_tiles(cg_, 1, channel_offset(1), nullptr), "gather b");
        cirrus_solve_params p;
        cirrus_solve_params_default(&p);
        p.max_iters = max_iters;
        p.relative_tolerance = relative_tolerance;
        p.level_iters = level_iters;
        p.coarsest_iters = coarsest_iters;
        p.sync_stride = sync_stride;
        p.is_pure_neumann = is_pure_neumann ? 1 : 0;
        p.one_over_alpha = one_over_alpha_;
        p.prolong_coeff = prolong_coeff_;
        cirrus_solve_result r;
        check(cirrus_gmg_solve(cg_, &p, nullptr, &r), "cirrus_gmg_solve");
        check(cirrus_grid_scatter_tiles(cg_, 0, channel_offset(0), nullptr), "scatter x");
        check(cirrus_grid_scatter_tiles(cg_, 1, channel_offset(1), nullptr), "scatter r");
        if (cudaDeviceSynchronize() != cudaSuccess) throw std::runtime_error("cirrus_dropin: CUDA error");
        if (verbose) std::printf("cirrus GMG-PCG: %d iterations, relative residual %.3e\n", r.iters, r.rel_residual);
        return std::make_tuple(r.iters, sync_stride > 0 ? r.rel_residual : -1.0);
    }

    /* GMGSolver::dampedJacobiSolve (src/GMGSolver.cu:449-531): b in channel 1, x to channel 0,
     * the last residual in channel 2 and the diagonal in channel 3 of LEAF|GHOST tiles (both
     * channels keep their previous contents on NONLEAF tiles, as in the reference). */
    std::tuple<int, double> dampedJacobiSolve(Grid& grid, bool verbose, int max_iters, double relative_tolerance, float omega) {
        bind(grid);
        for (int c : {1, 2, 3}) check(cirrus_grid_gather_tiles(cg_, c, channel_offset(c), nullptr), "gather");
        int iters = 0;
        double rel = 0.0;
        check(cirrus_damped_jacobi_solve(cg_, max_iters, relative_tolerance, omega, nullptr, &iters, &rel), "cirrus_damped_jacobi_solve");
        for (int c : {0, 2, 3}) check(cirrus_grid_scatter_tiles(cg_, c, channel_offset(c), nullptr), "scatter");
        if (cudaDeviceSynchronize() != cudaSuccess) throw std::runtime_error("cirrus_dropin: CUDA error");
        if (verbose) std::printf("cirrus damped Jacobi: %d iterations, relative residual %.3e\n", iters, rel);
        return std::make_tuple(iters, rel);
    }

private:
    using Info = typename std::decay<decltype(std::declval<Grid&>().hAllTiles[0])>::type;
    using Tile = typename std::decay<decltype(*std::declval<Info&>().mTilePtr)>::type;

    static size_t channel_offset(int c) {
        static const size_t base = [] {
            static Tile probe;
            return (size_t)((const char*)&probe.mData[0][0] - (const char*)&probe);
        }();
        return base + (size_t)c * sizeof(((Tile*)nullptr)->mData[0]);
    }
    static size_t types_offset() {
        static Tile probe;
        return (size_t)((const char*)&probe.mCellType[0] - (const char*)&probe);
    }

    void release() {
        if (cg_) cirrus_grid_destroy(cg_);
        if (topo_) cirrus_topology_destroy(topo_);
        cg_ = nullptr;
        topo_ = nullptr;
        ptrs_.clear();
        types_.clear();
    }

    void bind(Grid& grid) {
        const size_t n = grid.hAllTiles.size();
        std::vector<const void*> ptrs(n);
        std::vector<uint8_t> types(n);
        for (size_t i = 0; i < n; i++) {
            ptrs[i] = grid.hAllTiles[i].mTilePtr;
            types[i] = grid.hAllTiles[i].mType;
        }
        if (cg_ && ptrs == ptrs_ && types == types_) return;  // same tiles: reuse the pool
        release();
        std::vector<uint32_t> log2(grid.hLog2Hashes.begin(), grid.hLog2Hashes.end());
        check(cirrus_topology_create((int)grid.mNumLayers, log2.data(), (double)grid.mH0, &topo_), "topology");
        std::vector<int32_t> t5(5 * n);
        for (size_t i = 0; i < n; i++) {
            const auto& info = grid.hAllTiles[i];
            t5[5 * i] = info.mLevel;
            t5[5 * i + 1] = info.mTileCoord[0];
            t5[5 * i + 2] = info.mTileCoord[1];
            t5[5 * i + 3] = info.mTileCoord[2];
            t5[5 * i + 4] = info.mType;
        }
        check(cirrus_topology_import_tiles(topo_, t5.data(), (int)n), "import tiles");
        std::vector<uint8_t> ct(512 * n);
        for (size_t i = 0; i < n; i++)
            if (cudaMemcpy(ct.data() + 512 * i, (const char*)ptrs[i] + types_offset(), 512, cudaMemcpyDeviceToHost) != cudaSuccess)
                throw std::runtime_error("cirrus_dropin: reading cell types");
        check(cirrus_topology_set_cell_types(topo_, ct.data()), "cell types");
        check(cirrus_grid_create(topo_, &cg_), "grid");
        check(cirrus_grid_set_tile_pointers(cg_, ptrs.data()), "tile pointers");
        ptrs_ = std::move(ptrs);
        types_ = std::move(types);
    }

    float one_over_alpha_, prolong_coeff_;
    cirrus_topology* topo_ = nullptr;
    cirrus_grid* cg_ = nullptr;
    std::vector<const void*> ptrs_;
    std::vector<uint8_t> types_;
};

}  // namespace cirrus_dropin

#endif  // CIRRUS_GMG_DROPIN_HPP
