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
 * channel 0, channel 1 left holding the final residual.
 *
 * FluidEuler::project constructs a fresh solver object for every projection, so the device
 * state does not live in the object: a process-wide registry keeps, per grid object, the tile
 * pool built from it (topology tables, stencil masks, the captured solve graph).  A solve
 *   1. compares the grid's tile list (tile pointers, levels, coordinates, types) with the bound
 *      one and rebuilds the pool when it differs (a refined or coarsened grid);
 *   2. gathers every tile's mCellType on the device and compares it with the pool's (one kernel,
 *      1 byte per cell, and a 4-byte read-back): CalcCellTypesFromLeafs rewrites the cell types
 *      every step (src/FluidEuler.h:934) and can move NEUMANN/DIRICHLET cells without changing
 *      tiles, and the stencil masks derive from them, so a change rebuilds the pool's masks from
 *      the gathered types;
 *   3. gathers b, solves (one CUDA graph launch) and scatters x and r back, on the device.
 * A pool stays bound until release(grid) or release_all(); its memory is about 60 bytes per cell.
 * Template parameter Grid needs: hAllTiles (host array of infos with mTileCoord, mTilePtr,
 * mLevel, mType), hLog2Hashes, mNumLayers, mH0; its Tile needs mData[c][...] and mCellType[512].
 * Calls for one grid are serialised by the registry; the reference's solve is not re-entrant
 * for a grid either.
 *
 * cirrus_dropin::autotune(grid) tunes the bound pool's launch shapes once (optional).
 * cirrus_dropin::AMGSolver<Grid> (below) replaces the reference's AMGSolver on the same registry.
 */
#ifndef CIRRUS_GMG_DROPIN_HPP
#define CIRRUS_GMG_DROPIN_HPP

#include "cirrus_b200.h"

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <map>
#include <memory>
#include <mutex>
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

namespace detail {

// The device pool bound to one grid object, with the tile list it was built from.
struct Binding {
    std::vector<const void*> ptrs;
    std::vector<int32_t> tiles5;  // level, x, y, z, type per tile (all-tiles order)
    std::vector<uint8_t> ctypes;  // host staging of gathered cell types (num_tiles*512)
    int num_layers = 0;
    std::vector<uint32_t> log2;
    double h0 = 0;
    cirrus_topology* topo = nullptr;
    cirrus_grid* cg = nullptr;
    bool amg_ready = false;  // the AMG coefficients of this pool are prepared (AMGSolver)
    std::mutex mu;  // one solve at a time per grid
    ~Binding() { drop(); }
    void drop() {
        if (cg) cirrus_grid_destroy(cg);
        if (topo) cirrus_topology_destroy(topo);
        cg = nullptr;
        topo = nullptr;
        amg_ready = false;
    }
};

struct Registry {
    std::mutex mu;
    std::map<const void*, std::shared_ptr<Binding>> by_grid;
};
// Never destroyed: a static destructor would free device memory after the CUDA runtime may
// already have shut down at process exit.  release_all() frees the pools explicitly.
inline Registry& registry() {
    static Registry* r = new Registry();
    return *r;
}

}  // namespace detail

// Frees the device pool bound to `grid` (if any).  Call it before a grid object is destroyed
// when its memory matters; a later solve on the same object rebuilds the pool.
template <class Grid>
void release(const Grid& grid) {
    auto& reg = detail::registry();
    std::shared_ptr<detail::Binding> b;
    {
        std::lock_guard<std::mutex> lk(reg.mu);
        auto it = reg.by_grid.find(static_cast<const void*>(&grid));
        if (it == reg.by_grid.end()) return;
        b = it->second;
        reg.by_grid.erase(it);
    }
    std::lock_guard<std::mutex> lk(b->mu);
    b->drop();
}
// Frees every bound pool.
inline void release_all() {
    auto& reg = detail::registry();
    std::map<const void*, std::shared_ptr<detail::Binding>> all;
    {
        std::lock_guard<std::mutex> lk(reg.mu);
        all.swap(reg.by_grid);
    }
    for (auto& kv : all) {
        std::lock_guard<std::mutex> lk(kv.second->mu);
        kv.second->drop();
    }
}
// Number of grids with a bound pool.
inline int bound_grids() {
    auto& reg = detail::registry();
    std::lock_guard<std::mutex> lk(reg.mu);
    return (int)reg.by_grid.size();
}

namespace detail {
// Tile layout, registry lookup and (re)binding of a reference grid type, shared by the solver
// classes below.
template <class Grid>
struct Access {
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
        static const size_t off = [] {
            static Tile probe;
            return (size_t)((const char*)&probe.mCellType[0] - (const char*)&probe);
        }();
        return off;
    }

    static std::shared_ptr<detail::Binding> binding(Grid& grid) {
        auto& reg = detail::registry();
        std::lock_guard<std::mutex> lk(reg.mu);
        auto& slot = reg.by_grid[static_cast<const void*>(&grid)];
        if (!slot) slot = std::make_shared<detail::Binding>();
        return slot;
    }

    // Builds the topology and the device pool from the bound tile list and the cell types in
    // b.ctypes (all tiles, as the reference's CalcCellTypesFromLeafs left them).
    static void build_pool(detail::Binding& b) {
        b.drop();
        const int n = (int)b.ptrs.size();
        check(cirrus_topology_create(b.num_layers, b.log2.data(), b.h0, &b.topo), "topology");
        check(cirrus_topology_import_tiles(b.topo, b.tiles5.data(), n), "import tiles");
        check(cirrus_topology_set_cell_types(b.topo, b.ctypes.data()), "cell types");
        check(cirrus_grid_create(b.topo, &b.cg), "grid");
        check(cirrus_grid_set_tile_pointers(b.cg, b.ptrs.data()), "tile pointers");
    }

    static void bind(Grid& grid, detail::Binding& b) {
        if (grid.hAllTiles.empty()) throw std::runtime_error("cirrus_dropin: grid has no tiles");
        const size_t n = grid.hAllTiles.size();
        std::vector<const void*> ptrs(n);
        std::vector<int32_t> t5(5 * n);
        for (size_t i = 0; i < n; i++) {
            const auto& info = grid.hAllTiles[i];
            ptrs[i] = info.mTilePtr;
            t5[5 * i] = info.mLevel;
            t5[5 * i + 1] = info.mTileCoord[0];
            t5[5 * i + 2] = info.mTileCoord[1];
            t5[5 * i + 3] = info.mTileCoord[2];
            t5[5 * i + 4] = info.mType;
        }
        if (!b.cg || ptrs != b.ptrs || t5 != b.tiles5 || (int)grid.mNumLayers != b.num_layers || (double)grid.mH0 != b.h0) {
            // new or changed tile list: read the cell types (one gather kernel, one copy) and
            // build the pool from them
            b.ptrs = std::move(ptrs);
            b.tiles5 = std::move(t5);
            b.num_layers = (int)grid.mNumLayers;
            b.log2.assign(grid.hLog2Hashes.begin(), grid.hLog2Hashes.end());
            b.h0 = (double)grid.mH0;
            b.ctypes.resize(512 * n);
            check(cirrus_gather_tile_bytes(b.ptrs.data(), (int)n, types_offset(), b.ctypes.data(), nullptr), "read cell types");
            build_pool(b);
            return;
        }
        int changed = 0;
        check(cirrus_grid_compare_tile_cell_types(b.cg, types_offset(), nullptr, &changed, b.ctypes.data()), "cell types");
        if (changed) build_pool(b);
    }

};
}  // namespace detail

/* Tunes the launch shapes of the pool bound to `grid` (binding it first) on the grid's current
 * right-hand sides (channel 1 of its tiles): cirrus_grid_autotune, about 1-2 s for a
 * ring512-sized grid, for a caller whose tiles and cell types stay the same over many solves.
 * The shapes stay with the pool until its tile list or cell types change (a rebuilt pool starts
 * from the untuned shape again).  Results never change. */
template <class Grid>
void autotune(Grid& grid) {
    using A = detail::Access<Grid>;
    std::shared_ptr<detail::Binding> b = A::binding(grid);
    std::lock_guard<std::mutex> lk(b->mu);
    A::bind(grid, *b);
    check(cirrus_grid_gather_tiles(b->cg, 1, A::channel_offset(1), nullptr), "gather b");
    check(cirrus_grid_autotune(b->cg, 0, nullptr), "cirrus_grid_autotune");
    if (cudaDeviceSynchronize() != cudaSuccess) throw std::runtime_error("cirrus_dropin: CUDA error");
}

template <class Grid>
class GMGSolver {
public:
    explicit GMGSolver(float one_over_alpha = 1.f, float prolong_coeff = 1.f)
        : one_over_alpha_(one_over_alpha), prolong_coeff_(prolong_coeff) {}
    GMGSolver(const GMGSolver&) = delete;
    GMGSolver& operator=(const GMGSolver&) = delete;

    /* GMGSolver::solve (src/GMGSolver.cu:531-666): returns (iterations, relative residual). */
    std::tuple<int, double> solve(Grid& grid, bool verbose, int max_iters, double relative_tolerance, int level_iters,
                                  int coarsest_iters, int sync_stride, bool is_pure_neumann) {
        using A = detail::Access<Grid>;
        std::shared_ptr<detail::Binding> b = A::binding(grid);
        std::lock_guard<std::mutex> lk(b->mu);
        A::bind(grid, *b);
        cirrus_grid* cg = b->cg;
        check(cirrus_grid_gather_tiles(cg, 1, A::channel_offset(1), nullptr), "gather b");
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
        check(cirrus_gmg_solve(cg, &p, nullptr, &r), "cirrus_gmg_solve");
        check(cirrus_grid_scatter_tiles(cg, 0, A::channel_offset(0), nullptr), "scatter x");
        check(cirrus_grid_scatter_tiles(cg, 1, A::channel_offset(1), nullptr), "scatter r");
        if (cudaDeviceSynchronize() != cudaSuccess) throw std::runtime_error("cirrus_dropin: CUDA error");
        if (verbose) std::printf("cirrus GMG-PCG: %d iterations, relative residual %.3e\n", r.iters, r.rel_residual);
        return std::make_tuple(r.iters, sync_stride > 0 ? r.rel_residual : -1.0);
    }

    /* GMGSolver::dampedJacobiSolve (src/GMGSolver.cu:449-531): b in channel 1, x to channel 0,
     * the last residual in channel 2 and the diagonal in channel 3 of LEAF|GHOST tiles (both
     * channels keep their previous contents on NONLEAF tiles, as in the reference). */
    std::tuple<int, double> dampedJacobiSolve(Grid& grid, bool verbose, int max_iters, double relative_tolerance, float omega) {
        using A = detail::Access<Grid>;
        std::shared_ptr<detail::Binding> b = A::binding(grid);
        std::lock_guard<std::mutex> lk(b->mu);
        A::bind(grid, *b);
        cirrus_grid* cg = b->cg;
        for (int c : {1, 2, 3}) check(cirrus_grid_gather_tiles(cg, c, A::channel_offset(c), nullptr), "gather");
        int iters = 0;
        double rel = 0.0;
        check(cirrus_damped_jacobi_solve(cg, max_iters, relative_tolerance, omega, nullptr, &iters, &rel), "cirrus_damped_jacobi_solve");
        for (int c : {0, 2, 3}) check(cirrus_grid_scatter_tiles(cg, c, A::channel_offset(c), nullptr), "scatter");
        if (cudaDeviceSynchronize() != cudaSuccess) throw std::runtime_error("cirrus_dropin: CUDA error");
        if (verbose) std::printf("cirrus damped Jacobi: %d iterations, relative residual %.3e\n", iters, rel);
        return std::make_tuple(iters, rel);
    }

private:
    float one_over_alpha_, prolong_coeff_;
};

/* Drop-in for the reference's AMGSolver (src/AMGSolver.h:20-53; AMGSolver.cu:717-853) on the same
 * registry of bound pools: prepareTypesAndCoeffs(grid) forms the AMG cell types and coefficients
 * on the device pool (cirrus_amg_prepare), solve(...) runs the AMG-preconditioned CG
 * (cirrus_amg_solve) with b gathered from channel 1 and x / the final residual scattered to
 * channels 0 / 1.  The reference writes the coefficients into tile channels coeff_channel..+3
 * and rewrites NONLEAF cell types in place; here both stay on the device pool (the tiles'
 * channels other than 0 and 1 and their cell types are not written), so coeff_channel is kept
 * only for the signature.  A solve after the pool was rebuilt (new tiles or cell types) without
 * a new prepareTypesAndCoeffs throws, where the reference would use stale coefficients. */
template <class Grid>
class AMGSolver {
public:
    explicit AMGSolver(int coeff_channel, float one_over_alpha = 1.f, float prolong_coeff = 1.f)
        : coeff_channel(coeff_channel), one_over_alpha(one_over_alpha), prolong_coeff(prolong_coeff) {}
    AMGSolver(const AMGSolver&) = delete;
    AMGSolver& operator=(const AMGSolver&) = delete;

    void prepareTypesAndCoeffs(Grid& grid) {
        using A = detail::Access<Grid>;
        std::shared_ptr<detail::Binding> b = A::binding(grid);
        std::lock_guard<std::mutex> lk(b->mu);
        A::bind(grid, *b);
        check(cirrus_amg_prepare(b->cg, one_over_alpha, nullptr), "cirrus_amg_prepare");
        b->amg_ready = true;
    }

    std::tuple<int, double> solve(Grid& grid, bool verbose, int max_iters, double relative_tolerance, int level_iters,
                                  int coarsest_iters, int sync_stride, bool is_pure_neumann) {
        using A = detail::Access<Grid>;
        std::shared_ptr<detail::Binding> b = A::binding(grid);
        std::lock_guard<std::mutex> lk(b->mu);
        A::bind(grid, *b);
        if (!b->amg_ready) throw std::runtime_error("cirrus_dropin::AMGSolver: prepareTypesAndCoeffs first (the tiles or cell types changed)");
        cirrus_grid* cg = b->cg;
        check(cirrus_grid_gather_tiles(cg, 1, A::channel_offset(1), nullptr), "gather b");
        cirrus_solve_params p;
        cirrus_solve_params_default(&p);
        p.max_iters = max_iters;
        p.relative_tolerance = relative_tolerance;
        p.level_iters = level_iters;
        p.coarsest_iters = coarsest_iters;
        p.sync_stride = sync_stride;
        p.is_pure_neumann = is_pure_neumann ? 1 : 0;
        p.one_over_alpha = one_over_alpha;
        p.prolong_coeff = prolong_coeff;
        cirrus_solve_result r;
        check(cirrus_amg_solve(cg, &p, nullptr, &r), "cirrus_amg_solve");
        check(cirrus_grid_scatter_tiles(cg, 0, A::channel_offset(0), nullptr), "scatter x");
        check(cirrus_grid_scatter_tiles(cg, 1, A::channel_offset(1), nullptr), "scatter r");
        if (cudaDeviceSynchronize() != cudaSuccess) throw std::runtime_error("cirrus_dropin: CUDA error");
        if (verbose) std::printf("cirrus AMG-PCG: %d iterations, relative residual %.3e\n", r.iters, r.rel_residual);
        return std::make_tuple(r.iters, sync_stride > 0 ? r.rel_residual : -1.0);
    }

    int coeff_channel;
    float one_over_alpha, prolong_coeff;
};

}  // namespace cirrus_dropin

#endif  // CIRRUS_GMG_DROPIN_HPP
