// Harness that runs the product's header-only drop-in (include/cirrus_gmg_dropin.hpp) on a grid
// built by the reference's own code (oracle/ref_harness.cu, libcirrus_ref.so): what
// FluidEuler::project runs after switching its solver class.  TEST INFRASTRUCTURE ONLY: built
// by oracle/build_ref.sh into oracle/_ref/libcirrus_ref_dropin.so, which links both the
// reference harness and the product library; only tests load it (bench.py's reference arm
// loads libcirrus_ref.so alone).
//
// Each call constructs a fresh solver object, as FluidEuler::project does on every projection
// (src/FluidEuler.h:591), and times it the way FluidEuler::project times its solve
// (src/FluidEuler.h:595-601: host clock around the call, device synchronised on both sides).

#include "GMGSolver.h"
#include "PoissonSolver.h"

#include "cirrus_gmg_dropin.hpp"

#include <chrono>

extern "C" void* ref_grid(void* h);  // oracle/ref_harness.cu

extern "C" {

int refdrop_solve(void* h, int max_iters, double tol, int level_iters, int coarsest_iters, int sync_stride, int pure_neumann,
                  double* rel, double* ms) {
    auto& grid = *static_cast<HADeviceGrid<Tile>*>(ref_grid(h));
    cudaDeviceSynchronize();
    auto t0 = std::chrono::high_resolution_clock::now();
    int iters = -1;
    double err = 0.0;
    try {
        cirrus_dropin::GMGSolver<HADeviceGrid<Tile>> solver(1.f, 1.f);
        std::tie(iters, err) = solver.solve(grid, false, max_iters, tol, level_iters, coarsest_iters, sync_stride, pure_neumann != 0);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "refdrop_solve: %s\n", e.what());
        return -1;
    }
    cudaDeviceSynchronize();
    auto t1 = std::chrono::high_resolution_clock::now();
    if (rel) *rel = err;
    if (ms) *ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    return iters;
}

int refdrop_damped_jacobi(void* h, int max_iters, double tol, float omega, double* rel) {
    auto& grid = *static_cast<HADeviceGrid<Tile>*>(ref_grid(h));
    int iters = -1;
    double err = 0.0;
    try {
        cirrus_dropin::GMGSolver<HADeviceGrid<Tile>> solver(1.f, 1.f);
        std::tie(iters, err) = solver.dampedJacobiSolve(grid, false, max_iters, tol, omega);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "refdrop_damped_jacobi: %s\n", e.what());
        return -1;
    }
    cudaDeviceSynchronize();
    if (rel) *rel = err;
    return iters;
}

// The AMG drop-in on the reference grid: prepareTypesAndCoeffs (prepare != 0) then solve, fresh
// object per call.  Returns iterations, -1 on an exception (message on stderr).
int refdrop_amg_solve(void* h, int prepare, int max_iters, double tol, int level_iters, int coarsest_iters, int sync_stride,
                      int pure_neumann, double* rel) {
    auto& grid = *static_cast<HADeviceGrid<Tile>*>(ref_grid(h));
    int iters = -1;
    double err = 0.0;
    try {
        cirrus_dropin::AMGSolver<HADeviceGrid<Tile>> solver(6, 1.f, 1.f);
        if (prepare) solver.prepareTypesAndCoeffs(grid);
        std::tie(iters, err) = solver.solve(grid, false, max_iters, tol, level_iters, coarsest_iters, sync_stride, pure_neumann != 0);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "refdrop_amg_solve: %s\n", e.what());
        return -1;
    }
    cudaDeviceSynchronize();
    if (rel) *rel = err;
    return iters;
}

// cirrus_dropin::autotune on this grid (the bound pool's launch shapes); 0, or -1 on an exception.
int refdrop_autotune(void* h) {
    auto& grid = *static_cast<HADeviceGrid<Tile>*>(ref_grid(h));
    try {
        cirrus_dropin::autotune(grid);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "refdrop_autotune: %s\n", e.what());
        return -1;
    }
    return 0;
}

// Bound device pools held by the drop-in's process-wide registry.
int refdrop_bound_grids() { return cirrus_dropin::bound_grids(); }
void refdrop_release_all() { cirrus_dropin::release_all(); }

}  // extern "C"
