// Host-side structures of the device solver shared by the kernels, the grid builder, the
// PCG driver and the C ABI.
#pragma once

#include "common.cuh"

#include <cuda_runtime.h>
#include <cstdint>
#include <map>
#include <string>
#include <tuple>
#include <vector>

namespace cirrus {

class Topology;

// Scalar state of one PCG solve, resident in device memory (the reference keeps gamma, beta,
// alpha, gamma_old, fp, mean, count as 7 device doubles, src/GMGSolver.h:22-30).
struct Scalars {
    double rhs2, thr2, gamma, gamma_old, beta, alpha, fp, res2, mean, rel;
    int iter, iters, done, converged, nonfinite, pad;
};

// Per-solve constants passed by value to the reduction kernels.
struct SolveCtl {
    int sync_stride;
    int max_iters;
    double tol;
    double* history;       // optional per-iteration relative residuals (device)
    int history_cap;
    int use_cond;          // 1 when running inside a graph with a while-conditional node
    cudaGraphConditionalHandle cond;
};

enum { OP_DOT = 0, OP_INIT = 1, OP_COPY_DOT = 2, OP_XR = 3, OP_MEAN = 4, OP_PAP = 5 };
enum { EPI_NONE = -1, EPI_INIT = 0, EPI_GAMMA = 1, EPI_ALPHA = 2, EPI_CHECK = 3, EPI_BETA = 4, EPI_MEAN = 5, EPI_FINAL = 6 };

struct GraphKey {
    int max_iters, level_iters, coarsest_iters, sync_stride, pure_neumann;
    double tol;
    float one_over_alpha, prolong_coeff;
    int fused;
    bool operator<(const GraphKey& o) const {
        return std::tie(max_iters, level_iters, coarsest_iters, sync_stride, pure_neumann, tol, one_over_alpha, prolong_coeff, fused) <
               std::tie(o.max_iters, o.level_iters, o.coarsest_iters, o.sync_stride, o.pure_neumann, o.tol, o.one_over_alpha,
                        o.prolong_coeff, o.fused);
    }
};

struct DevGrid {
    int device = 0;
    int n = 0, num_layers = 0, max_level = -1;
    int sm_count = 148;
    int red_blocks = 1;          // CTAs of the leaf reductions (fixed per grid: deterministic sums)
    int64_t dof = 0;
    size_t bytes = 0;
    Topo topo{};
    float h0 = 0.125f;

    float* d_chbuf = nullptr;
    float* d_ch[kNumChannels] = {};
    uint8_t* d_u8 = nullptr;     // ctype | mask_lap | mask_mg
    TileMeta* d_meta = nullptr;
    uint32_t* d_fcls = nullptr;
    int* d_child = nullptr;      // n x 8 finer tiles per octant, -1 if absent
    int* d_edge = nullptr;       // n x 12 same-level edge neighbours, -1 if absent
    int* d_ghost_tables = nullptr;  // ghost slot per tile (n) | ghost slot per child octant (n x 8)
    float* d_gacc = nullptr;        // per GHOST tile: 64 partial sums of its A p (fused Laplacian)
    float* d_xpre = nullptr;        // n x 512: pre-smoothed x of the fused V-cycle (read by the upstroke)
    void** d_tile_ptrs = nullptr;  // optional external array-of-tiles storage (interop)
    int* d_lists = nullptr;
    const int* d_leaf = nullptr;
    const int* d_ghost = nullptr;
    const int* d_leafghost = nullptr;
    const int* d_mg = nullptr;
    int n_leaf = 0, n_ghost = 0, n_leafghost = 0;
    std::vector<int> mg_offset, mg_count, level_first, level_count;
    int* d_level_tables = nullptr;  // mg_offset | mg_count | level_first | level_count (num_layers each)
    int bottom_level = -1;          // levels 0..bottom_level fit the shared-memory small-level kernel (-1: none)
    std::vector<uint8_t> h_tile_type;

    double* d_partials = nullptr;
    unsigned int* d_counter = nullptr;
    Scalars* d_scalars = nullptr;
    Scalars* h_scalars = nullptr;  // pinned
    double* d_history = nullptr;
    int history_cap = 0;

    // FP64 defect-correction buffers (allocated on first mixed-precision solve)
    double* d_x64 = nullptr;
    double* d_ax64 = nullptr;
    double* d_r64 = nullptr;
    double* d_norm = nullptr;
    float* d_bsave = nullptr;
    bool x64_valid = false;      // the last solve was mixed precision: d_x64 holds its FP64 x

    struct SolveGraph {
        cudaGraphExec_t exec = nullptr;
        long long prologue = 0, body = 0, epilogue = 0;  // kernel launches per section
    };
    std::map<GraphKey, SolveGraph> graphs;
    mutable long long launch_count = 0;  // kernels launched (or recorded into graphs) so far
    long long last_solve_launches = 0;   // kernels executed by the last solve
    std::string last_error;
};

// Builds the device grid from a finalised topology (cell types set, CalcCellTypesFromLeafs done).
int grid_create(const Topology& topo, DevGrid** out, std::string* err);
void grid_destroy(DevGrid* g);

namespace launch {
template <class T> void full_laplacian(const DevGrid& g, T* X, T* Y, const int* done, cudaStream_t s);
// FullNegativeLaplacian as one launch; the ghost-to-parent sums are completed by OP_PAP.
void laplacian_fused(const DevGrid& g, const float* X, float* Y, const int* done, cudaStream_t s);
void gs_sweep(const DevGrid& g, int level, float* X, const float* R, int color, const int* done, cudaStream_t s);
void gs_sequence(const DevGrid& g, int level, float* X, const float* R, uint32_t colors, int nsweeps, const int* done,
                 cudaStream_t s);
void residual_restrict(const DevGrid& g, int level, const float* X, const float* RHS, float* C, float one_over_alpha,
                       const int* done, cudaStream_t s);
void prolongate(const DevGrid& g, int level, const float* CX, float* FX, float prolong_coeff, const int* done, cudaStream_t s);
void vcycle_init(const DevGrid& g, float* X, float* RHS, const float* F, const int* done, cudaStream_t s);
void leaf_reduce(int op, const DevGrid& g, float* A, float* B, float* C, float* D, Scalars* S, const SolveCtl& ctl, int epi,
                 int skip_if_done, cudaStream_t s);
// OP_DOT over an explicit leaf list with caller-provided scratch (partials: 2 doubles per block;
// counter 0 at launch); the sum goes to S->gamma.
void leaf_dot_raw(const float* A, const float* B, const int* leaves, int nleaf, int blocks, double* partials,
                  unsigned int* counter, Scalars* S, cudaStream_t s);
void update_p(const DevGrid& g, float* P, const float* Z, const Scalars* S, cudaStream_t s);
void recenter(const DevGrid& g, float* R, const Scalars* S, int skip_if_done, cudaStream_t s, float* RC = nullptr);
void residual64(const DevGrid& g, const float* B, const double* AX, double* R64, float* R32, cudaStream_t s);
void accumulate_correction(const DevGrid& g, double* X64, float* E, cudaStream_t s);
void norm64(const DevGrid& g, const double* A, const float* B32, double* out, cudaStream_t s);
void widen(const DevGrid& g, const float* a, double* b, size_t n, cudaStream_t s);
void narrow(const DevGrid& g, const double* a, float* b, size_t n, cudaStream_t s);
// right-hand side construction (rhs.cu)
void clear_neumann_faces(const DevGrid& g, int u_channel, cudaStream_t s);
void propagate_to_children(const DevGrid& g, int channel, cudaStream_t s);
void velocity_divergence(const DevGrid& g, int u_channel, int b_channel, cudaStream_t s);
// fused V-cycle (vcycle_fused.cu)
void presmooth(const DevGrid& g, int level, float* XP, const float* RHS, const int* done, cudaStream_t s);
void prolong_sweep(const DevGrid& g, int level, float* Z, const float* XP, const float* RHS, float prolong_coeff, const int* done,
                   cudaStream_t s);
void zero_ghost_tiles(const DevGrid& g, float* X, cudaStream_t s);
bool bottom(const DevGrid& g, int lb, int coarsest_iters, float* Z, const float* RHS, float one_over_alpha, float prolong_coeff,
            const int* done, cudaStream_t s);
bool bottom_supported(int coarsest_iters, int lb);
constexpr int kBottomTiles = 40;  // tiles the shared-memory small-level kernel holds
void init_kernel_attributes();
// array-of-tiles interop (interop.cu)
void gather_tiles(const DevGrid& g, int channel, size_t byte_offset, cudaStream_t s);
void scatter_tiles(const DevGrid& g, int channel, size_t byte_offset, cudaStream_t s);
}  // namespace launch

// V-cycle with the reference's schedule (src/GMGSolver.cu:383-447), one launch per kernel of the
// reference (any level_iters).
void vcycle(const DevGrid& g, float* X, const float* F, float* RHS, int level_iters, int coarsest_iters, float one_over_alpha,
            float prolong_coeff, const int* done, cudaStream_t s);
// The same V-cycle with fused kernels (level_iters == 1).  Precondition: RHS holds f on LEAF
// tiles (the PCG kernels that write r maintain this) and 0 on GHOST tiles; X needs no
// initialisation.
void vcycle_fused(const DevGrid& g, float* X, float* RHS, int coarsest_iters, float one_over_alpha, float prolong_coeff,
                  const int* done, cudaStream_t s);
bool use_fused(const DevGrid& g, int level_iters, int coarsest_iters);

struct SolveParams {
    int max_iters = 1000;
    double tol = 1e-6;
    int level_iters = 1, coarsest_iters = 10, sync_stride = 1, pure_neumann = 0;
    float one_over_alpha = 1.f, prolong_coeff = 1.f;
    int precision = 0, warm_start = 0;
    double inner_tol = 1e-3;
    int max_outer = 20;
};
struct SolveResult {
    int iters = 0, outer = 0, status = 0;
    double rel = 0, true_rel = -1;
    long long launches = 0;  // kernels executed by the solve
};

// Plain FP32 GMG-PCG (GMGSolver::solve).  b in channel 1, x to channel 0.
int pcg_solve(DevGrid& g, const SolveParams& p, cudaStream_t s, SolveResult* r);
// Mixed precision: FP64 defect correction around FP32 PCG solves.
int mixed_solve(DevGrid& g, const SolveParams& p, cudaStream_t s, SolveResult* r);
// FP64 true relative residual of the last solution against b (device FP32 leaf channel): the
// FP64 x of a mixed-precision solve, else channel 0 widened to FP64.
int true_residual(DevGrid& g, const float* d_b, double* rel, cudaStream_t s);
// Copy the last solution to the host in FP64 (num_tiles*512 doubles).
int solution_f64(DevGrid& g, double* host, cudaStream_t s);

}  // namespace cirrus
