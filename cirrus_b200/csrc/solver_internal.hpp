// Host-side structures of the device solver shared by the kernels, the grid builder, the
// PCG driver and the C ABI.
#pragma once

#include "common.cuh"

#include <cuda_runtime.h>
#include <array>
#include <cstdint>
#include <map>
#include <string>
#include <tuple>
#include <vector>

namespace cirrus {

class Topology;

// Per-solve constants passed by value to the reduction kernels (tolerances and iteration caps are
// per instance, in InstParams).
struct SolveCtl {
    int sync_stride;
    double* history;       // optional per-iteration relative residuals of instance 0 (device)
    int history_cap;
    int use_cond;          // 1 when running inside a graph with a while-conditional node
    cudaGraphConditionalHandle cond;
    int* active;           // instances still iterating; the last to stop ends the graph's loop
};

constexpr int kBottomMaxLevels = 16;
// Coarse-level boxes of one instance for the shared-memory coarse-level kernel: its tile records
// (rec_off.., level-major), its stencil codes (code_off.., cells, a multiple of 8), and per level
// the record range and the box strides.
struct BottomInst {
    int rec_off, nrec, code_off, cells;
    int first[kBottomMaxLevels], cnt[kBottomMaxLevels], sy[kBottomMaxLevels], sz[kBottomMaxLevels];
};

enum { OP_DOT = 0, OP_INIT = 1, OP_COPY_DOT = 2, OP_XR = 3, OP_MEAN = 4 };
enum { SKIP_INACTIVE = 0, SKIP_DONE = 1 };  // which instances a reduction leaves out
constexpr int kChunkVecs = 1024;            // 4-cell vectors per reduction chunk (one CTA)
enum { EPI_NONE = -1, EPI_INIT = 0, EPI_GAMMA = 1, EPI_ALPHA = 2, EPI_CHECK = 3, EPI_BETA = 4, EPI_MEAN = 5, EPI_FINAL = 6 };

struct GraphKey {
    int max_iters, level_iters, coarsest_iters, sync_stride, pure_neumann;
    float one_over_alpha, prolong_coeff;
    int fused;
    int preconditioner;
    bool operator<(const GraphKey& o) const {
        return std::tie(max_iters, level_iters, coarsest_iters, sync_stride, pure_neumann, one_over_alpha, prolong_coeff, fused,
                        preconditioner) < std::tie(o.max_iters, o.level_iters, o.coarsest_iters, o.sync_stride, o.pure_neumann,
                                                   o.one_over_alpha, o.prolong_coeff, o.fused, o.preconditioner);
    }
};

// Kernels with selectable launch shapes (tiles per CTA x tiles in flight per thread group); the
// choice per kernel and level is made by the autotuner (autotune.cu) and is bit-neutral: every
// shape computes each tile with the same operations.
enum { KS_GS_SWEEP = 0, KS_PRESMOOTH = 1, KS_PROLONG = 2, KS_RESIDUAL = 3, KS_LAPLACIAN = 4, KS_COUNT = 5 };
// shapes 0..7: (tiles per CTA, tiles in flight per group, minimum CTAs per SM); 8..11 four of
// them prefetching the tiles of CTAs one resident wave ahead into L2
constexpr int kNumShapes = 12;
constexpr int kCommonShapes = 8;
// The launch shape of an untuned grid: one tile per 128-thread CTA (faster than shape 1 for one
// ring512 instance up to sixteen: 4.30 against 4.96 ms, 27.4 against 29.0 ms).
constexpr int kDefaultShape = 4;
// Grids of at most this many tiles (one instance or a few) are chains of latency-bound launches:
// the autotuner refines their shapes with whole solves.
constexpr int kSmallGridTiles = 16384;
// the Laplacian's 8..11 are instead the TMA-staged pipeline (lap_tma.cu) with (consumer groups,
// stages) = (2, 8), (4, 16), (2, 12), (1, 6); then 12..15 eight cells per thread (lap8.cu), 16..19
// shapes 2, 3, 5, 1 prefetching into L2 the tiles of CTAs one resident wave ahead
constexpr int kNumLapShapes = 20;
constexpr int kFirstTmaShape = 8;
constexpr int kFirstLap8Shape = 12;
inline int num_shapes(int kind) { return kind == KS_LAPLACIAN ? kNumLapShapes : kNumShapes; }

// A contiguous run of one instance's tiles inside the merged pool: tiles local..local+count of
// the instance's all-tiles order are global..global+count (one run per level).
struct TileRun {
    int global, local, count;
};

struct DevGrid {
    int device = 0;
    int n = 0, num_layers = 0, max_level = -1;
    int num_inst = 1;
    int sm_count = 148;
    int red_blocks = 1;          // CTAs of the whole-grid leaf dot (cirrus_dot)
    int64_t dof = 0;
    size_t bytes = 0;
    Topo topo{};

    // instances
    std::vector<float> inst_h0;
    std::vector<int> inst_tiles, inst_leaves, inst_max_level;
    std::vector<int64_t> inst_dof;
    std::vector<std::vector<TileRun>> inst_runs;
    int* d_inst = nullptr;          // n: instance of each tile
    float* d_inst_h0 = nullptr;
    float4* d_lconst = nullptr;     // per instance x kLevelSlots: level constants

    float* d_chbuf = nullptr;
    float* d_ch[kNumChannels] = {};
    uint8_t* d_u8 = nullptr;     // ctype | mask_lap | mask_mg
    TileMeta* d_meta = nullptr;
    uint32_t* d_fcls = nullptr;
    int* d_child = nullptr;      // n x 8 finer tiles per octant, -1 if absent
    int* d_edge = nullptr;       // n x 12 same-level edge neighbours, -1 if absent
    int* d_ghost_tables = nullptr;  // ghost slot per tile (n) | ghost slot per child octant (n x 8)
    float* d_gacc = nullptr;        // per GHOST tile: 64 partial sums of its A p (fused Laplacian)
    uint8_t* d_ghost_faces = nullptr;  // per GHOST tile: faces whose p other tiles read (Topo::ghost_faces)
    float* d_xpre = nullptr;        // n x 512: pre-smoothed x of the fused V-cycle (read by the upstroke)
    void** d_tile_ptrs = nullptr;  // optional external array-of-tiles storage (interop)
    uint8_t* d_ct_gather = nullptr;       // n x 512 cell types gathered from the external tiles
    unsigned int* d_ct_flag = nullptr;    // set when a gathered cell type differs from the pool's
    int launch_mode = 0;                  // 0: solves run as one CUDA graph; 1: direct launches
    void* tile_map_cache = nullptr;       // tensor maps of the channel buffers (lap_tma.cu)
    unsigned int* d_err = nullptr;        // set by a kernel whose bounded wait gave up (0 otherwise)
    unsigned int* h_err = nullptr;        // pinned mirror, read back after each solve
    // the grid's own stream and join event for solves of several grids at once (created on first use)
    cudaStream_t side_stream = nullptr;
    cudaEvent_t side_join = nullptr;
    int* d_lists = nullptr;
    const int* d_leaf = nullptr;   // LEAF tiles, instance by instance, each in its all-tiles order
    const int* d_ghost = nullptr;
    const int* d_leafghost = nullptr;
    const int* d_mg = nullptr;
    int n_leaf = 0, n_ghost = 0, n_leafghost = 0;
    // fused Laplacian: LEAF tiles + GHOST tiles coupled inside (staged path); GHOST tiles coupled
    // only outward across their faces (face path): per coarse cell touching a coupled face an
    // item (tile, ghost slot << 6 | cell, coupled faces | face classes << 6, level-constant index)
    const int* d_lapmain = nullptr;
    int n_lapmain = 0;
    int4* d_lapitems = nullptr;
    int n_lapface = 0, n_lapitems = 0;
    // residual + restriction with GHOST x and right-hand sides 0: per level the tiles of the
    // staged path (all but the face-path GHOST tiles) and one item per coarse cell of each
    // face-path GHOST tile (tile, cell | coupled faces << 6 | face classes << 12 | octant << 24,
    // parent tile, level-constant index)
    std::vector<int> rr_off, rr_cnt, rri_off, rri_cnt;
    int* d_rrmain = nullptr;
    int4* d_rritems = nullptr;
    // prolongation of the fused V-cycle: per level the non-GHOST tiles (staged path) and one item
    // per GHOST face towards a non-GHOST neighbour (tile, face, parent tile, octant)
    std::vector<int> pr_off, pr_cnt, pri_off, pri_cnt;
    int* d_prmain = nullptr;
    int4* d_pritems = nullptr;
    std::vector<int> mg_offset, mg_count, level_first, level_count;
    std::vector<uint8_t> h_tile_type;
    std::vector<uint8_t> shapes;  // KS_COUNT x num_layers launch-shape choices
    int shape(int kind, int level) const { return shapes.empty() ? kDefaultShape : shapes[(size_t)kind * num_layers + level]; }

    // coarse levels 0..bottom_level of every instance in the shared-memory kernel (-1: none)
    int bottom_level = -1;
    size_t bottom_smem = 0;
    int4* d_bottom_tiles = nullptr;     // per record: box base, parent-cell base, type | level << 8, tile
    uint16_t* d_bottom_code = nullptr;  // per box cell: stencil mask byte | cross-level (c2) face flags << 7
    BottomInst* d_bottom_inst = nullptr;

    // per-instance reductions: chunk table (instance, first vector, end vector) and per instance
    // (first chunk, chunk count)
    // per-tile parts of the PCG dot products formed by the stencil kernels (the fused Laplacian for
    // p.Ap, the V-cycle's last colour sweeps for r.z): one FP64 value per LEAF tile in LEAF-list
    // order; per instance its first LEAF slot and count; the LEAF tiles at the shared-memory
    // kernel's levels (their r.z parts formed apart)
    int* d_leafslot = nullptr;
    double* d_wpart = nullptr;
    int2* d_inst_leafrange = nullptr;
    int* d_bottom_leaves = nullptr;
    int n_bottom_leaves = 0;
    int* d_gpar_leaves = nullptr;  // LEAF tiles with GHOST children
    int n_gpar_leaves = 0;
    int n_chunks = 0;
    int4* d_chunks = nullptr;
    int2* d_inst_chunks = nullptr;
    unsigned int* d_counters = nullptr;  // ticket counter per instance
    double* d_partials = nullptr;        // 2 doubles per chunk (and per cirrus_dot block)
    unsigned int* d_counter = nullptr;   // ticket counter of the whole-grid reductions
    Scalars* d_scalars = nullptr;        // per instance
    Scalars* h_scalars = nullptr;        // pinned mirror
    Scalars* d_dot = nullptr;            // result slot of the whole-grid reductions
    InstParams* d_iparams = nullptr;
    InstParams* h_iparams = nullptr;     // pinned
    int* d_active = nullptr;             // instances still iterating in the running solve
    double* d_history = nullptr;
    int history_cap = 0;

    // FP64 defect-correction buffers (allocated on first mixed-precision solve)
    double* d_x64 = nullptr;
    double* d_ax64 = nullptr;
    double* d_r64 = nullptr;
    double* d_norm = nullptr;      // per instance
    double* d_msum = nullptr;      // per instance: sum of the FP64 residual (pure-Neumann projection)
    double* d_dofd = nullptr;      // per instance: INTERIOR cells of LEAF tiles, as doubles
    float* d_bsave = nullptr;
    bool x64_valid = false;      // the last solve was mixed precision: d_x64 holds its FP64 x

    // AMG variant (amg.cu): 4 planes of n*512 coefficients (x-, y-, z- face off-diagonals,
    // diagonal) and the AMG cell types, allocated by the first amg_prepare
    float* d_amg = nullptr;
    uint8_t* d_amg_ct = nullptr;
    int2* d_amg_l0 = nullptr;  // per instance: (first entry, count) of its level-0 LEAF|NONLEAF tiles
    int amg_l0_max = 0;        // the largest count
    bool amg_ready = false;

    struct SolveGraph {
        cudaGraphExec_t exec = nullptr;
        long long prologue = 0, body = 0, epilogue = 0;  // kernel launches per section
    };
    std::map<GraphKey, SolveGraph> graphs;
    mutable long long launch_count = 0;  // kernels launched (or recorded into graphs) so far
    long long last_solve_launches = 0;   // kernels executed by the last solve
    std::string last_error;
};

// Builds the device grid of one or more instances from finalised topologies (cell types set,
// CalcCellTypesFromLeafs done).
int grid_create(const std::vector<const Topology*>& topos, DevGrid** out, std::string* err);
void grid_destroy(DevGrid* g);

namespace launch {
// Programmatic dependent launch of the solve kernels (on unless CIRRUS_NO_PDL=1).
bool pdl_enabled();
// Launches kernel k on stream s with programmatic stream serialisation: the kernel may be
// scheduled while its predecessor finishes; the kernel itself waits for the predecessor's
// completion (pdl_entry, or pdl_wait after its topology loads) before touching data that a
// kernel writes.
template <class... KArgs, class... Args>
inline void launch_kernel(void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl_enabled() ? 1 : 0;
    cudaLaunchKernelEx(&cfg, k, static_cast<KArgs>(args)...);
}
// The grid's kernel view for one launch of a staged kernel k (threads per CTA, dynamic shared
// memory, list entries per CTA): with prefetch, tp.pf = the list entries the CTAs resident at once
// cover, so each CTA prefetches into L2 the tiles of the CTA one resident wave later.
template <class K>
inline Topo prefetch_topo(const DevGrid& g, K k, int threads, size_t smem, int per_cta, bool prefetch) {
    Topo tp = g.topo;
    tp.pf = 0;
    if (prefetch) {
        int resident = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, k, threads, smem);
        tp.pf = (resident > 0 ? resident : 1) * g.sm_count * per_cta;
    }
    return tp;
}
// S (nullable): per-instance scalars; tiles of finished instances are skipped.
template <class T> void full_laplacian(const DevGrid& g, T* X, T* Y, const Scalars* S, cudaStream_t s);
// FullNegativeLaplacian with calc_diag: the diagonal of LEAF|GHOST cells, ghost rows accumulated.
void full_laplacian_diag(const DevGrid& g, float* X, float* D, cudaStream_t s);
// NegativeLaplacianSameLevel128 over the tiles of `level` (-1: all tiles) whose
// subtreeType(subtree_level) is in `types`.
void laplacian_same_level(const DevGrid& g, int level, int subtree_level, uint32_t types, const float* X, float* Y, bool diag,
                          cudaStream_t s);
// dampedJacobiSolve's residual (Ax = b - Ax) and update (x += omega r / D) on INTERIOR LEAF cells.
void jacobi_residual(const DevGrid& g, const float* B, float* AX, cudaStream_t s);
void jacobi_update(const DevGrid& g, float* X, const float* R, const float* D, float omega, cudaStream_t s);
// Dot over the 4-cell vectors of the tiles in `list` (synchronises s; result on the host).
double list_dot(const DevGrid& g, const float* A, const float* B, const int* list, int n, cudaStream_t s);
// FullNegativeLaplacian as one launch; the ghost-to-parent sums are completed by pap_ghost.
// with_pap: also store the p.Ap tile parts of LEAF tiles without GHOST children (d_wpart)
void laplacian_fused(const DevGrid& g, const float* X, float* Y, const Scalars* S, cudaStream_t s, bool with_pap = false);
// The same with the staged tiles moved by bulk asynchronous copies through a stage ring
// (lap_tma.cu); variant 0..3 = (consumer groups, stages) (2, 8), (4, 16), (2, 12), (1, 6).  False
// (nothing launched) when the tensor maps of X cannot be made.
bool laplacian_tma(const DevGrid& g, int variant, const float* X, float* Y, const Scalars* S, cudaStream_t s, bool with_pap);
// The same with a column of eight cells per thread (lap8.cu); variant 0..3 = (tile groups per
// CTA, tiles in flight per group) (2, 2), (4, 1), (1, 4), (2, 2) with at least 7 CTAs per SM.
// WP: as laplacian_fused's.
void laplacian8(const DevGrid& g, int variant, const float* X, float* Y, const Scalars* S, cudaStream_t s, double* WP);
// Ap += GHOST children's sums on the LEAF tiles that have them, and their p.Ap tile parts
void pap_ghost(const DevGrid& g, const float* P, float* AP, cudaStream_t s);
// RD: with the PCG residual r, also store the r.z tile parts of the level's LEAF tiles (d_wpart)
void gs_sweep(const DevGrid& g, int level, float* X, const float* R, int color, const Scalars* S, cudaStream_t s,
              const float* RD = nullptr);
// r.z tile parts (d_wpart) of the LEAF tiles at the shared-memory kernel's levels
void leaf_wpart(const DevGrid& g, const float* R, const float* Z, cudaStream_t s);
// per instance: the sum of its LEAF tiles' parts in d_wpart (fixed order), then the epilogue
void inst_wsum(const DevGrid& g, const SolveCtl& ctl, int epi, int skip, cudaStream_t s);
void gs_sequence(const DevGrid& g, int level, float* X, const float* R, uint32_t colors, int nsweeps, const Scalars* S,
                 cudaStream_t s);
// ghosts_zero: GHOST tiles hold x = 0 and right-hand side 0 (the fused V-cycle), so the
// face-path GHOST tiles of the level skip staging.
void residual_restrict(const DevGrid& g, int level, const float* X, const float* RHS, float* C, float one_over_alpha,
                       const Scalars* S, cudaStream_t s, bool ghosts_zero = false);
void prolongate(const DevGrid& g, int level, const float* CX, float* FX, float prolong_coeff, const Scalars* S, cudaStream_t s);
void vcycle_init(const DevGrid& g, float* X, float* RHS, const float* F, const Scalars* S, cudaStream_t s);
// Per-instance reduction over LEAF vectors with the fused elementwise work of `op`; the
// instance's epilogue `epi` runs on its scalars.
void inst_reduce(int op, const DevGrid& g, float* A, float* B, float* C, float* D, const SolveCtl& ctl, int epi, int skip,
                 cudaStream_t s);
// Whole-grid dot over all LEAF tiles into g.d_dot->gamma (cirrus_dot).
void grid_dot(const DevGrid& g, const float* A, const float* B, cudaStream_t s);
// OP_DOT over an explicit leaf list with caller-provided scratch (partials: 2 doubles per block;
// counter 0 at launch); the sum goes to S->gamma.
void leaf_dot_raw(const float* A, const float* B, const int* leaves, int nleaf, int blocks, double* partials,
                  unsigned int* counter, Scalars* S, cudaStream_t s);
// Sets up the per-instance scalars of a solve from g.d_iparams.
void begin_solve(const DevGrid& g, const SolveCtl& ctl, cudaStream_t s);
// x += alpha p and p = z + beta p (instances still iterating), p pushed to GHOST children
void update_p(const DevGrid& g, float* P, const float* Z, float* X, cudaStream_t s);
// the last iteration's x += alpha p, after the loop
void x_final(const DevGrid& g, float* X, const float* P, cudaStream_t s);
void recenter(const DevGrid& g, float* R, float* RC, cudaStream_t s);
void residual64(const DevGrid& g, const float* B, const double* AX, double* R64, float* R32, cudaStream_t s);
void accumulate_correction(const DevGrid& g, double* X64, float* E, cudaStream_t s);
// per-instance FP64 sums of squares into out[instance] (A, or B32 widened); plain_sum: sums of A
void norm64(const DevGrid& g, const double* A, const float* B32, double* out, cudaStream_t s, bool plain_sum = false);
// pure-Neumann active instances: R64 -= sums/counts on INTERIOR cells of LEAF tiles, R32 refreshed
void sub_mean64(const DevGrid& g, double* R64, float* R32, const double* sums, const double* counts, cudaStream_t s);
void widen(const DevGrid& g, const float* a, double* b, size_t n, cudaStream_t s);
void narrow(const DevGrid& g, const double* a, float* b, size_t n, cudaStream_t s);
// right-hand side construction (rhs.cu)
void clear_neumann_faces(const DevGrid& g, int u_channel, cudaStream_t s);
void propagate_to_children(const DevGrid& g, int channel, cudaStream_t s);
void velocity_divergence(const DevGrid& g, int u_channel, int b_channel, cudaStream_t s);
// AddGradientToFaceCenters (src/PoissonSolver.cu:144-206): p propagated to GHOST cells, face
// gradient terms, GHOST children accumulated into LEAF parents (1/4, INTERIOR|DIRICHLET).
void add_gradient(const DevGrid& g, int p_channel, int u_channel, cudaStream_t s);
// PropagateValuesToGhostTiles (src/PoissonGrid.cu:585-605) of channel X.
template <class T> void propagate_ghosts(const DevGrid& g, T* X, const Scalars* S, cudaStream_t s);
// fused V-cycle (vcycle_fused.cu)
void presmooth(const DevGrid& g, int level, float* XP, const float* RHS, const Scalars* S, cudaStream_t s);
void prolong_sweep(const DevGrid& g, int level, float* Z, const float* XP, const float* RHS, float prolong_coeff, const Scalars* S,
                   cudaStream_t s);
void zero_ghost_tiles(const DevGrid& g, float* X, cudaStream_t s);
bool bottom(const DevGrid& g, int lb, int coarsest_iters, float* Z, const float* RHS, float one_over_alpha, float prolong_coeff,
            const Scalars* S, cudaStream_t s);
bool bottom_supported(int coarsest_iters, int lb);
constexpr int kBottomSmemBudget = 224 * 1024;  // dynamic shared memory of the coarse-level kernel
size_t bottom_smem_bytes(long long cells, int tiles);
void init_kernel_attributes();
void init_stencil_attributes();
// array-of-tiles interop (interop.cu)
void gather_tiles(const DevGrid& g, int channel, size_t byte_offset, cudaStream_t s);
void scatter_tiles(const DevGrid& g, int channel, size_t byte_offset, cudaStream_t s);
// the 512 cell-type bytes at tile_ptr + byte_offset of every tile into d_ct_gather, and
// *d_ct_flag |= 1 where one differs from the pool's cell types (flag cleared first on s)
void compare_tile_cell_types(const DevGrid& g, size_t byte_offset, cudaStream_t s);
}  // namespace launch

// tensor-map cache of the TMA-staged kernels (lap_tma.cu)
void init_tile_map_cache(DevGrid& g);
void free_tile_map_cache(DevGrid& g);

// 512 bytes at tile_ptrs[i] + byte_offset of n device tiles into host_out, through temporary
// device buffers (interop.cu); synchronises s.  0, or 2 (CUDA error) / 3 (out of memory).
int gather_tile_bytes(const void* const* tile_ptrs, int n, size_t byte_offset, uint8_t* host_out, cudaStream_t s);

// V-cycle with the reference's schedule (src/GMGSolver.cu:383-447), one launch per kernel of the
// reference (any level_iters).
void vcycle(const DevGrid& g, float* X, const float* F, float* RHS, int level_iters, int coarsest_iters, float one_over_alpha,
            float prolong_coeff, const Scalars* S, cudaStream_t s);
// The same V-cycle with fused kernels (level_iters == 1).  Precondition: RHS holds f on LEAF
// tiles (the PCG kernels that write r maintain this) and 0 on GHOST tiles; X needs no
// initialisation.  dot_r (the PCG residual r, optional): also leave the r.z part of every LEAF
// tile in d_wpart for inst_wsum.
void vcycle_fused(const DevGrid& g, float* X, float* RHS, int coarsest_iters, float one_over_alpha, float prolong_coeff,
                  const Scalars* S, cudaStream_t s, const float* dot_r = nullptr);
bool use_fused(const DevGrid& g, int level_iters, int coarsest_iters);

// AMG variant (amg.cu).  AMGSolver::prepareTypesAndCoeffs (src/AMGSolver.cu:717-720): the AMG
// cell types and coefficients of every tile.  0, 2 (CUDA error) or 3 (out of memory).
int amg_prepare(DevGrid& g, float one_over_alpha, cudaStream_t s);
// the 4 coefficient planes (4 * n * 512 floats) and the AMG cell types (n * 512), either may be
// null; synchronises s.  1 when amg_prepare has not run.
int amg_download(const DevGrid& g, float* coeffs, uint8_t* types, cudaStream_t s);
// VCycleAMG(grid, x, f, tmp, rhs, ...) (src/AMGSolver.cu:610-715), after amg_prepare
void vcycle_amg(const DevGrid& g, float* X, const float* F, float* TMP, float* RHS, int level_iters, int coarsest_iters,
                float one_over_alpha, float prolong_coeff, const Scalars* S, cudaStream_t s);

struct SolveParams {
    int preconditioner = 0;  // 0: the GMG V-cycle (GMGSolver); 1: the AMG V-cycle (AMGSolver, amg_prepare first)
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
    long long launches = 0;  // kernels executed by the solve (the whole batch's)
};
// Per-instance part of a batched solve request (defaults: the shared SolveParams).
struct InstRequest {
    int active = 1;
    double tol = -1;          // < 0: SolveParams::tol
    int pure_neumann = -1;    // < 0: SolveParams::pure_neumann
};

// Plain FP32 GMG-PCG (GMGSolver::solve) of every active instance: b in channel 1, x to channel 0.
// r: one result per instance; req: one request per instance or null (all active).
int pcg_solve(DevGrid& g, const SolveParams& p, cudaStream_t s, SolveResult* r, const InstRequest* req = nullptr);
// Mixed precision: FP64 defect correction around FP32 PCG solves.
int mixed_solve(DevGrid& g, const SolveParams& p, cudaStream_t s, SolveResult* r, const InstRequest* req = nullptr);
// pcg_solve in two halves for asynchronous callers: pcg_launch enqueues the solve on s (the graph
// launch, or direct launches with their per-iteration host checks, then the copy of the
// instances' scalars into the pinned mirror); pcg_collect turns that mirror into results once s
// has completed.  `direct` carries the direct path's launch count (-1: graph) from one to the other.
int pcg_launch(DevGrid& g, const SolveParams& p, cudaStream_t s, const InstRequest* req, long long* direct);
void pcg_collect(DevGrid& g, const SolveParams& p, long long direct, SolveResult* r);
// Plain FP32 solves of several grids at once: each grid's solve is launched on the grid's own
// stream, forked from s after s's pending work and joined back into s; results per grid, in grid
// order.  Mixed precision drives each grid from a host thread of its own (its outer loop reads
// residuals on the host).
int solve_grids(const std::vector<DevGrid*>& grids, const SolveParams& p, cudaStream_t s, std::vector<std::vector<SolveResult>>& r);
// GMGSolver::dampedJacobiSolve (src/GMGSolver.cu:449-531): b in channel 1, x to channel 0,
// channels 2 (residual) and 3 (diagonal) as the reference leaves them.  Single-instance grids.
int damped_jacobi(DevGrid& g, int max_iters, double tol, float omega, cudaStream_t s, int* iters, double* rel);
// FP64 true relative residual of the last solution of each instance against b (device FP32
// channel): the FP64 x of a mixed-precision solve, else channel 0 widened to FP64.
int true_residual(DevGrid& g, const float* d_b, double* rel, cudaStream_t s);
// Times every launch shape of the shape-selectable kernels on this grid and keeps the fastest per
// kernel and level (autotune.cu); overwrites the scratch channels 2-5.  report (optional) gets one
// line per choice.
int autotune(DevGrid& g, cudaStream_t s, int reps, std::string* report);
// Destroys the grid's cached solve graphs (after a change of launch shapes).
void drop_graphs(DevGrid& g);
// Fastest converging (level_iters, coarsest_iters) for `base` on the grid's current right-hand
// sides (autotune.cu); 5 if no candidate converged (base's values are returned).
int autotune_sweeps(DevGrid& g, const SolveParams& base, cudaStream_t s, int* level_iters, int* coarsest_iters,
                    std::string* report);
// Copy the last solution to the host in FP64 (num_tiles*512 doubles, pool order).
int solution_f64(DevGrid& g, double* host, cudaStream_t s);

}  // namespace cirrus
