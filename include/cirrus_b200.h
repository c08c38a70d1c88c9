/*
 * cirrus_b200.h -- C ABI of the B200-native GMG-PCG Poisson solver for adaptive octree-tile
 * grids (8^3-cell tiles).  Drop-in for the pressure-projection solve of wang-mengdi/Cirrus.
 *
 * Conventions
 *   - Every function returns cirrus_status and never throws across the ABI.
 *   - Plain pointers and sizes only; `stream` is a cudaStream_t passed as void* (NULL = the
 *     legacy default stream).
 *   - Host arrays are owned by the caller; device state is owned by the library until the
 *     matching *_destroy call.
 *   - Tiles are addressed in "all-tiles order": level-major, and inside a level in the order of
 *     the level's open-addressing hash table, exactly as the reference's dAllTiles
 *     (src/HAGrid.h:538-556).  Cell c of a tile is local (i,j,k) with c = i*64 + j*8 + k
 *     (src/HAAccessor.h:32-34).
 *   - Channel ids follow PoissonTile (src/PoissonTile.h:12-24): 0 x, 1 b (= r), 2 p, 3 Ap,
 *     4 z, 5 tmp, 6 u, 7 v, 8 w.
 *   - Calls on distinct grids are thread-safe; calls on one grid must be serialised.
 */
#ifndef CIRRUS_B200_H
#define CIRRUS_B200_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum cirrus_status {
    CIRRUS_OK = 0,
    CIRRUS_ERR_INVALID_ARGUMENT = 1,
    CIRRUS_ERR_CUDA = 2,
    CIRRUS_ERR_OUT_OF_MEMORY = 3,
    CIRRUS_ERR_TOPOLOGY = 4,        /* hash table full, bad level, inconsistent tree      */
    CIRRUS_ERR_NOT_CONVERGED = 5,   /* iteration cap reached before the tolerance          */
    CIRRUS_ERR_NONFINITE = 6,       /* NaN/Inf residual or CG scalar                       */
    CIRRUS_ERR_BUDGET = 7,          /* admission refused: HBM budget exceeded              */
    CIRRUS_ERR_NO_DEVICE = 8,
    CIRRUS_ERR_STATE = 9            /* call out of order (e.g. grid not finalised)         */
} cirrus_status;

/* Tile types (src/HATileInfo.h:19) and cell types (src/PoissonTile.h:6). */
enum { CIRRUS_LEAF = 1, CIRRUS_NONLEAF = 2, CIRRUS_GHOST = 4 };
enum { CIRRUS_DIRICHLET = 1, CIRRUS_INTERIOR = 2, CIRRUS_NEUMANN = 4 };

/* Returns a static, NUL-terminated description of a status code. */
const char* cirrus_status_string(cirrus_status s);
/* Library version string. */
const char* cirrus_version(void);

/* ------------------------------------------------------------------------------------------
 * Host topology: the octree of tiles, built exactly as the reference builds it.
 * ---------------------------------------------------------------------------------------- */
typedef struct cirrus_topology cirrus_topology;

/* level_target callback: returns the target level of a LEAF tile (src/PoissonGrid.h:63). */
typedef int (*cirrus_level_target_fn)(void* user, int level, int x, int y, int z);

/* Replaces HADeviceGrid(h0, levels_log2_hash) (src/HAGrid.h:265-293). */
cirrus_status cirrus_topology_create(int num_layers, const uint32_t* log2_hash, double h0, cirrus_topology** out);
void cirrus_topology_destroy(cirrus_topology* topo);
/* Replaces HADeviceGrid::setTileHost(level, b_ijk, Tile(), type) (src/HAGrid.h:387-407). */
cirrus_status cirrus_topology_set_tile(cirrus_topology* topo, int level, int x, int y, int z, int type);
/* Adopts an existing tile list in the given all-tiles order (5 int32 per tile: level, x, y, z,
 * type; level-major), e.g. a reference grid's hAllTiles (src/HAGrid.h:538-556): the order is
 * kept as given so channel data can be exchanged tile for tile.  Replaces any previous content. */
cirrus_status cirrus_topology_import_tiles(cirrus_topology* topo, const int32_t* tiles5, int num_tiles);
/* Replaces compressHost() + syncHostAndDevice() (src/HAGrid.h:491-561). */
cirrus_status cirrus_topology_compress(cirrus_topology* topo);
/* Replaces SpawnGhostTiles(grid) (src/PoissonGrid.cu:30-60). */
cirrus_status cirrus_topology_spawn_ghost_tiles(cirrus_topology* topo);
/* Replaces RefineLeafsOneStep(grid, level_target) (src/PoissonGrid.h:35-162).
 * refined_per_level (optional, num_layers ints) receives the refined-tile counts. */
cirrus_status cirrus_topology_refine_leafs_one_step(cirrus_topology* topo, cirrus_level_target_fn fn, void* user,
                                                    int* refined_per_level);
/* Replaces IterativeRefine(grid, level_target) (src/PoissonGrid.h:316-326). */
cirrus_status cirrus_topology_iterative_refine(cirrus_topology* topo, cirrus_level_target_fn fn, void* user);
/* IterativeRefine with level_target(tile) = level + (mask[level][(x*dy+y)*dz+z] != 0); masks[l]
 * may be NULL (never refine level l); dims holds 3 ints per layer. */
cirrus_status cirrus_topology_iterative_refine_masks(cirrus_topology* topo, const uint8_t* const* masks, const int* dims);
cirrus_status cirrus_topology_num_tiles(const cirrus_topology* topo, int* num_tiles);
cirrus_status cirrus_topology_max_level(const cirrus_topology* topo, int* max_level);
/* Tiles in all-tiles order, 5 int32 each: level, x, y, z, type (src/HAGrid.h:538-556). */
cirrus_status cirrus_topology_tiles(const cirrus_topology* topo, int32_t* out5);
/* Hash slot of each tile inside its level's table (src/HAAccessor.h:225-242). */
cirrus_status cirrus_topology_hash_slots(const cirrus_topology* topo, int32_t* out);
/* Cell types, num_tiles*512 bytes in all-tiles order.  set: only LEAF tiles' entries are used. */
cirrus_status cirrus_topology_set_cell_types(cirrus_topology* topo, const uint8_t* ctypes);
cirrus_status cirrus_topology_cell_types(const cirrus_topology* topo, uint8_t* ctypes);
/* Replaces CalcCellTypesFromLeafs(grid) (src/PoissonSolver.cu:7-61). */
cirrus_status cirrus_topology_calc_cell_types_from_leafs(cirrus_topology* topo);
/* Replaces CalculateNeighborTiles(grid) (src/PoissonGrid.cu:121-134): 6 int32 per tile
 * (x-, y-, z-, x+, y+, z+), the neighbour's all-tiles index or -1. */
cirrus_status cirrus_topology_neighbor_tiles(const cirrus_topology* topo, int32_t* out6);

/* ------------------------------------------------------------------------------------------
 * Device-resident topology: the same octree construction on the GPU.  The reference rebuilds
 * its grid every step with device kernels for the per-tile decisions and host loops for the
 * hash-table edits, one cudaMalloc per new tile (RefineLeafsOneStep and CoarsenStep,
 * src/PoissonGrid.h:35-314; SpawnGhostTiles, src/PoissonGrid.cu:30-60; compressHost /
 * syncHostAndDevice, src/HAGrid.h:491-561; CalcCellTypesFromLeafs, src/PoissonSolver.cu:7-61).
 * Here the tables, tile statuses and cell types stay in device memory: decisions are parallel
 * kernels, the order-dependent table edits (linear-probing insertion, removeTileHost's
 * backward-shift deletion) are applied in the reference's order by one warp, and the host reads
 * back only per-level counts.  Tile order (hash-slot order), statuses and cell types are those of
 * the host topology and of the reference.  Level targets come as dense per-level masks (as
 * cirrus_topology_iterative_refine_masks): refine when mask != 0 (target = level + 1); for
 * CoarsenStep a LEAF tile with mask != 0 has target level - 1.  Calls synchronise the device.
 * ---------------------------------------------------------------------------------------- */
typedef struct cirrus_dtopology cirrus_dtopology;

cirrus_status cirrus_dtopology_create(int num_layers, const uint32_t* log2_hash, double h0, cirrus_dtopology** out);
void cirrus_dtopology_destroy(cirrus_dtopology* topo);
/* setTileHost(level, (x, y, z), blank tile, type) for n tiles of one level, in order. */
cirrus_status cirrus_dtopology_set_tiles(cirrus_dtopology* topo, int level, const int32_t* xyz, const uint8_t* types, int n);
cirrus_status cirrus_dtopology_compress(cirrus_dtopology* topo);
cirrus_status cirrus_dtopology_spawn_ghost_tiles(cirrus_dtopology* topo);
cirrus_status cirrus_dtopology_refine_leafs_one_step(cirrus_dtopology* topo, const uint8_t* const* masks, const int* dims,
                                                     int* refined_per_level);
cirrus_status cirrus_dtopology_iterative_refine(cirrus_dtopology* topo, const uint8_t* const* masks, const int* dims);
cirrus_status cirrus_dtopology_coarsen_step(cirrus_dtopology* topo, const uint8_t* const* masks, const int* dims,
                                            int* deleted_per_level);
/* Cell types of all tiles in all-tiles order (num_tiles*512 bytes). */
cirrus_status cirrus_dtopology_set_cell_types(cirrus_dtopology* topo, const uint8_t* ctypes);
cirrus_status cirrus_dtopology_calc_cell_types_from_leafs(cirrus_dtopology* topo);
cirrus_status cirrus_dtopology_num_tiles(const cirrus_dtopology* topo, int* num_tiles);
cirrus_status cirrus_dtopology_max_level(const cirrus_dtopology* topo, int* max_level);
/* Exports in all-tiles order: tiles (level, x, y, z, type), hash slots, cell types, status words
 * (the reference's mStatus: REFINE 1, DELETE 2, COARSEN 4). */
cirrus_status cirrus_dtopology_tiles(const cirrus_dtopology* topo, int32_t* out5);
cirrus_status cirrus_dtopology_hash_slots(const cirrus_dtopology* topo, int32_t* out);
cirrus_status cirrus_dtopology_cell_types(const cirrus_dtopology* topo, uint8_t* ctypes);
cirrus_status cirrus_dtopology_statuses(const cirrus_dtopology* topo, int32_t* out);
/* A host topology holding the device topology's tiles (in its order) and cell types, from which
 * cirrus_grid_create builds the solver's tile pool. */
cirrus_status cirrus_dtopology_to_topology(const cirrus_dtopology* topo, cirrus_topology** out);

/* ------------------------------------------------------------------------------------------
 * Device grid: the tile pool resident in HBM (SoA channels, int32 topology tables).
 * ---------------------------------------------------------------------------------------- */
typedef struct cirrus_grid cirrus_grid;

/* Uploads a finalised topology (cell types set) to the current CUDA device. */
cirrus_status cirrus_grid_create(const cirrus_topology* topo, cirrus_grid** out);
/* Batched grid: `count` independent instances (finalised topologies, any sizes, depths and h0)
 * in one tile pool, solved together by cirrus_gmg_solve_batch.  No counterpart in the reference
 * (one HADeviceGrid per solve).  Pool order is level-major across the instances; inside a level,
 * instance by instance in each one's all-tiles order (a batch of one is the plain grid). */
cirrus_status cirrus_grid_create_batch(const cirrus_topology* const* topos, int count, cirrus_grid** out);
cirrus_status cirrus_grid_num_instances(const cirrus_grid* grid, int* count);
/* Tiles and DoF (INTERIOR cells of LEAF tiles) of one instance; either output may be NULL. */
cirrus_status cirrus_grid_instance_info(const cirrus_grid* grid, int instance, int* num_tiles, int64_t* dof);
/* Channel transfer of one instance: its num_tiles*512 floats in its own all-tiles order. */
cirrus_status cirrus_grid_set_channel_instance(cirrus_grid* grid, int instance, int channel, const float* host, void* stream);
cirrus_status cirrus_grid_get_channel_instance(const cirrus_grid* grid, int instance, int channel, float* host, void* stream);
void cirrus_grid_destroy(cirrus_grid* grid);
/* Grid descriptor: a reference grid's content as plain arrays -- its tile list per level in the
 * reference's compacted order (the dAllTiles order, src/HAGrid.h:538-556), tile types, cell types
 * (CalcCellTypesFromLeafs applied, src/PoissonSolver.cu:7-61) and optionally b and x0.  The
 * library builds its own neighbour, parent and child tables from the coordinates. */
typedef struct cirrus_grid_desc {
    double h0;                       /* voxel size of level 0 (HADeviceGrid's h0) */
    int num_layers;
    const uint32_t* log2_hash;       /* num_layers: log2 of each level's hash-table size */
    const int32_t* tiles_per_level;  /* num_layers */
    const int32_t* coords;           /* 3 int32 (x, y, z) per tile: level 0's tiles first */
    const uint8_t* types;            /* per tile: CIRRUS_LEAF, CIRRUS_NONLEAF or CIRRUS_GHOST */
    const uint8_t* cell_types;       /* 512 per tile */
    const float* b;                  /* optional (NULL): 512 per tile, loaded into channel 1 */
    const float* x0;                 /* optional (NULL): 512 per tile, loaded into channel 0 */
} cirrus_grid_desc;
/* One call from a descriptor to a device grid: cirrus_topology_create + _import_tiles +
 * _set_cell_types + cirrus_grid_create (+ the channel uploads, synchronous).  Replaces building a
 * HADeviceGrid tile by tile when the tiles already exist elsewhere. */
cirrus_status cirrus_grid_create_from_desc(const cirrus_grid_desc* desc, cirrus_grid** out);
cirrus_status cirrus_grid_num_tiles(const cirrus_grid* grid, int* num_tiles);
/* Device bytes held by the grid. */
cirrus_status cirrus_grid_device_bytes(const cirrus_grid* grid, size_t* bytes);
/* Number of DoF: INTERIOR cells of LEAF tiles. */
cirrus_status cirrus_grid_dof(const cirrus_grid* grid, int64_t* dof);
/* Channel transfer, num_tiles*512 floats in all-tiles order (host pointers; ordered on stream). */
cirrus_status cirrus_grid_set_channel(cirrus_grid* grid, int channel, const float* host, void* stream);
cirrus_status cirrus_grid_get_channel(const cirrus_grid* grid, int channel, float* host, void* stream);
/* Array-of-tiles interop: register one device pointer per tile (all-tiles order; 16-byte
 * aligned), e.g. the reference's HATileInfo::mTilePtr of every tile (src/HATileInfo.h:66-72).
 * The table is copied to the device; the tiles stay owned by the caller. */
cirrus_status cirrus_grid_set_tile_pointers(cirrus_grid* grid, const void* const* tile_ptrs);
/* Copy 512 floats at tile_ptr + byte_offset of every registered tile into `channel`, or back
 * (scatter), on the device.  For the reference's PoissonTile<float> channel c lies at
 * c * 736 * 4 bytes (src/PoissonTile.h:39,51). */
cirrus_status cirrus_grid_gather_tiles(cirrus_grid* grid, int channel, size_t byte_offset, void* stream);
cirrus_status cirrus_grid_scatter_tiles(cirrus_grid* grid, int channel, size_t byte_offset, void* stream);
/* Array-of-tiles cell types: copies the 512 cell-type bytes at tile_ptr + byte_offset of every
 * registered tile (the reference's PoissonTile<float>::mCellType, src/PoissonTile.h:54) into a
 * device buffer of the grid and compares them, on the device, with the cell types the grid was
 * built from.  *changed = 1 if any byte differs, else 0.  When it differs and host_types is not
 * NULL, the gathered types (num_tiles*512 bytes, all-tiles order) are copied to host_types, ready
 * for cirrus_topology_set_cell_types and a rebuild of the grid (the stencil masks derive from
 * them).  byte_offset must be a multiple of 4.  Synchronises `stream`.  The reference rewrites
 * mCellType every step (CalcCellTypesFromLeafs, src/FluidEuler.h:934) without changing tiles, so
 * a caller that keeps a grid across steps checks this before each solve. */
cirrus_status cirrus_grid_compare_tile_cell_types(cirrus_grid* grid, size_t byte_offset, void* stream, int* changed,
                                                 uint8_t* host_types);
/* The 512 bytes at tile_ptrs[i] + byte_offset of num_tiles device tiles (e.g. every tile's
 * mCellType) into host_out (num_tiles*512 bytes), with one gather kernel and one copy through
 * temporary device buffers, instead of a copy per tile.  byte_offset a multiple of 4, tile
 * pointers 4-byte aligned.  Synchronises `stream`. */
cirrus_status cirrus_gather_tile_bytes(const void* const* tile_ptrs, int num_tiles, size_t byte_offset, uint8_t* host_out,
                                       void* stream);
/* Device-to-device copy of a whole channel, ordered on `stream` (asynchronous). */
cirrus_status cirrus_grid_copy_channel(cirrus_grid* grid, int dst_channel, int src_channel, void* stream);
/* Device pointer of a channel (num_tiles*512 floats), for zero-copy integration. */
cirrus_status cirrus_grid_channel_ptr(cirrus_grid* grid, int channel, float** device_ptr);

/* ------------------------------------------------------------------------------------------
 * Operators (the reference's public solver functions)
 * ---------------------------------------------------------------------------------------- */
/* FullNegativeLaplacian(grid, x_channel, Ax_channel) (src/GMGSolver.cu:203-213). */
cirrus_status cirrus_full_negative_laplacian(cirrus_grid* grid, int x_channel, int Ax_channel, void* stream);
/* FullNegativeLaplacian(grid, x_channel, Ax_channel, calc_diag) with the reference's calc_diag
 * argument (src/GMGSolver.h:13): calc_diag != 0 gives the diagonal of the same operator
 * (GHOST rows accumulated into their parents as for A x). */
cirrus_status cirrus_full_negative_laplacian_ex(cirrus_grid* grid, int x_channel, int Ax_channel, int calc_diag, void* stream);
/* NegativeLaplacianSameLevel128(grid, tiles, n, subtree_level, launch_tile_types, x_channel,
 * Ax_channel, calc_diag) (src/GMGSolver.h:7, src/GMGSolver.cu:145-201).  tile_level selects the
 * tile array: -1 = all tiles (grid.dAllTiles), l >= 0 = the tiles of level l
 * (grid.dTileArrays[l]).  A tile is computed when its subtreeType(subtree_level) -- NONLEAF at
 * that level counts as LEAF -- is in launch_tile_types (CIRRUS_LEAF | CIRRUS_NONLEAF |
 * CIRRUS_GHOST bits); it gets A x (or the diagonal) on all 512 cells, 0 on non-INTERIOR cells.
 * No ghost propagation or accumulation (FullNegativeLaplacian adds those). */
cirrus_status cirrus_negative_laplacian_same_level(cirrus_grid* grid, int tile_level, int subtree_level, int launch_tile_types,
                                                   int x_channel, int Ax_channel, int calc_diag, void* stream);
/* One red-black colour sweep on LEAF|NONLEAF tiles of `level`
 * (NegativeLaplacianAndGaussSeidelSameLevel128, src/GMGSolver.cu:216-274). */
cirrus_status cirrus_gauss_seidel_sweep(cirrus_grid* grid, int level, int x_channel, int rhs_channel, int color, void* stream);
/* ResidualAndRestrict (src/GMGSolver.cu:284-343) from `level` into level-1. */
cirrus_status cirrus_residual_and_restrict(cirrus_grid* grid, int level, int x_channel, int rhs_channel,
                                           int coarse_channel, float one_over_alpha, void* stream);
/* ProlongateAndUpdate128 (src/GMGSolver.cu:345-380) into `fine_level`. */
cirrus_status cirrus_prolongate_and_update(cirrus_grid* grid, int fine_level, int coarse_channel, int fine_channel,
                                           float prolong_coeff, void* stream);
/* GMGSolver::VCycle (src/GMGSolver.cu:383-447). */
cirrus_status cirrus_vcycle(cirrus_grid* grid, int x_channel, int f_channel, int rhs_channel, int level_iters,
                            int coarsest_iters, void* stream);
/* Dot over LEAF tiles (src/PoissonGrid.cu:199-228); synchronises `stream`. */
cirrus_status cirrus_dot(cirrus_grid* grid, int a_channel, int b_channel, double* result, void* stream);

/* Allocation-free LEAF dot product.  No counterpart in the reference: its Dot reduces through
 * buffers allocated with the grid.  For callers that cannot call cudaMalloc at this point --
 * cudaMalloc/cudaFree may synchronise the device, fail when the memory budget is spent, or be
 * off-limits inside a caller's allocator or memory-pool callbacks -- and for callers that keep
 * their tiles in their own memory and hold no cirrus_grid.  The result is bit-identical to
 * cirrus_dot on a grid whose LEAF tiles are leaf_tiles (same kernel, same block count).
 *   a, b        device pointers, 512 floats per tile (tile t at a + 512*t), 16-byte aligned
 *   leaf_tiles  device array of n_leaf tile indices (the LEAF tiles in all-tiles order)
 *   result      host pointer; the call synchronises `stream`
 * All reduction scratch is one static device array of the library (about 17 KB per device):
 * per-block partial sums for at most CIRRUS_NOALLOC_MAX_BLOCKS blocks, a result slot and a
 * ticket counter that must be 0 when the kernel starts (the call zeroes it on `stream` first).
 * The call needs min(ceil(n_leaf/2), 4 x SM count) blocks and returns
 * CIRRUS_ERR_INVALID_ARGUMENT, doing nothing, when that exceeds CIRRUS_NOALLOC_MAX_BLOCKS
 * (only on devices with more than 256 SMs).  The first call on each device looks up the
 * scratch address (cudaGetSymbolAddress); make it before any stream capture on that device.
 * The address is kept for the life of the process: after cudaDeviceReset (or any reset of the
 * device's primary context) it is stale, so do not call this function on that device again.
 * Calls that can overlap on one device (several host threads, or streams not ordered with each
 * other) share the scratch and race: serialise them.  Calls from one host thread never overlap,
 * since each returns only after its stream is synchronised. */
#define CIRRUS_NOALLOC_MAX_BLOCKS 1024
cirrus_status cirrus_leaf_dot_noalloc(const float* a, const float* b, const int32_t* leaf_tiles, int n_leaf,
                                      double* result, void* stream);

/* Right-hand side of the projection (the callers either side of the solve in FluidEuler::project).
 * Velocities are the three lower-face components in channels u, u+1, u+2. */
/* ClearAllNeumannNeighborFaces (src/FluidEuler.cu:43-60) on LEAF tiles. */
cirrus_status cirrus_clear_neumann_neighbor_faces(cirrus_grid* grid, int u_channel, void* stream);
/* PropagateToChildren(c, c, -1, GHOST, LAUNCH_SUBTREE, I|D|N) (src/PoissonGrid.cu:635-661). */
cirrus_status cirrus_propagate_to_children(cirrus_grid* grid, int channel, void* stream);
/* VelocityVolumeDivergenceOnLeafs (src/PoissonSolver.cu:66-142), including the accumulation of
 * GHOST fluxes into their LEAF parents. */
cirrus_status cirrus_velocity_volume_divergence_on_leafs(cirrus_grid* grid, int u_channel, int div_channel, void* stream);
/* AddGradientToFaceCenters(grid, p_channel, u_channel) (src/PoissonSolver.cu:144-206), the step
 * after the solve in FluidEuler::project (src/FluidEuler.h:607): p is propagated to GHOST cells,
 * the lower-face velocities of LEAF and GHOST tiles get (p1 - p0)/dh, and GHOST children are
 * accumulated into their LEAF parents. */
cirrus_status cirrus_add_gradient_to_face_centers(cirrus_grid* grid, int p_channel, int u_channel, void* stream);

/* ------------------------------------------------------------------------------------------
 * GMG-PCG solve (GMGSolver::solve, src/GMGSolver.cu:531-666)
 * ---------------------------------------------------------------------------------------- */
enum {
    CIRRUS_PRECISION_FP32 = 0,          /* the reference's arithmetic: FP32 vectors, FP64 scalars */
    CIRRUS_PRECISION_MIXED_FP64 = 1     /* FP32 V-cycle/matvec + FP64 defect correction           */
};

typedef struct cirrus_solve_params {
    int max_iters;              /* 1000 at the reference call site (src/FluidEuler.h:598) */
    double relative_tolerance;  /* 1e-6 */
    int level_iters;            /* 1 */
    int coarsest_iters;         /* 10 */
    int sync_stride;            /* 1 */
    int is_pure_neumann;        /* 0 / 1 */
    float one_over_alpha;       /* 1 (GMGSolver constructor) */
    float prolong_coeff;        /* 1 */
    int precision;              /* CIRRUS_PRECISION_* */
    int warm_start;             /* mixed mode: start from the x channel instead of 0 */
    double inner_tolerance;     /* mixed mode: the tightest relative tolerance an FP32 inner solve
                                   is asked for (each targets max(this, 0.9*tol/current residual));
                                   default 1e-7: the inner solves stop on FP32's recursive residual,
                                   which keeps falling, so a 1e-6 solve takes one inner solve */
    int max_outer_iters;        /* mixed mode: cap on defect-correction steps */
} cirrus_solve_params;

typedef struct cirrus_solve_result {
    int iters;                  /* PCG iterations (summed over inner solves in mixed mode) */
    int outer_iters;            /* defect-correction steps (0 in FP32 mode) */
    double rel_residual;        /* ||r||/||b|| of the recursively updated residual (FP32 mode),
                                   or of the FP64 true residual (mixed mode) */
    double true_rel_residual;   /* ||b - A x||/||b|| evaluated in FP64 (or -1 if not computed) */
    int status;                 /* cirrus_status of the solve */
    long long kernel_launches;  /* CUDA kernels the solve executed on the device */
} cirrus_solve_result;

/* How a grid's solves reach the GPU (no counterpart in the reference, which launches every kernel
 * from the host and reads the residual back each iteration).  CIRRUS_LAUNCH_GRAPH (the default):
 * the whole PCG loop is one CUDA graph with a device-side while node, captured on first use per
 * parameter set.  CIRRUS_LAUNCH_DIRECT: the same kernels launched one by one from the host, which
 * reads the per-instance scalars after each iteration -- for profilers and launch tracers that do
 * not follow kernels inside conditional graph nodes.  Results are bit-identical in both modes. */
enum { CIRRUS_LAUNCH_GRAPH = 0, CIRRUS_LAUNCH_DIRECT = 1 };
cirrus_status cirrus_grid_set_launch_mode(cirrus_grid* grid, int mode);
cirrus_status cirrus_grid_get_launch_mode(const cirrus_grid* grid, int* mode);

/* Fills params with the reference call site's values (src/FluidEuler.h:591-598). */
void cirrus_solve_params_default(cirrus_solve_params* params);

/* Solves -lap(x) = b on the device-resident grid: b in channel 1 of LEAF tiles, x written to
 * channel 0.  As in the reference, channel 1 is overwritten with the final residual and
 * channels 2-4 are scratch.  The solve runs as one CUDA graph launch on `stream`; the call
 * returns after the result scalars are on the host. */
cirrus_status cirrus_gmg_solve(cirrus_grid* grid, const cirrus_solve_params* params, void* stream,
                               cirrus_solve_result* result);

/* Solves every instance of a (batched) grid in one graph launch: one kernel per step for the whole
 * batch, per-instance CG scalars and stopping, the loop running until the last instance stops.
 * active (NULL = all): instances with 0 take no part and keep their channels; tolerances (NULL =
 * params->relative_tolerance): per-instance relative tolerance; pure_neumann (NULL =
 * params->is_pure_neumann): per-instance projection of r to zero mean.  results: one per
 * instance.  An instance's result is bit-identical whatever else is in the batch (per-instance
 * reductions in a fixed order).  cirrus_gmg_solve on a batched grid solves all instances and
 * reports instance 0. */
cirrus_status cirrus_gmg_solve_batch(cirrus_grid* grid, const cirrus_solve_params* params, const int* active,
                                     const double* tolerances, const int* pure_neumann, void* stream,
                                     cirrus_solve_result* results);

/* Solves every instance of `count` distinct grids at once: each grid's solve graph is launched on
 * a stream of the grid's own, forked from `stream` after its pending work and joined back into
 * it, so the grids' kernels share the GPU (one grid's latency-bound coarse-level launches overlap
 * another's large ones: 32 ring512 instances as two grids of 16 solve about 4 % faster than as
 * one grid of 32).  results: one per instance, grid after grid.  Each result is bit-identical to
 * that grid's cirrus_gmg_solve_batch.  Mixed precision (params->precision), whose outer loop
 * reads residuals on the host, drives each grid from a host thread of its own.  Returns after
 * every result is on the host.  No counterpart in the reference. */
cirrus_status cirrus_gmg_solve_grids(cirrus_grid* const* grids, int count, const cirrus_solve_params* params, void* stream,
                                     cirrus_solve_result* results);

/* ------------------------------------------------------------------------------------------
 * AMG variant of the preconditioner: replaces AMGSolver (src/AMGSolver.h:20-53).  Explicit
 * per-cell face coefficients (CalculateAMGCoefficients, src/AMGSolver.cu:37-108), coarse-level
 * coefficients and cell types formed from the children (CoarsenTypesAndAMGCoeffs, :110-204), the
 * V-cycle on them (VCycleAMG, :610-715) and GMGSolver::solve's PCG around it
 * (AMGSolver::solve, :722-853).  The reference keeps the coefficients in four tile channels and
 * rewrites the NONLEAF cell types in place; here both live in separate device planes, so the
 * grid's channels and cell types are untouched.  The reference's AMG file does not build in this
 * project's environment, so these results are checked against a CPU restatement only.
 * ---------------------------------------------------------------------------------------- */
/* AMGSolver::prepareTypesAndCoeffs (src/AMGSolver.cu:717-720); one_over_alpha as the
 * AMGSolver constructor's (1).  Required before the other AMG calls (CIRRUS_ERR_STATE). */
cirrus_status cirrus_amg_prepare(cirrus_grid* grid, float one_over_alpha, void* stream);
/* The prepared coefficients: coeffs (optional) 4 * num_tiles * 512 floats (the off-diagonal
 * coefficient of each cell's x-, y- and z- face, then the diagonal, each plane in all-tiles
 * order); types (optional) num_tiles * 512 AMG cell types.  Synchronises `stream`. */
cirrus_status cirrus_amg_coefficients(cirrus_grid* grid, float* coeffs, uint8_t* types, void* stream);
/* VCycleAMG(grid, x, f, tmp, rhs, level_iters, coarsest_iters, one_over_alpha, prolong_coeff)
 * (src/AMGSolver.cu:610-715); the four channels must differ. */
cirrus_status cirrus_amg_vcycle(cirrus_grid* grid, int x_channel, int f_channel, int tmp_channel, int rhs_channel, int level_iters,
                                int coarsest_iters, float one_over_alpha, float prolong_coeff, void* stream);
/* AMGSolver::solve(grid, verbose, max_iters, relative_tolerance, level_iters, coarsest_iters,
 * sync_stride, is_pure_neumann) (src/AMGSolver.cu:722-853): b in channel 1, x to channel 0, the
 * V-cycle using channels 3 and 5 as its scratch; params->one_over_alpha / prolong_coeff are the
 * AMGSolver's.  Precision, graphs and batches as cirrus_gmg_solve / _batch. */
cirrus_status cirrus_amg_solve(cirrus_grid* grid, const cirrus_solve_params* params, void* stream, cirrus_solve_result* result);
cirrus_status cirrus_amg_solve_batch(cirrus_grid* grid, const cirrus_solve_params* params, const int* active, const double* tolerances,
                                     const int* pure_neumann, void* stream, cirrus_solve_result* results);
/* cirrus_gmg_solve_grids with the AMG preconditioner: every grid prepared by cirrus_amg_prepare
 * (CIRRUS_ERR_STATE otherwise). */
cirrus_status cirrus_amg_solve_grids(cirrus_grid* const* grids, int count, const cirrus_solve_params* params, void* stream,
                                     cirrus_solve_result* results);

/* End-to-end variant for callers holding host arrays: copies b (num_tiles*512 floats, pinned or
 * pageable) to the device, solves, and copies x back into x_host. */
cirrus_status cirrus_gmg_solve_host(cirrus_grid* grid, const cirrus_solve_params* params, const float* b_host,
                                    float* x_host, void* stream, cirrus_solve_result* result);

/* Asynchronous form of cirrus_gmg_solve_host for pipelines (no counterpart in the reference):
 * enqueues on `stream` the copy of b_host to the device, the solve (one graph launch for every
 * instance of the grid) and the copy of x into x_host, and returns without waiting.  Both host
 * arrays must stay valid and untouched until cirrus_gmg_solve_host_wait returns; pinned memory
 * makes the copies asynchronous.  cirrus_gmg_solve_host_wait synchronises the stream and writes
 * one result per instance.  One solve in flight per grid (a second submit first waits for the
 * previous one, discarding its results); to overlap one batch's transfers with another batch's
 * solve, alternate between two grids of the same problems, each with its own stream.  Mixed
 * precision runs to completion inside the submit (its outer loop reads residuals on the host). */
cirrus_status cirrus_gmg_solve_host_submit(cirrus_grid* grid, const cirrus_solve_params* params, const float* b_host,
                                           float* x_host, void* stream);
cirrus_status cirrus_gmg_solve_host_wait(cirrus_grid* grid, cirrus_solve_result* results);

/* The last solution in FP64 (num_tiles*512 doubles, all-tiles order): the FP64 iterate of a
 * mixed-precision solve, else channel 0 widened.  Channel 0 always holds its FP32 rounding. */
cirrus_status cirrus_grid_get_solution_f64(cirrus_grid* grid, double* host, void* stream);

/* Autotuner (no counterpart in the reference): times every launch shape (tiles per CTA, tiles in
 * flight per thread group) of the staged stencil kernels on this grid -- per kernel and level --
 * and keeps the fastest for the following solves.  On grids of at most 16,384 tiles (one
 * instance or a few, where a solve is a chain of latency-bound launches) it then refines the
 * choice with whole solves: 8-iteration solves of the grid's own right-hand sides (channel 1),
 * trying the eight common shapes for every kernel, per kernel each shape on all its levels, then
 * per V-cycle kernel and level each shape (about 1-2 s for one ring512 instance); b and x are
 * restored afterwards (skipped when the right-hand sides end a solve at once).  Shapes never
 * change results.  Overwrites channels 2-5 (the solve's scratch); synchronises `stream`; takes
 * about reps x (number of kernels x levels x shapes) launches plus, on small grids, a few hundred
 * short solves.  reps <= 0 picks 20. */
cirrus_status cirrus_grid_autotune(cirrus_grid* grid, int reps, void* stream);

/* Sweep-count tuner (no counterpart in the reference, which always runs the caller's
 * level_iters and coarsest_iters): solves the grid's current right-hand sides (channel 1, every
 * instance) with `params` -- its precision, tolerance and pure-Neumann flag -- once per candidate
 * (level_iters, coarsest_iters) in {(1,2), (1,4), (1,6), (1,10), (1,16), (1,24), (2,10)}, first
 * untimed (building that solve's graph) then timed, and writes to *best a copy of params with the
 * fastest pair whose solves all converged (CIRRUS_ERR_NOT_CONVERGED and params' own pair if none
 * did).  Sweep counts change the preconditioner and so the iterates: the reference's bits come
 * only from (1, 10).  Meant for the mixed-precision solver, whose result is set by its FP64
 * tolerance.  Channel 1 is restored; channels 0 and 2-5 keep the last trial's values.
 * Synchronises `stream`; holds one channel of scratch device memory while it runs. */
cirrus_status cirrus_grid_autotune_sweeps(cirrus_grid* grid, const cirrus_solve_params* params, void* stream,
                                          cirrus_solve_params* best);

/* Measurement hook: launches one kernel of the solve `reps` times back to back on `stream` (no
 * synchronisation), so a caller can time it with its own CUDA events on that stream.  Uses
 * channels 2-5 (the solve's scratch) and overwrites them.  level: the level of the per-level
 * kernels (ignored by the others).  No counterpart in the reference. */
enum {
    CIRRUS_KERNEL_LAPLACIAN = 0,        /* fused FullNegativeLaplacian over LEAF|GHOST tiles, with
                                           the p.Ap tile parts it forms in the solve                */
    CIRRUS_KERNEL_GS_SWEEP = 1,         /* one red-black colour sweep of a level, with the r.z tile
                                           parts it forms in the solve                              */
    CIRRUS_KERNEL_PRESMOOTH = 2,        /* two-colour pre-smoothing from x = 0 of a level           */
    CIRRUS_KERNEL_PROLONG_SWEEP = 3,    /* prolongation + first post-smoothing colour of a level    */
    CIRRUS_KERNEL_RESIDUAL_RESTRICT = 4,/* residual and restriction of a level                      */
    CIRRUS_KERNEL_COARSE = 5,           /* the shared-memory coarse-level V-cycle                   */
    CIRRUS_KERNEL_DOT = 6               /* whole-grid LEAF dot product                              */
};
cirrus_status cirrus_bench_launch(cirrus_grid* grid, int kernel, int level, int reps, void* stream);

/* Launch shapes of the staged stencil kernels, as the autotuner sets them: kernel one of
 * CIRRUS_KERNEL_LAPLACIAN / _GS_SWEEP / _PRESMOOTH / _PROLONG_SWEEP / _RESIDUAL_RESTRICT (or -1:
 * all of them, shapes 0..7 only), level a level of the grid (or -1: all levels; the Laplacian
 * has one entry, level 0).  Shapes 0..7 (tiles per CTA, tiles in flight per thread group, minimum CTAs per SM)
 * exist for every kernel.  The V-cycle kernels add 8..11 (four of them also prefetching into L2
 * the tiles of the CTAs one resident wave later).  The Laplacian adds 8..11, its TMA-staged
 * pipeline (persistent CTAs, one producer warp issuing bulk tensor copies of each tile and its
 * halos into a ring of shared-memory stages, 1-4 consumer groups), 12..15, a column of eight cells
 * per thread (64 threads per tile), and 16..19, shapes 2, 3, 5 and 1 prefetching into L2.  Lets a
 * caller reuse tuned shapes for grids of the same structure or pin one.  Before any tuning a grid
 * runs shape 4 (one tile per 128-thread CTA).
 * Shapes never change results.  No counterpart in the reference. */
#define CIRRUS_NUM_LAUNCH_SHAPES 20
cirrus_status cirrus_grid_set_launch_shape(cirrus_grid* grid, int kernel, int level, int shape);
cirrus_status cirrus_grid_get_launch_shape(cirrus_grid* grid, int kernel, int level, int* shape);

/* Replaces GMGSolver::dampedJacobiSolve(grid, verbose, max_iters, relative_tolerance, omega)
 * (src/GMGSolver.cu:449-531; FluidEuler::project's commented-out alternative,
 * src/FluidEuler.h:599): x = 0; per iteration r = b - A x on INTERIOR cells of LEAF tiles
 * (channel 2), stop when ||r|| < relative_tolerance * ||b|| (||b|| over LEAF|NONLEAF|GHOST
 * tiles), else D = the diagonal (channel 3) and x += omega * r / D.  b in channel 1, x to
 * channel 0.  *iters and *rel: the reference's returned pair.  Grids of one instance. */
cirrus_status cirrus_damped_jacobi_solve(cirrus_grid* grid, int max_iters, double relative_tolerance, float omega, void* stream,
                                         int* iters, double* rel);

/* FP64 true residual ||b - A x||/||b|| over INTERIOR cells of LEAF tiles for a given b (host,
 * num_tiles*512 floats) and the last solution (FP64 after a mixed-precision solve, else the
 * FP32 channel 0); one value per instance (rel holds num_instances doubles). */
cirrus_status cirrus_true_residual(cirrus_grid* grid, const float* b_host, double* rel, void* stream);

/* ------------------------------------------------------------------------------------------
 * Tile-holder files: the reference's on-disk form of a grid's tiles, its checkpoint, warm-start
 * and interchange format (IOFunc::WriteHAHostTileHolderToFile / ReadHAHostTileHolderFromFile,
 * src/PoissonIOFunc.cu:38-121, over HAHostTileHolder<PoissonTile<float>>, src/HAGrid.h:74-92).
 * The file holds h0, the layer count and the finest level, the raw 33104-byte PoissonTile<float>
 * records (11 channels of 736 floats, neighbour infos, 512 cell types, flags) and per level the
 * tile infos (coordinates, level, type, record index).  Files written here are read by the
 * reference's reader and the other way round.
 * ---------------------------------------------------------------------------------------- */
typedef struct cirrus_holder cirrus_holder;

/* Reads a holder file (ReadHAHostTileHolderFromFile); CIRRUS_ERR_INVALID_ARGUMENT if it cannot be
 * opened or is truncated or inconsistent. */
cirrus_status cirrus_holder_read(const char* path, cirrus_holder** out);
/* Writes a holder file (WriteHAHostTileHolderToFile). */
cirrus_status cirrus_holder_write(const cirrus_holder* holder, const char* path);
void cirrus_holder_destroy(cirrus_holder* holder);
/* Any output may be NULL.  num_tiles counts the tile infos of all levels. */
cirrus_status cirrus_holder_info(const cirrus_holder* holder, double* h0, int* num_layers, int* max_level, int* num_tiles);
/* The holder's tiles level by level, each level in file order: level, x, y, z, type (5 int32). */
cirrus_status cirrus_holder_tiles(const cirrus_holder* holder, int32_t* tiles5);
/* Cell types (num_tiles*512 bytes) and one channel (0..10; num_tiles*512 floats, the first 512
 * of the record's 736), in the order of cirrus_holder_tiles. */
cirrus_status cirrus_holder_cell_types(const cirrus_holder* holder, uint8_t* out);
cirrus_status cirrus_holder_channel(const cirrus_holder* holder, int channel, float* out);
/* HADeviceGrid(h0, log2_hash) + setTilesFromHolder + compressHost (src/HAGrid.h:316-331, 491-561):
 * a topology of the holder's tiles, inserted level by level in file order into hash tables of the
 * given sizes, then compressed; cell types from the records.  order (optional, num_tiles int32)
 * receives each holder tile's index in the topology's all-tiles order. */
cirrus_status cirrus_topology_from_holder(const cirrus_holder* holder, const uint32_t* log2_hash, int num_layers, cirrus_topology** out,
                                          int32_t* order);
/* HADeviceGrid::getHostTileHolder(tile_types) (src/HAGrid.h:433-462) of a single-instance grid
 * and the topology it was created from: the tiles whose type is in tile_types, level by level in
 * all-tiles order, with channels 0..8 and the cell types copied from the device (channels 9, 10,
 * the neighbour infos and the flags zero).  Synchronous. */
cirrus_status cirrus_holder_from_grid(const cirrus_topology* topo, const cirrus_grid* grid, int tile_types, cirrus_holder** out);
/* Copies the holder's channels selected by channel_mask (bit c: channel c, 0..8) into the grid's
 * tiles at order[i] (from cirrus_topology_from_holder); other tiles keep their values.  A warm
 * start: load channel 0 and solve in mixed precision with warm_start = 1.  Synchronous. */
cirrus_status cirrus_grid_load_holder(cirrus_grid* grid, const cirrus_holder* holder, const int32_t* order, uint32_t channel_mask,
                                      void* stream);

/* ------------------------------------------------------------------------------------------
 * Serving loop with continuous batching (no counterpart in the reference): independent problems
 * ("sessions") whose solves arrive over time.  Sessions of similar size (classes of < 256,
 * < 1024 and < 4096 tiles) registered together share one batched tile pool of up to `pool_size`
 * instances and 8192 tiles; a session of 4096 tiles or more has a pool of its own (its solve fills
 * the GPU by itself).  Each launch serves one pool and takes the oldest waiting request of each
 * of its sessions, so requests that arrive while a pool is busy are merged into its next launch
 * -- one mixed-precision batched solve (FP64 defect correction from the session's previous
 * pressure to params->relative_tolerance) with the other instances inactive.  Per-instance
 * results do not depend on which other requests share the launch.  `slots` worker threads, each
 * with its own CUDA stream, run launches of different pools concurrently.  Pools are admitted
 * against an HBM budget; idle pools are evicted least recently used first, their sessions'
 * pressures kept on the host for the next warm start.  A session's solves run one at a time, in
 * submission order.
 * ---------------------------------------------------------------------------------------- */
typedef struct cirrus_server cirrus_server;

typedef struct cirrus_completion {
    uint64_t ticket;
    int session;
    int slot;
    int status;               /* cirrus_status of the solve (CIRRUS_ERR_BUDGET: larger than the budget) */
    int iters;                /* FP32 PCG iterations summed over the defect-correction steps */
    int outer_iters;
    int warm;                 /* 1 if the solve started from the session's previous pressure */
    double rel_residual;      /* FP64 true relative residual */
    double latency_ms;        /* submission to completion (host clock) */
    double device_ms;         /* its launch on the stream, b uploads to x downloads (CUDA events) */
    int batch;                /* requests solved together in that launch */
} cirrus_completion;

/* hbm_budget_bytes: device memory the pools may occupy; slots: concurrent launches; pool_size:
 * sessions per batched pool (1: every session in a pool of its own, no merging).
 * cirrus_server_create uses pool_size 8. */
cirrus_status cirrus_server_create_ex(size_t hbm_budget_bytes, int slots, int pool_size, cirrus_server** out);
cirrus_status cirrus_server_create(size_t hbm_budget_bytes, int slots, cirrus_server** out);
/* Launches run so far and the requests they carried (requests / launches = mean batch). */
cirrus_status cirrus_server_batch_stats(cirrus_server* server, long long* launches, long long* requests);
/* Finishes running solves, drops queued ones, frees every session's device state. */
void cirrus_server_destroy(cirrus_server* server);
/* Registers a problem (a finalised topology, which must stay valid while the server exists: its
 * pool may be re-created from it after an eviction); no device memory is taken until its pool is
 * first admitted. */
cirrus_status cirrus_server_add_session(cirrus_server* server, const cirrus_topology* topo, int* session);
/* Waits for the session's queued and running solves, then frees its device state. */
cirrus_status cirrus_server_close_session(cirrus_server* server, int session);
/* Queues a solve of the session: b_host (the session's num_tiles*512 floats, all-tiles order)
 * is read and x_host written when the solve runs; both must stay valid until its completion is
 * polled. */
cirrus_status cirrus_server_submit(cirrus_server* server, int session, const cirrus_solve_params* params, const float* b_host,
                                   float* x_host, uint64_t* ticket);
/* Up to max completions (oldest first); waits up to wait_ms for the first if none is ready. */
cirrus_status cirrus_server_poll(cirrus_server* server, cirrus_completion* out, int max, int* count, int wait_ms);
/* Resident bytes now and at peak, resident sessions, queued solves, evictions so far (any may be NULL). */
cirrus_status cirrus_server_stats(cirrus_server* server, size_t* resident_bytes, size_t* peak_bytes, int* resident_sessions,
                                  int* pending, long long* evictions);

#ifdef __cplusplus
}
#endif

#endif /* CIRRUS_B200_H */
