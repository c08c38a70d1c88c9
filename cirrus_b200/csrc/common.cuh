// Shared definitions of the device solver: constants, the per-tile metadata layout and the
// kernel-side view of a grid.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace cirrus {

constexpr int kTileCells = 512;
constexpr int kNumChannels = 9;       // x, b/r, p, Ap, z, tmp, u, v, w (PoissonTile channel ids)
constexpr int kChX = 0, kChB = 1, kChR = 1, kChP = 2, kChAp = 3, kChZ = 4, kChTmp = 5, kChU = 6;

constexpr uint8_t LEAF_T = 1, NONLEAF_T = 2, GHOST_T = 4;
constexpr uint8_t DIRICHLET_C = 1, INTERIOR_C = 2, NEUMANN_C = 4;

// Per-tile metadata, 8 int32: [0..5] same-level neighbour in the reference's stencil face order
// (x-, x+, y-, y+, z-, z+) or -1, [6] parent tile or -1, [7] packed = level | type << 8 |
// octant << 16 | (neighbour f is GHOST) << (24 + f)  (octant = child offset inside the parent,
// bit0 x, bit1 y, bit2 z).
struct __align__(16) TileMeta {
    int nb[6];
    int parent;
    int packed;
};
__host__ __device__ inline int meta_level(int packed) { return packed & 0xff; }
__host__ __device__ inline int meta_type(int packed) { return (packed >> 8) & 0xff; }
__host__ __device__ inline int meta_octant(int packed) { return (packed >> 16) & 0x7; }
__host__ __device__ inline bool meta_nb_ghost(int packed, int f) { return (packed >> (24 + f)) & 1; }

// Per-cell stencil mask byte: bit f (f in x-, x+, y-, y+, z-, z+) set when the face carries a
// non-zero coefficient, bit 6 set for INTERIOR cells.  Two contexts exist: the full-tree
// Laplacian (tile types as stored) and the multigrid level context (NONLEAF counts as LEAF at
// its own level).  Per tile, fcls holds the coefficient class of the six cross-tile faces:
// 2 bits per face, context lap in bits 0..11, mg in bits 12..23; class 1 = 1/h^2 (same level),
// class 2 = (2/3)/h^2 (leaf-ghost T-junction).
// Bit 7 is set when at least one face of the cell carries the (2/3)/h^2 coefficient, so a byte of
// exactly kMaskFull marks an INTERIOR cell with six 1/h^2 faces (the kernels' uniform fast path).
constexpr int kMaskInterior = 64;
constexpr int kMaskC2 = 128;
constexpr int kMaskFull = 0x7F;

// Scalar state of one PCG solve of one instance, resident in device memory (the reference keeps
// gamma, beta, alpha, gamma_old, fp, mean, count as 7 device doubles, src/GMGSolver.h:22-30).
struct Scalars {
    double rhs2, thr2, gamma, gamma_old, beta, alpha, fp, res2, mean, rel;
    int iter, iters, done, converged, nonfinite;
    int capped;  // reached max_iters unconverged; pure Neumann: stops after this iteration's recentring
};

// Per-instance parameters of one solve of a (batched) grid, written by the host before each solve.
struct InstParams {
    double tol;           // relative residual tolerance
    int max_iters;
    int active;           // 0: the instance takes no part in this solve (its channels stay untouched)
    int pure_neumann;     // project r to zero mean each iteration (ReCenterLeafVoxels)
    int pad;
};

// Kernel-side view of the topology tables of a device grid.  A grid holds one or more independent
// instances (a batch); tiles are ordered level-major across the batch and, inside a level and
// instance, in the instance's all-tiles order.
struct Topo {
    const uint8_t* ctype;        // n*512 cell types
    const uint8_t* mask_lap;     // n*512 stencil masks, full-tree Laplacian context
    const uint8_t* mask_mg;      // n*512 stencil masks, multigrid level context
    const TileMeta* meta;        // n
    const uint32_t* fcls;        // n cross-face coefficient classes
    const int* edge;             // n x 12 same-level edge neighbours (see Topology::edge_tiles)
    const int* ghost_slot;       // n: index of a GHOST tile in the ghost list, else -1
    const int* ghost_child;      // n x 8: ghost slot of the GHOST child in each octant, else -1
    const int* ghost_list;       // GHOST tile of each ghost slot
    const uint8_t* ghost_faces;  // per ghost slot: faces other tiles read (bit f: toward a non-GHOST
                                 // neighbour), bit 6: every cell is read
    const int* inst;             // n: instance of each tile
    const float* inst_h0;        // per instance: voxel size of level 0, stored in FP32 as the reference does
    const float4* lconst;        // per instance x kLevelSlots levels: h, c1, c2, fast-path diagonal
    const int* leafslot;         // n: position s of a LEAF tile in the LEAF list, stored as s for a
                                 // tile without GHOST children and as -2 - s for one with them; -1
                                 // for every other tile
    int pf;                      // per launch: the staged kernels also prefetch into L2 the tiles pf
                                 // list entries ahead of their own (0: no prefetching)
};
constexpr int kLevelSlots = 16;

__host__ __device__ inline float tile_h0(const Topo& tp, int tile) { return tp.inst_h0[tp.inst[tile]]; }
// true when the tile's instance has finished (or takes no part in) the running solve
__host__ __device__ inline bool tile_done(const Topo& tp, const Scalars* S, int tile) {
    return S != nullptr && S[tp.inst[tile]].done != 0;
}
}  // namespace cirrus
