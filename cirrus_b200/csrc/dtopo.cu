// Device-resident octree topology.  The reference rebuilds its adaptive grid every step with
// device kernels for the per-tile decisions and host loops for the hash-table edits (one
// cudaMalloc per new tile and host round trips in between): RefineLeafsOneStep and CoarsenStep
// (src/PoissonGrid.h:35-314), SpawnGhostTiles (src/PoissonGrid.cu:30-60), compressHost /
// syncHostAndDevice (src/HAGrid.h:491-561), CalcCellTypesFromLeafs (src/PoissonSolver.cu:7-61).
// Here everything stays on the GPU:
//   * per level two open-addressing tables of DSlot (the reference's host table, which edits go
//     to, and the device copy taken at the last sync, which the decision kernels read), with the
//     reference's hash and linear probing (src/HAAccessor.h:214-242); a tile's status word and
//     cell types live in device tile memory indexed by the slot's memory id;
//   * the per-tile decisions (refine / coarsen / delete flags, ghost candidates, cell types) are
//     data-parallel kernels;
//   * the table edits whose result depends on their order -- linear-probing insertion and the
//     backward-shift deletion of removeTileHost (src/HAGrid.h:409-431) -- are applied in the
//     reference's order by one warp, which probes 32 slots per step;
//   * compaction into hash-slot order (the reference's copy_if) is one ordered block scan per level.
// The host only reads back per-level counts.  Results: the same tiles, hash slots, statuses and
// cell types as the host Topology and the reference build (tests).
#include "dtopo.hpp"

#include "common.cuh"

#include <algorithm>
#include <cstring>

namespace cirrus {

namespace {

constexpr int kRefineFlag = 1, kDeleteFlag = 2, kCoarsenFlag = 4;  // src/PoissonTile.h:7
constexpr int kTypeShift = 24;
constexpr int kMemMask = (1 << kTypeShift) - 1;
__constant__ int c_nb[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};

__host__ __device__ __forceinline__ uint32_t slot_hash(int x, int y, int z, uint32_t log2) {
    uint32_t r = 0;
    r ^= (uint32_t)x * 1u;
    r ^= (uint32_t)y * 2654435761u;
    r ^= (uint32_t)z * 805459861u;
    return r & ((1u << log2) - 1u);
}
__device__ __forceinline__ int slot_type(const DSlot& s) { return s.meta < 0 ? 0 : (s.meta >> kTypeShift) & 0xff; }
__device__ __forceinline__ int slot_mem(const DSlot& s) { return s.meta & kMemMask; }

// Linear probing by one thread: the slot holding (x, y, z), or -1 (HATileAccessor::tileIdx +
// empty test).  At most `size` probes.
__device__ __forceinline__ int find_slot(const DSlot* t, uint32_t log2, int x, int y, int z) {
    const uint32_t mask = (1u << log2) - 1u;
    uint32_t k = slot_hash(x, y, z, log2);
    for (uint32_t n = 0; n <= mask; n++, k = (k + 1) & mask) {
        const DSlot s = t[k];
        if (s.meta < 0) return -1;
        if (s.x == x && s.y == y && s.z == z) return (int)k;
    }
    return -1;
}

// level target from dense per-level masks: mask[l][(x*dy + y)*dz + z] != 0, 0 outside
__device__ __forceinline__ bool mask_at(uint8_t* const* masks, const int* dims, int l, int x, int y, int z) {
    const uint8_t* m = masks[l];
    if (!m) return false;
    const int dx = dims[3 * l], dy = dims[3 * l + 1], dz = dims[3 * l + 2];
    if (x < 0 || y < 0 || z < 0 || x >= dx || y >= dy || z >= dz) return false;
    return m[((size_t)x * dy + y) * dz + z] != 0;
}

// Ordered compaction of the occupied slots of one table into `out`, one block of 1024 threads
// walking the table in chunks (the reference's thrust::copy_if keeps slot order).
__global__ void __launch_bounds__(1024) k_compact_table(const DSlot* __restrict__ t, uint32_t size, DSlot* out, int* count) {
    __shared__ int warp_tot[32];
    __shared__ int base;
    if (threadIdx.x == 0) base = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (uint32_t c0 = 0; c0 < size; c0 += 1024) {
        const uint32_t i = c0 + threadIdx.x;
        DSlot s;
        s.meta = -1;
        if (i < size) s = t[i];
        const bool occ = s.meta >= 0;
        const unsigned b = __ballot_sync(0xffffffffu, occ);
        if (lane == 0) warp_tot[w] = __popc(b);
        __syncthreads();
        int before = 0, total = 0;
        for (int k = 0; k < 32; k++) {
            const int v = warp_tot[k];
            if (k < w) before += v;
            total += v;
        }
        if (occ) out[base + before + __popc(b & ((1u << lane) - 1u))] = s;
        __syncthreads();
        if (threadIdx.x == 0) base += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) *count = base;
}

// Ordered compaction of flag indices: out[k] = the k-th i with flags[i] != 0 (one block).
__global__ void __launch_bounds__(1024) k_compact_flags(const int* __restrict__ flags, int n, int* out, int* count) {
    __shared__ int warp_tot[32];
    __shared__ int base;
    if (threadIdx.x == 0) base = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int c0 = 0; c0 < n; c0 += 1024) {
        const int i = c0 + (int)threadIdx.x;
        const bool on = i < n && flags[i] != 0;
        const unsigned b = __ballot_sync(0xffffffffu, on);
        if (lane == 0) warp_tot[w] = __popc(b);
        __syncthreads();
        int before = 0, total = 0;
        for (int k = 0; k < 32; k++) {
            const int v = warp_tot[k];
            if (k < w) before += v;
            total += v;
        }
        if (on) out[base + before + __popc(b & ((1u << lane) - 1u))] = i;
        __syncthreads();
        if (threadIdx.x == 0) base += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) *count = base;
}

enum { kInsSet = 0, kInsIfAbsent = 1 };

// setTileHost (src/HAGrid.h:387-407) for a sequence of requests, in order, by one warp.  Request
// r: coordinates and type req[r] = {x, y, z, type | octant << 8}, source tile memory src[r] (-1:
// a blank tile; else the parent whose childTile(octant) the new tile receives, src/PoissonTile.h:170-191:
// its status and, per child cell, the parent cell's type).  kInsSet: an existing tile is
// overwritten (type and memory); kInsIfAbsent: an existing tile is left alone (SpawnGhostTiles'
// empty test).  Each probe step reads 32 consecutive slots; the first that is empty or holds the
// coordinates ends the probe, as in linear probing.
__global__ void __launch_bounds__(32) k_insert(DSlot* table, uint32_t log2, const int4* __restrict__ req, const int* __restrict__ src,
                                               int n, int mode, int32_t* status, uint8_t* ctype, int* mem_count, int mem_cap,
                                               unsigned int* err) {
    const int lane = threadIdx.x;
    const uint32_t size = 1u << log2, mask = size - 1u;
    int mc = *mem_count;
    for (int r = 0; r < n; r++) {
        const int4 q = req[r];
        const int type = q.w & 0xff, oct = (q.w >> 8) & 7;
        const uint32_t h = slot_hash(q.x, q.y, q.z, log2);
        int found = -1;
        bool empty = false;
        for (uint32_t base = 0; base < size; base += 32) {
            const uint32_t k = (h + base + (uint32_t)lane) & mask;
            const DSlot s = table[k];
            const bool e = s.meta < 0, hit = !e && s.x == q.x && s.y == q.y && s.z == q.z;
            const unsigned b = __ballot_sync(0xffffffffu, (e || hit) && base + (uint32_t)lane < size);
            if (b) {
                const int first = __ffs(b) - 1;
                found = (int)((h + base + (uint32_t)first) & mask);
                empty = __shfl_sync(0xffffffffu, e, first);
                break;
            }
        }
        if (found < 0) {  // table full
            if (lane == 0) atomicOr(err, 1u);
            break;
        }
        if (!empty && mode == kInsIfAbsent) continue;
        int mem;
        if (empty) {
            if (mc >= mem_cap) {
                if (lane == 0) atomicOr(err, 2u);
                break;
            }
            mem = mc++;
        } else {
            mem = slot_mem(table[found]);
        }
        // the tile memory: blank, or the parent's childTile(octant)
        const int sm = src[r];
        int32_t st = 0;
        uint8_t bytes[16];
        if (sm >= 0) {
            st = status[sm];
            const int ox = oct & 1, oy = (oct >> 1) & 1, oz = (oct >> 2) & 1;
#pragma unroll
            for (int e = 0; e < 16; e++) {
                const int c = lane * 16 + e, a = c >> 6, bb = (c >> 3) & 7, cc = c & 7;
                const int pc = (((ox * 8 + a) >> 1) << 6) | (((oy * 8 + bb) >> 1) << 3) | ((oz * 8 + cc) >> 1);
                bytes[e] = ctype[(size_t)sm * kTileCells + pc];
            }
        } else {
#pragma unroll
            for (int e = 0; e < 16; e++) bytes[e] = 0;
        }
        __syncwarp();  // every lane has read the source before the destination is written
        uint4 v;
        memcpy(&v, bytes, 16);
        *reinterpret_cast<uint4*>(ctype + (size_t)mem * kTileCells + lane * 16) = v;
        if (lane == 0) {
            status[mem] = st;
            DSlot s;
            s.x = q.x;
            s.y = q.y;
            s.z = q.z;
            s.meta = mem | (type << kTypeShift);
            table[found] = s;
        }
        __syncwarp();
    }
    if (lane == 0) *mem_count = mc;
}

// CoarsenStep's table edits for one level, in array order, by one thread (src/PoissonGrid.h:280-305):
// op[r] = {x, y, z, 1: removeTileHost with its backward shift (src/HAGrid.h:409-431) | 2: set LEAF}.
__global__ void k_edit_serial(DSlot* table, uint32_t log2, const int4* __restrict__ op, int n, unsigned int* err) {
    if (threadIdx.x != 0) return;
    const uint32_t mask = (1u << log2) - 1u;
    for (int r = 0; r < n; r++) {
        const int4 q = op[r];
        const int s = find_slot(table, log2, q.x, q.y, q.z);
        if (s < 0) continue;
        if (q.w == 2) {
            table[s].meta = slot_mem(table[s]) | (LEAF_T << kTypeShift);
            continue;
        }
        uint32_t i = (uint32_t)s, j = i;
        for (uint32_t guard = 0; guard <= mask; guard++) {
            j = (j + 1) & mask;
            const DSlot sj = table[j];
            if (sj.meta < 0) break;
            const uint32_t k = slot_hash(sj.x, sj.y, sj.z, log2);
            if ((j > i && (k <= i || k > j)) || (j < i && (k <= i && k > j))) {
                const DSlot si = table[i];
                table[i] = sj;
                table[j] = si;
                i = j;
            }
            if (guard == mask) atomicOr(err, 4u);
        }
        table[i].meta = -1;
    }
}

// ------------------------------------------------------------------ decision kernels
struct LevelView {
    const DSlot* const* snap;  // per level
    DSlot* const* live;
    const uint32_t* log2;
    int num_layers;
};

__device__ __forceinline__ const DSlot* snap_find(const LevelView& v, int l, int x, int y, int z) {
    if (l < 0 || l >= v.num_layers) return nullptr;
    const int s = find_slot(v.snap[l], v.log2[l], x, y, z);
    return s < 0 ? nullptr : &v.snap[l][s];
}
__device__ __forceinline__ DSlot* live_find(const LevelView& v, int l, int x, int y, int z) {
    if (l < 0 || l >= v.num_layers) return nullptr;
    const int s = find_slot(v.live[l], v.log2[l], x, y, z);
    return s < 0 ? nullptr : &v.live[l][s];
}

// RefineLeafsOneStep pass 1 (src/PoissonGrid.h:50-84): LEAF tiles of level i
__global__ void k_refine_leaf_flags(LevelView v, const DSlot* __restrict__ arr, int n, int i, int dev_max, uint8_t* const* masks,
                                    const int* dims, int32_t* status, int* flags) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const DSlot t = arr[j];
    flags[j] = 0;
    if (!(slot_type(t) & LEAF_T)) return;
    bool to_refine = mask_at(masks, dims, i, t.x, t.y, t.z);  // target level i + 1 > i
    if (i < dev_max)
        for (int ci = 0; ci < 8; ci++) {
            const DSlot* c = snap_find(v, i + 1, t.x * 2 + (ci & 1), t.y * 2 + ((ci >> 1) & 1), t.z * 2 + ((ci >> 2) & 1));
            if (c && (slot_type(*c) & GHOST_T) && (status[slot_mem(*c)] & kRefineFlag)) to_refine = true;
        }
    if (i + 1 >= v.num_layers) to_refine = false;
    int32_t& st = status[slot_mem(t)];
    st = to_refine ? (st | kRefineFlag) : (st & ~kRefineFlag);
    flags[j] = to_refine ? 1 : 0;
}
// pass 2 (:86-102): GHOST tiles of level i take the flag of any refined LEAF neighbour
__global__ void k_refine_ghost_flags(LevelView v, const DSlot* __restrict__ arr, int n, int i, int32_t* status) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const DSlot t = arr[j];
    if (!(slot_type(t) & GHOST_T)) return;
    bool rf = false;
    for (int f = 0; f < 6; f++) {
        const DSlot* nb = snap_find(v, i, t.x + c_nb[f][0], t.y + c_nb[f][1], t.z + c_nb[f][2]);
        if (nb && (slot_type(*nb) & LEAF_T) && (status[slot_mem(*nb)] & kRefineFlag)) rf = true;
    }
    int32_t& st = status[slot_mem(t)];
    st = rf ? (st | kRefineFlag) : (st & ~kRefineFlag);
}
// the host loop of the refine step (:104-129) for the refined tiles `idx`: the live entry becomes
// NONLEAF, and 8 child requests (childTile of the parent's memory) in child order
__global__ void k_refine_requests(LevelView v, const DSlot* __restrict__ arr, const int* __restrict__ idx, int n, int i, int4* req,
                                  int* src) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const DSlot t = arr[idx[r]];
    DSlot* h = live_find(v, i, t.x, t.y, t.z);
    int mem = slot_mem(t);
    if (h) {
        h->meta = slot_mem(*h) | (NONLEAF_T << kTypeShift);
        mem = slot_mem(*h);
    }
    for (int ci = 0; ci < 8; ci++) {
        req[8 * r + ci] = make_int4(t.x * 2 + (ci & 1), t.y * 2 + ((ci >> 1) & 1), t.z * 2 + ((ci >> 2) & 1), LEAF_T | (ci << 8));
        src[8 * r + ci] = mem;
    }
}
// SpawnGhostTiles candidates of level l (src/PoissonGrid.cu:36-56): for every LEAF|NONLEAF tile
// of the compacted array and each face neighbour whose parent is a LEAF of the live level l-1
// table; the insertion skips those that exist by then.
__global__ void k_ghost_candidates(LevelView v, const DSlot* __restrict__ arr, int n, int l, int* flags, int4* cand) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= 6 * n) return;
    const int j = q / 6, f = q % 6;
    const DSlot t = arr[j];
    flags[q] = 0;
    if (!(slot_type(t) & (LEAF_T | NONLEAF_T))) return;
    const int nx = t.x + c_nb[f][0], ny = t.y + c_nb[f][1], nz = t.z + c_nb[f][2];
    const DSlot* p = live_find(v, l - 1, nx >> 1, ny >> 1, nz >> 1);
    if (p && (slot_type(*p) & LEAF_T)) {
        flags[q] = 1;
        cand[q] = make_int4(nx, ny, nz, GHOST_T);
    }
}
__global__ void k_gather_requests(const int* __restrict__ idx, int n, const int4* __restrict__ cand, int4* req, int* src) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    req[r] = cand[idx[r]];
    src[r] = -1;
}

// CoarsenStep flags (src/PoissonGrid.h:172-276)
__device__ __forceinline__ void set_mask(int32_t& st, int m, bool on) { st = on ? (st | m) : (st & ~m); }
__global__ void k_coarsen_nonleaf(LevelView v, const DSlot* __restrict__ arr, int n, int l, int32_t* status) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const DSlot t = arr[j];
    if (!(slot_type(t) & NONLEAF_T)) return;
    bool to_coarsen = true;
    for (int ci = 0; ci < 8; ci++) {
        const DSlot* c = snap_find(v, l + 1, t.x * 2 + (ci & 1), t.y * 2 + ((ci >> 1) & 1), t.z * 2 + ((ci >> 2) & 1));
        const int ct = c ? slot_type(*c) : 0;
        if (ct & LEAF_T) {
            if (!(status[slot_mem(*c)] & kDeleteFlag)) to_coarsen = false;
        } else {
            to_coarsen = false;
        }
    }
    int32_t& st = status[slot_mem(t)];
    set_mask(st, kCoarsenFlag, to_coarsen);
    set_mask(st, kDeleteFlag, false);
}
__global__ void k_coarsen_leaf(LevelView v, const DSlot* __restrict__ arr, int n, int l, uint8_t* const* masks, const int* dims,
                               int32_t* status) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const DSlot t = arr[j];
    if (!(slot_type(t) & LEAF_T)) return;
    bool to_delete = mask_at(masks, dims, l, t.x, t.y, t.z);  // target level l - 1 < l
    for (int f = 0; f < 6; f++) {
        const DSlot* nb = snap_find(v, l, t.x + c_nb[f][0], t.y + c_nb[f][1], t.z + c_nb[f][2]);
        if (nb && (slot_type(*nb) & NONLEAF_T) && !(status[slot_mem(*nb)] & kCoarsenFlag)) to_delete = false;
    }
    int32_t& st = status[slot_mem(t)];
    set_mask(st, kCoarsenFlag, false);
    set_mask(st, kDeleteFlag, to_delete);
}
__global__ void k_coarsen_down(LevelView v, const DSlot* __restrict__ arr, int n, int l, int32_t* status) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const DSlot t = arr[j];
    if (!(slot_type(t) & (LEAF_T | GHOST_T))) return;
    bool to_delete = false;
    const DSlot* p = snap_find(v, l - 1, t.x >> 1, t.y >> 1, t.z >> 1);
    if (p && (status[slot_mem(*p)] & kCoarsenFlag)) to_delete = true;
    int32_t& st = status[slot_mem(t)];
    set_mask(st, kDeleteFlag, to_delete);
    if (to_delete) set_mask(st, kCoarsenFlag, true);
}
__global__ void k_coarsen_ghost(LevelView v, const DSlot* __restrict__ arr, int n, int l, int32_t* status) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const DSlot t = arr[j];
    if (!(slot_type(t) & GHOST_T)) return;
    bool to_delete = true;
    for (int f = 0; f < 6; f++) {
        const DSlot* nb = snap_find(v, l, t.x + c_nb[f][0], t.y + c_nb[f][1], t.z + c_nb[f][2]);
        if (nb && (slot_type(*nb) & LEAF_T) && !(status[slot_mem(*nb)] & kDeleteFlag)) to_delete = false;
    }
    if (to_delete) status[slot_mem(t)] |= kDeleteFlag;
}
// the deletion loop's requests for one level, in array order (:280-305)
__global__ void k_coarsen_ops(const DSlot* __restrict__ arr, int n, const int32_t* __restrict__ status, int* flags, int4* ops) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const DSlot t = arr[j];
    const int32_t st = status[slot_mem(t)];
    flags[j] = 0;
    if (st & kDeleteFlag) {
        flags[j] = 1;
        ops[j] = make_int4(t.x, t.y, t.z, 1);
    } else if (st & kCoarsenFlag) {
        flags[j] = 1;
        ops[j] = make_int4(t.x, t.y, t.z, 2);
    }
}
__global__ void k_gather_ops(const int* __restrict__ idx, int n, const int4* __restrict__ ops, int4* out) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < n) out[r] = ops[idx[r]];
}

// CalcCellTypesFromLeafs (src/PoissonSolver.cu:7-61).  Step 1, one level at a time from fine to
// coarse, one block per NONLEAF tile: a cell is DIRICHLET if any LEAF|NONLEAF child cell is, else
// INTERIOR if any is, else NEUMANN.
__global__ void __launch_bounds__(128) k_celltypes_nonleaf(LevelView v, const DSlot* __restrict__ arr, int n, int l, uint8_t* ctype) {
    __shared__ int child_mem[8];
    const int j = blockIdx.x;
    if (j >= n) return;
    const DSlot t = arr[j];
    if (!(slot_type(t) & NONLEAF_T)) return;
    if (threadIdx.x < 8) {
        const int ci = threadIdx.x;
        const DSlot* c = snap_find(v, l + 1, t.x * 2 + (ci & 1), t.y * 2 + ((ci >> 1) & 1), t.z * 2 + ((ci >> 2) & 1));
        child_mem[ci] = (c && (slot_type(*c) & (LEAF_T | NONLEAF_T))) ? slot_mem(*c) : -1;
    }
    __syncthreads();
    uint8_t* out = ctype + (size_t)slot_mem(t) * kTileCells;
    for (int o = threadIdx.x; o < kTileCells; o += blockDim.x) {
        const int i = o >> 6, jj = (o >> 3) & 7, k = o & 7;
        int dcnt = 0, icnt = 0;
        for (int c = 0; c < 8; c++) {
            const int gx = (i * 2 + (c & 1)), gy = (jj * 2 + ((c >> 1) & 1)), gz = (k * 2 + ((c >> 2) & 1));
            // the child tile holding fine cell (gx, gy, gz) of this tile's 16^3 refinement
            const int cm = child_mem[(gx >> 3) | ((gy >> 3) << 1) | ((gz >> 3) << 2)];
            if (cm < 0) continue;
            const uint8_t tt = ctype[(size_t)cm * kTileCells + ((gx & 7) << 6) + ((gy & 7) << 3) + (gz & 7)];
            if (tt & DIRICHLET_C) dcnt++;
            else if (tt & INTERIOR_C) icnt++;
        }
        out[o] = dcnt > 0 ? DIRICHLET_C : (icnt > 0 ? INTERIOR_C : NEUMANN_C);
    }
}
// Step 2: a GHOST cell takes its parent cell's type, DIRICHLET without a parent tile.
__global__ void __launch_bounds__(128) k_celltypes_ghost(LevelView v, const DSlot* __restrict__ arr, int n, int l, uint8_t* ctype) {
    const int j = blockIdx.x;
    if (j >= n) return;
    const DSlot t = arr[j];
    if (!(slot_type(t) & GHOST_T)) return;
    const DSlot* p = snap_find(v, l - 1, t.x >> 1, t.y >> 1, t.z >> 1);
    const int pm = p ? slot_mem(*p) : -1;
    uint8_t* out = ctype + (size_t)slot_mem(t) * kTileCells;
    const int ox = t.x & 1, oy = t.y & 1, oz = t.z & 1;
    for (int o = threadIdx.x; o < kTileCells; o += blockDim.x) {
        const int i = o >> 6, jj = (o >> 3) & 7, k = o & 7;
        const int pc = (((ox * 8 + i) >> 1) << 6) | (((oy * 8 + jj) >> 1) << 3) | ((oz * 8 + k) >> 1);
        out[o] = pm >= 0 ? ctype[(size_t)pm * kTileCells + pc] : DIRICHLET_C;
    }
}

// exports: per compacted tile its memory id, hash slot (probe of the live table)
__global__ void k_slots_of(const DSlot* __restrict__ arr, int n, const DSlot* __restrict__ live, uint32_t log2, int32_t* slot, int32_t* mem) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const DSlot t = arr[j];
    slot[j] = find_slot(live, log2, t.x, t.y, t.z);
    mem[j] = slot_mem(t);
}
__global__ void k_copy_types(const int32_t* __restrict__ mem, int n, const uint8_t* __restrict__ ctype, uint8_t* out, int to_mem) {
    const int j = blockIdx.x;
    if (j >= n) return;
    const size_t m = (size_t)mem[j] * kTileCells, a = (size_t)j * kTileCells;
    for (int o = threadIdx.x * 4; o < kTileCells; o += blockDim.x * 4) {
        if (to_mem) *reinterpret_cast<uint32_t*>(const_cast<uint8_t*>(ctype) + m + o) = *reinterpret_cast<const uint32_t*>(out + a + o);
        else *reinterpret_cast<uint32_t*>(out + a + o) = *reinterpret_cast<const uint32_t*>(ctype + m + o);
    }
}
__global__ void k_gather_status(const int32_t* __restrict__ mem, int n, const int32_t* __restrict__ status, int32_t* out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < n) out[j] = status[mem[j]];
}

inline int blocks(int n, int b = 256) { return std::max(1, (n + b - 1) / b); }

#define DT_CK(x)                                                           \
    do {                                                                   \
        cudaError_t e_ = (x);                                              \
        if (e_ != cudaSuccess) {                                           \
            last_error = std::string(#x ": ") + cudaGetErrorString(e_);    \
            return e_ == cudaErrorMemoryAllocation ? 3 : 2;                \
        }                                                                  \
    } while (0)

}  // namespace

DevTopology::DevTopology(int num_layers, const uint32_t* log2_hash, double h0)
    : num_layers_(num_layers), h0_(h0), log2_(log2_hash, log2_hash + num_layers) {
    live_.assign(num_layers, nullptr);
    snap_.assign(num_layers, nullptr);
    arr_.assign(num_layers, nullptr);
    count_.assign(num_layers, 0);
    mask_bufs_.assign(num_layers, nullptr);
    bool ok = true;
    for (int l = 0; l < num_layers && ok; l++) {
        const size_t sz = sizeof(DSlot) << log2_[l];
        ok = cudaMalloc(&live_[l], sz) == cudaSuccess && cudaMalloc(&snap_[l], sz) == cudaSuccess &&
             cudaMalloc(&arr_[l], sz) == cudaSuccess;
        if (ok) {
            cudaMemset(live_[l], 0xff, sz);  // meta = -1: empty
            cudaMemset(snap_[l], 0xff, sz);
        }
    }
    ok = ok && cudaMalloc(&d_live_, sizeof(DSlot*) * num_layers) == cudaSuccess &&
         cudaMalloc(&d_snap_, sizeof(DSlot*) * num_layers) == cudaSuccess && cudaMalloc(&d_arr_, sizeof(DSlot*) * num_layers) == cudaSuccess &&
         cudaMalloc(&d_log2_, sizeof(uint32_t) * num_layers) == cudaSuccess && cudaMalloc(&d_count_, sizeof(int) * num_layers) == cudaSuccess &&
         cudaMalloc(&d_nflag_, sizeof(int) * 4) == cudaSuccess && cudaMalloc(&d_mem_count_, sizeof(int)) == cudaSuccess &&
         cudaMalloc(&d_masks_, sizeof(uint8_t*) * num_layers) == cudaSuccess &&
         cudaMalloc(&d_mask_dims_, sizeof(int) * 3 * num_layers) == cudaSuccess && cudaMalloc(&d_err_, sizeof(unsigned int)) == cudaSuccess;
    if (ok) {
        cudaMemcpy(d_live_, live_.data(), sizeof(DSlot*) * num_layers, cudaMemcpyHostToDevice);
        cudaMemcpy(d_snap_, snap_.data(), sizeof(DSlot*) * num_layers, cudaMemcpyHostToDevice);
        cudaMemcpy(d_arr_, arr_.data(), sizeof(DSlot*) * num_layers, cudaMemcpyHostToDevice);
        cudaMemcpy(d_log2_, log2_.data(), sizeof(uint32_t) * num_layers, cudaMemcpyHostToDevice);
        cudaMemset(d_count_, 0, sizeof(int) * num_layers);
        cudaMemset(d_mem_count_, 0, sizeof(int));
        cudaMemset(d_err_, 0, sizeof(unsigned int));
    }
    if (!ok) last_error = "device topology: allocation failed";
}

DevTopology::~DevTopology() {
    for (int l = 0; l < num_layers_; l++) {
        cudaFree(live_[l]);
        cudaFree(snap_[l]);
        cudaFree(arr_[l]);
        cudaFree(mask_bufs_[l]);
    }
    cudaFree(d_live_);
    cudaFree(d_snap_);
    cudaFree(d_arr_);
    cudaFree(d_log2_);
    cudaFree(d_count_);
    cudaFree(d_scratch_);
    cudaFree(d_nflag_);
    cudaFree(status_);
    cudaFree(ctype_);
    cudaFree(d_mem_count_);
    cudaFree(d_masks_);
    cudaFree(d_mask_dims_);
    cudaFree(d_err_);
}

int DevTopology::num_tiles() const {
    int n = 0;
    for (int c : count_) n += c;
    return n;
}

int DevTopology::ensure_mem(int extra) {
    if (mem_count_ + extra <= mem_cap_) return 0;
    const int cap = std::max(mem_count_ + extra, std::max(1024, mem_cap_ * 2));
    int32_t* st = nullptr;
    uint8_t* ct = nullptr;
    DT_CK(cudaMalloc(&st, sizeof(int32_t) * cap));
    DT_CK(cudaMalloc(&ct, (size_t)cap * kTileCells));
    if (mem_count_ > 0) {
        DT_CK(cudaMemcpy(st, status_, sizeof(int32_t) * mem_count_, cudaMemcpyDeviceToDevice));
        DT_CK(cudaMemcpy(ct, ctype_, (size_t)mem_count_ * kTileCells, cudaMemcpyDeviceToDevice));
    }
    cudaFree(status_);
    cudaFree(ctype_);
    status_ = st;
    ctype_ = ct;
    mem_cap_ = cap;
    return 0;
}

// scratch layout (int4 units): [0, cap) requests | [cap, 2cap) candidates/ops | then int arrays
// (flags, indices, sources) of cap entries each
static size_t scratch_int4(size_t cap) { return 2 * cap + (3 * cap + 3) / 4; }

int DevTopology::insert_requests(int level, int n, int mode, int /*src_level*/) {
    if (n <= 0) return 0;
    int rc = ensure_mem(n);
    if (rc) return rc;
    int4* req = reinterpret_cast<int4*>(d_scratch_);
    int* src = reinterpret_cast<int*>(reinterpret_cast<int4*>(d_scratch_) + 2 * scratch_cap_) + 2 * scratch_cap_;
    k_insert<<<1, 32>>>(live_[level], log2_[level], req, src, n, mode, status_, ctype_, d_mem_count_, mem_cap_, d_err_);
    DT_CK(cudaMemcpy(&mem_count_, d_mem_count_, sizeof(int), cudaMemcpyDeviceToHost));
    unsigned int err = 0;
    DT_CK(cudaMemcpy(&err, d_err_, sizeof(err), cudaMemcpyDeviceToHost));
    if (err) {
        last_error = (err & 1) ? "hash table full at level " + std::to_string(level) : "device topology: insertion failed";
        cudaMemset(d_err_, 0, sizeof(unsigned int));
        return 4;
    }
    return 0;
}

int DevTopology::set_tiles(int level, const int32_t* xyz, const uint8_t* types, int n) {
    if (level < 0 || level >= num_layers_ || n < 0) {
        last_error = "level out of range";
        return 1;
    }
    if ((size_t)n > scratch_cap_) {
        cudaFree(d_scratch_);
        d_scratch_ = nullptr;
        scratch_cap_ = std::max<size_t>(n, 1024);
        DT_CK(cudaMalloc(&d_scratch_, sizeof(int4) * scratch_int4(scratch_cap_)));
    }
    std::vector<int4> req(n);
    std::vector<int> src(n, -1);
    for (int i = 0; i < n; i++) req[i] = make_int4(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], types[i]);
    int4* dreq = reinterpret_cast<int4*>(d_scratch_);
    int* dsrc = reinterpret_cast<int*>(reinterpret_cast<int4*>(d_scratch_) + 2 * scratch_cap_) + 2 * scratch_cap_;
    DT_CK(cudaMemcpy(dreq, req.data(), sizeof(int4) * n, cudaMemcpyHostToDevice));
    DT_CK(cudaMemcpy(dsrc, src.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
    return insert_requests(level, n, kInsSet, -1);
}

int DevTopology::counts_from_device() {
    DT_CK(cudaMemcpy(count_.data(), d_count_, sizeof(int) * num_layers_, cudaMemcpyDeviceToHost));
    max_level_ = -1;
    for (int l = 0; l < num_layers_; l++)
        if (count_[l] > 0) max_level_ = l;
    // scratch must hold 8 requests per tile of the largest level
    size_t need = 1024;
    for (int c : count_) need = std::max<size_t>(need, (size_t)8 * c);
    if (need > scratch_cap_) {
        cudaFree(d_scratch_);
        d_scratch_ = nullptr;
        scratch_cap_ = need;
        DT_CK(cudaMalloc(&d_scratch_, sizeof(int4) * scratch_int4(scratch_cap_)));
    }
    return 0;
}

int DevTopology::compress_and_sync() {
    for (int l = 0; l < num_layers_; l++) {
        k_compact_table<<<1, 1024>>>(live_[l], 1u << log2_[l], arr_[l], d_count_ + l);
        DT_CK(cudaMemcpyAsync(snap_[l], live_[l], sizeof(DSlot) << log2_[l], cudaMemcpyDeviceToDevice));
    }
    DT_CK(cudaGetLastError());
    return counts_from_device();
}

int DevTopology::spawn_ghost_tiles() {
    LevelView v{d_snap_, d_live_, d_log2_, num_layers_};
    int4* req = reinterpret_cast<int4*>(d_scratch_);
    int4* cand = req + scratch_cap_;
    int* flags = reinterpret_cast<int*>(req + 2 * scratch_cap_);
    int* idx = flags + scratch_cap_;
    int* src = idx + scratch_cap_;
    for (int level = max_level_; level > 0; level--) {
        const int n = count_[level];
        if (n == 0) continue;
        k_ghost_candidates<<<blocks(6 * n), 256>>>(v, arr_[level], n, level, flags, cand);
        k_compact_flags<<<1, 1024>>>(flags, 6 * n, idx, d_nflag_);
        int m = 0;
        DT_CK(cudaMemcpy(&m, d_nflag_, sizeof(int), cudaMemcpyDeviceToHost));
        if (m == 0) continue;
        k_gather_requests<<<blocks(m), 256>>>(idx, m, cand, req, src);
        int rc = insert_requests(level, m, kInsIfAbsent, -1);
        if (rc) return rc;
    }
    return compress_and_sync();
}

int DevTopology::upload_masks(const std::vector<const uint8_t*>& masks, const std::vector<int>& dims) {
    std::vector<uint8_t*> ptrs(num_layers_, nullptr);
    for (int l = 0; l < num_layers_; l++) {
        cudaFree(mask_bufs_[l]);
        mask_bufs_[l] = nullptr;
        const size_t n = (size_t)dims[3 * l] * dims[3 * l + 1] * dims[3 * l + 2];
        if (l < (int)masks.size() && masks[l] && n > 0) {
            DT_CK(cudaMalloc(&mask_bufs_[l], n));
            DT_CK(cudaMemcpy(mask_bufs_[l], masks[l], n, cudaMemcpyHostToDevice));
            ptrs[l] = mask_bufs_[l];
        }
    }
    DT_CK(cudaMemcpy(d_masks_, ptrs.data(), sizeof(uint8_t*) * num_layers_, cudaMemcpyHostToDevice));
    DT_CK(cudaMemcpy(d_mask_dims_, dims.data(), sizeof(int) * 3 * num_layers_, cudaMemcpyHostToDevice));
    return 0;
}

int DevTopology::refine_leafs_one_step(const std::vector<const uint8_t*>& masks, const std::vector<int>& dims, std::vector<int>* counts) {
    int rc = upload_masks(masks, dims);
    if (rc) return rc;
    LevelView v{d_snap_, d_live_, d_log2_, num_layers_};
    int4* req = reinterpret_cast<int4*>(d_scratch_);
    int* flags = reinterpret_cast<int*>(req + 2 * scratch_cap_);
    int* idx = flags + scratch_cap_;
    int* src = idx + scratch_cap_;
    std::vector<int> cnt(num_layers_, 0);
    const int dev_max = max_level_;
    for (int i = max_level_; i >= 0; i--) {
        const int n = count_[i];
        if (n == 0) continue;
        k_refine_leaf_flags<<<blocks(n), 256>>>(v, arr_[i], n, i, dev_max, d_masks_, d_mask_dims_, status_, flags);
        k_refine_ghost_flags<<<blocks(n), 256>>>(v, arr_[i], n, i, status_);
        k_compact_flags<<<1, 1024>>>(flags, n, idx, d_nflag_);
        int m = 0;
        DT_CK(cudaMemcpy(&m, d_nflag_, sizeof(int), cudaMemcpyDeviceToHost));
        cnt[i] = m;
        if (m == 0) continue;
        k_refine_requests<<<blocks(m), 256>>>(v, arr_[i], idx, m, i, req, src);
        rc = insert_requests(i + 1, 8 * m, kInsSet, i);
        if (rc) return rc;
    }
    if (counts) *counts = cnt;
    return compress_and_sync();
}

int DevTopology::iterative_refine(const std::vector<const uint8_t*>& masks, const std::vector<int>& dims) {
    // src/PoissonGrid.h:316-326
    for (int guard = 0; guard < 64; guard++) {
        std::vector<int> c;
        int rc = refine_leafs_one_step(masks, dims, &c);
        if (rc) return rc;
        rc = spawn_ghost_tiles();
        if (rc) return rc;
        int tot = 0;
        for (int x : c) tot += x;
        if (tot == 0) return 0;
    }
    last_error = "iterative refine did not settle";
    return 4;
}

int DevTopology::coarsen_step(const std::vector<const uint8_t*>& masks, const std::vector<int>& dims, std::vector<int>* deleted) {
    int rc = upload_masks(masks, dims);
    if (rc) return rc;
    LevelView v{d_snap_, d_live_, d_log2_, num_layers_};
    int4* req = reinterpret_cast<int4*>(d_scratch_);
    int4* ops = req + scratch_cap_;
    int* flags = reinterpret_cast<int*>(req + 2 * scratch_cap_);
    int* idx = flags + scratch_cap_;
    for (int l = num_layers_ - 1; l >= 0; l--) {
        const int n = count_[l];
        if (n == 0) continue;
        k_coarsen_nonleaf<<<blocks(n), 256>>>(v, arr_[l], n, l, status_);
        k_coarsen_leaf<<<blocks(n), 256>>>(v, arr_[l], n, l, d_masks_, d_mask_dims_, status_);
    }
    for (int l = 0; l < num_layers_; l++) {
        const int n = count_[l];
        if (n == 0) continue;
        k_coarsen_down<<<blocks(n), 256>>>(v, arr_[l], n, l, status_);
        k_coarsen_ghost<<<blocks(n), 256>>>(v, arr_[l], n, l, status_);
    }
    std::vector<int> del(num_layers_, 0);
    for (int l = 0; l < num_layers_; l++) {
        const int n = count_[l];
        if (n == 0) continue;
        k_coarsen_ops<<<blocks(n), 256>>>(arr_[l], n, status_, flags, ops);
        k_compact_flags<<<1, 1024>>>(flags, n, idx, d_nflag_);
        int m = 0;
        DT_CK(cudaMemcpy(&m, d_nflag_, sizeof(int), cudaMemcpyDeviceToHost));
        if (m == 0) continue;
        k_gather_ops<<<blocks(m), 256>>>(idx, m, ops, req);
        std::vector<int4> h(m);
        DT_CK(cudaMemcpy(h.data(), req, sizeof(int4) * m, cudaMemcpyDeviceToHost));
        for (const int4& q : h) del[l] += q.w == 1;
        k_edit_serial<<<1, 32>>>(live_[l], log2_[l], req, m, d_err_);
    }
    unsigned int err = 0;
    DT_CK(cudaMemcpy(&err, d_err_, sizeof(err), cudaMemcpyDeviceToHost));
    if (err) {
        last_error = "device topology: deletion did not terminate";
        cudaMemset(d_err_, 0, sizeof(unsigned int));
        return 4;
    }
    if (deleted) *deleted = del;
    return compress_and_sync();
}

int DevTopology::calc_cell_types_from_leafs() {
    LevelView v{d_snap_, d_live_, d_log2_, num_layers_};
    for (int l = num_layers_ - 1; l >= 0; l--)
        if (count_[l] > 0) k_celltypes_nonleaf<<<count_[l], 128>>>(v, arr_[l], count_[l], l, ctype_);
    for (int l = 0; l < num_layers_; l++)
        if (count_[l] > 0) k_celltypes_ghost<<<count_[l], 128>>>(v, arr_[l], count_[l], l, ctype_);
    DT_CK(cudaDeviceSynchronize());
    return 0;
}

int DevTopology::tiles(int32_t* out5) const {
    size_t i = 0;
    for (int l = 0; l < num_layers_; l++) {
        std::vector<DSlot> a(count_[l]);
        if (count_[l] && cudaMemcpy(a.data(), arr_[l], sizeof(DSlot) * count_[l], cudaMemcpyDeviceToHost) != cudaSuccess) return 2;
        for (const DSlot& s : a) {
            out5[5 * i] = l;
            out5[5 * i + 1] = s.x;
            out5[5 * i + 2] = s.y;
            out5[5 * i + 3] = s.z;
            out5[5 * i + 4] = (s.meta >> kTypeShift) & 0xff;
            i++;
        }
    }
    return 0;
}

int DevTopology::hash_slots(int32_t* out) const {
    const int n = num_tiles();
    int32_t *slot = nullptr, *mem = nullptr;
    if (cudaMalloc(&slot, sizeof(int32_t) * std::max(n, 1)) != cudaSuccess || cudaMalloc(&mem, sizeof(int32_t) * std::max(n, 1)) != cudaSuccess) {
        cudaFree(slot);
        return 3;
    }
    int off = 0;
    for (int l = 0; l < num_layers_; l++) {
        if (count_[l]) k_slots_of<<<blocks(count_[l]), 256>>>(arr_[l], count_[l], live_[l], log2_[l], slot + off, mem + off);
        off += count_[l];
    }
    const bool ok = cudaMemcpy(out, slot, sizeof(int32_t) * n, cudaMemcpyDeviceToHost) == cudaSuccess;
    cudaFree(slot);
    cudaFree(mem);
    return ok ? 0 : 2;
}

// memory ids of the compacted tiles, all-tiles order (device buffer of n)
static int32_t* mem_ids(const std::vector<DSlot*>& arr, const std::vector<int>& count, const std::vector<DSlot*>& live,
                        const std::vector<uint32_t>& log2, int n) {
    int32_t *slot = nullptr, *mem = nullptr;
    if (cudaMalloc(&slot, sizeof(int32_t) * std::max(n, 1)) != cudaSuccess) return nullptr;
    if (cudaMalloc(&mem, sizeof(int32_t) * std::max(n, 1)) != cudaSuccess) {
        cudaFree(slot);
        return nullptr;
    }
    int off = 0;
    for (size_t l = 0; l < arr.size(); l++) {
        if (count[l]) k_slots_of<<<blocks(count[l]), 256>>>(arr[l], count[l], live[l], log2[l], slot + off, mem + off);
        off += count[l];
    }
    cudaFree(slot);
    return mem;
}

int DevTopology::cell_types(uint8_t* out) const {
    const int n = num_tiles();
    if (n == 0) return 0;
    int32_t* mem = mem_ids(arr_, count_, live_, log2_, n);
    uint8_t* buf = nullptr;
    if (!mem || cudaMalloc(&buf, (size_t)n * kTileCells) != cudaSuccess) {
        cudaFree(mem);
        return 3;
    }
    k_copy_types<<<n, 128>>>(mem, n, ctype_, buf, 0);
    const bool ok = cudaMemcpy(out, buf, (size_t)n * kTileCells, cudaMemcpyDeviceToHost) == cudaSuccess;
    cudaFree(buf);
    cudaFree(mem);
    return ok ? 0 : 2;
}

int DevTopology::set_cell_types(const uint8_t* host_ct) {
    const int n = num_tiles();
    if (n == 0) return 0;
    int32_t* mem = mem_ids(arr_, count_, live_, log2_, n);
    uint8_t* buf = nullptr;
    if (!mem || cudaMalloc(&buf, (size_t)n * kTileCells) != cudaSuccess) {
        cudaFree(mem);
        return 3;
    }
    bool ok = cudaMemcpy(buf, host_ct, (size_t)n * kTileCells, cudaMemcpyHostToDevice) == cudaSuccess;
    if (ok) k_copy_types<<<n, 128>>>(mem, n, ctype_, buf, 1);
    ok = ok && cudaDeviceSynchronize() == cudaSuccess;
    cudaFree(buf);
    cudaFree(mem);
    return ok ? 0 : 2;
}

int DevTopology::statuses(int32_t* out) const {
    const int n = num_tiles();
    if (n == 0) return 0;
    int32_t* mem = mem_ids(arr_, count_, live_, log2_, n);
    int32_t* buf = nullptr;
    if (!mem || cudaMalloc(&buf, sizeof(int32_t) * n) != cudaSuccess) {
        cudaFree(mem);
        return 3;
    }
    k_gather_status<<<blocks(n), 256>>>(mem, n, status_, buf);
    const bool ok = cudaMemcpy(out, buf, sizeof(int32_t) * n, cudaMemcpyDeviceToHost) == cudaSuccess;
    cudaFree(buf);
    cudaFree(mem);
    return ok ? 0 : 2;
}

}  // namespace cirrus
