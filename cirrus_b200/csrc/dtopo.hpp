// Device-resident octree topology (dtopo.cu): the reference's per-level hash tables, their
// compaction and the refinement / coarsening / ghost-spawning / cell-type steps run on the GPU,
// bit-exact with the host Topology and the reference (tile order = hash-slot order).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

namespace cirrus {

// One hash slot on the device: tile coordinates and meta = tile-memory id | type << 24, or -1
// when empty.
struct __align__(16) DSlot {
    int x, y, z, meta;
};

class DevTopology {
public:
    DevTopology(int num_layers, const uint32_t* log2_hash, double h0);
    ~DevTopology();
    DevTopology(const DevTopology&) = delete;
    DevTopology& operator=(const DevTopology&) = delete;

    int num_layers() const { return num_layers_; }
    double h0() const { return h0_; }
    int max_level() const { return max_level_; }
    const uint32_t* log2_hash() const { return log2_.data(); }
    int num_tiles() const;

    // setTileHost with blank tiles, in the given order (one level per call)
    int set_tiles(int level, const int32_t* xyz, const uint8_t* types, int n);
    int compress_and_sync();                          // compressHost + syncHostAndDevice
    int spawn_ghost_tiles();                          // SpawnGhostTiles
    // RefineLeafsOneStep / CoarsenStep with level targets from dense per-level masks:
    // refine: target = level + (mask != 0); coarsen: target = level - (mask != 0)
    int refine_leafs_one_step(const std::vector<const uint8_t*>& masks, const std::vector<int>& dims, std::vector<int>* counts);
    int iterative_refine(const std::vector<const uint8_t*>& masks, const std::vector<int>& dims);
    int coarsen_step(const std::vector<const uint8_t*>& masks, const std::vector<int>& dims, std::vector<int>* deleted);
    int set_cell_types(const uint8_t* host_ct);       // all tiles, all-tiles order
    int calc_cell_types_from_leafs();                 // CalcCellTypesFromLeafs

    // all-tiles order exports (host arrays)
    int tiles(int32_t* out5) const;
    int hash_slots(int32_t* out) const;
    int cell_types(uint8_t* out) const;
    int statuses(int32_t* out) const;
    std::string last_error;

private:
    int ensure_mem(int extra);
    int insert_requests(int level, int n, int mode, int src_level);
    int upload_masks(const std::vector<const uint8_t*>& masks, const std::vector<int>& dims);
    int counts_from_device();

    int num_layers_;
    double h0_;
    int max_level_ = -1;
    std::vector<uint32_t> log2_;
    std::vector<DSlot*> live_, snap_;   // per level: the edited table and the synced copy
    std::vector<DSlot*> arr_;           // per level: compacted snapshot (hash-slot order)
    std::vector<int> count_;            // per level: tiles in arr_
    DSlot** d_live_ = nullptr;          // device arrays of the per-level pointers
    DSlot** d_snap_ = nullptr;
    DSlot** d_arr_ = nullptr;
    uint32_t* d_log2_ = nullptr;
    int* d_count_ = nullptr;            // per level, written by the compaction
    int* d_scratch_ = nullptr;          // request / flag buffers (int4 per entry)
    size_t scratch_cap_ = 0;            // in int4
    int* d_nflag_ = nullptr;            // counters of the request builders
    int32_t* status_ = nullptr;         // per tile memory
    uint8_t* ctype_ = nullptr;          // 512 per tile memory
    int mem_count_ = 0, mem_cap_ = 0;
    int* d_mem_count_ = nullptr;
    uint8_t** d_masks_ = nullptr;       // device copies of the level-target masks
    std::vector<uint8_t*> mask_bufs_;
    int* d_mask_dims_ = nullptr;
    unsigned int* d_err_ = nullptr;     // hash table full / bounded loop gave up
};

}  // namespace cirrus
