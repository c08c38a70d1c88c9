// Host-side octree topology of 8^3-cell tiles, bit-exact with the reference's construction.
//
// The reference keeps, per octree level, an open-addressing hash table of tile infos on the
// host and a copy of it on the device (src/HAGrid.h:229-255).  Topology edits go to the host
// table while the refinement kernels read the device copy taken at the last sync; tile memory
// (refinement status, cell types) is shared.  Tile order everywhere is the compacted hash-slot
// order (src/HAGrid.h:491-509), concatenated level-major (src/HAGrid.h:538-556).  This class
// reproduces those semantics on the host with flat arrays, then emits the int32 tables the
// device solver consumes.
#pragma once

#include <array>
#include <cstdint>
#include <functional>
#include <string>
#include <vector>

namespace cirrus {

constexpr uint8_t kLeaf = 1, kNonLeaf = 2, kGhost = 4;
constexpr uint8_t kDirichlet = 1, kInterior = 2, kNeumann = 4;
constexpr int kCells = 512;

// One hash slot: a copy of the tile's identity (HATileInfo without the pointer).
struct Slot {
    int32_t x = 0, y = 0, z = 0;
    int32_t mem = -1;  // tile-memory id, -1 = empty slot
    uint8_t type = 0;
    bool empty() const { return mem < 0; }
};

struct LevelTable {
    uint32_t log2 = 0;
    std::vector<Slot> slots;
    // src/HAAccessor.h:214-223
    static uint32_t hash(int32_t x, int32_t y, int32_t z, uint32_t log2) {
        uint32_t r = 0;
        r ^= (uint32_t)x * 1u;
        r ^= (uint32_t)y * 2654435761u;
        r ^= (uint32_t)z * 805459861u;
        return r & ((1u << log2) - 1u);
    }
    // src/HAAccessor.h:225-242: first slot that is empty or holds the coordinate; -1 if full.
    int64_t probe(int32_t x, int32_t y, int32_t z) const {
        const uint32_t mask = (1u << log2) - 1u;
        uint32_t k0 = hash(x, y, z, log2), k1 = k0;
        do {
            const Slot& s = slots[k1];
            if (s.mem < 0 || (s.x == x && s.y == y && s.z == z)) return k1;
            k1 = (k1 + 1) & mask;
        } while (k1 != k0);
        return -1;
    }
    const Slot* find(int32_t x, int32_t y, int32_t z) const {
        int64_t s = probe(x, y, z);
        return (s < 0 || slots[s].mem < 0) ? nullptr : &slots[s];
    }
};

using LevelTargetFn = std::function<int(int level, int x, int y, int z)>;

class Topology {
public:
    Topology(int num_layers, const uint32_t* log2_hash, double h0);

    int num_layers() const { return num_layers_; }
    double h0() const { return h0_; }
    int max_level() const { return max_level_; }

    bool set_tile(int level, int x, int y, int z, uint8_t type);  // setTileHost with a blank tile
    // Adopt an existing tile list in the given all-tiles order (level-major), e.g. the
    // reference's hAllTiles: tables are filled for lookups, the order is kept as given.
    bool import_tiles(const int32_t* tiles5, int n);
    void compress_and_sync();                                     // compressHost + syncHostAndDevice
    void spawn_ghost_tiles();                                     // SpawnGhostTiles
    std::vector<int> refine_leafs_one_step(const LevelTargetFn& target);
    void iterative_refine(const LevelTargetFn& target);

    // all-tiles order views (valid after compress_and_sync)
    int num_tiles() const { return (int)all_.size(); }
    void tiles(int32_t* out5) const;
    void hash_slots(int32_t* out) const;
    void neighbor_tiles(int32_t* out6) const;  // CalculateNeighborTiles
    void set_cell_types(const uint8_t* ct);
    void cell_types(uint8_t* ct) const;
    void calc_cell_types_from_leafs();       // CalcCellTypesFromLeafs

    // parent tile (all-tiles index) of each tile, or -1
    void parent_tiles(int32_t* out) const;
    // the 8 tiles one level finer inside each tile (octant o = x | y<<1 | z<<2), or -1
    void child_tiles(int32_t* out8) const;
    // the 12 same-level edge neighbours of each tile, or -1.  Edge e = 4*p + 2*(sa>0) + (sb>0)
    // for axis pair p in {(x,y), (x,z), (y,z)} with offsets sa, sb in {-1,+1} on its two axes.
    void edge_tiles(int32_t* out12) const;

    std::string last_error;

private:
    struct Mem {
        int32_t status = 0;
        std::array<uint8_t, kCells> ctype{};
    };
    bool put_host(int level, int x, int y, int z, const Mem& data, uint8_t type);
    const Slot* dev_find(int level, int x, int y, int z) const {
        if (level < 0 || level >= num_layers_) return nullptr;
        return dev_[level].find(x, y, z);
    }
    const Slot* host_find(int level, int x, int y, int z) const {
        if (level < 0 || level >= num_layers_) return nullptr;
        return host_[level].find(x, y, z);
    }
    int all_index_of_voxel(int level, int gx, int gy, int gz, int* cell) const;

    int num_layers_;
    double h0_;
    int max_level_ = -1;
    std::vector<LevelTable> host_, dev_;
    std::vector<std::vector<Slot>> arrays_;  // compacted per level
    std::vector<Slot> all_;                  // dAllTiles
    std::vector<Mem> mem_;
    std::vector<int32_t> mem_to_all_;        // tile-memory id -> all-tiles index
};

}  // namespace cirrus
