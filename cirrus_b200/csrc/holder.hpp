// Tile-holder files (holder.cpp): the reference's on-disk form of a grid's tiles.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace cirrus {

class Topology;

// PoissonTile<float> record layout (src/PoissonTile.h:51-56): 11 channels of 736 floats, 6 tile
// infos of 32 bytes, 512 cell types, two flags, status, serial, padding.
constexpr size_t kRecordBytes = 33104;
constexpr size_t kRecordData = 0;
constexpr int kRecordChannels = 11;
constexpr size_t kChannelStride = 736;  // floats
constexpr size_t kRecordNeighbors = 32384;
constexpr size_t kRecordCellType = 32576;
constexpr size_t kRecordStatus = 33092;
constexpr size_t kRecordSerial = 33096;

// One tile info as the file stores it (HATileInfo without the pointer, plus the record index).
struct HolderInfo {
    int32_t x = 0, y = 0, z = 0, level = 0;
    uint8_t type = 0;
    int64_t record = -1;
};

struct Holder {
    float h0 = 0.f;
    int32_t num_layers = 0, max_level = -1;
    std::vector<uint8_t> records;                 // num_records x kRecordBytes
    std::vector<std::vector<HolderInfo>> levels;  // per level, in file order
    int num_tiles() const;                        // infos over all levels
    std::vector<const HolderInfo*> ordered() const;  // level by level, file order
    float* channel_of(int record, int c);
    const float* channel_of(int record, int c) const;
    uint8_t* types_of(int record);
    const uint8_t* types_of(int record) const;
};

int holder_read(const char* path, Holder* h, std::string* err);
int holder_write(const Holder& h, const char* path, std::string* err);
// setTilesFromHolder + compressHost into a new topology with the given hash sizes; order[i] = the
// all-tiles index of the holder's i-th tile (level by level, file order); cell types from the records.
int holder_to_topology(const Holder& h, const uint32_t* log2_hash, int num_layers, Topology** out, std::vector<int32_t>* order,
                       std::string* err);

}  // namespace cirrus
