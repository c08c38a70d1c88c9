// Tile-holder files: the reference's on-disk form of a grid's tiles, used as its checkpoint,
// warm-start and interchange format (IOFunc::WriteHAHostTileHolderToFile and
// ReadHAHostTileHolderFromFile, src/PoissonIOFunc.cu:38-121, over HAHostTileHolder<PoissonTile<float>>,
// src/HAGrid.h:74-92, filled by HADeviceGrid::getHostTileHolder, src/HAGrid.h:433-462, and read back
// by setTilesFromHolder, src/HAGrid.h:316-331).
//
// File layout (the writing machine's byte order; x86-64 little-endian here):
//   float h0 | int32 num_layers | int32 max_level
//   uint64 num_tiles, then num_tiles tile records of kRecordBytes bytes each
//   uint64 num_levels, then per level: uint64 count, then per tile info:
//       int32 x, y, z | int32 level | uint8 type | int64 record index (-1: no tile)
// A tile record is a PoissonTile<float> as laid out in memory (src/PoissonTile.h:51-56):
//   float data[11][736] (channel c, cell i*64 + j*8 + k at data[c][cell]; entries 512..735 unused)
//   6 neighbour infos of 32 bytes (pointers of the writing process, meaningless in a file)
//   uint8 cell_type[512] | bool interest | bool locked | 2 bytes padding | int32 status | int32 serial
//   | 4 bytes padding.
// The layout constants are checked against the reference's compiled structs by the tests.
#include "holder.hpp"

#include "topology.hpp"

#include <cstdio>
#include <cstring>
#include <map>
#include <tuple>

namespace cirrus {

namespace {

template <class T> bool put(std::FILE* f, const T& v) { return std::fwrite(&v, sizeof(T), 1, f) == 1; }
template <class T> bool get(std::FILE* f, T& v) { return std::fread(&v, sizeof(T), 1, f) == 1; }

struct FileCloser {
    std::FILE* f;
    ~FileCloser() {
        if (f) std::fclose(f);
    }
};

}  // namespace

float* Holder::channel_of(int record, int c) {
    return reinterpret_cast<float*>(records.data() + (size_t)record * kRecordBytes + kRecordData + (size_t)c * kChannelStride * 4);
}
const float* Holder::channel_of(int record, int c) const {
    return reinterpret_cast<const float*>(records.data() + (size_t)record * kRecordBytes + kRecordData +
                                          (size_t)c * kChannelStride * 4);
}
uint8_t* Holder::types_of(int record) { return records.data() + (size_t)record * kRecordBytes + kRecordCellType; }
const uint8_t* Holder::types_of(int record) const { return records.data() + (size_t)record * kRecordBytes + kRecordCellType; }

int Holder::num_tiles() const {
    int n = 0;
    for (const auto& lv : levels) n += (int)lv.size();
    return n;
}

std::vector<const HolderInfo*> Holder::ordered() const {
    std::vector<const HolderInfo*> out;
    for (const auto& lv : levels)
        for (const HolderInfo& h : lv) out.push_back(&h);
    return out;
}

int holder_write(const Holder& h, const char* path, std::string* err) {
    FileCloser fc{std::fopen(path, "wb")};
    if (!fc.f) {
        if (err) *err = std::string("cannot open for writing: ") + path;
        return 1;
    }
    const uint64_t nrec = h.records.size() / kRecordBytes;
    bool ok = put(fc.f, h.h0) && put(fc.f, h.num_layers) && put(fc.f, h.max_level) && put(fc.f, nrec);
    ok = ok && (nrec == 0 || std::fwrite(h.records.data(), kRecordBytes, nrec, fc.f) == nrec);
    ok = ok && put(fc.f, (uint64_t)h.levels.size());
    for (const auto& lv : h.levels) {
        ok = ok && put(fc.f, (uint64_t)lv.size());
        for (const HolderInfo& t : lv)
            ok = ok && put(fc.f, t.x) && put(fc.f, t.y) && put(fc.f, t.z) && put(fc.f, t.level) && put(fc.f, t.type) &&
                 put(fc.f, t.record);
    }
    if (!ok && err) *err = std::string("write failed: ") + path;
    return ok ? 0 : 1;
}

int holder_read(const char* path, Holder* h, std::string* err) {
    FileCloser fc{std::fopen(path, "rb")};
    auto fail = [&](const char* what) {
        if (err) *err = std::string(what) + ": " + path;
        return 1;
    };
    if (!fc.f) return fail("cannot open");
    std::fseek(fc.f, 0, SEEK_END);
    const long long fsize = std::ftell(fc.f);
    std::fseek(fc.f, 0, SEEK_SET);
    uint64_t nrec = 0, nlev = 0;
    if (!get(fc.f, h->h0) || !get(fc.f, h->num_layers) || !get(fc.f, h->max_level) || !get(fc.f, nrec)) return fail("truncated header");
    if (h->num_layers <= 0 || h->num_layers > 64 || nrec > (uint64_t)fsize / kRecordBytes) return fail("implausible header");
    h->records.resize(nrec * kRecordBytes);
    if (nrec && std::fread(h->records.data(), kRecordBytes, nrec, fc.f) != nrec) return fail("truncated tile records");
    if (!get(fc.f, nlev) || nlev > 64) return fail("bad level count");
    h->levels.assign(nlev, {});
    for (auto& lv : h->levels) {
        uint64_t cnt = 0;
        if (!get(fc.f, cnt) || cnt > (uint64_t)fsize) return fail("bad level size");
        lv.resize(cnt);
        for (HolderInfo& t : lv) {
            if (!get(fc.f, t.x) || !get(fc.f, t.y) || !get(fc.f, t.z) || !get(fc.f, t.level) || !get(fc.f, t.type) || !get(fc.f, t.record))
                return fail("truncated tile infos");
            if (t.record < -1 || t.record >= (int64_t)nrec) return fail("tile index out of range");
        }
    }
    return 0;
}

int holder_to_topology(const Holder& h, const uint32_t* log2_hash, int num_layers, Topology** out, std::vector<int32_t>* order,
                       std::string* err) {
    if (num_layers != h.num_layers || num_layers != (int)h.levels.size()) {
        if (err) *err = "holder: number of layers differs from the grid's";
        return 1;
    }
    Topology* t = new Topology(num_layers, log2_hash, (double)h.h0);
    // setTilesFromHolder: every level's tiles in file order, then compressHost
    for (int l = 0; l < num_layers; l++)
        for (const HolderInfo& i : h.levels[l])
            if (!t->set_tile(l, i.x, i.y, i.z, i.type)) {
                if (err) *err = "holder: " + t->last_error;
                delete t;
                return 4;
            }
    t->compress_and_sync();
    const int n = t->num_tiles();
    std::vector<int32_t> t5((size_t)n * 5);
    t->tiles(t5.data());
    std::map<std::tuple<int, int, int, int>, int> at;
    for (int i = 0; i < n; i++) at[{t5[5 * i], t5[5 * i + 1], t5[5 * i + 2], t5[5 * i + 3]}] = i;
    std::vector<uint8_t> ct((size_t)n * kCells, 0);
    std::vector<int32_t> ord;
    for (int l = 0; l < num_layers; l++)
        for (const HolderInfo& i : h.levels[l]) {
            const int a = at.at({l, i.x, i.y, i.z});
            ord.push_back(a);
            if (i.record >= 0) std::memcpy(&ct[(size_t)a * kCells], h.types_of((int)i.record), kCells);
        }
    t->set_cell_types(ct.data());
    if (order) *order = std::move(ord);
    *out = t;
    return 0;
}

}  // namespace cirrus
