// Host octree topology; semantics follow the reference line by line where order matters
// (see topology.hpp).  Citations are paths inside the reference project.
#include "topology.hpp"

#include <cstring>

namespace cirrus {

namespace {
// HACoordAccessor::neighborOffset order: x-, x+, y-, y+, z-, z+ (src/HAAccessor.h:161-168)
const int kNb[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
inline int loc(int i, int j, int k) { return (i << 6) | (j << 3) | k; }
}  // namespace

Topology::Topology(int num_layers, const uint32_t* log2_hash, double h0) : num_layers_(num_layers), h0_(h0) {
    host_.resize(num_layers);
    for (int l = 0; l < num_layers; l++) {
        host_[l].log2 = log2_hash[l];
        host_[l].slots.assign(size_t(1) << log2_hash[l], Slot());
    }
    dev_ = host_;
    arrays_.assign(num_layers, {});
}

bool Topology::put_host(int level, int x, int y, int z, const Mem& data, uint8_t type) {
    // src/HAGrid.h:387-407: probe; new slot gets new tile memory; memory overwritten; info reset
    LevelTable& t = host_[level];
    int64_t s = t.probe(x, y, z);
    if (s < 0) {
        last_error = "hash table full at level " + std::to_string(level);
        return false;
    }
    Slot& slot = t.slots[s];
    if (slot.mem < 0) {
        mem_.push_back(Mem());
        slot.mem = (int32_t)mem_.size() - 1;
    }
    mem_[slot.mem] = data;
    slot.x = x; slot.y = y; slot.z = z; slot.type = type;
    return true;
}

bool Topology::set_tile(int level, int x, int y, int z, uint8_t type) {
    if (level < 0 || level >= num_layers_) {
        last_error = "level out of range";
        return false;
    }
    return put_host(level, x, y, z, Mem(), type);
}

bool Topology::import_tiles(const int32_t* t5, int n) {
    for (int l = 0; l < num_layers_; l++) {
        host_[l].slots.assign(host_[l].slots.size(), Slot());
        arrays_[l].clear();
    }
    mem_.clear();
    int prev = 0;
    for (int i = 0; i < n; i++) {
        const int level = t5[5 * i];
        const uint8_t type = (uint8_t)t5[5 * i + 4];
        if (level < prev || level >= num_layers_ || !(type == kLeaf || type == kNonLeaf || type == kGhost)) {
            last_error = "import: tiles must be level-major with valid levels and types";
            return false;
        }
        prev = level;
        if (host_find(level, t5[5 * i + 1], t5[5 * i + 2], t5[5 * i + 3])) {
            last_error = "import: duplicate tile";
            return false;
        }
        if (!put_host(level, t5[5 * i + 1], t5[5 * i + 2], t5[5 * i + 3], Mem(), type)) return false;
        const int64_t s = host_[level].probe(t5[5 * i + 1], t5[5 * i + 2], t5[5 * i + 3]);
        arrays_[level].push_back(host_[level].slots[s]);
    }
    max_level_ = -1;
    for (int l = 0; l < num_layers_; l++)
        if (!arrays_[l].empty()) max_level_ = l;
    dev_ = host_;
    all_.clear();
    for (int l = 0; l < num_layers_; l++) all_.insert(all_.end(), arrays_[l].begin(), arrays_[l].end());
    mem_to_all_.assign(mem_.size(), -1);
    for (size_t i = 0; i < all_.size(); i++) mem_to_all_[all_[i].mem] = (int32_t)i;
    return true;
}

void Topology::compress_and_sync() {
    // src/HAGrid.h:491-509 then :510-561
    max_level_ = -1;
    for (int l = 0; l < num_layers_; l++) {
        arrays_[l].clear();
        for (const Slot& s : host_[l].slots)
            if (s.mem >= 0) arrays_[l].push_back(s);
        if (!arrays_[l].empty()) max_level_ = l;
    }
    dev_ = host_;
    all_.clear();
    for (int l = 0; l < num_layers_; l++) all_.insert(all_.end(), arrays_[l].begin(), arrays_[l].end());
    mem_to_all_.assign(mem_.size(), -1);
    for (size_t i = 0; i < all_.size(); i++) mem_to_all_[all_[i].mem] = (int32_t)i;
}

void Topology::spawn_ghost_tiles() {
    // src/PoissonGrid.cu:30-60: iterate the compacted arrays (not the live table), consult the
    // live host table, create GHOST tiles whose parent is a LEAF.
    for (int level = max_level_; level > 0; level--) {
        const std::vector<Slot> arr = arrays_[level];
        for (const Slot& info : arr) {
            if (!(info.type & (kLeaf | kNonLeaf))) continue;
            for (int n = 0; n < 6; n++) {
                int nx = info.x + kNb[n][0], ny = info.y + kNb[n][1], nz = info.z + kNb[n][2];
                if (host_find(level, nx, ny, nz)) continue;
                const Slot* p = host_find(level - 1, nx >> 1, ny >> 1, nz >> 1);
                if (p && (p->type & kLeaf)) put_host(level, nx, ny, nz, Mem(), kGhost);
            }
        }
    }
    compress_and_sync();
}

std::vector<int> Topology::refine_leafs_one_step(const LevelTargetFn& target) {
    // src/PoissonGrid.h:35-162
    constexpr int32_t kRefine = 1;
    std::vector<int> counts(num_layers_, 0);
    const int dev_max = max_level_;
    for (int i = max_level_; i >= 0; i--) {
        const std::vector<Slot> arr = arrays_[i];
        std::vector<uint8_t> flag(arr.size(), 0);
        // device pass 1: LEAF tiles of level i
        for (size_t j = 0; j < arr.size(); j++) {
            const Slot& info = arr[j];
            if (!(info.type & kLeaf)) continue;
            bool to_refine = target(i, info.x, info.y, info.z) > i;
            if (i < dev_max) {
                for (int ci = 0; ci < 8; ci++) {
                    const Slot* c = dev_find(i + 1, info.x * 2 + (ci & 1), info.y * 2 + ((ci >> 1) & 1),
                                             info.z * 2 + ((ci >> 2) & 1));
                    if (c && (c->type & kGhost) && (mem_[c->mem].status & kRefine)) to_refine = true;
                }
            }
            if (i + 1 >= num_layers_) to_refine = false;
            int32_t& st = mem_[info.mem].status;
            st = to_refine ? (st | kRefine) : (st & ~kRefine);
            flag[j] = to_refine;
        }
        // device pass 2: GHOST tiles of level i
        for (size_t j = 0; j < arr.size(); j++) {
            const Slot& info = arr[j];
            if (!(info.type & kGhost)) continue;
            bool rf = false;
            for (int n = 0; n < 6; n++) {
                const Slot* nb = dev_find(i, info.x + kNb[n][0], info.y + kNb[n][1], info.z + kNb[n][2]);
                if (nb && (nb->type & kLeaf) && (mem_[nb->mem].status & kRefine)) rf = true;
            }
            int32_t& st = mem_[info.mem].status;
            st = rf ? (st | kRefine) : (st & ~kRefine);
        }
        // host: mark NONLEAF in the live table, create the 8 children (childTile copies the
        // parent's cell types and status, src/PoissonTile.h:170-191)
        for (size_t j = 0; j < arr.size(); j++) {
            if (!flag[j]) continue;
            counts[i]++;
            int64_t s = host_[i].probe(arr[j].x, arr[j].y, arr[j].z);
            Slot& h = host_[i].slots[s];
            h.type = kNonLeaf;
            const Mem parent = mem_[h.mem];
            const int px = h.x, py = h.y, pz = h.z;
            for (int ci = 0; ci < 8; ci++) {
                int ox = ci & 1, oy = (ci >> 1) & 1, oz = (ci >> 2) & 1;
                Mem child;
                child.status = parent.status;
                for (int a = 0; a < 8; a++)
                    for (int b = 0; b < 8; b++)
                        for (int c = 0; c < 8; c++)
                            child.ctype[loc(a, b, c)] = parent.ctype[loc((ox * 8 + a) >> 1, (oy * 8 + b) >> 1, (oz * 8 + c) >> 1)];
                put_host(i + 1, px * 2 + ox, py * 2 + oy, pz * 2 + oz, child, kLeaf);
            }
        }
    }
    compress_and_sync();
    return counts;
}

void Topology::iterative_refine(const LevelTargetFn& target) {
    // src/PoissonGrid.h:316-326
    while (true) {
        std::vector<int> c = refine_leafs_one_step(target);
        spawn_ghost_tiles();
        int tot = 0;
        for (int v : c) tot += v;
        if (tot == 0) break;
    }
}

void Topology::tiles(int32_t* out) const {
    size_t i = 0;
    for (int l = 0; l < num_layers_; l++) {
        for (const Slot& s : arrays_[l]) {
            out[5 * i] = l; out[5 * i + 1] = s.x; out[5 * i + 2] = s.y; out[5 * i + 3] = s.z; out[5 * i + 4] = s.type;
            i++;
        }
    }
}

void Topology::hash_slots(int32_t* out) const {
    size_t i = 0;
    for (int l = 0; l < num_layers_; l++)
        for (const Slot& s : arrays_[l]) out[i++] = (int32_t)host_[l].probe(s.x, s.y, s.z);
}

void Topology::neighbor_tiles(int32_t* out6) const {
    // src/PoissonGrid.cu:121-134 with the device tables: mNeighbors[axis] = b - e_axis,
    // mNeighbors[axis + 3] = b + e_axis.
    size_t i = 0;
    for (int l = 0; l < num_layers_; l++) {
        for (const Slot& s : arrays_[l]) {
            for (int a = 0; a < 3; a++) {
                int m[3] = {s.x, s.y, s.z}, p[3] = {s.x, s.y, s.z};
                m[a]--; p[a]++;
                const Slot* nm = dev_find(l, m[0], m[1], m[2]);
                const Slot* np = dev_find(l, p[0], p[1], p[2]);
                out6[6 * i + a] = nm ? mem_to_all_[nm->mem] : -1;
                out6[6 * i + a + 3] = np ? mem_to_all_[np->mem] : -1;
            }
            i++;
        }
    }
}

void Topology::parent_tiles(int32_t* out) const {
    size_t i = 0;
    for (int l = 0; l < num_layers_; l++) {
        for (const Slot& s : arrays_[l]) {
            const Slot* p = dev_find(l - 1, s.x >> 1, s.y >> 1, s.z >> 1);
            out[i++] = p ? mem_to_all_[p->mem] : -1;
        }
    }
}

void Topology::child_tiles(int32_t* out8) const {
    size_t i = 0;
    for (int l = 0; l < num_layers_; l++) {
        for (const Slot& s : arrays_[l]) {
            for (int o = 0; o < 8; o++) {
                const Slot* c = dev_find(l + 1, s.x * 2 + (o & 1), s.y * 2 + ((o >> 1) & 1), s.z * 2 + ((o >> 2) & 1));
                out8[8 * i + o] = c ? mem_to_all_[c->mem] : -1;
            }
            i++;
        }
    }
}

void Topology::edge_tiles(int32_t* out12) const {
    static const int pairs[3][2] = {{0, 1}, {0, 2}, {1, 2}};
    size_t i = 0;
    for (int l = 0; l < num_layers_; l++) {
        for (const Slot& s : arrays_[l]) {
            for (int e = 0; e < 12; e++) {
                int c[3] = {s.x, s.y, s.z};
                c[pairs[e >> 2][0]] += (e & 2) ? 1 : -1;
                c[pairs[e >> 2][1]] += (e & 1) ? 1 : -1;
                const Slot* t = dev_find(l, c[0], c[1], c[2]);
                out12[12 * i + e] = t ? mem_to_all_[t->mem] : -1;
            }
            i++;
        }
    }
}

void Topology::set_cell_types(const uint8_t* ct) {
    for (size_t i = 0; i < all_.size(); i++) std::memcpy(mem_[all_[i].mem].ctype.data(), ct + i * kCells, kCells);
}

void Topology::cell_types(uint8_t* ct) const {
    for (size_t i = 0; i < all_.size(); i++) std::memcpy(ct + i * kCells, mem_[all_[i].mem].ctype.data(), kCells);
}

int Topology::all_index_of_voxel(int level, int gx, int gy, int gz, int* cell) const {
    const Slot* s = dev_find(level, gx >> 3, gy >> 3, gz >> 3);
    *cell = loc(gx & 7, gy & 7, gz & 7);
    return s ? s->mem : -1;
}

void Topology::calc_cell_types_from_leafs() {
    // src/PoissonSolver.cu:7-61.  Step 1, fine to coarse over NONLEAF tiles: DIRICHLET if any
    // active child cell is Dirichlet, else INTERIOR if any is interior, else NEUMANN.
    for (int l = num_layers_ - 1; l >= 0; l--) {
        for (const Slot& s : arrays_[l]) {
            if (!(s.type & kNonLeaf)) continue;
            auto& ct = mem_[s.mem].ctype;
            for (int o = 0; o < kCells; o++) {
                int gx = s.x * 8 + (o >> 6), gy = s.y * 8 + ((o >> 3) & 7), gz = s.z * 8 + (o & 7);
                int dcnt = 0, icnt = 0;
                for (int c = 0; c < 8; c++) {
                    int cell;
                    const Slot* cs = dev_find(l + 1, (gx * 2 + (c & 1)) >> 3, (gy * 2 + ((c >> 1) & 1)) >> 3,
                                              (gz * 2 + ((c >> 2) & 1)) >> 3);
                    if (!cs || !(cs->type & (kLeaf | kNonLeaf))) continue;
                    cell = loc((gx * 2 + (c & 1)) & 7, (gy * 2 + ((c >> 1) & 1)) & 7, (gz * 2 + ((c >> 2) & 1)) & 7);
                    uint8_t t = mem_[cs->mem].ctype[cell];
                    if (t & kDirichlet) dcnt++;
                    else if (t & kInterior) icnt++;
                }
                ct[o] = dcnt > 0 ? kDirichlet : (icnt > 0 ? kInterior : kNeumann);
            }
        }
    }
    // Step 2: GHOST cells take their parent cell's type, DIRICHLET without a parent.
    for (int l = 0; l < num_layers_; l++) {
        for (const Slot& s : arrays_[l]) {
            if (!(s.type & kGhost)) continue;
            auto& ct = mem_[s.mem].ctype;
            for (int o = 0; o < kCells; o++) {
                int gx = s.x * 8 + (o >> 6), gy = s.y * 8 + ((o >> 3) & 7), gz = s.z * 8 + (o & 7);
                int cell;
                int pm = all_index_of_voxel(l - 1, gx >> 1, gy >> 1, gz >> 1, &cell);
                ct[o] = pm >= 0 ? mem_[pm].ctype[cell] : kDirichlet;
            }
        }
    }
}

}  // namespace cirrus
