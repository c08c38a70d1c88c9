// C ABI (include/cirrus_b200.h).  Every entry point validates its arguments, maps internal
// failures to cirrus_status and never lets an exception cross the boundary.
#include "../../include/cirrus_b200.h"
#include "dtopo.hpp"
#include "holder.hpp"
#include "serve.hpp"
#include "solver_internal.hpp"
#include "topology.hpp"

#include <algorithm>
#include <cstring>
#include <exception>
#include <new>
#include <vector>

struct cirrus_topology {
    cirrus::Topology* t;
};
struct cirrus_grid {
    cirrus::DevGrid* g;
    // the asynchronous end-to-end solve in flight (cirrus_gmg_solve_host_submit), if any
    struct Pending {
        bool active = false, collected = false;
        cudaStream_t stream = nullptr;
        cirrus::SolveParams p;
        long long direct = -1;
        int rc = 0;
        std::vector<cirrus::SolveResult> r;
    } pending;
};
struct cirrus_server {
    cirrus::Server* s;
};

namespace {

cirrus_status map_rc(int rc) {
    switch (rc) {
    case 0: return CIRRUS_OK;
    case 1: return CIRRUS_ERR_INVALID_ARGUMENT;
    case 2: return CIRRUS_ERR_CUDA;
    case 3: return CIRRUS_ERR_OUT_OF_MEMORY;
    case 4: return CIRRUS_ERR_TOPOLOGY;
    case 5: return CIRRUS_ERR_NOT_CONVERGED;
    case 6: return CIRRUS_ERR_NONFINITE;
    case 7: return CIRRUS_ERR_BUDGET;
    default: return CIRRUS_ERR_STATE;
    }
}

inline bool channel_ok(int c) { return c >= 0 && c < cirrus::kNumChannels; }
inline cudaStream_t S(void* s) { return reinterpret_cast<cudaStream_t>(s); }

template <class F>
cirrus_status guard(F&& f) {
    try {
        return f();
    } catch (const std::bad_alloc&) {
        return CIRRUS_ERR_OUT_OF_MEMORY;
    } catch (...) {
        return CIRRUS_ERR_STATE;
    }
}

cirrus_status cuda_status() {
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) return CIRRUS_OK;
    return e == cudaErrorMemoryAllocation ? CIRRUS_ERR_OUT_OF_MEMORY : CIRRUS_ERR_CUDA;
}

void to_internal(const cirrus_solve_params* p, cirrus::SolveParams* q) {
    q->max_iters = p->max_iters;
    q->tol = p->relative_tolerance;
    q->level_iters = p->level_iters;
    q->coarsest_iters = p->coarsest_iters;
    q->sync_stride = p->sync_stride;
    q->pure_neumann = p->is_pure_neumann ? 1 : 0;
    q->one_over_alpha = p->one_over_alpha;
    q->prolong_coeff = p->prolong_coeff;
    q->precision = p->precision;
    q->warm_start = p->warm_start;
    q->inner_tol = p->inner_tolerance;
    q->max_outer = p->max_outer_iters;
}

bool params_ok(const cirrus_solve_params* p) {
    return p && p->max_iters >= 0 && p->relative_tolerance >= 0 && p->level_iters >= 0 && p->coarsest_iters >= 0 &&
           (p->precision == CIRRUS_PRECISION_FP32 || p->precision == CIRRUS_PRECISION_MIXED_FP64) && p->max_outer_iters >= 0;
}

}  // namespace

extern "C" {

const char* cirrus_status_string(cirrus_status s) {
    switch (s) {
    case CIRRUS_OK: return "ok";
    case CIRRUS_ERR_INVALID_ARGUMENT: return "invalid argument";
    case CIRRUS_ERR_CUDA: return "CUDA error";
    case CIRRUS_ERR_OUT_OF_MEMORY: return "out of device memory";
    case CIRRUS_ERR_TOPOLOGY: return "topology error";
    case CIRRUS_ERR_NOT_CONVERGED: return "not converged";
    case CIRRUS_ERR_NONFINITE: return "non-finite residual";
    case CIRRUS_ERR_BUDGET: return "HBM budget exceeded";
    case CIRRUS_ERR_NO_DEVICE: return "no CUDA device";
    case CIRRUS_ERR_STATE: return "invalid state";
    }
    return "unknown status";
}

const char* cirrus_version(void) { return "cirrus-b200 0.1.0 (sm_100a)"; }

// ---------------------------------------------------------------- topology
cirrus_status cirrus_topology_create(int num_layers, const uint32_t* log2_hash, double h0, cirrus_topology** out) {
    if (!out || !log2_hash || num_layers < 1 || num_layers > 16 || !(h0 > 0)) return CIRRUS_ERR_INVALID_ARGUMENT;
    for (int l = 0; l < num_layers; l++)
        if (log2_hash[l] < 1 || log2_hash[l] > 28) return CIRRUS_ERR_INVALID_ARGUMENT;
    return guard([&] {
        *out = new cirrus_topology{new cirrus::Topology(num_layers, log2_hash, h0)};
        return CIRRUS_OK;
    });
}
void cirrus_topology_destroy(cirrus_topology* topo) {
    if (!topo) return;
    delete topo->t;
    delete topo;
}
cirrus_status cirrus_topology_set_tile(cirrus_topology* topo, int level, int x, int y, int z, int type) {
    if (!topo || level < 0 || level >= topo->t->num_layers()) return CIRRUS_ERR_INVALID_ARGUMENT;
    if (type != CIRRUS_LEAF && type != CIRRUS_NONLEAF && type != CIRRUS_GHOST) return CIRRUS_ERR_INVALID_ARGUMENT;
    return guard([&] { return topo->t->set_tile(level, x, y, z, (uint8_t)type) ? CIRRUS_OK : CIRRUS_ERR_TOPOLOGY; });
}
cirrus_status cirrus_topology_import_tiles(cirrus_topology* topo, const int32_t* tiles5, int num_tiles) {
    if (!topo || !tiles5 || num_tiles <= 0) return CIRRUS_ERR_INVALID_ARGUMENT;
    return guard([&] {
        topo->t->last_error.clear();
        return topo->t->import_tiles(tiles5, num_tiles) ? CIRRUS_OK : CIRRUS_ERR_TOPOLOGY;
    });
}
cirrus_status cirrus_topology_compress(cirrus_topology* topo) {
    if (!topo) return CIRRUS_ERR_INVALID_ARGUMENT;
    return guard([&] { topo->t->compress_and_sync(); return CIRRUS_OK; });
}
cirrus_status cirrus_topology_spawn_ghost_tiles(cirrus_topology* topo) {
    if (!topo) return CIRRUS_ERR_INVALID_ARGUMENT;
    return guard([&] {
        topo->t->last_error.clear();
        topo->t->spawn_ghost_tiles();
        return topo->t->last_error.empty() ? CIRRUS_OK : CIRRUS_ERR_TOPOLOGY;
    });
}
cirrus_status cirrus_topology_refine_leafs_one_step(cirrus_topology* topo, cirrus_level_target_fn fn, void* user,
                                                    int* refined_per_level) {
    if (!topo || !fn) return CIRRUS_ERR_INVALID_ARGUMENT;
    return guard([&] {
        topo->t->last_error.clear();
        auto c = topo->t->refine_leafs_one_step([&](int l, int x, int y, int z) { return fn(user, l, x, y, z); });
        if (refined_per_level)
            for (size_t i = 0; i < c.size(); i++) refined_per_level[i] = c[i];
        return topo->t->last_error.empty() ? CIRRUS_OK : CIRRUS_ERR_TOPOLOGY;
    });
}
cirrus_status cirrus_topology_iterative_refine(cirrus_topology* topo, cirrus_level_target_fn fn, void* user) {
    if (!topo || !fn) return CIRRUS_ERR_INVALID_ARGUMENT;
    return guard([&] {
        topo->t->last_error.clear();
        topo->t->iterative_refine([&](int l, int x, int y, int z) { return fn(user, l, x, y, z); });
        return topo->t->last_error.empty() ? CIRRUS_OK : CIRRUS_ERR_TOPOLOGY;
    });
}
cirrus_status cirrus_topology_iterative_refine_masks(cirrus_topology* topo, const uint8_t* const* masks, const int* dims) {
    if (!topo || !masks || !dims) return CIRRUS_ERR_INVALID_ARGUMENT;
    const int nl = topo->t->num_layers();
    return guard([&] {
        topo->t->last_error.clear();
        topo->t->iterative_refine([&](int l, int x, int y, int z) {
            if (l < 0 || l >= nl || !masks[l]) return l;
            const int* d = dims + 3 * l;
            if (x < 0 || y < 0 || z < 0 || x >= d[0] || y >= d[1] || z >= d[2]) return l;
            return masks[l][((size_t)x * d[1] + y) * d[2] + z] ? l + 1 : l;
        });
        return topo->t->last_error.empty() ? CIRRUS_OK : CIRRUS_ERR_TOPOLOGY;
    });
}
cirrus_status cirrus_topology_num_tiles(const cirrus_topology* topo, int* num_tiles) {
    if (!topo || !num_tiles) return CIRRUS_ERR_INVALID_ARGUMENT;
    *num_tiles = topo->t->num_tiles();
    return CIRRUS_OK;
}
cirrus_status cirrus_topology_max_level(const cirrus_topology* topo, int* max_level) {
    if (!topo || !max_level) return CIRRUS_ERR_INVALID_ARGUMENT;
    *max_level = topo->t->max_level();
    return CIRRUS_OK;
}
cirrus_status cirrus_topology_tiles(const cirrus_topology* topo, int32_t* out5) {
    if (!topo || !out5) return CIRRUS_ERR_INVALID_ARGUMENT;
    topo->t->tiles(out5);
    return CIRRUS_OK;
}
cirrus_status cirrus_topology_hash_slots(const cirrus_topology* topo, int32_t* out) {
    if (!topo || !out) return CIRRUS_ERR_INVALID_ARGUMENT;
    topo->t->hash_slots(out);
    return CIRRUS_OK;
}
cirrus_status cirrus_topology_set_cell_types(cirrus_topology* topo, const uint8_t* ctypes) {
    if (!topo || !ctypes) return CIRRUS_ERR_INVALID_ARGUMENT;
    topo->t->set_cell_types(ctypes);
    return CIRRUS_OK;
}
cirrus_status cirrus_topology_cell_types(const cirrus_topology* topo, uint8_t* ctypes) {
    if (!topo || !ctypes) return CIRRUS_ERR_INVALID_ARGUMENT;
    topo->t->cell_types(ctypes);
    return CIRRUS_OK;
}
cirrus_status cirrus_topology_calc_cell_types_from_leafs(cirrus_topology* topo) {
    if (!topo) return CIRRUS_ERR_INVALID_ARGUMENT;
    return guard([&] { topo->t->calc_cell_types_from_leafs(); return CIRRUS_OK; });
}
cirrus_status cirrus_topology_neighbor_tiles(const cirrus_topology* topo, int32_t* out6) {
    if (!topo || !out6) return CIRRUS_ERR_INVALID_ARGUMENT;
    topo->t->neighbor_tiles(out6);
    return CIRRUS_OK;
}

// ---------------------------------------------------------------- device grid
cirrus_status cirrus_grid_create(const cirrus_topology* topo, cirrus_grid** out) {
    if (!topo || !out) return CIRRUS_ERR_INVALID_ARGUMENT;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return CIRRUS_ERR_NO_DEVICE;
    }
    return guard([&] {
        cirrus::DevGrid* g = nullptr;
        std::string err;
        int rc = cirrus::grid_create({topo->t}, &g, &err);
        if (rc) return map_rc(rc);
        *out = new cirrus_grid{g};
        return CIRRUS_OK;
    });
}
cirrus_status cirrus_grid_create_from_desc(const cirrus_grid_desc* d, cirrus_grid** out) {
    if (!d || !out || d->num_layers <= 0 || !d->log2_hash || !d->tiles_per_level || !d->coords || !d->types || !d->cell_types)
        return CIRRUS_ERR_INVALID_ARGUMENT;
    long long n = 0;
    for (int l = 0; l < d->num_layers; l++) {
        if (d->tiles_per_level[l] < 0) return CIRRUS_ERR_INVALID_ARGUMENT;
        n += d->tiles_per_level[l];
    }
    if (n <= 0 || n > (1LL << 30)) return CIRRUS_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    cirrus_topology* topo = nullptr;
    cirrus_status st = cirrus_topology_create(d->num_layers, d->log2_hash, d->h0, &topo);
    if (st != CIRRUS_OK) return st;
    st = guard([&] {
        std::vector<int32_t> t5((size_t)n * 5);
        size_t q = 0;
        for (int l = 0; l < d->num_layers; l++)
            for (int k = 0; k < d->tiles_per_level[l]; k++, q++) {
                t5[5 * q] = l;
                t5[5 * q + 1] = d->coords[3 * q];
                t5[5 * q + 2] = d->coords[3 * q + 1];
                t5[5 * q + 3] = d->coords[3 * q + 2];
                t5[5 * q + 4] = d->types[q];
            }
        cirrus_status r = cirrus_topology_import_tiles(topo, t5.data(), (int)n);
        if (r == CIRRUS_OK) r = cirrus_topology_set_cell_types(topo, d->cell_types);
        if (r == CIRRUS_OK) r = cirrus_grid_create(topo, out);
        if (r == CIRRUS_OK && d->b) r = cirrus_grid_set_channel(*out, 1, d->b, nullptr);
        if (r == CIRRUS_OK && d->x0) r = cirrus_grid_set_channel(*out, 0, d->x0, nullptr);
        if (r == CIRRUS_OK && cudaStreamSynchronize(nullptr) != cudaSuccess) r = cuda_status();
        if (r != CIRRUS_OK && *out) {
            cirrus_grid_destroy(*out);
            *out = nullptr;
        }
        return r;
    });
    cirrus_topology_destroy(topo);
    return st;
}

cirrus_status cirrus_grid_create_batch(const cirrus_topology* const* topos, int count, cirrus_grid** out) {
    if (!topos || count <= 0 || !out) return CIRRUS_ERR_INVALID_ARGUMENT;
    for (int i = 0; i < count; i++)
        if (!topos[i]) return CIRRUS_ERR_INVALID_ARGUMENT;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return CIRRUS_ERR_NO_DEVICE;
    }
    return guard([&] {
        std::vector<const cirrus::Topology*> ts;
        for (int i = 0; i < count; i++) ts.push_back(topos[i]->t);
        cirrus::DevGrid* g = nullptr;
        std::string err;
        int rc = cirrus::grid_create(ts, &g, &err);
        if (rc) return map_rc(rc);
        *out = new cirrus_grid{g};
        return CIRRUS_OK;
    });
}
cirrus_status cirrus_grid_num_instances(const cirrus_grid* grid, int* count) {
    if (!grid || !count) return CIRRUS_ERR_INVALID_ARGUMENT;
    *count = grid->g->num_inst;
    return CIRRUS_OK;
}
cirrus_status cirrus_grid_instance_info(const cirrus_grid* grid, int instance, int* num_tiles, int64_t* dof) {
    if (!grid || instance < 0 || instance >= grid->g->num_inst) return CIRRUS_ERR_INVALID_ARGUMENT;
    if (num_tiles) *num_tiles = grid->g->inst_tiles[instance];
    if (dof) *dof = grid->g->inst_dof[instance];
    return CIRRUS_OK;
}
cirrus_status cirrus_grid_set_channel_instance(cirrus_grid* grid, int instance, int channel, const float* host, void* stream) {
    if (!grid || !host || !channel_ok(channel) || instance < 0 || instance >= grid->g->num_inst) return CIRRUS_ERR_INVALID_ARGUMENT;
    for (const cirrus::TileRun& r : grid->g->inst_runs[instance])
        if (cudaMemcpyAsync(grid->g->d_ch[channel] + (size_t)r.global * cirrus::kTileCells, host + (size_t)r.local * cirrus::kTileCells,
                            (size_t)r.count * cirrus::kTileCells * sizeof(float), cudaMemcpyHostToDevice, S(stream)) != cudaSuccess)
            return cuda_status();
    return cudaStreamSynchronize(S(stream)) == cudaSuccess ? CIRRUS_OK : cuda_status();
}
cirrus_status cirrus_grid_get_channel_instance(const cirrus_grid* grid, int instance, int channel, float* host, void* stream) {
    if (!grid || !host || !channel_ok(channel) || instance < 0 || instance >= grid->g->num_inst) return CIRRUS_ERR_INVALID_ARGUMENT;
    for (const cirrus::TileRun& r : grid->g->inst_runs[instance])
        if (cudaMemcpyAsync(host + (size_t)r.local * cirrus::kTileCells, grid->g->d_ch[channel] + (size_t)r.global * cirrus::kTileCells,
                            (size_t)r.count * cirrus::kTileCells * sizeof(float), cudaMemcpyDeviceToHost, S(stream)) != cudaSuccess)
            return cuda_status();
    return cudaStreamSynchronize(S(stream)) == cudaSuccess ? CIRRUS_OK : cuda_status();
}
void cirrus_grid_destroy(cirrus_grid* grid) {
    if (!grid) return;
    if (grid->pending.active) cudaStreamSynchronize(grid->pending.stream);
    cirrus::grid_destroy(grid->g);
    delete grid;
}
cirrus_status cirrus_grid_num_tiles(const cirrus_grid* grid, int* num_tiles) {
    if (!grid || !num_tiles) return CIRRUS_ERR_INVALID_ARGUMENT;
    *num_tiles = grid->g->n;
    return CIRRUS_OK;
}
cirrus_status cirrus_grid_device_bytes(const cirrus_grid* grid, size_t* bytes) {
    if (!grid || !bytes) return CIRRUS_ERR_INVALID_ARGUMENT;
    *bytes = grid->g->bytes;
    return CIRRUS_OK;
}
cirrus_status cirrus_grid_dof(const cirrus_grid* grid, int64_t* dof) {
    if (!grid || !dof) return CIRRUS_ERR_INVALID_ARGUMENT;
    *dof = grid->g->dof;
    return CIRRUS_OK;
}
cirrus_status cirrus_grid_set_channel(cirrus_grid* grid, int channel, const float* host, void* stream) {
    if (!grid || !host || !channel_ok(channel)) return CIRRUS_ERR_INVALID_ARGUMENT;
    const size_t bytes = (size_t)grid->g->n * cirrus::kTileCells * sizeof(float);
    if (cudaMemcpyAsync(grid->g->d_ch[channel], host, bytes, cudaMemcpyHostToDevice, S(stream)) != cudaSuccess) return cuda_status();
    return cudaStreamSynchronize(S(stream)) == cudaSuccess ? CIRRUS_OK : cuda_status();
}
cirrus_status cirrus_grid_get_channel(const cirrus_grid* grid, int channel, float* host, void* stream) {
    if (!grid || !host || !channel_ok(channel)) return CIRRUS_ERR_INVALID_ARGUMENT;
    const size_t bytes = (size_t)grid->g->n * cirrus::kTileCells * sizeof(float);
    if (cudaMemcpyAsync(host, grid->g->d_ch[channel], bytes, cudaMemcpyDeviceToHost, S(stream)) != cudaSuccess) return cuda_status();
    return cudaStreamSynchronize(S(stream)) == cudaSuccess ? CIRRUS_OK : cuda_status();
}
cirrus_status cirrus_grid_copy_channel(cirrus_grid* grid, int dst_channel, int src_channel, void* stream) {
    if (!grid || !channel_ok(dst_channel) || !channel_ok(src_channel)) return CIRRUS_ERR_INVALID_ARGUMENT;
    if (dst_channel == src_channel) return CIRRUS_OK;
    const size_t bytes = (size_t)grid->g->n * cirrus::kTileCells * sizeof(float);
    if (cudaMemcpyAsync(grid->g->d_ch[dst_channel], grid->g->d_ch[src_channel], bytes, cudaMemcpyDeviceToDevice, S(stream)) !=
        cudaSuccess)
        return cuda_status();
    return CIRRUS_OK;
}
cirrus_status cirrus_grid_set_tile_pointers(cirrus_grid* grid, const void* const* tile_ptrs) {
    if (!grid || !tile_ptrs) return CIRRUS_ERR_INVALID_ARGUMENT;
    auto& g = *grid->g;
    for (int i = 0; i < g.n; i++)
        if (!tile_ptrs[i] || (reinterpret_cast<uintptr_t>(tile_ptrs[i]) & 15u)) return CIRRUS_ERR_INVALID_ARGUMENT;
    if (!g.d_tile_ptrs && cudaMalloc(&g.d_tile_ptrs, sizeof(void*) * g.n) != cudaSuccess) return cuda_status();
    if (cudaMemcpy(g.d_tile_ptrs, tile_ptrs, sizeof(void*) * g.n, cudaMemcpyHostToDevice) != cudaSuccess) return cuda_status();
    return CIRRUS_OK;
}
cirrus_status cirrus_grid_gather_tiles(cirrus_grid* grid, int channel, size_t byte_offset, void* stream) {
    if (!grid || !channel_ok(channel) || (byte_offset & 15u)) return CIRRUS_ERR_INVALID_ARGUMENT;
    if (!grid->g->d_tile_ptrs) return CIRRUS_ERR_STATE;
    cirrus::launch::gather_tiles(*grid->g, channel, byte_offset, S(stream));
    return cuda_status();
}
cirrus_status cirrus_grid_scatter_tiles(cirrus_grid* grid, int channel, size_t byte_offset, void* stream) {
    if (!grid || !channel_ok(channel) || (byte_offset & 15u)) return CIRRUS_ERR_INVALID_ARGUMENT;
    if (!grid->g->d_tile_ptrs) return CIRRUS_ERR_STATE;
    cirrus::launch::scatter_tiles(*grid->g, channel, byte_offset, S(stream));
    return cuda_status();
}
cirrus_status cirrus_grid_compare_tile_cell_types(cirrus_grid* grid, size_t byte_offset, void* stream, int* changed,
                                                 uint8_t* host_types) {
    if (!grid || !changed || (byte_offset & 3u)) return CIRRUS_ERR_INVALID_ARGUMENT;
    auto& g = *grid->g;
    if (!g.d_tile_ptrs) return CIRRUS_ERR_STATE;
    const size_t cells = (size_t)g.n * cirrus::kTileCells;
    if (!g.d_ct_gather) {
        if (cudaMalloc(&g.d_ct_gather, cells) != cudaSuccess) return cuda_status();
        if (cudaMalloc(&g.d_ct_flag, sizeof(unsigned int)) != cudaSuccess) return cuda_status();
        g.bytes += cells + sizeof(unsigned int);
    }
    cirrus::launch::compare_tile_cell_types(g, byte_offset, S(stream));
    unsigned int flag = 0;
    if (cudaMemcpyAsync(&flag, g.d_ct_flag, sizeof(flag), cudaMemcpyDeviceToHost, S(stream)) != cudaSuccess) return cuda_status();
    if (cudaStreamSynchronize(S(stream)) != cudaSuccess) return cuda_status();
    *changed = flag ? 1 : 0;
    if (flag && host_types &&
        cudaMemcpyAsync(host_types, g.d_ct_gather, cells, cudaMemcpyDeviceToHost, S(stream)) != cudaSuccess)
        return cuda_status();
    return cudaStreamSynchronize(S(stream)) == cudaSuccess ? CIRRUS_OK : cuda_status();
}
cirrus_status cirrus_gather_tile_bytes(const void* const* tile_ptrs, int num_tiles, size_t byte_offset, uint8_t* host_out,
                                       void* stream) {
    if (!tile_ptrs || num_tiles <= 0 || !host_out || (byte_offset & 3u)) return CIRRUS_ERR_INVALID_ARGUMENT;
    for (int i = 0; i < num_tiles; i++)
        if (!tile_ptrs[i] || (reinterpret_cast<uintptr_t>(tile_ptrs[i]) & 3u)) return CIRRUS_ERR_INVALID_ARGUMENT;
    return map_rc(cirrus::gather_tile_bytes(tile_ptrs, num_tiles, byte_offset, host_out, S(stream)));
}
cirrus_status cirrus_grid_set_launch_mode(cirrus_grid* grid, int mode) {
    if (!grid || (mode != CIRRUS_LAUNCH_GRAPH && mode != CIRRUS_LAUNCH_DIRECT)) return CIRRUS_ERR_INVALID_ARGUMENT;
    grid->g->launch_mode = mode;
    return CIRRUS_OK;
}
cirrus_status cirrus_grid_get_launch_mode(const cirrus_grid* grid, int* mode) {
    if (!grid || !mode) return CIRRUS_ERR_INVALID_ARGUMENT;
    *mode = grid->g->launch_mode;
    return CIRRUS_OK;
}
cirrus_status cirrus_grid_channel_ptr(cirrus_grid* grid, int channel, float** device_ptr) {
    if (!grid || !device_ptr || !channel_ok(channel)) return CIRRUS_ERR_INVALID_ARGUMENT;
    *device_ptr = grid->g->d_ch[channel];
    return CIRRUS_OK;
}

// ---------------------------------------------------------------- operators
cirrus_status cirrus_full_negative_laplacian(cirrus_grid* grid, int x_channel, int Ax_channel, void* stream) {
    if (!grid || !channel_ok(x_channel) || !channel_ok(Ax_channel) || x_channel == Ax_channel) return CIRRUS_ERR_INVALID_ARGUMENT;
    auto& g = *grid->g;
    cirrus::launch::full_laplacian<float>(g, g.d_ch[x_channel], g.d_ch[Ax_channel], nullptr, S(stream));
    return cuda_status();
}
cirrus_status cirrus_full_negative_laplacian_ex(cirrus_grid* grid, int x_channel, int Ax_channel, int calc_diag, void* stream) {
    if (!calc_diag) return cirrus_full_negative_laplacian(grid, x_channel, Ax_channel, stream);
    if (!grid || !channel_ok(x_channel) || !channel_ok(Ax_channel) || x_channel == Ax_channel) return CIRRUS_ERR_INVALID_ARGUMENT;
    auto& g = *grid->g;
    cirrus::launch::full_laplacian_diag(g, g.d_ch[x_channel], g.d_ch[Ax_channel], S(stream));
    return cuda_status();
}
cirrus_status cirrus_negative_laplacian_same_level(cirrus_grid* grid, int tile_level, int subtree_level, int launch_tile_types,
                                                   int x_channel, int Ax_channel, int calc_diag, void* stream) {
    if (!grid || !channel_ok(x_channel) || !channel_ok(Ax_channel) || x_channel == Ax_channel) return CIRRUS_ERR_INVALID_ARGUMENT;
    auto& g = *grid->g;
    if (tile_level < -1 || tile_level >= (int)g.level_count.size() || subtree_level < -1 || (launch_tile_types & ~7) != 0)
        return CIRRUS_ERR_INVALID_ARGUMENT;
    cirrus::launch::laplacian_same_level(g, tile_level, subtree_level, (uint32_t)launch_tile_types, g.d_ch[x_channel],
                                         g.d_ch[Ax_channel], calc_diag != 0, S(stream));
    return cuda_status();
}
cirrus_status cirrus_gauss_seidel_sweep(cirrus_grid* grid, int level, int x_channel, int rhs_channel, int color, void* stream) {
    if (!grid || !channel_ok(x_channel) || !channel_ok(rhs_channel) || (color != 0 && color != 1)) return CIRRUS_ERR_INVALID_ARGUMENT;
    auto& g = *grid->g;
    if (level < 0 || level >= g.num_layers) return CIRRUS_ERR_INVALID_ARGUMENT;
    cirrus::launch::gs_sweep(g, level, g.d_ch[x_channel], g.d_ch[rhs_channel], color, nullptr, S(stream));
    return cuda_status();
}
cirrus_status cirrus_residual_and_restrict(cirrus_grid* grid, int level, int x_channel, int rhs_channel, int coarse_channel,
                                           float one_over_alpha, void* stream) {
    if (!grid || !channel_ok(x_channel) || !channel_ok(rhs_channel) || !channel_ok(coarse_channel)) return CIRRUS_ERR_INVALID_ARGUMENT;
    auto& g = *grid->g;
    if (level < 1 || level >= g.num_layers) return CIRRUS_ERR_INVALID_ARGUMENT;
    cirrus::launch::residual_restrict(g, level, g.d_ch[x_channel], g.d_ch[rhs_channel], g.d_ch[coarse_channel], one_over_alpha, nullptr,
                                      S(stream));
    return cuda_status();
}
cirrus_status cirrus_prolongate_and_update(cirrus_grid* grid, int fine_level, int coarse_channel, int fine_channel,
                                           float prolong_coeff, void* stream) {
    if (!grid || !channel_ok(coarse_channel) || !channel_ok(fine_channel)) return CIRRUS_ERR_INVALID_ARGUMENT;
    auto& g = *grid->g;
    if (fine_level < 1 || fine_level >= g.num_layers) return CIRRUS_ERR_INVALID_ARGUMENT;
    cirrus::launch::prolongate(g, fine_level, g.d_ch[coarse_channel], g.d_ch[fine_channel], prolong_coeff, nullptr, S(stream));
    return cuda_status();
}
cirrus_status cirrus_vcycle(cirrus_grid* grid, int x_channel, int f_channel, int rhs_channel, int level_iters, int coarsest_iters,
                            void* stream) {
    if (!grid || !channel_ok(x_channel) || !channel_ok(f_channel) || !channel_ok(rhs_channel) || level_iters < 0 || coarsest_iters < 0)
        return CIRRUS_ERR_INVALID_ARGUMENT;
    auto& g = *grid->g;
    if (cirrus::use_fused(g, level_iters, coarsest_iters) && x_channel != rhs_channel && f_channel != rhs_channel &&
        x_channel != f_channel) {
        // the fused schedule takes f already copied into the right-hand-side channel
        cirrus::launch::vcycle_init(g, g.d_ch[x_channel], g.d_ch[rhs_channel], g.d_ch[f_channel], nullptr, S(stream));
        cirrus::vcycle_fused(g, g.d_ch[x_channel], g.d_ch[rhs_channel], coarsest_iters, 1.f, 1.f, nullptr, S(stream));
    } else {
        cirrus::vcycle(g, g.d_ch[x_channel], g.d_ch[f_channel], g.d_ch[rhs_channel], level_iters, coarsest_iters, 1.f, 1.f,
                       nullptr, S(stream));
    }
    return cuda_status();
}
cirrus_status cirrus_dot(cirrus_grid* grid, int a_channel, int b_channel, double* result, void* stream) {
    if (!grid || !result || !channel_ok(a_channel) || !channel_ok(b_channel)) return CIRRUS_ERR_INVALID_ARGUMENT;
    auto& g = *grid->g;
    cirrus::launch::grid_dot(g, g.d_ch[a_channel], g.d_ch[b_channel], S(stream));
    if (cudaMemcpyAsync(result, &g.d_dot->gamma, sizeof(double), cudaMemcpyDeviceToHost, S(stream)) != cudaSuccess)
        return cuda_status();
    if (cudaStreamSynchronize(S(stream)) != cudaSuccess) return cuda_status();
    return cuda_status();
}

cirrus_status cirrus_clear_neumann_neighbor_faces(cirrus_grid* grid, int u_channel, void* stream) {
    if (!grid || u_channel < 0 || u_channel + 2 >= cirrus::kNumChannels) return CIRRUS_ERR_INVALID_ARGUMENT;
    cirrus::launch::clear_neumann_faces(*grid->g, u_channel, S(stream));
    return cuda_status();
}
cirrus_status cirrus_propagate_to_children(cirrus_grid* grid, int channel, void* stream) {
    if (!grid || !channel_ok(channel)) return CIRRUS_ERR_INVALID_ARGUMENT;
    cirrus::launch::propagate_to_children(*grid->g, channel, S(stream));
    return cuda_status();
}
cirrus_status cirrus_velocity_volume_divergence_on_leafs(cirrus_grid* grid, int u_channel, int div_channel, void* stream) {
    if (!grid || u_channel < 0 || u_channel + 2 >= cirrus::kNumChannels || !channel_ok(div_channel) ||
        (div_channel >= u_channel && div_channel <= u_channel + 2))
        return CIRRUS_ERR_INVALID_ARGUMENT;
    cirrus::launch::velocity_divergence(*grid->g, u_channel, div_channel, S(stream));
    return cuda_status();
}

cirrus_status cirrus_add_gradient_to_face_centers(cirrus_grid* grid, int p_channel, int u_channel, void* stream) {
    if (!grid || !channel_ok(p_channel) || u_channel < 0 || u_channel + 2 >= cirrus::kNumChannels ||
        (p_channel >= u_channel && p_channel <= u_channel + 2))
        return CIRRUS_ERR_INVALID_ARGUMENT;
    cirrus::launch::add_gradient(*grid->g, p_channel, u_channel, S(stream));
    return cuda_status();
}

// ---------------------------------------------------------------- solve
void cirrus_solve_params_default(cirrus_solve_params* p) {
    if (!p) return;
    p->max_iters = 1000;
    p->relative_tolerance = 1e-6;
    p->level_iters = 1;
    p->coarsest_iters = 10;
    p->sync_stride = 1;
    p->is_pure_neumann = 0;
    p->one_over_alpha = 1.f;
    p->prolong_coeff = 1.f;
    p->precision = CIRRUS_PRECISION_FP32;
    p->warm_start = 0;
    p->inner_tolerance = 1e-7;
    p->max_outer_iters = 20;
}

namespace {
// the batched solve with the GMG (0) or the AMG (1) preconditioner
cirrus_status solve_batch_with(int preconditioner, cirrus_grid* grid, const cirrus_solve_params* params, const int* active,
                               const double* tolerances, const int* pure_neumann, void* stream, cirrus_solve_result* results) {
    if (!grid || !params_ok(params) || !results) return CIRRUS_ERR_INVALID_ARGUMENT;
    const int K = grid->g->num_inst;
    if (tolerances)
        for (int i = 0; i < K; i++)
            if (!(tolerances[i] >= 0)) return CIRRUS_ERR_INVALID_ARGUMENT;
    return guard([&] {
        cirrus::SolveParams p;
        to_internal(params, &p);
        p.preconditioner = preconditioner;
        std::vector<cirrus::InstRequest> req(K);
        for (int i = 0; i < K; i++) {
            req[i].active = active ? (active[i] ? 1 : 0) : 1;
            if (tolerances) req[i].tol = tolerances[i];
            if (pure_neumann) req[i].pure_neumann = pure_neumann[i] ? 1 : 0;
        }
        std::vector<cirrus::SolveResult> r(K);
        if (p.precision != CIRRUS_PRECISION_MIXED_FP64) grid->g->x64_valid = false;
        int rc = p.precision == CIRRUS_PRECISION_MIXED_FP64 ? cirrus::mixed_solve(*grid->g, p, S(stream), r.data(), req.data())
                                                            : cirrus::pcg_solve(*grid->g, p, S(stream), r.data(), req.data());
        if (rc) return map_rc(rc);
        for (int i = 0; i < K; i++) {
            results[i].iters = r[i].iters;
            results[i].outer_iters = r[i].outer;
            results[i].rel_residual = r[i].rel;
            results[i].true_rel_residual = r[i].true_rel;
            results[i].status = (int)map_rc(r[i].status);
            results[i].kernel_launches = r[i].launches;
        }
        return CIRRUS_OK;
    });
}
}  // namespace

cirrus_status cirrus_gmg_solve_batch(cirrus_grid* grid, const cirrus_solve_params* params, const int* active,
                                     const double* tolerances, const int* pure_neumann, void* stream,
                                     cirrus_solve_result* results) {
    return solve_batch_with(0, grid, params, active, tolerances, pure_neumann, stream, results);
}

namespace {
cirrus_status solve_grids_with(int preconditioner, cirrus_grid* const* grids, int count, const cirrus_solve_params* params,
                               void* stream, cirrus_solve_result* results) {
    if (!grids || count <= 0 || !params_ok(params) || !results) return CIRRUS_ERR_INVALID_ARGUMENT;
    std::vector<cirrus::DevGrid*> gs(count);
    for (int k = 0; k < count; k++) {
        if (!grids[k]) return CIRRUS_ERR_INVALID_ARGUMENT;
        gs[k] = grids[k]->g;
        for (int j = 0; j < k; j++)
            if (gs[j] == gs[k]) return CIRRUS_ERR_INVALID_ARGUMENT;  // one solve in flight per grid
    }
    if (preconditioner == 1)
        for (cirrus::DevGrid* g : gs)
            if (!g->amg_ready) return CIRRUS_ERR_STATE;
    return guard([&] {
        cirrus::SolveParams p;
        to_internal(params, &p);
        p.preconditioner = preconditioner;
        std::vector<std::vector<cirrus::SolveResult>> r;
        const int rc = cirrus::solve_grids(gs, p, S(stream), r);
        if (rc) return map_rc(rc);
        int o = 0;
        for (int k = 0; k < count; k++)
            for (const cirrus::SolveResult& x : r[k]) {
                results[o].iters = x.iters;
                results[o].outer_iters = x.outer;
                results[o].rel_residual = x.rel;
                results[o].true_rel_residual = x.true_rel;
                results[o].status = (int)map_rc(x.status);
                results[o].kernel_launches = x.launches;
                o++;
            }
        return CIRRUS_OK;
    });
}
}  // namespace

cirrus_status cirrus_gmg_solve_grids(cirrus_grid* const* grids, int count, const cirrus_solve_params* params, void* stream,
                                     cirrus_solve_result* results) {
    return solve_grids_with(0, grids, count, params, stream, results);
}
cirrus_status cirrus_amg_solve_grids(cirrus_grid* const* grids, int count, const cirrus_solve_params* params, void* stream,
                                     cirrus_solve_result* results) {
    return solve_grids_with(1, grids, count, params, stream, results);
}

cirrus_status cirrus_gmg_solve(cirrus_grid* grid, const cirrus_solve_params* params, void* stream, cirrus_solve_result* result) {
    if (!grid || !params_ok(params) || !result) return CIRRUS_ERR_INVALID_ARGUMENT;
    return guard([&] {
        std::vector<cirrus_solve_result> all(grid->g->num_inst);
        cirrus_status st = cirrus_gmg_solve_batch(grid, params, nullptr, nullptr, nullptr, stream, all.data());
        if (st == CIRRUS_OK) *result = all[0];
        return st;
    });
}

cirrus_status cirrus_amg_prepare(cirrus_grid* grid, float one_over_alpha, void* stream) {
    if (!grid || !(one_over_alpha == one_over_alpha)) return CIRRUS_ERR_INVALID_ARGUMENT;
    return guard([&] {
        const int rc = cirrus::amg_prepare(*grid->g, one_over_alpha, S(stream));
        return rc ? map_rc(rc) : cuda_status();
    });
}
cirrus_status cirrus_amg_coefficients(cirrus_grid* grid, float* coeffs, uint8_t* types, void* stream) {
    if (!grid) return CIRRUS_ERR_INVALID_ARGUMENT;
    const int rc = cirrus::amg_download(*grid->g, coeffs, types, S(stream));
    return rc == 1 ? CIRRUS_ERR_STATE : map_rc(rc);
}
cirrus_status cirrus_amg_vcycle(cirrus_grid* grid, int x_channel, int f_channel, int tmp_channel, int rhs_channel, int level_iters,
                                int coarsest_iters, float one_over_alpha, float prolong_coeff, void* stream) {
    if (!grid || !channel_ok(x_channel) || !channel_ok(f_channel) || !channel_ok(tmp_channel) || !channel_ok(rhs_channel) ||
        level_iters < 0 || coarsest_iters < 0)
        return CIRRUS_ERR_INVALID_ARGUMENT;
    const int ch[4] = {x_channel, f_channel, tmp_channel, rhs_channel};
    for (int a = 0; a < 4; a++)
        for (int b = a + 1; b < 4; b++)
            if (ch[a] == ch[b]) return CIRRUS_ERR_INVALID_ARGUMENT;
    auto& g = *grid->g;
    if (!g.amg_ready) return CIRRUS_ERR_STATE;
    cirrus::vcycle_amg(g, g.d_ch[x_channel], g.d_ch[f_channel], g.d_ch[tmp_channel], g.d_ch[rhs_channel], level_iters, coarsest_iters,
                       one_over_alpha, prolong_coeff, nullptr, S(stream));
    return cuda_status();
}
cirrus_status cirrus_amg_solve_batch(cirrus_grid* grid, const cirrus_solve_params* params, const int* active, const double* tolerances,
                                     const int* pure_neumann, void* stream, cirrus_solve_result* results) {
    if (grid && !grid->g->amg_ready) return CIRRUS_ERR_STATE;
    return solve_batch_with(1, grid, params, active, tolerances, pure_neumann, stream, results);
}
cirrus_status cirrus_amg_solve(cirrus_grid* grid, const cirrus_solve_params* params, void* stream, cirrus_solve_result* result) {
    if (!grid || !params_ok(params) || !result) return CIRRUS_ERR_INVALID_ARGUMENT;
    return guard([&] {
        std::vector<cirrus_solve_result> all(grid->g->num_inst);
        cirrus_status st = cirrus_amg_solve_batch(grid, params, nullptr, nullptr, nullptr, stream, all.data());
        if (st == CIRRUS_OK) *result = all[0];
        return st;
    });
}

cirrus_status cirrus_gmg_solve_host(cirrus_grid* grid, const cirrus_solve_params* params, const float* b_host, float* x_host,
                                    void* stream, cirrus_solve_result* result) {
    if (!grid || !params_ok(params) || !b_host || !x_host || !result) return CIRRUS_ERR_INVALID_ARGUMENT;
    auto& g = *grid->g;
    const size_t bytes = (size_t)g.n * cirrus::kTileCells * sizeof(float);
    if (cudaMemcpyAsync(g.d_ch[cirrus::kChB], b_host, bytes, cudaMemcpyHostToDevice, S(stream)) != cudaSuccess) return cuda_status();
    cirrus_status st = cirrus_gmg_solve(grid, params, stream, result);
    if (st != CIRRUS_OK) return st;
    if (cudaMemcpyAsync(x_host, g.d_ch[cirrus::kChX], bytes, cudaMemcpyDeviceToHost, S(stream)) != cudaSuccess) return cuda_status();
    return cudaStreamSynchronize(S(stream)) == cudaSuccess ? CIRRUS_OK : cuda_status();
}

cirrus_status cirrus_gmg_solve_host_wait(cirrus_grid* grid, cirrus_solve_result* results) {
    if (!grid || !results || !grid->pending.active) return CIRRUS_ERR_INVALID_ARGUMENT;
    auto& pd = grid->pending;
    auto& g = *grid->g;
    pd.active = false;
    if (!pd.collected) {
        if (cudaStreamSynchronize(pd.stream) != cudaSuccess) return cuda_status();
        pd.r.assign(g.num_inst, cirrus::SolveResult());
        cirrus::pcg_collect(g, pd.p, pd.direct, pd.r.data());
    }
    if (pd.rc) return map_rc(pd.rc);
    for (int i = 0; i < g.num_inst; i++) {
        results[i].iters = pd.r[i].iters;
        results[i].outer_iters = pd.r[i].outer;
        results[i].rel_residual = pd.r[i].rel;
        results[i].true_rel_residual = pd.r[i].true_rel;
        results[i].status = (int)map_rc(pd.r[i].status);
        results[i].kernel_launches = pd.r[i].launches;
    }
    return CIRRUS_OK;
}

cirrus_status cirrus_gmg_solve_host_submit(cirrus_grid* grid, const cirrus_solve_params* params, const float* b_host, float* x_host,
                                           void* stream) {
    if (!grid || !params_ok(params) || !b_host || !x_host) return CIRRUS_ERR_INVALID_ARGUMENT;
    if (grid->pending.active) {  // one solve in flight per grid: finish the previous one first
        std::vector<cirrus_solve_result> prev(grid->g->num_inst);
        cirrus_gmg_solve_host_wait(grid, prev.data());
    }
    return guard([&] {
        auto& g = *grid->g;
        auto& pd = grid->pending;
        const size_t bytes = (size_t)g.n * cirrus::kTileCells * sizeof(float);
        if (cudaMemcpyAsync(g.d_ch[cirrus::kChB], b_host, bytes, cudaMemcpyHostToDevice, S(stream)) != cudaSuccess) return cuda_status();
        to_internal(params, &pd.p);
        pd.stream = S(stream);
        pd.direct = -1;
        pd.rc = 0;
        pd.collected = false;
        if (pd.p.precision == CIRRUS_PRECISION_MIXED_FP64) {
            // the outer refinement loop reads residuals on the host: runs to completion here
            pd.r.assign(g.num_inst, cirrus::SolveResult());
            pd.rc = cirrus::mixed_solve(g, pd.p, pd.stream, pd.r.data(), nullptr);
            pd.collected = true;
        } else {
            g.x64_valid = false;
            const int rc = cirrus::pcg_launch(g, pd.p, pd.stream, nullptr, &pd.direct);
            if (rc) return map_rc(rc);
        }
        if (!pd.rc && cudaMemcpyAsync(x_host, g.d_ch[cirrus::kChX], bytes, cudaMemcpyDeviceToHost, pd.stream) != cudaSuccess)
            return cuda_status();
        pd.active = true;
        return CIRRUS_OK;
    });
}

cirrus_status cirrus_grid_autotune(cirrus_grid* grid, int reps, void* stream) {
    if (!grid) return CIRRUS_ERR_INVALID_ARGUMENT;
    return guard([&] { return map_rc(cirrus::autotune(*grid->g, S(stream), reps > 0 ? reps : 20, nullptr)); });
}

namespace {
// CIRRUS_KERNEL_* of a kernel with launch shapes -> its row in DevGrid::shapes (-1: none)
int shape_kind(int kernel) {
    switch (kernel) {
    case CIRRUS_KERNEL_LAPLACIAN: return cirrus::KS_LAPLACIAN;
    case CIRRUS_KERNEL_GS_SWEEP: return cirrus::KS_GS_SWEEP;
    case CIRRUS_KERNEL_PRESMOOTH: return cirrus::KS_PRESMOOTH;
    case CIRRUS_KERNEL_PROLONG_SWEEP: return cirrus::KS_PROLONG;
    case CIRRUS_KERNEL_RESIDUAL_RESTRICT: return cirrus::KS_RESIDUAL;
    default: return -1;
    }
}
}  // namespace

cirrus_status cirrus_grid_set_launch_shape(cirrus_grid* grid, int kernel, int level, int shape) {
    if (!grid || shape < 0 || shape >= CIRRUS_NUM_LAUNCH_SHAPES) return CIRRUS_ERR_INVALID_ARGUMENT;
    auto& g = *grid->g;
    if (kernel != -1 && shape_kind(kernel) < 0) return CIRRUS_ERR_INVALID_ARGUMENT;
    // shapes past the common eight exist for the Laplacian only
    // kernel -1 (all kernels): the shapes every kernel shares, 0..7
    if (shape >= (kernel == -1 ? cirrus::kCommonShapes : cirrus::num_shapes(shape_kind(kernel)))) return CIRRUS_ERR_INVALID_ARGUMENT;
    if (level < -1 || level >= g.num_layers) return CIRRUS_ERR_INVALID_ARGUMENT;
    return guard([&] {
        for (int k = 0; k < cirrus::KS_COUNT; k++) {
            if (kernel != -1 && k != shape_kind(kernel)) continue;
            for (int l = 0; l < g.num_layers; l++)
                if (level == -1 || l == level) g.shapes[(size_t)k * g.num_layers + l] = (uint8_t)shape;
        }
        cirrus::drop_graphs(g);  // graphs captured with the previous shapes
        return CIRRUS_OK;
    });
}

cirrus_status cirrus_grid_get_launch_shape(cirrus_grid* grid, int kernel, int level, int* shape) {
    if (!grid || !shape || shape_kind(kernel) < 0) return CIRRUS_ERR_INVALID_ARGUMENT;
    const auto& g = *grid->g;
    if (level < 0 || level >= g.num_layers) return CIRRUS_ERR_INVALID_ARGUMENT;
    *shape = g.shape(shape_kind(kernel), level);
    return CIRRUS_OK;
}

cirrus_status cirrus_damped_jacobi_solve(cirrus_grid* grid, int max_iters, double relative_tolerance, float omega, void* stream,
                                         int* iters, double* rel) {
    if (!grid || !iters || !rel || max_iters < 0 || !(relative_tolerance >= 0)) return CIRRUS_ERR_INVALID_ARGUMENT;
    if (grid->g->num_inst != 1) return CIRRUS_ERR_INVALID_ARGUMENT;
    return guard([&] { return map_rc(cirrus::damped_jacobi(*grid->g, max_iters, relative_tolerance, omega, S(stream), iters, rel)); });
}

cirrus_status cirrus_grid_autotune_sweeps(cirrus_grid* grid, const cirrus_solve_params* params, void* stream,
                                          cirrus_solve_params* best) {
    if (!grid || !params_ok(params) || !best) return CIRRUS_ERR_INVALID_ARGUMENT;
    return guard([&] {
        cirrus::SolveParams p;
        to_internal(params, &p);
        int li = p.level_iters, ci = p.coarsest_iters;
        const int rc = cirrus::autotune_sweeps(*grid->g, p, S(stream), &li, &ci, nullptr);
        *best = *params;
        best->level_iters = li;
        best->coarsest_iters = ci;
        return map_rc(rc);
    });
}

cirrus_status cirrus_bench_launch(cirrus_grid* grid, int kernel, int level, int reps, void* stream) {
    if (!grid || reps < 0) return CIRRUS_ERR_INVALID_ARGUMENT;
    auto& g = *grid->g;
    const bool per_level = kernel >= CIRRUS_KERNEL_GS_SWEEP && kernel <= CIRRUS_KERNEL_RESIDUAL_RESTRICT;
    if (per_level && (level < 0 || level > g.max_level)) return CIRRUS_ERR_INVALID_ARGUMENT;
    if (kernel == CIRRUS_KERNEL_RESIDUAL_RESTRICT && level < 1) return CIRRUS_ERR_INVALID_ARGUMENT;
    if ((kernel == CIRRUS_KERNEL_PRESMOOTH || kernel == CIRRUS_KERNEL_PROLONG_SWEEP || kernel == CIRRUS_KERNEL_COARSE) &&
        g.bottom_level < 0)
        return CIRRUS_ERR_STATE;
    float *p = g.d_ch[2], *ap = g.d_ch[3], *z = g.d_ch[4], *tmp = g.d_ch[5];
    cudaStream_t s = S(stream);
    for (int i = 0; i < reps; i++) {
        switch (kernel) {
        case CIRRUS_KERNEL_LAPLACIAN: cirrus::launch::laplacian_fused(g, p, tmp, nullptr, s, true); break;
        case CIRRUS_KERNEL_GS_SWEEP: cirrus::launch::gs_sweep(g, level, z, ap, i & 1, nullptr, s, p); break;
        case CIRRUS_KERNEL_PRESMOOTH: cirrus::launch::presmooth(g, level, g.d_xpre, ap, nullptr, s); break;
        case CIRRUS_KERNEL_PROLONG_SWEEP: cirrus::launch::prolong_sweep(g, level, z, g.d_xpre, ap, 1.f, nullptr, s); break;
        case CIRRUS_KERNEL_RESIDUAL_RESTRICT: cirrus::launch::residual_restrict(g, level, g.d_xpre, ap, tmp, 1.f, nullptr, s, true); break;
        case CIRRUS_KERNEL_COARSE: cirrus::launch::bottom(g, g.bottom_level, 10, z, ap, 1.f, 1.f, nullptr, s); break;
        case CIRRUS_KERNEL_DOT: cirrus::launch::grid_dot(g, p, z, s); break;
        default: return CIRRUS_ERR_INVALID_ARGUMENT;
        }
    }
    return cuda_status();
}

cirrus_status cirrus_grid_get_solution_f64(cirrus_grid* grid, double* host, void* stream) {
    if (!grid || !host) return CIRRUS_ERR_INVALID_ARGUMENT;
    return guard([&] { return map_rc(cirrus::solution_f64(*grid->g, host, S(stream))); });
}

cirrus_status cirrus_true_residual(cirrus_grid* grid, const float* b_host, double* rel, void* stream) {
    if (!grid || !b_host || !rel) return CIRRUS_ERR_INVALID_ARGUMENT;
    auto& g = *grid->g;
    return guard([&] {
        const size_t bytes = (size_t)g.n * cirrus::kTileCells * sizeof(float);
        float* d_b = g.d_ch[cirrus::kChTmp];
        // channel 5 (tmp) carries b for the evaluation
        if (cudaMemcpyAsync(d_b, b_host, bytes, cudaMemcpyHostToDevice, S(stream)) != cudaSuccess) return cuda_status();
        int rc = cirrus::true_residual(g, d_b, rel, S(stream));
        return map_rc(rc);
    });
}

// ---------------------------------------------------------------- serving loop
cirrus_status cirrus_server_create_ex(size_t hbm_budget_bytes, int slots, int pool_size, cirrus_server** out) {
    if (!out || slots < 1 || slots > 64 || hbm_budget_bytes == 0 || pool_size < 1 || pool_size > 1024) return CIRRUS_ERR_INVALID_ARGUMENT;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return CIRRUS_ERR_NO_DEVICE;
    }
    return guard([&] {
        *out = new cirrus_server{new cirrus::Server(hbm_budget_bytes, slots, pool_size)};
        return CIRRUS_OK;
    });
}
cirrus_status cirrus_server_create(size_t hbm_budget_bytes, int slots, cirrus_server** out) {
    return cirrus_server_create_ex(hbm_budget_bytes, slots, 8, out);
}
cirrus_status cirrus_server_batch_stats(cirrus_server* server, long long* launches, long long* requests) {
    if (!server) return CIRRUS_ERR_INVALID_ARGUMENT;
    if (launches) *launches = server->s->batches();
    if (requests) *requests = server->s->merged_requests();
    return CIRRUS_OK;
}
void cirrus_server_destroy(cirrus_server* server) {
    if (!server) return;
    delete server->s;
    delete server;
}
cirrus_status cirrus_server_add_session(cirrus_server* server, const cirrus_topology* topo, int* session) {
    if (!server || !topo || !session || topo->t->num_tiles() <= 0) return CIRRUS_ERR_INVALID_ARGUMENT;
    return guard([&] {
        *session = server->s->add_session(topo->t);
        return CIRRUS_OK;
    });
}
cirrus_status cirrus_server_close_session(cirrus_server* server, int session) {
    if (!server) return CIRRUS_ERR_INVALID_ARGUMENT;
    return guard([&] { return server->s->close_session(session) ? CIRRUS_ERR_INVALID_ARGUMENT : CIRRUS_OK; });
}
cirrus_status cirrus_server_submit(cirrus_server* server, int session, const cirrus_solve_params* params, const float* b_host,
                                   float* x_host, uint64_t* ticket) {
    if (!server || !params_ok(params) || !b_host || !ticket) return CIRRUS_ERR_INVALID_ARGUMENT;
    return guard([&] {
        cirrus::SolveParams p;
        to_internal(params, &p);
        return server->s->submit(session, p, b_host, x_host, ticket) ? CIRRUS_ERR_INVALID_ARGUMENT : CIRRUS_OK;
    });
}
cirrus_status cirrus_server_poll(cirrus_server* server, cirrus_completion* out, int max, int* count, int wait_ms) {
    if (!server || !out || max < 1 || !count) return CIRRUS_ERR_INVALID_ARGUMENT;
    return guard([&] {
        std::vector<cirrus::Server::Completion> v;
        server->s->poll(v, max, wait_ms);
        for (size_t i = 0; i < v.size(); i++) {
            cirrus_completion& c = out[i];
            c.ticket = v[i].ticket;
            c.session = v[i].session;
            c.slot = v[i].slot;
            c.status = (int)map_rc(v[i].status);
            c.iters = v[i].iters;
            c.outer_iters = v[i].outer;
            c.warm = v[i].warm;
            c.rel_residual = v[i].rel;
            c.latency_ms = v[i].latency_ms;
            c.device_ms = v[i].device_ms;
            c.batch = v[i].batch;
        }
        *count = (int)v.size();
        return CIRRUS_OK;
    });
}
cirrus_status cirrus_server_stats(cirrus_server* server, size_t* resident_bytes, size_t* peak_bytes, int* resident_sessions,
                                  int* pending, long long* evictions) {
    if (!server) return CIRRUS_ERR_INVALID_ARGUMENT;
    server->s->stats(resident_bytes, peak_bytes, resident_sessions, pending);
    if (evictions) *evictions = server->s->evictions();
    return CIRRUS_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- tile-holder files
struct cirrus_holder {
    cirrus::Holder h;
};

cirrus_status cirrus_holder_read(const char* path, cirrus_holder** out) {
    if (!path || !out) return CIRRUS_ERR_INVALID_ARGUMENT;
    return guard([&] {
        auto* h = new cirrus_holder();
        std::string err;
        if (cirrus::holder_read(path, &h->h, &err)) {
            delete h;
            return CIRRUS_ERR_INVALID_ARGUMENT;
        }
        *out = h;
        return CIRRUS_OK;
    });
}
cirrus_status cirrus_holder_write(const cirrus_holder* holder, const char* path) {
    if (!holder || !path) return CIRRUS_ERR_INVALID_ARGUMENT;
    return guard([&] {
        std::string err;
        return cirrus::holder_write(holder->h, path, &err) ? CIRRUS_ERR_INVALID_ARGUMENT : CIRRUS_OK;
    });
}
void cirrus_holder_destroy(cirrus_holder* holder) { delete holder; }
cirrus_status cirrus_holder_info(const cirrus_holder* holder, double* h0, int* num_layers, int* max_level, int* num_tiles) {
    if (!holder) return CIRRUS_ERR_INVALID_ARGUMENT;
    if (h0) *h0 = (double)holder->h.h0;
    if (num_layers) *num_layers = holder->h.num_layers;
    if (max_level) *max_level = holder->h.max_level;
    if (num_tiles) *num_tiles = holder->h.num_tiles();
    return CIRRUS_OK;
}
cirrus_status cirrus_holder_tiles(const cirrus_holder* holder, int32_t* tiles5) {
    if (!holder || !tiles5) return CIRRUS_ERR_INVALID_ARGUMENT;
    size_t i = 0;
    for (const cirrus::HolderInfo* t : holder->h.ordered()) {
        tiles5[5 * i] = t->level;
        tiles5[5 * i + 1] = t->x;
        tiles5[5 * i + 2] = t->y;
        tiles5[5 * i + 3] = t->z;
        tiles5[5 * i + 4] = t->type;
        i++;
    }
    return CIRRUS_OK;
}
cirrus_status cirrus_holder_cell_types(const cirrus_holder* holder, uint8_t* out) {
    if (!holder || !out) return CIRRUS_ERR_INVALID_ARGUMENT;
    size_t i = 0;
    for (const cirrus::HolderInfo* t : holder->h.ordered()) {
        if (t->record >= 0) std::memcpy(out + i * cirrus::kTileCells, holder->h.types_of((int)t->record), cirrus::kTileCells);
        else std::memset(out + i * cirrus::kTileCells, 0, cirrus::kTileCells);
        i++;
    }
    return CIRRUS_OK;
}
cirrus_status cirrus_holder_channel(const cirrus_holder* holder, int channel, float* out) {
    if (!holder || !out || channel < 0 || channel >= cirrus::kRecordChannels) return CIRRUS_ERR_INVALID_ARGUMENT;
    size_t i = 0;
    for (const cirrus::HolderInfo* t : holder->h.ordered()) {
        if (t->record >= 0)
            std::memcpy(out + i * cirrus::kTileCells, holder->h.channel_of((int)t->record, channel), sizeof(float) * cirrus::kTileCells);
        else std::memset(out + i * cirrus::kTileCells, 0, sizeof(float) * cirrus::kTileCells);
        i++;
    }
    return CIRRUS_OK;
}
cirrus_status cirrus_topology_from_holder(const cirrus_holder* holder, const uint32_t* log2_hash, int num_layers, cirrus_topology** out,
                                          int32_t* order) {
    if (!holder || !log2_hash || !out || num_layers <= 0) return CIRRUS_ERR_INVALID_ARGUMENT;
    return guard([&] {
        cirrus::Topology* t = nullptr;
        std::vector<int32_t> ord;
        std::string err;
        const int rc = cirrus::holder_to_topology(holder->h, log2_hash, num_layers, &t, &ord, &err);
        if (rc) return map_rc(rc);
        auto* topo = new cirrus_topology();
        topo->t = t;
        if (order) std::copy(ord.begin(), ord.end(), order);
        *out = topo;
        return CIRRUS_OK;
    });
}
cirrus_status cirrus_holder_from_grid(const cirrus_topology* topo, const cirrus_grid* grid, int tile_types, cirrus_holder** out) {
    if (!topo || !grid || !out || grid->g->num_inst != 1 || (tile_types & ~7) || !tile_types) return CIRRUS_ERR_INVALID_ARGUMENT;
    const auto& g = *grid->g;
    if (topo->t->num_tiles() != g.n) return CIRRUS_ERR_INVALID_ARGUMENT;
    return guard([&] {
        const size_t cells = (size_t)g.n * cirrus::kTileCells;
        std::vector<float> ch(cells * cirrus::kNumChannels);
        std::vector<uint8_t> ct(cells);
        if (cudaMemcpy(ch.data(), g.d_chbuf, ch.size() * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess) return cuda_status();
        if (cudaMemcpy(ct.data(), g.topo.ctype, cells, cudaMemcpyDeviceToHost) != cudaSuccess) return cuda_status();
        std::vector<int32_t> t5((size_t)g.n * 5);
        topo->t->tiles(t5.data());
        auto* h = new cirrus_holder();
        cirrus::Holder& H = h->h;
        H.h0 = (float)topo->t->h0();
        H.num_layers = topo->t->num_layers();
        H.max_level = topo->t->max_level();
        H.levels.assign(H.num_layers, {});
        int nrec = 0;
        for (int i = 0; i < g.n; i++) nrec += (t5[5 * i + 4] & tile_types) ? 1 : 0;
        H.records.assign((size_t)nrec * cirrus::kRecordBytes, 0);
        int r = 0;
        for (int i = 0; i < g.n; i++) {  // getHostTileHolder: level by level, all-tiles order
            if (!(t5[5 * i + 4] & tile_types)) continue;
            cirrus::HolderInfo info;
            info.level = t5[5 * i];
            info.x = t5[5 * i + 1];
            info.y = t5[5 * i + 2];
            info.z = t5[5 * i + 3];
            info.type = (uint8_t)t5[5 * i + 4];
            info.record = r;
            for (int c = 0; c < cirrus::kNumChannels; c++)
                std::memcpy(H.channel_of(r, c), ch.data() + (size_t)c * cells + (size_t)i * cirrus::kTileCells,
                            sizeof(float) * cirrus::kTileCells);
            std::memcpy(H.types_of(r), ct.data() + (size_t)i * cirrus::kTileCells, cirrus::kTileCells);
            H.levels[info.level].push_back(info);
            r++;
        }
        *out = h;
        return CIRRUS_OK;
    });
}
cirrus_status cirrus_grid_load_holder(cirrus_grid* grid, const cirrus_holder* holder, const int32_t* order, uint32_t channel_mask,
                                      void* stream) {
    if (!grid || !holder || !order || grid->g->num_inst != 1 || (channel_mask >> cirrus::kNumChannels)) return CIRRUS_ERR_INVALID_ARGUMENT;
    auto& g = *grid->g;
    return guard([&] {
        const auto tiles = holder->h.ordered();
        for (size_t i = 0; i < tiles.size(); i++)
            if (order[i] < 0 || order[i] >= g.n) return CIRRUS_ERR_INVALID_ARGUMENT;
        std::vector<float> buf((size_t)g.n * cirrus::kTileCells);
        for (int c = 0; c < cirrus::kNumChannels; c++) {
            if (!(channel_mask & (1u << c))) continue;
            if (cudaMemcpyAsync(buf.data(), g.d_ch[c], buf.size() * sizeof(float), cudaMemcpyDeviceToHost, S(stream)) != cudaSuccess ||
                cudaStreamSynchronize(S(stream)) != cudaSuccess)
                return cuda_status();
            for (size_t i = 0; i < tiles.size(); i++)
                if (tiles[i]->record >= 0)
                    std::memcpy(buf.data() + (size_t)order[i] * cirrus::kTileCells, holder->h.channel_of((int)tiles[i]->record, c),
                                sizeof(float) * cirrus::kTileCells);
            if (cudaMemcpyAsync(g.d_ch[c], buf.data(), buf.size() * sizeof(float), cudaMemcpyHostToDevice, S(stream)) != cudaSuccess ||
                cudaStreamSynchronize(S(stream)) != cudaSuccess)
                return cuda_status();
        }
        g.x64_valid = false;
        return CIRRUS_OK;
    });
}

// ---------------------------------------------------------------- device-resident topology
struct cirrus_dtopology {
    cirrus::DevTopology* t;
};

namespace {
int dt_masks(const cirrus_dtopology* dt, const uint8_t* const* masks, const int* dims, std::vector<const uint8_t*>& m,
             std::vector<int>& d) {
    const int nl = dt->t->num_layers();
    m.assign(masks, masks + nl);
    d.assign(dims, dims + 3 * nl);
    return 0;
}
cirrus_status dt_status(cirrus::DevTopology* t, int rc) { return rc == 0 ? CIRRUS_OK : map_rc(rc); }
}  // namespace

cirrus_status cirrus_dtopology_create(int num_layers, const uint32_t* log2_hash, double h0, cirrus_dtopology** out) {
    if (num_layers <= 0 || num_layers > 32 || !log2_hash || !out) return CIRRUS_ERR_INVALID_ARGUMENT;
    for (int l = 0; l < num_layers; l++)
        if (log2_hash[l] < 1 || log2_hash[l] > 26) return CIRRUS_ERR_INVALID_ARGUMENT;
    return guard([&] {
        auto* t = new cirrus::DevTopology(num_layers, log2_hash, h0);
        if (!t->last_error.empty()) {
            delete t;
            return CIRRUS_ERR_OUT_OF_MEMORY;
        }
        *out = new cirrus_dtopology{t};
        return CIRRUS_OK;
    });
}
void cirrus_dtopology_destroy(cirrus_dtopology* dt) {
    if (!dt) return;
    delete dt->t;
    delete dt;
}
cirrus_status cirrus_dtopology_set_tiles(cirrus_dtopology* dt, int level, const int32_t* xyz, const uint8_t* types, int n) {
    if (!dt || (n > 0 && (!xyz || !types)) || n < 0) return CIRRUS_ERR_INVALID_ARGUMENT;
    for (int i = 0; i < n; i++)
        if (types[i] != CIRRUS_LEAF && types[i] != CIRRUS_NONLEAF && types[i] != CIRRUS_GHOST) return CIRRUS_ERR_INVALID_ARGUMENT;
    return guard([&] { return dt_status(dt->t, dt->t->set_tiles(level, xyz, types, n)); });
}
cirrus_status cirrus_dtopology_compress(cirrus_dtopology* dt) {
    if (!dt) return CIRRUS_ERR_INVALID_ARGUMENT;
    return guard([&] { return dt_status(dt->t, dt->t->compress_and_sync()); });
}
cirrus_status cirrus_dtopology_spawn_ghost_tiles(cirrus_dtopology* dt) {
    if (!dt) return CIRRUS_ERR_INVALID_ARGUMENT;
    return guard([&] { return dt_status(dt->t, dt->t->spawn_ghost_tiles()); });
}
cirrus_status cirrus_dtopology_refine_leafs_one_step(cirrus_dtopology* dt, const uint8_t* const* masks, const int* dims,
                                                     int* refined_per_level) {
    if (!dt || !masks || !dims) return CIRRUS_ERR_INVALID_ARGUMENT;
    return guard([&] {
        std::vector<const uint8_t*> m;
        std::vector<int> d, c;
        dt_masks(dt, masks, dims, m, d);
        const int rc = dt->t->refine_leafs_one_step(m, d, &c);
        if (rc == 0 && refined_per_level) std::copy(c.begin(), c.end(), refined_per_level);
        return dt_status(dt->t, rc);
    });
}
cirrus_status cirrus_dtopology_iterative_refine(cirrus_dtopology* dt, const uint8_t* const* masks, const int* dims) {
    if (!dt || !masks || !dims) return CIRRUS_ERR_INVALID_ARGUMENT;
    return guard([&] {
        std::vector<const uint8_t*> m;
        std::vector<int> d;
        dt_masks(dt, masks, dims, m, d);
        return dt_status(dt->t, dt->t->iterative_refine(m, d));
    });
}
cirrus_status cirrus_dtopology_coarsen_step(cirrus_dtopology* dt, const uint8_t* const* masks, const int* dims, int* deleted_per_level) {
    if (!dt || !masks || !dims) return CIRRUS_ERR_INVALID_ARGUMENT;
    return guard([&] {
        std::vector<const uint8_t*> m;
        std::vector<int> d, c;
        dt_masks(dt, masks, dims, m, d);
        const int rc = dt->t->coarsen_step(m, d, &c);
        if (rc == 0 && deleted_per_level) std::copy(c.begin(), c.end(), deleted_per_level);
        return dt_status(dt->t, rc);
    });
}
cirrus_status cirrus_dtopology_set_cell_types(cirrus_dtopology* dt, const uint8_t* ctypes) {
    if (!dt || !ctypes) return CIRRUS_ERR_INVALID_ARGUMENT;
    return guard([&] { return dt_status(dt->t, dt->t->set_cell_types(ctypes)); });
}
cirrus_status cirrus_dtopology_calc_cell_types_from_leafs(cirrus_dtopology* dt) {
    if (!dt) return CIRRUS_ERR_INVALID_ARGUMENT;
    return guard([&] { return dt_status(dt->t, dt->t->calc_cell_types_from_leafs()); });
}
cirrus_status cirrus_dtopology_num_tiles(const cirrus_dtopology* dt, int* num_tiles) {
    if (!dt || !num_tiles) return CIRRUS_ERR_INVALID_ARGUMENT;
    *num_tiles = dt->t->num_tiles();
    return CIRRUS_OK;
}
cirrus_status cirrus_dtopology_max_level(const cirrus_dtopology* dt, int* max_level) {
    if (!dt || !max_level) return CIRRUS_ERR_INVALID_ARGUMENT;
    *max_level = dt->t->max_level();
    return CIRRUS_OK;
}
cirrus_status cirrus_dtopology_tiles(const cirrus_dtopology* dt, int32_t* out5) {
    if (!dt || !out5) return CIRRUS_ERR_INVALID_ARGUMENT;
    return guard([&] { return dt_status(dt->t, dt->t->tiles(out5)); });
}
cirrus_status cirrus_dtopology_hash_slots(const cirrus_dtopology* dt, int32_t* out) {
    if (!dt || !out) return CIRRUS_ERR_INVALID_ARGUMENT;
    return guard([&] { return dt_status(dt->t, dt->t->hash_slots(out)); });
}
cirrus_status cirrus_dtopology_cell_types(const cirrus_dtopology* dt, uint8_t* out) {
    if (!dt || !out) return CIRRUS_ERR_INVALID_ARGUMENT;
    return guard([&] { return dt_status(dt->t, dt->t->cell_types(out)); });
}
cirrus_status cirrus_dtopology_statuses(const cirrus_dtopology* dt, int32_t* out) {
    if (!dt || !out) return CIRRUS_ERR_INVALID_ARGUMENT;
    return guard([&] { return dt_status(dt->t, dt->t->statuses(out)); });
}
cirrus_status cirrus_dtopology_to_topology(const cirrus_dtopology* dt, cirrus_topology** out) {
    if (!dt || !out) return CIRRUS_ERR_INVALID_ARGUMENT;
    return guard([&] {
        const int n = dt->t->num_tiles();
        if (n <= 0) return CIRRUS_ERR_STATE;
        std::vector<int32_t> t5((size_t)n * 5);
        std::vector<uint8_t> ct((size_t)n * cirrus::kTileCells);
        int rc = dt->t->tiles(t5.data());
        if (!rc) rc = dt->t->cell_types(ct.data());
        if (rc) return map_rc(rc);
        cirrus_topology* topo = nullptr;
        cirrus_status st = CIRRUS_OK;
        {
            auto* t = new cirrus::Topology(dt->t->num_layers(), dt->t->log2_hash(), dt->t->h0());
            if (!t->import_tiles(t5.data(), n)) {
                delete t;
                return CIRRUS_ERR_TOPOLOGY;
            }
            t->set_cell_types(ct.data());
            topo = new cirrus_topology{t};
        }
        *out = topo;
        return st;
    });
}
