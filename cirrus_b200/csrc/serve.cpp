// Serving loop with continuous batching: solves of independent problems ("sessions") are
// submitted as they arrive; sessions of similar size share one batched tile pool (a DevGrid of
// several instances, sessions of one size class grouped in registration order up to a tile cap;
// the largest sessions alone), and every launch
// takes, for the pool it serves, the oldest waiting request of each of its sessions -- requests
// that arrived while the pool was busy join the next launch of that pool, whichever sessions
// they come from.  Each launch is one mixed-precision batched solve (FP32 V-cycle, FP64 defect
// correction) with only the requested instances active; per-instance results do not depend on
// the others in the launch, so a request's pressure is the same alone and in any mix.  A fixed
// number of slots (one worker thread and one CUDA stream each) runs launches of different pools
// concurrently on the GPU.  Pools are admitted against an HBM budget; idle pools are evicted
// least recently used first, their sessions' pressures kept on the host for the next warm start.
// Victims are chosen under the scheduler lock; their pressure copies and pool releases run on the
// evicting worker's stream after the lock is dropped.  No counterpart in the reference.
#include "serve.hpp"

#include "solver_internal.hpp"
#include "topology.hpp"

#include <algorithm>
#include <chrono>
#include <set>

namespace cirrus {

namespace {
double now_ms() {
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

// channel `c` of one instance of a batched grid <-> a host array in that instance's own order
bool instance_copy(const DevGrid& g, int inst, int c, float* host, bool to_device, cudaStream_t s) {
    for (const TileRun& r : g.inst_runs[inst]) {
        float* d = g.d_ch[c] + (size_t)r.global * kTileCells;
        float* h = host + (size_t)r.local * kTileCells;
        const size_t bytes = (size_t)r.count * kTileCells * sizeof(float);
        const cudaError_t e = to_device ? cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, s)
                                        : cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, s);
        if (e != cudaSuccess) return false;
    }
    return true;
}
}  // namespace

size_t Server::estimate_bytes(const Topology& t) {
    // channels (9) + pre-smoothed x + FP64 defect-correction buffers (3 doubles + 1 float) per
    // cell, masks/types, per-tile tables, plus fixed scratch
    const size_t tiles = (size_t)t.num_tiles();
    return tiles * (kTileCells * (10 * sizeof(float) + 3 * sizeof(double) + sizeof(float) + 3) + 512) + (size_t)(4 << 20);
}

// Size classes of the pools: a launch over a pool costs about as long as its largest member's
// solve, so only sessions of similar size are merged, and a session of kSoloTiles tiles or more
// (whose solve fills the GPU by itself) gets a pool of its own.
int Server::size_class(size_t tiles) { return tiles < 256 ? 0 : tiles < 1024 ? 1 : tiles < kSoloTiles ? 2 : 3; }

Server::Server(size_t budget, int slots, int pool_size) : budget_(budget), pool_size_(std::max(1, pool_size)) {
    cudaGetDevice(&device_);
    for (int i = 0; i < slots; i++) workers_.emplace_back([this, i] { worker(i); });
}

Server::~Server() {
    {
        std::lock_guard<std::mutex> lk(mu_);
        stop_ = true;
    }
    cv_.notify_all();
    for (auto& w : workers_) w.join();
    for (Pool& p : pools_)
        if (p.grid) grid_destroy(p.grid);
}

int Server::add_session(const Topology* topo) {
    std::lock_guard<std::mutex> lk(mu_);
    const int id = next_session_++;
    Session& s = sessions_[id];
    s.topo = topo;
    s.estimate = estimate_bytes(*topo);
    const int cls = size_class((size_t)topo->num_tiles());
    int p = -1;
    for (size_t i = 0; i < pools_.size(); i++)
        if (!pools_[i].sealed && pools_[i].size_class == cls && cls < 3 && (int)pools_[i].members.size() < pool_size_ &&
            pools_[i].tiles + (size_t)topo->num_tiles() <= kPoolTiles) {
            p = (int)i;
            break;
        }
    if (p < 0) {
        pools_.emplace_back();
        p = (int)pools_.size() - 1;
        pools_[p].size_class = cls;
    }
    s.pool = p;
    s.member = (int)pools_[p].members.size();
    pools_[p].members.push_back(id);
    pools_[p].estimate += s.estimate;
    pools_[p].tiles += (size_t)topo->num_tiles();
    return id;
}

int Server::close_session(int id) {
    std::unique_lock<std::mutex> lk(mu_);
    auto it = sessions_.find(id);
    if (it == sessions_.end()) return 1;
    it->second.closing = true;
    // wait until no request of the session is running or queued
    cv_.wait(lk, [&] {
        if (it->second.running) return false;
        for (const Request& r : pending_)
            if (r.session == id) return false;
        return true;
    });
    const int p = it->second.pool;
    sessions_.erase(it);
    // the last session of a pool frees its device state
    bool any = false;
    for (int m : pools_[p].members) any = any || sessions_.count(m);
    cv_.wait(lk, [&] { return !pools_[p].busy && !pools_[p].evicting; });
    if (!any && pools_[p].grid) {
        grid_destroy(pools_[p].grid);
        pools_[p].grid = nullptr;
        used_ -= pools_[p].bytes;
        pools_[p].bytes = 0;
    }
    cv_.notify_all();
    return 0;
}

int Server::submit(int session, const SolveParams& p, const float* b, float* x, uint64_t* ticket) {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = sessions_.find(session);
    if (it == sessions_.end() || it->second.closing) return 1;
    Request r;
    r.ticket = next_ticket_++;
    r.session = session;
    r.params = p;
    r.b = b;
    r.x = x;
    r.t_submit = now_ms();
    pending_.push_back(r);
    *ticket = r.ticket;
    cv_.notify_all();
    return 0;
}

int Server::poll(std::vector<Completion>& out, int max, int wait_ms) {
    std::unique_lock<std::mutex> lk(mu_);
    if (done_.empty() && wait_ms > 0) cv_.wait_for(lk, std::chrono::milliseconds(wait_ms), [&] { return !done_.empty(); });
    const int n = std::min<int>(max, (int)done_.size());
    out.assign(done_.begin(), done_.begin() + n);
    done_.erase(done_.begin(), done_.begin() + n);
    return 0;
}

void Server::stats(size_t* resident, size_t* peak, int* resident_sessions, int* pending) {
    std::lock_guard<std::mutex> lk(mu_);
    if (resident) *resident = used_;
    if (peak) *peak = peak_;
    if (resident_sessions) {
        int c = 0;
        for (auto& kv : sessions_) c += pools_[kv.second.pool].grid != nullptr;
        *resident_sessions = c;
    }
    if (pending) *pending = (int)pending_.size();
}

// Under the lock: the pool of the oldest queued request that can run now, with the oldest queued
// request of each of its sessions.  The pool must be idle; if it is not resident, its bytes must
// fit after evicting idle pools (chosen here, least recently used first, released by the caller
// outside the lock).  A pool larger than the whole budget fails its requests at once.
bool Server::take_runnable(Batch& b, std::vector<Victim>& victims) {
    for (auto it = pending_.begin(); it != pending_.end(); ++it) {
        const int pi = sessions_[it->session].pool;
        Pool& P = pools_[pi];
        if (P.busy || P.evicting) continue;
        if (!P.grid) {
            if (P.estimate > budget_) {
                Completion c{};
                c.ticket = it->ticket;
                c.session = it->session;
                c.status = 7;  // budget
                c.latency_ms = now_ms() - it->t_submit;
                done_.push_back(c);
                pending_.erase(it);
                cv_.notify_all();
                return take_runnable(b, victims);
            }
            size_t freeable = 0;
            for (const Pool& q : pools_)
                if (q.grid && !q.busy) freeable += q.bytes;
            if (used_ + P.estimate > budget_ + freeable) continue;
            while (used_ + P.estimate > budget_ && pick_lru(victims, pi)) {
            }
            used_ += P.estimate;  // reserved now, corrected to the grid's bytes after the launch
            P.bytes = P.estimate;
            peak_ = std::max(peak_, used_);
            b.need_create = true;
        } else {
            b.need_create = false;
        }
        P.busy = true;
        P.sealed = true;
        b.pool = pi;
        b.reqs.clear();
        std::set<int> taken;
        for (auto jt = pending_.begin(); jt != pending_.end();) {
            if (sessions_[jt->session].pool == pi && taken.insert(jt->session).second) {
                b.reqs.push_back(*jt);
                sessions_[jt->session].running = true;
                jt = pending_.erase(jt);
            } else {
                ++jt;
            }
        }
        return true;
    }
    return false;
}

// Under the lock: detach the least recently used idle resident pool (other than keep_pool) as a
// victim; its bytes count as freed from now on.  False if there is none.
bool Server::pick_lru(std::vector<Victim>& victims, int keep_pool) {
    int lru = -1;
    for (size_t i = 0; i < pools_.size(); i++) {
        const Pool& q = pools_[i];
        if ((int)i != keep_pool && q.grid && !q.busy && !q.evicting && (lru < 0 || q.last_used < pools_[lru].last_used)) lru = (int)i;
    }
    if (lru < 0) return false;
    Pool& q = pools_[lru];
    victims.push_back({lru, q.grid});
    q.grid = nullptr;
    q.evicting = true;
    used_ -= q.bytes;
    q.bytes = 0;
    evictions_++;
    return true;
}

// Outside the lock: save every live session's pressure of each victim pool to the host (for its
// next warm start) and free the pool; then mark it evicted.
void Server::finish_evictions(std::vector<Victim>& victims, cudaStream_t stream) {
    if (victims.empty()) return;
    for (Victim& v : victims) {
        std::vector<std::pair<int, int>> live;  // (session, member)
        {
            std::lock_guard<std::mutex> lk(mu_);
            for (int m : pools_[v.pool].members) {
                auto it = sessions_.find(m);
                if (it != sessions_.end()) live.push_back({m, it->second.member});
            }
        }
        for (auto& sm : live) {
            std::vector<float> x((size_t)v.grid->inst_tiles[sm.second] * kTileCells);
            instance_copy(*v.grid, sm.second, kChX, x.data(), false, stream);
            cudaStreamSynchronize(stream);
            std::lock_guard<std::mutex> lk(mu_);
            auto it = sessions_.find(sm.first);
            if (it != sessions_.end()) {
                it->second.x_saved = std::move(x);
                it->second.has_saved = true;
            }
        }
        grid_destroy(v.grid);
    }
    {
        std::lock_guard<std::mutex> lk(mu_);
        for (Victim& v : victims) pools_[v.pool].evicting = false;
    }
    victims.clear();
    cv_.notify_all();
}

void Server::worker(int slot) {
    cudaSetDevice(device_);
    cudaStream_t stream = nullptr;
    cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (;;) {
        Batch b;
        std::vector<Victim> victims;
        bool got = false;
        std::vector<const Topology*> topos;        // per instance of the pool
        std::vector<std::vector<float>> restore;   // saved pressures per instance (pool re-created)
        std::vector<int> req_member;               // instance of each request
        Pool* P = nullptr;
        {
            std::unique_lock<std::mutex> lk(mu_);
            cv_.wait(lk, [&] {
                if (stop_) return true;
                got = take_runnable(b, victims);
                return got;
            });
            if (!got) break;
            P = &pools_[b.pool];
            restore.resize(P->members.size());
            for (size_t i = 0; i < P->members.size(); i++) {
                auto it = sessions_.find(P->members[i]);
                topos.push_back(it != sessions_.end() ? it->second.topo : nullptr);
                if (b.need_create && it != sessions_.end() && it->second.has_saved) restore[i] = it->second.x_saved;
            }
            for (const Request& r : b.reqs) req_member.push_back(sessions_[r.session].member);
            batches_++;
            merged_ += (long long)b.reqs.size();
        }
        finish_evictions(victims, stream);  // before the new pool is allocated
        int rc = 0;
        if (b.need_create) {
            // a session closed before its pool was created keeps its instance, sized by a live
            // member's topology (it is never active)
            const Topology* any = nullptr;
            for (const Topology* t : topos)
                if (t) any = t;
            for (auto& t : topos)
                if (!t) t = any;
            std::string err;
            DevGrid* g = nullptr;
            rc = any ? grid_create(topos, &g, &err) : 1;
            if (rc == 0) {
                P->grid = g;
                for (size_t i = 0; i < restore.size(); i++)
                    if (!restore[i].empty()) instance_copy(*g, (int)i, kChX, restore[i].data(), true, stream);
            }
        }
        std::vector<SolveResult> res;
        double device_ms = 0.0;
        if (rc == 0) {
            DevGrid& g = *P->grid;
            cudaEventRecord(e0, stream);
            std::vector<InstRequest> inst(g.num_inst);
            for (InstRequest& q : inst) q.active = 0;
            for (size_t k = 0; k < b.reqs.size(); k++) {
                const Request& r = b.reqs[k];
                const int m = req_member[k];
                if (!instance_copy(g, m, kChB, const_cast<float*>(r.b), true, stream)) rc = 2;
                inst[m].active = 1;
                inst[m].tol = r.params.tol;
                inst[m].pure_neumann = r.params.pure_neumann;
            }
            // the pool's instances hold their sessions' last pressures (0 before a first solve,
            // the saved one after an eviction): every solve starts from them
            SolveParams p = b.reqs.front().params;
            p.precision = 1;
            p.warm_start = 1;
            res.resize(g.num_inst);
            if (rc == 0) rc = mixed_solve(g, p, stream, res.data(), inst.data());
            for (size_t k = 0; rc == 0 && k < b.reqs.size(); k++)
                if (b.reqs[k].x && !instance_copy(g, req_member[k], kChX, b.reqs[k].x, false, stream)) rc = 2;
            cudaEventRecord(e1, stream);
            if (cudaStreamSynchronize(stream) != cudaSuccess) rc = 2;
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            device_ms = ms;
        }
        {
            std::lock_guard<std::mutex> lk(mu_);
            const double t = now_ms();
            for (size_t k = 0; k < b.reqs.size(); k++) {
                const Request& r = b.reqs[k];
                Session& s = sessions_[r.session];
                Completion c{};
                c.ticket = r.ticket;
                c.session = r.session;
                c.slot = slot;
                c.batch = (int)b.reqs.size();
                const SolveResult* sr = (rc == 0 && !res.empty()) ? &res[req_member[k]] : nullptr;
                c.status = sr ? sr->status : rc;
                if (sr) {
                    c.iters = sr->iters;
                    c.outer = sr->outer;
                    c.rel = sr->true_rel;
                }
                c.latency_ms = t - r.t_submit;
                c.device_ms = device_ms;
                c.warm = s.solves > 0 || s.has_saved;
                s.solves++;
                s.running = false;
                done_.push_back(c);
            }
            if (P->grid) {
                used_ -= P->bytes;
                P->bytes = P->grid->bytes;
                used_ += P->bytes;
                // the pool's real size (FP64 buffers, graphs) can exceed the reservation: evict
                // idle pools until the resident bytes fit the budget again
                while (used_ > budget_ && pick_lru(victims, b.pool)) {
                }
                peak_ = std::max(peak_, used_);
            } else {
                used_ -= P->bytes;  // creation failed: release the reservation
                P->bytes = 0;
            }
            P->busy = false;
            P->last_used = ++clock_;
        }
        cv_.notify_all();
        finish_evictions(victims, stream);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamDestroy(stream);
}

}  // namespace cirrus
