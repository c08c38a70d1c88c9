// Serving loop: solves of independent problems ("sessions") submitted as they arrive, run
// concurrently on a fixed number of slots (one worker thread and one CUDA stream per slot, so the
// GPU overlaps the solves' kernels), admitted against an HBM budget.  A session's tile pool and
// its last pressure stay resident on the device between its solves; each solve after the first
// starts from that pressure (FP64 defect correction from the warm start).  When a session must be
// made resident and the budget is spent, idle sessions are evicted least recently used first,
// their pressure kept on the host for the next warm start.  Victims are chosen under the
// scheduler lock, but their pressure copy and pool release (a device synchronisation) run on the
// evicting worker's stream after the lock is dropped, so other slots keep scheduling meanwhile.
// No counterpart in the reference.
#include "serve.hpp"

#include "solver_internal.hpp"
#include "topology.hpp"

#include <algorithm>
#include <chrono>

namespace cirrus {

namespace {
double now_ms() {
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}
}  // namespace

size_t Server::estimate_bytes(const Topology& t) {
    // channels (9) + pre-smoothed x + FP64 defect-correction buffers (3 doubles + 1 float) per
    // cell, masks/types, per-tile tables, plus fixed scratch
    const size_t tiles = (size_t)t.num_tiles();
    return tiles * (kTileCells * (10 * sizeof(float) + 3 * sizeof(double) + sizeof(float) + 3) + 512) + (size_t)(4 << 20);
}

Server::Server(size_t budget, int slots) : budget_(budget) {
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
    for (auto& kv : sessions_)
        if (kv.second.grid) grid_destroy(kv.second.grid);
}

int Server::add_session(const Topology* topo) {
    std::lock_guard<std::mutex> lk(mu_);
    const int id = next_session_++;
    Session& s = sessions_[id];
    s.topo = topo;
    s.estimate = estimate_bytes(*topo);
    return id;
}

int Server::close_session(int id) {
    std::unique_lock<std::mutex> lk(mu_);
    auto it = sessions_.find(id);
    if (it == sessions_.end()) return 1;
    it->second.closing = true;
    // wait until no request of the session is running or queued
    cv_.wait(lk, [&] {
        if (it->second.busy || it->second.evicting) return false;
        for (const Request& r : pending_)
            if (r.session == id) return false;
        return true;
    });
    if (it->second.grid) {
        grid_destroy(it->second.grid);
        used_ -= it->second.bytes;
    }
    sessions_.erase(it);
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
        for (auto& kv : sessions_) c += kv.second.grid != nullptr;
        *resident_sessions = c;
    }
    if (pending) *pending = (int)pending_.size();
}

// Under the lock: the first queued request that can start now.  Its session must be idle; if it
// is not resident, the bytes it needs must fit after evicting idle sessions (chosen here, least
// recently used first, and released by the caller outside the lock).  A session larger than the
// whole budget fails its requests at once.
bool Server::take_runnable(Request& r, bool& need_create, std::vector<Victim>& victims) {
    for (auto it = pending_.begin(); it != pending_.end(); ++it) {
        Session& s = sessions_[it->session];
        if (s.busy || s.evicting) continue;
        if (s.grid) {
            need_create = false;
        } else {
            if (s.estimate > budget_) {
                Completion c{};
                c.ticket = it->ticket;
                c.session = it->session;
                c.status = 7;  // budget
                c.latency_ms = now_ms() - it->t_submit;
                done_.push_back(c);
                pending_.erase(it);
                cv_.notify_all();
                return take_runnable(r, need_create, victims);
            }
            size_t freeable = 0;
            for (auto& kv : sessions_)
                if (kv.second.grid && !kv.second.busy) freeable += kv.second.bytes;
            if (used_ + s.estimate > budget_ + freeable) continue;
            while (used_ + s.estimate > budget_ && pick_lru(victims, &s)) {
            }
            used_ += s.estimate;  // reserved now, corrected to the grid's bytes after its first solve
            s.bytes = s.estimate;
            peak_ = std::max(peak_, used_);
            need_create = true;
        }
        s.busy = true;
        r = *it;
        pending_.erase(it);
        return true;
    }
    return false;
}

// Under the lock: detach the least recently used idle resident session (other than `keep`) as a
// victim; its bytes count as freed from now on.  False if there is none.
bool Server::pick_lru(std::vector<Victim>& victims, const Session* keep) {
    Session* lru = nullptr;
    for (auto& kv : sessions_) {
        Session& c = kv.second;
        if (&c != keep && c.grid && !c.busy && !c.evicting && (!lru || c.last_used < lru->last_used)) lru = &c;
    }
    if (!lru) return false;
    choose_victim(*lru, victims);
    return true;
}

void Server::choose_victim(Session& s, std::vector<Victim>& victims) {
    victims.push_back({&s, s.grid});
    s.grid = nullptr;
    s.evicting = true;
    used_ -= s.bytes;
    s.bytes = 0;
    evictions_++;
}

// Outside the lock: save each victim's pressure to the host (for its next warm start) and free
// its pool; then mark it evicted.
void Server::finish_evictions(std::vector<Victim>& victims, cudaStream_t stream) {
    if (victims.empty()) return;
    for (Victim& v : victims) {
        const size_t cells = (size_t)v.grid->n * kTileCells;
        v.s->x_saved.resize(cells);
        cudaMemcpyAsync(v.s->x_saved.data(), v.grid->d_ch[kChX], cells * sizeof(float), cudaMemcpyDeviceToHost, stream);
        cudaStreamSynchronize(stream);
        grid_destroy(v.grid);
    }
    {
        std::lock_guard<std::mutex> lk(mu_);
        for (Victim& v : victims) {
            v.s->has_saved = true;
            v.s->evicting = false;
        }
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
        Request r;
        bool need_create = false, got = false;
        Session* s = nullptr;
        std::vector<Victim> victims;
        {
            std::unique_lock<std::mutex> lk(mu_);
            cv_.wait(lk, [&] {
                if (stop_) return true;
                got = take_runnable(r, need_create, victims);
                return got;
            });
            if (!got) break;
            s = &sessions_[r.session];
        }
        finish_evictions(victims, stream);  // before the new pool is allocated
        Completion c{};
        c.ticket = r.ticket;
        c.session = r.session;
        c.slot = slot;
        int rc = 0;
        if (need_create) {
            std::string err;
            DevGrid* g = nullptr;
            rc = grid_create({s->topo}, &g, &err);
            if (rc == 0) {
                s->grid = g;
                if (s->has_saved)
                    cudaMemcpyAsync(g->d_ch[kChX], s->x_saved.data(), s->x_saved.size() * sizeof(float), cudaMemcpyHostToDevice,
                                    stream);
            }
        }
        SolveResult res;
        if (rc == 0) {
            DevGrid& g = *s->grid;
            const size_t bytes = (size_t)g.n * kTileCells * sizeof(float);
            cudaEventRecord(e0, stream);
            cudaMemcpyAsync(g.d_ch[kChB], r.b, bytes, cudaMemcpyHostToDevice, stream);
            SolveParams p = r.params;
            p.precision = 1;
            p.warm_start = (s->solves > 0 || s->has_saved) ? 1 : 0;
            rc = mixed_solve(g, p, stream, &res, nullptr);
            if (rc == 0 && r.x) cudaMemcpyAsync(r.x, g.d_ch[kChX], bytes, cudaMemcpyDeviceToHost, stream);
            cudaEventRecord(e1, stream);
            if (cudaStreamSynchronize(stream) != cudaSuccess) rc = 2;
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            c.device_ms = ms;
        }
        c.status = rc ? rc : res.status;
        c.iters = res.iters;
        c.outer = res.outer;
        c.rel = res.true_rel;
        {
            std::lock_guard<std::mutex> lk(mu_);
            c.latency_ms = now_ms() - r.t_submit;
            c.warm = s->solves > 0 || s->has_saved;
            if (s->grid) {
                used_ -= s->bytes;
                s->bytes = s->grid->bytes;
                used_ += s->bytes;
                // the pool's real size (FP64 buffers, graphs) can exceed the reservation: evict
                // idle sessions until the resident bytes fit the budget again
                while (used_ > budget_ && pick_lru(victims, s)) {
                }
                peak_ = std::max(peak_, used_);
            } else {
                used_ -= s->bytes;  // creation failed: release the reservation
                s->bytes = 0;
            }
            s->solves++;
            s->busy = false;
            s->last_used = ++clock_;
            done_.push_back(c);
        }
        cv_.notify_all();
        finish_evictions(victims, stream);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamDestroy(stream);
}

}  // namespace cirrus
