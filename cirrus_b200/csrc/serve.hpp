// Serving loop (serve.cpp): sessions (independent problems) with resident device state, solves
// submitted as they arrive and merged into batched launches, admitted against an HBM budget.
#pragma once

#include "solver_internal.hpp"

#include <condition_variable>
#include <cstdint>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

namespace cirrus {

class Topology;

class Server {
public:
    struct Completion {
        uint64_t ticket = 0;
        int session = -1, slot = -1, status = 0, iters = 0, outer = 0, warm = 0;
        int batch = 0;  // requests solved together in the launch that carried this one
        double rel = 0, latency_ms = 0, device_ms = 0;
    };

    // pool_size: sessions of one size class that share a batched tile pool (1: every session alone)
    Server(size_t budget, int slots, int pool_size = 8);
    ~Server();
    int add_session(const Topology* topo);
    int close_session(int id);
    int submit(int session, const SolveParams& p, const float* b, float* x, uint64_t* ticket);
    int poll(std::vector<Completion>& out, int max, int wait_ms);
    void stats(size_t* resident, size_t* peak, int* resident_sessions, int* pending);
    long long evictions() const { return evictions_; }
    long long batches() const { return batches_; }
    long long merged_requests() const { return merged_; }
    static size_t estimate_bytes(const Topology& t);

private:
    struct Request {
        uint64_t ticket = 0;
        int session = -1;
        SolveParams params;
        const float* b = nullptr;
        float* x = nullptr;
        double t_submit = 0;
    };
    struct Session {
        const Topology* topo = nullptr;
        int pool = -1, member = -1;  // its pool and instance index in the pool's batched grid
        size_t estimate = 0;
        bool closing = false, running = false;
        long long solves = 0;
        std::vector<float> x_saved;  // the pressure kept on the host while its pool is evicted
        bool has_saved = false;
    };
    // Sessions of one size class registered together share one batched grid (instances in
    // registration order), created when the first of them is admitted; a pool takes no new
    // members once created.
    struct Pool {
        std::vector<int> members;
        int size_class = 0;
        DevGrid* grid = nullptr;
        size_t estimate = 0, bytes = 0, tiles = 0;
        bool busy = false, evicting = false, sealed = false;
        uint64_t last_used = 0;
    };
    struct Victim {
        int pool;
        DevGrid* grid;
    };
    struct Batch {
        int pool = -1;
        bool need_create = false;
        std::vector<Request> reqs;  // at most one per member session, oldest first
    };
    static constexpr size_t kSoloTiles = 4096;  // sessions this large are not pooled
    static constexpr size_t kPoolTiles = 8192;  // tiles of all members of one pool at most
    static int size_class(size_t tiles);
    bool take_runnable(Batch& b, std::vector<Victim>& victims);
    bool pick_lru(std::vector<Victim>& victims, int keep_pool);
    void finish_evictions(std::vector<Victim>& victims, cudaStream_t stream);
    void worker(int slot);

    size_t budget_, used_ = 0, peak_ = 0;
    int pool_size_ = 8;
    int device_ = 0;
    int next_session_ = 0;
    uint64_t next_ticket_ = 1, clock_ = 0;
    long long evictions_ = 0, batches_ = 0, merged_ = 0;
    bool stop_ = false;
    std::mutex mu_;
    std::condition_variable cv_;
    std::deque<Request> pending_;
    std::vector<Completion> done_;
    std::map<int, Session> sessions_;
    std::deque<Pool> pools_;  // references stay valid while pools are added
    std::vector<std::thread> workers_;
};

}  // namespace cirrus
