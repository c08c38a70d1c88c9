// Serving loop (serve.cpp): sessions (independent problems) with resident device state, solves
// submitted as they arrive, run concurrently on slots, admitted against an HBM budget.
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
        double rel = 0, latency_ms = 0, device_ms = 0;
    };

    Server(size_t budget, int slots);
    ~Server();
    int add_session(const Topology* topo);
    int close_session(int id);
    int submit(int session, const SolveParams& p, const float* b, float* x, uint64_t* ticket);
    int poll(std::vector<Completion>& out, int max, int wait_ms);
    void stats(size_t* resident, size_t* peak, int* resident_sessions, int* pending);
    long long evictions() const { return evictions_; }
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
        DevGrid* grid = nullptr;
        size_t estimate = 0, bytes = 0;
        bool busy = false, closing = false, has_saved = false;
        bool evicting = false;  // chosen for eviction: its pressure is being saved, its pool freed
        std::vector<float> x_saved;
        long long solves = 0;
        uint64_t last_used = 0;
    };
    // a session chosen for eviction under the lock; its pressure is copied out and its pool freed
    // outside the lock (finish_evictions)
    struct Victim {
        Session* s;
        DevGrid* grid;
    };
    bool take_runnable(Request& r, bool& need_create, std::vector<Victim>& victims);
    void choose_victim(Session& s, std::vector<Victim>& victims);
    bool pick_lru(std::vector<Victim>& victims, const Session* keep);
    void finish_evictions(std::vector<Victim>& victims, cudaStream_t stream);
    void worker(int slot);

    size_t budget_, used_ = 0, peak_ = 0;
    int device_ = 0;
    int next_session_ = 0;
    uint64_t next_ticket_ = 1, clock_ = 0;
    long long evictions_ = 0;
    bool stop_ = false;
    std::mutex mu_;
    std::condition_variable cv_;
    std::deque<Request> pending_;
    std::vector<Completion> done_;
    std::map<int, Session> sessions_;
    std::vector<std::thread> workers_;
};

}  // namespace cirrus
