// Autotuner of the launch shapes: for every kernel with selectable shapes and every level it runs
// on, each shape is timed on the grid itself (back-to-back launches captured in a CUDA graph,
// CUDA events around one graph launch) and the fastest is kept.  The shapes compute every tile
// with the same operations, so the choice changes timing only, never results.
#include "solver_internal.hpp"

#include <cstdio>
#include <vector>

namespace cirrus {

namespace {

template <class F>
float time_graph(F launch, int reps, cudaStream_t s) {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    float ms = -1.f;
    launch();  // first run outside the graph (lazy loading of the kernel)
    if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return -1.f;
    for (int i = 0; i < reps; i++) launch();
    if (cudaStreamEndCapture(s, &graph) != cudaSuccess || !graph) return -1.f;
    if (cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess) {
        cudaEvent_t a, b;
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        cudaGraphLaunch(exec, s);  // warm
        // the best of three timed graph launches (transients on a shared GPU only add time)
        for (int k = 0; k < 3; k++) {
            cudaEventRecord(a, s);
            cudaGraphLaunch(exec, s);
            cudaEventRecord(b, s);
            float t = -1.f;
            if (cudaEventSynchronize(b) == cudaSuccess) cudaEventElapsedTime(&t, a, b);
            if (t > 0.f && (ms < 0.f || t < ms)) ms = t;
        }
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        cudaGraphExecDestroy(exec);
    }
    cudaGraphDestroy(graph);
    return ms;
}

}  // namespace

// Whole-solve refinement of the shapes, for grids small enough that a solve is a chain of
// launches each bound by its own latency (one instance or a few): there, timing a kernel alone in
// back-to-back launches measures overlapped throughput, not its place in the chain.  Candidates:
// the per-kernel picks; each of the eight common shapes for every kernel; then, per kernel kind,
// each of its shapes on all its levels; then, level by level from the finest, each shape of each
// V-cycle kernel.  Each is timed as a fixed-length solve (8 PCG iterations
// of the grid's own right-hand sides, graph-launched, best of 3) and kept if it gains more than
// 0.5 %.  b and x are saved first and restored after; a grid whose right-hand sides end a solve
// early (zero or non-finite) is left as tuned.
static void refine_by_solve(DevGrid& g, cudaStream_t s) {
    const size_t bytes = (size_t)g.n * kTileCells * sizeof(float);
    float *bsave = nullptr, *xsave = nullptr;
    if (cudaMalloc(&bsave, bytes) != cudaSuccess || cudaMalloc(&xsave, bytes) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(bsave);
        return;
    }
    cudaMemcpyAsync(bsave, g.d_ch[kChB], bytes, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(xsave, g.d_ch[kChX], bytes, cudaMemcpyDeviceToDevice, s);
    SolveParams prm;
    prm.max_iters = 8;
    prm.tol = 0.0;  // never met: every trial runs the same 8 iterations
    std::vector<SolveResult> res(g.num_inst);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    auto trial = [&]() -> float {
        drop_graphs(g);
        float best = -1.f;
        for (int rep = 0; rep < 4; rep++) {  // the first builds the graph
            cudaMemcpyAsync(g.d_ch[kChB], bsave, bytes, cudaMemcpyDeviceToDevice, s);
            cudaEventRecord(e0, s);
            if (pcg_solve(g, prm, s, res.data()) != 0) return -1.f;
            cudaEventRecord(e1, s);
            float t = -1.f;
            if (cudaEventSynchronize(e1) != cudaSuccess) return -1.f;
            cudaEventElapsedTime(&t, e0, e1);
            if (rep > 0 && t > 0.f && (best < 0.f || t < best)) best = t;
        }
        return best;
    };
    std::vector<uint8_t> kept = g.shapes;
    float best = trial();
    bool iterated = false;
    for (const SolveResult& r : res) iterated = iterated || r.iters == prm.max_iters;
    if (!iterated) best = -1.f;
    auto consider = [&](const std::vector<uint8_t>& cand) {
        g.shapes = cand;
        const float t = trial();
        if (t > 0.f && best > 0.f && t < 0.995f * best) {
            best = t;
            kept = cand;
        }
    };
    if (best > 0.f) {
        const std::vector<uint8_t> tuned = kept;
        for (int sh = 0; sh < kCommonShapes; sh++) consider(std::vector<uint8_t>(tuned.size(), (uint8_t)sh));
        for (int kind = 0; kind < KS_COUNT; kind++) {
            const std::vector<uint8_t> base = kept;
            for (int sh = 0; sh < num_shapes(kind); sh++) {
                std::vector<uint8_t> cand = base;
                for (int l = 0; l < g.num_layers; l++) cand[(size_t)kind * g.num_layers + l] = (uint8_t)sh;
                consider(cand);
            }
        }
        // then the V-cycle kernels level by level, finest first
        const int lo = g.bottom_level + 1;
        for (int l = g.max_level; l >= lo; l--)
            for (int kind : {KS_GS_SWEEP, KS_PRESMOOTH, KS_PROLONG, KS_RESIDUAL}) {
                const std::vector<uint8_t> base = kept;
                for (int sh = 0; sh < num_shapes(kind); sh++) {
                    if (sh == base[(size_t)kind * g.num_layers + l]) continue;
                    std::vector<uint8_t> cand = base;
                    cand[(size_t)kind * g.num_layers + l] = (uint8_t)sh;
                    consider(cand);
                }
            }
    }
    g.shapes = kept;
    cudaMemcpyAsync(g.d_ch[kChB], bsave, bytes, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(g.d_ch[kChX], xsave, bytes, cudaMemcpyDeviceToDevice, s);
    cudaStreamSynchronize(s);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(bsave);
    cudaFree(xsave);
}

void drop_graphs(DevGrid& g) {
    // solve graphs captured with the previous shapes are rebuilt on the next solve
    for (auto& kv : g.graphs) cudaGraphExecDestroy(kv.second.exec);
    g.graphs.clear();
}

int autotune(DevGrid& g, cudaStream_t user, int reps, std::string* report) {
    if (reps < 1) reps = 1;
    // timing runs on a private stream (the caller's may be the legacy default stream, which
    // cannot be captured), after the caller's pending work
    if (cudaStreamSynchronize(user) != cudaSuccess) return 2;
    cudaStream_t s = nullptr;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return 2;
    float *p = g.d_ch[kChP], *ap = g.d_ch[kChAp], *z = g.d_ch[kChZ], *tmp = g.d_ch[kChTmp];
    const long long count0 = g.launch_count;
    const int lo = g.bottom_level >= 0 ? g.bottom_level + 1 : 0;
    auto pick = [&](int kind, int level, auto&& launch) {
        float best = 0.f;
        int best_shape = g.shape(kind, level);
        for (int sh = 0; sh < num_shapes(kind); sh++) {
            g.shapes[(size_t)kind * g.num_layers + level] = (uint8_t)sh;
            const float ms = time_graph(launch, reps, s);
            if (ms > 0.f && (best == 0.f || ms < best)) {
                best = ms;
                best_shape = sh;
            }
        }
        g.shapes[(size_t)kind * g.num_layers + level] = (uint8_t)best_shape;
        if (report) {
            char line[128];
            std::snprintf(line, sizeof line, "kind %d level %d shape %d %.2f us\n", kind, level, best_shape, 1e3f * best / reps);
            *report += line;
        }
    };
    for (int l = lo; l <= g.max_level; l++) {
        // the colour sweep as the solve runs it: with the r.z tile parts (r taken from channel p here)
        if (g.mg_count[l] > 0) pick(KS_GS_SWEEP, l, [&] { launch::gs_sweep(g, l, z, ap, 0, nullptr, s, p); });
        if (g.mg_count[l] > 0 && g.bottom_level >= 0)
            pick(KS_PRESMOOTH, l, [&] { launch::presmooth(g, l, g.d_xpre, ap, nullptr, s); });
        if (l >= 1 && g.level_count[l] > 0)
            pick(KS_RESIDUAL, l, [&] { launch::residual_restrict(g, l, g.d_xpre, ap, tmp, 1.f, nullptr, s, true); });
        if (l >= 1 && g.level_count[l] > 0 && g.bottom_level >= 0)
            pick(KS_PROLONG, l, [&] { launch::prolong_sweep(g, l, z, g.d_xpre, ap, 1.f, nullptr, s); });
    }
    if (g.n_lapmain + g.n_lapitems > 0) pick(KS_LAPLACIAN, 0, [&] { launch::laplacian_fused(g, p, tmp, nullptr, s, true); });
    if (g.n <= kSmallGridTiles && g.bottom_level >= 0) refine_by_solve(g, s);
    g.launch_count = count0;
    drop_graphs(g);
    const bool ok = cudaStreamSynchronize(s) == cudaSuccess;
    cudaStreamDestroy(s);
    return ok ? 0 : 2;
}

// Sweep-count tuner: each candidate (level_iters, coarsest_iters) solves the grid's current
// right-hand sides with `base` (precision, tolerance, flags), once to build its solve graph and
// once timed with CUDA events on a private stream; the fastest candidate whose every instance
// converged wins.  Sweep counts change the preconditioner (so the iterates), not the stopping
// rule: a mixed-precision solve still ends at its FP64 tolerance.  b is restored after every
// trial and at the end; x and the scratch channels keep the last trial's values.
int autotune_sweeps(DevGrid& g, const SolveParams& base, cudaStream_t user, int* level_iters, int* coarsest_iters,
                    std::string* report) {
    static const int kCand[][2] = {{1, 2}, {1, 4}, {1, 6}, {1, 10}, {1, 16}, {1, 24}, {2, 10}};
    *level_iters = base.level_iters;
    *coarsest_iters = base.coarsest_iters;
    if (cudaStreamSynchronize(user) != cudaSuccess) return 2;
    cudaStream_t s = nullptr;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return 2;
    const size_t bytes = (size_t)g.n * kTileCells * sizeof(float);
    float* bsave = nullptr;
    if (cudaMalloc(&bsave, bytes) != cudaSuccess) {
        cudaGetLastError();
        cudaStreamDestroy(s);
        return 3;
    }
    cudaMemcpyAsync(bsave, g.d_ch[kChB], bytes, cudaMemcpyDeviceToDevice, s);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    std::vector<SolveResult> r(g.num_inst);
    float best = -1.f;
    int rc = 0;
    for (const auto& c : kCand) {
        SolveParams p = base;
        p.level_iters = c[0];
        p.coarsest_iters = c[1];
        p.warm_start = 0;
        float ms = -1.f;
        bool ok = true;
        for (int rep = 0; rep < 2 && ok; rep++) {
            cudaMemcpyAsync(g.d_ch[kChB], bsave, bytes, cudaMemcpyDeviceToDevice, s);
            cudaEventRecord(e0, s);
            rc = base.precision ? mixed_solve(g, p, s, r.data()) : pcg_solve(g, p, s, r.data());
            cudaEventRecord(e1, s);
            if (rc || cudaEventSynchronize(e1) != cudaSuccess) {
                ok = false;
                break;
            }
            for (const SolveResult& x : r) ok = ok && x.status == 0;
            if (rep == 1) cudaEventElapsedTime(&ms, e0, e1);
        }
        if (rc) break;
        if (report) {
            char line[128];
            std::snprintf(line, sizeof line, "level_iters %d coarsest_iters %d: %s %.3f ms\n", c[0], c[1], ok ? "converged" : "not converged",
                          ms);
            *report += line;
        }
        if (ok && ms > 0.f && (best < 0.f || ms < best)) {
            best = ms;
            *level_iters = c[0];
            *coarsest_iters = c[1];
        }
    }
    cudaMemcpyAsync(g.d_ch[kChB], bsave, bytes, cudaMemcpyDeviceToDevice, s);
    const bool synced = cudaStreamSynchronize(s) == cudaSuccess;
    cudaFree(bsave);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamDestroy(s);
    drop_graphs(g);  // the trials' graphs; the next solve builds the one it needs
    g.x64_valid = false;
    if (rc) return rc;
    if (!synced) return 2;
    return best < 0.f ? 5 : 0;
}

}  // namespace cirrus
