// GMG-PCG driver: V-cycle schedule, the PCG loop captured as one CUDA graph with a device-side
// while-conditional (no host round trip per iteration), and the FP64 defect-correction loop.
// Every solve runs all active instances of a grid together: per-instance scalars and done flags,
// one kernel per step for the whole batch; the loop ends when the last instance stops.
#include "solver_internal.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <thread>

namespace cirrus {

// GMGSolver::VCycle (src/GMGSolver.cu:383-447): x = 0, rhs = f (0 on ghosts); downstroke
// GS(level_iters, order 0) + residual/restrict per level; coarsest GS(ci/2, 0) + GS(ci/2, 1);
// upstroke prolongate + GS(level_iters, order 1).
void vcycle(const DevGrid& g, float* X, const float* F, float* RHS, int level_iters, int coarsest_iters, float one_over_alpha,
            float prolong_coeff, const Scalars* S, cudaStream_t s) {
    launch::vcycle_init(g, X, RHS, F, S, s);
    auto smooth = [&](int level, int iters, int order) {
        // GaussSeidelGMG: colours (order, 1-order) per iteration
        uint32_t colors = 0;
        int ns = 0;
        for (int it = 0; it < iters; it++) {
            for (int c : {order, 1 - order}) {
                if (ns == 32) {
                    launch::gs_sequence(g, level, X, RHS, colors, ns, S, s);
                    colors = 0;
                    ns = 0;
                }
                colors |= (uint32_t)c << ns;
                ns++;
            }
        }
        if (ns) launch::gs_sequence(g, level, X, RHS, colors, ns, S, s);
    };
    for (int l = g.max_level; l > 0; l--) {
        smooth(l, level_iters, 0);
        launch::residual_restrict(g, l, X, RHS, RHS, one_over_alpha, S, s);
    }
    {
        uint32_t colors = 0;
        int ns = 0;
        auto push = [&](int c) {
            if (ns == 32) {
                launch::gs_sequence(g, 0, X, RHS, colors, ns, S, s);
                colors = 0;
                ns = 0;
            }
            colors |= (uint32_t)c << ns;
            ns++;
        };
        for (int it = 0; it < coarsest_iters / 2; it++) { push(0); push(1); }
        for (int it = 0; it < coarsest_iters / 2; it++) { push(1); push(0); }
        if (ns) launch::gs_sequence(g, 0, X, RHS, colors, ns, S, s);
    }
    for (int l = 1; l <= g.max_level; l++) {
        launch::prolongate(g, l, X, X, prolong_coeff, S, s);
        smooth(l, level_iters, 1);
    }
}

bool use_fused(const DevGrid& g, int level_iters, int coarsest_iters) {
    const char* e = std::getenv("CIRRUS_VCYCLE");
    if (e && std::strcmp(e, "generic") == 0) return false;
    return level_iters == 1 && g.bottom_level >= 0 && launch::bottom_supported(coarsest_iters, g.bottom_level);
}

void vcycle_fused(const DevGrid& g, float* X, float* RHS, int coarsest_iters, float one_over_alpha, float prolong_coeff,
                  const Scalars* S, cudaStream_t s, const float* dot_r) {
    const int lb = g.bottom_level;
    for (int l = g.max_level; l > lb; l--) {
        launch::presmooth(g, l, g.d_xpre, RHS, S, s);
        launch::residual_restrict(g, l, g.d_xpre, RHS, RHS, one_over_alpha, S, s, true);
    }
    launch::bottom(g, lb, coarsest_iters, X, RHS, one_over_alpha, prolong_coeff, S, s);
    for (int l = lb + 1; l <= g.max_level; l++) {
        launch::prolong_sweep(g, l, X, g.d_xpre, RHS, prolong_coeff, S, s);
        launch::gs_sweep(g, l, X, RHS, 0, S, s, dot_r);
    }
    if (dot_r) launch::leaf_wpart(g, dot_r, X, s);
}

namespace {

// the fused GMG V-cycle applies (the AMG preconditioner always runs its own V-cycle)
bool fused(const DevGrid& g, const SolveParams& p) {
    return p.preconditioner == 0 && use_fused(g, p.level_iters, p.coarsest_iters);
}

struct Ch {
    float *x, *r, *p, *ap, *z;
};
Ch channels(const DevGrid& g) { return {g.d_ch[kChX], g.d_ch[kChR], g.d_ch[kChP], g.d_ch[kChAp], g.d_ch[kChZ]}; }

// z <- M^-1 r with the fused kernels when level_iters == 1 (RHS already holds r on LEAF tiles).
// with_dot: the fused V-cycle also leaves the r.z tile parts in d_wpart (see k_gs_sweep_body).
void precondition(const DevGrid& g, const SolveParams& p, cudaStream_t s, bool with_dot = false) {
    const Ch c = channels(g);
    const Scalars* S = g.d_scalars;
    if (p.preconditioner == 1)  // AMGSolver::solve's VCycleAMG(z, r, tmp = Ap, rhs = tmp channel)
        vcycle_amg(g, c.z, c.r, c.ap, g.d_ch[kChTmp], p.level_iters, p.coarsest_iters, p.one_over_alpha, p.prolong_coeff, S, s);
    else if (fused(g, p))
        vcycle_fused(g, c.z, c.ap, p.coarsest_iters, p.one_over_alpha, p.prolong_coeff, S, s, with_dot ? c.r : nullptr);
    else vcycle(g, c.z, c.r, c.ap, p.level_iters, p.coarsest_iters, p.one_over_alpha, p.prolong_coeff, S, s);
}

// GMGSolver::solve, src/GMGSolver.cu:535-568
void record_prologue(const DevGrid& g, const SolveParams& p, const SolveCtl& ctl, cudaStream_t s) {
    const Ch c = channels(g);
    launch::begin_solve(g, ctl, s);
    // the fused V-cycle reads GHOST right-hand sides (channel Ap) as stored: 0; nothing in the
    // fused iteration writes them
    if (fused(g, p)) launch::zero_ghost_tiles(g, c.ap, s);
    launch::inst_reduce(OP_INIT, g, c.x, c.r, nullptr, c.ap, ctl, EPI_INIT, SKIP_INACTIVE, s);
    if (p.pure_neumann) {
        launch::inst_reduce(OP_MEAN, g, c.r, nullptr, nullptr, nullptr, ctl, EPI_MEAN, SKIP_DONE, s);
        launch::recenter(g, c.r, c.ap, s);
    }
    precondition(g, p, s);
    launch::inst_reduce(OP_COPY_DOT, g, c.z, c.r, c.p, nullptr, ctl, EPI_GAMMA, SKIP_DONE, s);
}

// One PCG iteration, src/GMGSolver.cu:573-653
void record_body(const DevGrid& g, const SolveParams& p, const SolveCtl& ctl, cudaStream_t s) {
    const Ch c = channels(g);
    if (fused(g, p)) {
        // p.Ap tile parts: from the Laplacian for LEAF tiles without GHOST children, from
        // pap_ghost (after adding the children's sums to Ap) for the others
        launch::laplacian_fused(g, c.p, c.ap, g.d_scalars, s, true);
        launch::pap_ghost(g, c.p, c.ap, s);
        launch::inst_wsum(g, ctl, EPI_ALPHA, SKIP_DONE, s);
    } else {
        launch::full_laplacian<float>(g, c.p, c.ap, g.d_scalars, s);
        launch::inst_reduce(OP_DOT, g, c.p, c.ap, nullptr, nullptr, ctl, EPI_ALPHA, SKIP_DONE, s);
    }
    launch::inst_reduce(OP_XR, g, c.x, c.p, c.r, c.ap, ctl, EPI_CHECK, SKIP_DONE, s);
    if (p.pure_neumann) {
        launch::inst_reduce(OP_MEAN, g, c.r, nullptr, nullptr, nullptr, ctl, EPI_MEAN, SKIP_DONE, s);
        launch::recenter(g, c.r, c.ap, s);
    }
    if (fused(g, p)) {
        precondition(g, p, s, true);  // r.z tile parts formed by the V-cycle's last colour sweeps
        launch::inst_wsum(g, ctl, EPI_BETA, SKIP_DONE, s);
    } else {
        precondition(g, p, s);
        launch::inst_reduce(OP_DOT, g, c.r, c.z, nullptr, nullptr, ctl, EPI_BETA, SKIP_DONE, s);
    }
    launch::update_p(g, c.p, c.z, c.x, s);
}

void record_epilogue(const DevGrid& g, const SolveCtl& ctl, cudaStream_t s) {
    const Ch c = channels(g);
    launch::x_final(g, c.x, c.p, s);
    launch::inst_reduce(OP_DOT, g, c.r, c.r, nullptr, nullptr, ctl, EPI_FINAL, SKIP_INACTIVE, s);
}

SolveCtl make_ctl(const DevGrid& g, const SolveParams& p) {
    SolveCtl c{};
    c.sync_stride = p.sync_stride;
    c.history = g.d_history;
    c.history_cap = g.history_cap;
    c.use_cond = 0;
    c.cond = 0;
    c.active = g.d_active;
    return c;
}

bool graphs_enabled() {
    const char* e = std::getenv("CIRRUS_NO_GRAPH");
    return !(e && e[0] == '1');
}

#define GK(x)                                                                      \
    do {                                                                           \
        cudaError_t e_ = (x);                                                      \
        if (e_ != cudaSuccess) {                                                   \
            g.last_error = std::string("graph build: " #x ": ") + cudaGetErrorString(e_); \
            ok = false;                                                            \
        }                                                                          \
    } while (0)

// Build the whole solve as one graph: prologue -> while(cond){ body } -> epilogue.
DevGrid::SolveGraph build_graph(DevGrid& g, const SolveParams& p) {
    bool ok = true;
    DevGrid::SolveGraph out;
    cudaStream_t cs = nullptr, cs2 = nullptr;
    GK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    GK(cudaStreamCreateWithFlags(&cs2, cudaStreamNonBlocking));
    if (!ok) return out;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    GK(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    cudaStreamCaptureStatus st;
    GK(cudaStreamGetCaptureInfo(cs, &st, nullptr, &graph, nullptr, nullptr));
    cudaGraphConditionalHandle handle = 0;
    GK(cudaGraphConditionalHandleCreate(&handle, graph, 1, cudaGraphCondAssignDefault));
    SolveCtl ctl = make_ctl(g, p);
    ctl.use_cond = 1;
    ctl.cond = handle;
    long long c0 = g.launch_count;
    record_prologue(g, p, ctl, cs);
    out.prologue = g.launch_count - c0;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    GK(cudaStreamGetCaptureInfo(cs, &st, nullptr, &graph, &deps, &ndeps));
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = handle;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t cnode = nullptr;
    GK(cudaGraphAddNode(&cnode, graph, deps, ndeps, &cp));
    if (ok) {
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        GK(cudaStreamBeginCaptureToGraph(cs2, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        c0 = g.launch_count;
        record_body(g, p, ctl, cs2);
        out.body = g.launch_count - c0;
        GK(cudaStreamEndCapture(cs2, &body));
        GK(cudaStreamUpdateCaptureDependencies(cs, &cnode, 1, cudaStreamSetCaptureDependencies));
    }
    c0 = g.launch_count;
    record_epilogue(g, ctl, cs);
    out.epilogue = g.launch_count - c0;
    cudaGraph_t outg = nullptr;
    cudaError_t ee = cudaStreamEndCapture(cs, &outg);
    if (ee != cudaSuccess) {
        g.last_error = std::string("graph build: end capture: ") + cudaGetErrorString(ee);
        ok = false;
    }
    if (ok) GK(cudaGraphInstantiate(&exec, outg, 0));
    if (outg) cudaGraphDestroy(outg);
    cudaStreamDestroy(cs);
    cudaStreamDestroy(cs2);
    if (!ok) {
        cudaGetLastError();
        if (exec) cudaGraphExecDestroy(exec);
        return DevGrid::SolveGraph();
    }
    out.exec = exec;
    return out;
}

// Per-instance parameters of a solve into the pinned mirror and onto the device (ordered on s).
void upload_params(DevGrid& g, const SolveParams& p, const InstRequest* req, cudaStream_t s) {
    for (int i = 0; i < g.num_inst; i++) {
        InstParams& q = g.h_iparams[i];
        q.tol = (req && req[i].tol >= 0) ? req[i].tol : p.tol;
        q.max_iters = p.max_iters;
        q.active = req ? (req[i].active ? 1 : 0) : 1;
        q.pure_neumann = (req && req[i].pure_neumann >= 0) ? req[i].pure_neumann : p.pure_neumann;
        q.pad = 0;
    }
    cudaMemcpyAsync(g.d_iparams, g.h_iparams, sizeof(InstParams) * g.num_inst, cudaMemcpyHostToDevice, s);
}

bool any_pure_neumann(const DevGrid& g) {
    for (int i = 0; i < g.num_inst; i++)
        if (g.h_iparams[i].active && g.h_iparams[i].pure_neumann) return true;
    return false;
}

}  // namespace

int pcg_solve(DevGrid& g, const SolveParams& p0, cudaStream_t s, SolveResult* r, const InstRequest* req) {
    long long direct = -1;
    int rc = pcg_launch(g, p0, s, req, &direct);
    if (rc) return rc;
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        g.last_error = std::string("solve: ") + cudaGetErrorString(e);
        return 2;
    }
    pcg_collect(g, p0, direct, r);
    return 0;
}

int solve_grids(const std::vector<DevGrid*>& grids, const SolveParams& p, cudaStream_t s, std::vector<std::vector<SolveResult>>& r) {
    r.assign(grids.size(), {});
    for (size_t k = 0; k < grids.size(); k++) r[k].resize(grids[k]->num_inst);
    for (DevGrid* g : grids) {
        if (!g->side_stream && cudaStreamCreateWithFlags(&g->side_stream, cudaStreamNonBlocking) != cudaSuccess) {
            g->side_stream = nullptr;
            return 2;
        }
        if (!g->side_join && cudaEventCreateWithFlags(&g->side_join, cudaEventDisableTiming) != cudaSuccess) {
            g->side_join = nullptr;
            return 2;
        }
    }
    cudaEvent_t fork = nullptr;
    if (cudaEventCreateWithFlags(&fork, cudaEventDisableTiming) != cudaSuccess) return 2;
    cudaEventRecord(fork, s);
    if (p.precision != 0) {
        // the mixed-precision outer loop reads residuals on the host: one host thread per grid,
        // each driving its grid's own stream
        std::vector<int> rcs(grids.size(), 0);
        std::vector<std::thread> th;
        for (size_t k = 0; k < grids.size(); k++) {
            cudaStreamWaitEvent(grids[k]->side_stream, fork, 0);
            th.emplace_back([&, k] { rcs[k] = mixed_solve(*grids[k], p, grids[k]->side_stream, r[k].data()); });
        }
        for (std::thread& t : th) t.join();
        for (DevGrid* g : grids) {
            cudaEventRecord(g->side_join, g->side_stream);
            cudaStreamWaitEvent(s, g->side_join, 0);
        }
        const cudaError_t e = cudaStreamSynchronize(s);
        cudaEventDestroy(fork);
        for (int rc : rcs)
            if (rc) return rc;
        return e == cudaSuccess ? 0 : 2;
    }
    std::vector<long long> direct(grids.size(), -1);
    int rc = 0;
    size_t launched = 0;
    for (; launched < grids.size(); launched++) {
        DevGrid& g = *grids[launched];
        g.x64_valid = false;
        cudaStreamWaitEvent(g.side_stream, fork, 0);
        rc = pcg_launch(g, p, g.side_stream, nullptr, &direct[launched]);
        cudaEventRecord(g.side_join, g.side_stream);
        cudaStreamWaitEvent(s, g.side_join, 0);
        if (rc) {
            launched++;
            break;
        }
    }
    const cudaError_t e = cudaStreamSynchronize(s);
    cudaEventDestroy(fork);
    if (rc) return rc;
    if (e != cudaSuccess) {
        grids[0]->last_error = std::string("solve: ") + cudaGetErrorString(e);
        return 2;
    }
    for (size_t k = 0; k < grids.size(); k++) pcg_collect(*grids[k], p, direct[k], r[k].data());
    return 0;
}

int pcg_launch(DevGrid& g, const SolveParams& p0, cudaStream_t s, const InstRequest* req, long long* direct_out) {
    if (p0.preconditioner == 1 && !g.amg_ready) {
        g.last_error = "AMG solve before its coefficients were prepared (amg_prepare)";
        return 1;
    }
    upload_params(g, p0, req, s);
    SolveParams p = p0;
    p.pure_neumann = any_pure_neumann(g) ? 1 : 0;
    GraphKey key{0, p.level_iters, p.coarsest_iters, p.sync_stride, p.pure_neumann, p.one_over_alpha, p.prolong_coeff,
                 fused(g, p) ? 1 : 0, p.preconditioner};
    DevGrid::SolveGraph sg;
    if (graphs_enabled() && g.launch_mode == 0) {
        auto it = g.graphs.find(key);
        if (it != g.graphs.end()) sg = it->second;
        else {
            sg = build_graph(g, p);
            if (sg.exec) g.graphs[key] = sg;
        }
    }
    long long direct = -1;
    if (sg.exec) {
        cudaError_t e = cudaGraphLaunch(sg.exec, s);
        if (e != cudaSuccess) {
            g.last_error = std::string("cudaGraphLaunch: ") + cudaGetErrorString(e);
            return 2;
        }
    } else {
        // Direct launches with a host-checked loop (the reference's sync_stride behaviour).
        const long long c0 = g.launch_count;
        SolveCtl ctl = make_ctl(g, p);
        record_prologue(g, p, ctl, s);
        for (int i = 0; i < p.max_iters; i++) {
            cudaMemcpyAsync(g.h_scalars, g.d_scalars, sizeof(Scalars) * g.num_inst, cudaMemcpyDeviceToHost, s);
            cudaStreamSynchronize(s);
            bool all_done = true;
            for (int k = 0; k < g.num_inst; k++) all_done = all_done && g.h_scalars[k].done;
            if (all_done) break;
            record_body(g, p, ctl, s);
        }
        record_epilogue(g, ctl, s);
        direct = g.launch_count - c0;
    }
    cudaMemcpyAsync(g.h_scalars, g.d_scalars, sizeof(Scalars) * g.num_inst, cudaMemcpyDeviceToHost, s);
    // a kernel whose bounded wait gave up (a stage that never filled) leaves a flag; read with the scalars
    cudaMemcpyAsync(g.h_err, g.d_err, sizeof(unsigned int), cudaMemcpyDeviceToHost, s);
    *direct_out = direct;
    return 0;
}

void pcg_collect(DevGrid& g, const SolveParams& p, long long direct, SolveResult* r) {
    const DevGrid::SolveGraph* sgp = nullptr;
    if (direct < 0) {
        GraphKey key{0, p.level_iters, p.coarsest_iters, p.sync_stride, any_pure_neumann(g) ? 1 : 0, p.one_over_alpha,
                     p.prolong_coeff, fused(g, p) ? 1 : 0, p.preconditioner};
        auto it = g.graphs.find(key);
        if (it != g.graphs.end()) sgp = &it->second;
    }
    // bodies executed = the largest iteration count of the instances (each body advances every
    // iterating instance's counter once)
    int loops = 0;
    for (int k = 0; k < g.num_inst; k++)
        if (g.h_iparams[k].active) loops = std::max(loops, g.h_scalars[k].iter);
    g.last_solve_launches = direct >= 0 ? direct : sgp ? sgp->prologue + (long long)loops * sgp->body + sgp->epilogue : 0;
    const bool wait_failed = *g.h_err != 0;
    if (wait_failed) {
        g.last_error = "a staged kernel gave up waiting for its copies (bounded wait)";
        *g.h_err = 0;
        cudaMemset(g.d_err, 0, sizeof(unsigned int));
    }
    for (int k = 0; k < g.num_inst; k++) {
        const Scalars& S = g.h_scalars[k];
        SolveResult& o = r[k];
        o = SolveResult();
        o.iters = S.iters;
        o.rel = S.rel;
        o.status = S.nonfinite ? 6 : (S.converged ? 0 : 5);
        if (p.sync_stride <= 0) o.status = 0;
        if (!g.h_iparams[k].active) o.status = 0;
        if (wait_failed) o.status = 2;
        o.launches = g.last_solve_launches;
    }
}

namespace {
int ensure_fp64(DevGrid& g) {
    if (g.d_x64) return 0;
    const size_t cells = (size_t)g.n * kTileCells;
    if (cudaMalloc(&g.d_x64, cells * sizeof(double)) != cudaSuccess) return 3;
    if (cudaMalloc(&g.d_ax64, cells * sizeof(double)) != cudaSuccess) return 3;
    if (cudaMalloc(&g.d_r64, cells * sizeof(double)) != cudaSuccess) return 3;
    if (cudaMalloc(&g.d_bsave, cells * sizeof(float)) != cudaSuccess) return 3;
    cudaMemset(g.d_x64, 0, cells * sizeof(double));
    cudaMemset(g.d_ax64, 0, cells * sizeof(double));
    if (cudaMalloc(&g.d_msum, sizeof(double) * g.num_inst) != cudaSuccess) return 3;
    if (cudaMalloc(&g.d_dofd, sizeof(double) * g.num_inst) != cudaSuccess) return 3;
    std::vector<double> dofd(g.inst_dof.begin(), g.inst_dof.end());
    if (cudaMemcpy(g.d_dofd, dofd.data(), sizeof(double) * g.num_inst, cudaMemcpyHostToDevice) != cudaSuccess) return 2;
    g.bytes += cells * (3 * sizeof(double) + sizeof(float)) + 2 * sizeof(double) * g.num_inst;
    return 0;
}

// Per-instance norms computed on the device into host doubles.
void read_norms(DevGrid& g, std::vector<double>& out, cudaStream_t s) {
    out.assign(g.num_inst, 0.0);
    cudaMemcpyAsync(out.data(), g.d_norm, sizeof(double) * g.num_inst, cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
}

void set_active(DevGrid& g, const std::vector<uint8_t>& active, cudaStream_t s, const std::vector<uint8_t>* pure = nullptr) {
    for (int i = 0; i < g.num_inst; i++) {
        g.h_iparams[i].active = active[i];
        if (pure) g.h_iparams[i].pure_neumann = (*pure)[i];
    }
    cudaMemcpyAsync(g.d_iparams, g.h_iparams, sizeof(InstParams) * g.num_inst, cudaMemcpyHostToDevice, s);
}
}  // namespace

int true_residual(DevGrid& g, const float* d_b, double* rel, cudaStream_t s) {
    int rc = ensure_fp64(g);
    if (rc) return rc;
    const size_t cells = (size_t)g.n * kTileCells;
    set_active(g, std::vector<uint8_t>(g.num_inst, 1), s);
    std::vector<double> bb, rr;
    launch::norm64(g, nullptr, d_b, g.d_norm, s);
    read_norms(g, bb, s);
    if (!g.x64_valid) launch::widen(g, g.d_ch[kChX], g.d_x64, cells, s);
    launch::full_laplacian<double>(g, g.d_x64, g.d_ax64, nullptr, s);
    launch::residual64(g, d_b, g.d_ax64, g.d_r64, g.d_bsave, s);
    launch::norm64(g, g.d_r64, nullptr, g.d_norm, s);
    read_norms(g, rr, s);
    for (int i = 0; i < g.num_inst; i++) rel[i] = bb[i] > 0 ? std::sqrt(rr[i] / bb[i]) : 0.0;
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

// FP64 defect correction of every active instance: x64 accumulates FP32 PCG corrections e
// solving A e = r, with r = b - A x64 formed in FP64 on the device; an instance stops when its
// ||r||/||b|| < tol (FP64 true residual).  All instances still correcting share each inner solve.
// A pure-Neumann instance's r is projected off A's null space (its mean over INTERIOR cells of
// LEAF tiles removed) before the norm and the inner solve, which also recentres as the
// reference's does; ||b|| is the unprojected norm, as the reference's rhs_norm2.
int damped_jacobi(DevGrid& g, int max_iters, double tol, float omega, cudaStream_t s, int* iters, double* rel) {
    float *X = g.d_ch[kChX], *B = g.d_ch[kChB], *AX = g.d_ch[2], *D = g.d_ch[3];
    cudaMemsetAsync(X, 0, (size_t)g.n * kTileCells * sizeof(float), s);  // x = 0 on LEAF|NONLEAF|GHOST tiles
    const int n_mg = g.mg_offset.empty() ? 0 : g.mg_offset.back() + g.mg_count.back();
    // ||b|| over LEAF|NONLEAF|GHOST tiles (src/GMGSolver.cu:467): the multigrid lists of all
    // levels hold every LEAF and NONLEAF tile once
    const double rhs_norm =
        std::sqrt(launch::list_dot(g, B, B, g.d_mg, n_mg, s) + launch::list_dot(g, B, B, g.d_ghost, g.n_ghost, s));
    const double threshold = std::max(tol * rhs_norm, std::numeric_limits<double>::min());
    double res = rhs_norm;
    int i = 0;
    for (i = 0; i < max_iters; i++) {
        launch::full_laplacian<float>(g, X, AX, nullptr, s);
        launch::jacobi_residual(g, B, AX, s);
        res = std::sqrt(launch::list_dot(g, AX, AX, g.d_leaf, g.n_leaf, s));
        if (res < threshold) break;
        launch::full_laplacian_diag(g, X, D, s);
        launch::jacobi_update(g, X, AX, D, omega, s);
    }
    g.x64_valid = false;
    *iters = i;
    *rel = res / rhs_norm;
    return cudaStreamSynchronize(s) == cudaSuccess ? 0 : 2;
}

int mixed_solve(DevGrid& g, const SolveParams& p, cudaStream_t s, SolveResult* r, const InstRequest* req) {
    int rc = ensure_fp64(g);
    if (rc) return rc;
    const int K = g.num_inst;
    const size_t cells = (size_t)g.n * kTileCells;
    const long long own0 = g.launch_count;
    long long inner_recorded = 0, inner_executed = 0;
    std::vector<uint8_t> want(K), active(K), pure(K);
    std::vector<double> tol(K);
    bool any_pure = false;
    for (int i = 0; i < K; i++) {
        want[i] = req ? (req[i].active ? 1 : 0) : 1;
        tol[i] = (req && req[i].tol >= 0) ? req[i].tol : p.tol;
        pure[i] = (req && req[i].pure_neumann >= 0) ? (req[i].pure_neumann ? 1 : 0) : (p.pure_neumann ? 1 : 0);
        any_pure = any_pure || (want[i] && pure[i]);
        r[i] = SolveResult();
        r[i].status = want[i] ? 5 : 0;
    }
    cudaMemcpyAsync(g.d_bsave, g.d_ch[kChB], cells * sizeof(float), cudaMemcpyDeviceToDevice, s);
    if (p.warm_start) launch::widen(g, g.d_ch[kChX], g.d_x64, cells, s);
    else cudaMemsetAsync(g.d_x64, 0, cells * sizeof(double), s);
    std::vector<double> bb, rr;
    launch::norm64(g, nullptr, g.d_bsave, g.d_norm, s);
    read_norms(g, bb, s);
    for (int i = 0; i < K; i++) {
        active[i] = want[i] && bb[i] != 0.0;
        if (want[i] && bb[i] == 0.0) {  // zero right-hand side: x = 0
            r[i].status = 0;
            r[i].rel = 0;
            r[i].true_rel = 0;
        }
    }
    std::vector<double> rel(K, 1.0);
    for (int k = 0; k <= p.max_outer; k++) {
        set_active(g, active, s, &pure);
        // from x = 0 the first residual is b itself: no FP64 Laplacian
        const bool cold = k == 0 && !p.warm_start;
        if (!cold) launch::full_laplacian<double>(g, g.d_x64, g.d_ax64, nullptr, s);
        launch::residual64(g, g.d_bsave, cold ? nullptr : g.d_ax64, g.d_r64, g.d_ch[kChB], s);
        if (any_pure) {
            launch::norm64(g, g.d_r64, nullptr, g.d_msum, s, true);
            launch::sub_mean64(g, g.d_r64, g.d_ch[kChB], g.d_msum, g.d_dofd, s);
        }
        launch::norm64(g, g.d_r64, nullptr, g.d_norm, s);
        read_norms(g, rr, s);
        bool any = false;
        std::vector<InstRequest> inner(K);
        for (int i = 0; i < K; i++) {
            inner[i].active = 0;
            if (!active[i]) continue;
            rel[i] = std::sqrt(rr[i] / bb[i]);
            if (!(rel[i] == rel[i])) { r[i].status = 6; active[i] = 0; continue; }
            if (rel[i] < tol[i]) { r[i].status = 0; active[i] = 0; continue; }
            if (k == p.max_outer) { active[i] = 0; continue; }
            // each inner FP32 solve targets the defect that leaves the outer residual just under
            // tol (0.9 of it: the FP32 recursive residual the inner solve stops on stays within a
            // few percent of the true one at these tolerances, and an outer step that falls short
            // costs one more short inner solve), but never tighter than inner_tol (where FP32
            // stalls) nor looser than 0.1
            double tau = 0.9 * tol[i] / rel[i];
            tau = std::min(0.1, std::max(p.inner_tol, tau));
            inner[i].active = 1;
            inner[i].tol = tau;
            inner[i].pure_neumann = pure[i];
            any = true;
        }
        if (!any) break;
        SolveParams ip = p;
        ip.precision = 0;
        std::vector<SolveResult> ir(K);
        const long long a = g.launch_count;
        int e = pcg_solve(g, ip, s, ir.data(), inner.data());
        if (e) return e;
        inner_recorded += g.launch_count - a;
        inner_executed += ir[0].launches;
        for (int i = 0; i < K; i++)
            if (inner[i].active) {
                r[i].iters += ir[i].iters;
                r[i].outer++;
            }
        // the inner solve left the active flags of this step on the device
        launch::accumulate_correction(g, g.d_x64, g.d_ch[kChX], s);
    }
    launch::narrow(g, g.d_x64, g.d_ch[kChX], cells, s);
    g.x64_valid = true;
    const long long launches = (g.launch_count - own0 - inner_recorded) + inner_executed;
    g.last_solve_launches = launches;
    for (int i = 0; i < K; i++) {
        if (want[i] && bb[i] != 0.0) {
            r[i].rel = rel[i];
            r[i].true_rel = rel[i];
        }
        r[i].launches = launches;
    }
    // b channel ends as the last FP32 defect, mirroring "b channel will be modified"
    return cudaStreamSynchronize(s) == cudaSuccess ? 0 : 2;
}

int solution_f64(DevGrid& g, double* host, cudaStream_t s) {
    int rc = ensure_fp64(g);
    if (rc) return rc;
    const size_t cells = (size_t)g.n * kTileCells;
    if (!g.x64_valid) launch::widen(g, g.d_ch[kChX], g.d_x64, cells, s);
    cudaMemcpyAsync(host, g.d_x64, cells * sizeof(double), cudaMemcpyDeviceToHost, s);
    return cudaStreamSynchronize(s) == cudaSuccess ? 0 : 2;
}

}  // namespace cirrus
