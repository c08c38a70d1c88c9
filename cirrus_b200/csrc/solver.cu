// GMG-PCG driver: V-cycle schedule, the PCG loop captured as one CUDA graph with a device-side
// while-conditional (no host round trip per iteration), and the FP64 defect-correction loop.
#include "solver_internal.hpp"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

namespace cirrus {

// GMGSolver::VCycle (src/GMGSolver.cu:383-447): x = 0, rhs = f (0 on ghosts); downstroke
// GS(level_iters, order 0) + residual/restrict per level; coarsest GS(ci/2, 0) + GS(ci/2, 1);
// upstroke prolongate + GS(level_iters, order 1).
void vcycle(const DevGrid& g, float* X, const float* F, float* RHS, int level_iters, int coarsest_iters, float one_over_alpha,
            float prolong_coeff, const int* done, cudaStream_t s) {
    launch::vcycle_init(g, X, RHS, F, done, s);
    auto smooth = [&](int level, int iters, int order) {
        // GaussSeidelGMG: colours (order, 1-order) per iteration
        uint32_t colors = 0;
        int ns = 0;
        for (int it = 0; it < iters; it++) {
            for (int c : {order, 1 - order}) {
                if (ns == 32) {
                    launch::gs_sequence(g, level, X, RHS, colors, ns, done, s);
                    colors = 0;
                    ns = 0;
                }
                colors |= (uint32_t)c << ns;
                ns++;
            }
        }
        if (ns) launch::gs_sequence(g, level, X, RHS, colors, ns, done, s);
    };
    for (int l = g.max_level; l > 0; l--) {
        smooth(l, level_iters, 0);
        launch::residual_restrict(g, l, X, RHS, RHS, one_over_alpha, done, s);
    }
    {
        uint32_t colors = 0;
        int ns = 0;
        auto push = [&](int c) {
            if (ns == 32) {
                launch::gs_sequence(g, 0, X, RHS, colors, ns, done, s);
                colors = 0;
                ns = 0;
            }
            colors |= (uint32_t)c << ns;
            ns++;
        };
        for (int it = 0; it < coarsest_iters / 2; it++) { push(0); push(1); }
        for (int it = 0; it < coarsest_iters / 2; it++) { push(1); push(0); }
        if (ns) launch::gs_sequence(g, 0, X, RHS, colors, ns, done, s);
    }
    for (int l = 1; l <= g.max_level; l++) {
        launch::prolongate(g, l, X, X, prolong_coeff, done, s);
        smooth(l, level_iters, 1);
    }
}

bool use_fused(const DevGrid& g, int level_iters, int coarsest_iters) {
    const char* e = std::getenv("CIRRUS_VCYCLE");
    if (e && std::strcmp(e, "generic") == 0) return false;
    return level_iters == 1 && g.bottom_level >= 0 && launch::bottom_supported(coarsest_iters, std::min(g.bottom_level, g.max_level));
}

void vcycle_fused(const DevGrid& g, float* X, float* RHS, int coarsest_iters, float one_over_alpha, float prolong_coeff,
                  const int* done, cudaStream_t s) {
    const int lb = std::min(g.bottom_level, g.max_level);
    for (int l = g.max_level; l > lb; l--) {
        launch::presmooth(g, l, g.d_xpre, RHS, done, s);
        launch::residual_restrict(g, l, g.d_xpre, RHS, RHS, one_over_alpha, done, s);
    }
    launch::bottom(g, lb, coarsest_iters, X, RHS, one_over_alpha, prolong_coeff, done, s);
    for (int l = lb + 1; l <= g.max_level; l++) {
        launch::prolong_sweep(g, l, X, g.d_xpre, RHS, prolong_coeff, done, s);
        launch::gs_sweep(g, l, X, RHS, 0, done, s);
    }
}

namespace {

struct Ch {
    float *x, *r, *p, *ap, *z;
};

// z <- M^-1 r with the fused kernels when level_iters == 1 (RHS already holds r on LEAF tiles).
void precondition(const DevGrid& g, const SolveParams& p, const int* done, cudaStream_t s) {
    const Ch c{g.d_ch[kChX], g.d_ch[kChR], g.d_ch[kChP], g.d_ch[kChAp], g.d_ch[kChZ]};
    if (use_fused(g, p.level_iters, p.coarsest_iters)) vcycle_fused(g, c.z, c.ap, p.coarsest_iters, p.one_over_alpha, p.prolong_coeff, done, s);
    else vcycle(g, c.z, c.r, c.ap, p.level_iters, p.coarsest_iters, p.one_over_alpha, p.prolong_coeff, done, s);
}
Ch channels(const DevGrid& g) { return {g.d_ch[kChX], g.d_ch[kChR], g.d_ch[kChP], g.d_ch[kChAp], g.d_ch[kChZ]}; }

// GMGSolver::solve, src/GMGSolver.cu:535-568
void record_prologue(const DevGrid& g, const SolveParams& p, const SolveCtl& ctl, cudaStream_t s) {
    const Ch c = channels(g);
    Scalars* S = g.d_scalars;
    const int* done = &S->done;
    cudaMemsetAsync(S, 0, sizeof(Scalars), s);
    // the fused V-cycle reads GHOST right-hand sides (channel Ap) as stored: 0; nothing in the
    // fused iteration writes them
    if (use_fused(g, p.level_iters, p.coarsest_iters)) launch::zero_ghost_tiles(g, c.ap, s);
    launch::leaf_reduce(OP_INIT, g, c.x, c.r, nullptr, c.ap, S, ctl, EPI_INIT, 0, s);
    if (p.pure_neumann) {
        launch::leaf_reduce(OP_MEAN, g, c.r, nullptr, nullptr, nullptr, S, ctl, EPI_MEAN, 1, s);
        launch::recenter(g, c.r, S, 1, s, c.ap);
    }
    precondition(g, p, done, s);
    launch::leaf_reduce(OP_COPY_DOT, g, c.z, c.r, c.p, nullptr, S, ctl, EPI_GAMMA, 1, s);
}

// One PCG iteration, src/GMGSolver.cu:573-653
void record_body(const DevGrid& g, const SolveParams& p, const SolveCtl& ctl, cudaStream_t s) {
    const Ch c = channels(g);
    Scalars* S = g.d_scalars;
    const int* done = &S->done;
    if (use_fused(g, p.level_iters, p.coarsest_iters)) {
        launch::laplacian_fused(g, c.p, c.ap, done, s);
        launch::leaf_reduce(OP_PAP, g, c.p, c.ap, g.d_gacc, nullptr, S, ctl, EPI_ALPHA, 1, s);
    } else {
        launch::full_laplacian<float>(g, c.p, c.ap, done, s);
        launch::leaf_reduce(OP_DOT, g, c.p, c.ap, nullptr, nullptr, S, ctl, EPI_ALPHA, 1, s);
    }
    launch::leaf_reduce(OP_XR, g, c.x, c.p, c.r, c.ap, S, ctl, EPI_CHECK, 1, s);
    if (p.pure_neumann) {
        launch::leaf_reduce(OP_MEAN, g, c.r, nullptr, nullptr, nullptr, S, ctl, EPI_MEAN, 1, s);
        launch::recenter(g, c.r, S, 1, s, c.ap);
    }
    precondition(g, p, done, s);
    launch::leaf_reduce(OP_DOT, g, c.r, c.z, nullptr, nullptr, S, ctl, EPI_BETA, 1, s);
    launch::update_p(g, c.p, c.z, S, s);
}

void record_epilogue(const DevGrid& g, const SolveCtl& ctl, cudaStream_t s) {
    const Ch c = channels(g);
    launch::leaf_reduce(OP_DOT, g, c.r, c.r, nullptr, nullptr, g.d_scalars, ctl, EPI_FINAL, 0, s);
}

SolveCtl make_ctl(const DevGrid& g, const SolveParams& p) {
    SolveCtl c{};
    c.sync_stride = p.sync_stride;
    c.max_iters = p.max_iters;
    c.tol = p.tol;
    c.history = g.d_history;
    c.history_cap = g.history_cap;
    c.use_cond = 0;
    c.cond = 0;
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

void fill_result(const DevGrid& g, SolveResult* r) {
    const Scalars& S = *g.h_scalars;
    r->iters = S.iters;
    r->rel = S.rel;
    r->status = S.nonfinite ? 6 : (S.converged ? 0 : 5);
}

}  // namespace

int pcg_solve(DevGrid& g, const SolveParams& p, cudaStream_t s, SolveResult* r) {
    GraphKey key{p.max_iters, p.level_iters, p.coarsest_iters, p.sync_stride, p.pure_neumann, p.tol, p.one_over_alpha, p.prolong_coeff,
                 use_fused(g, p.level_iters, p.coarsest_iters) ? 1 : 0};
    DevGrid::SolveGraph sg;
    if (graphs_enabled()) {
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
            cudaMemcpyAsync(g.h_scalars, g.d_scalars, sizeof(Scalars), cudaMemcpyDeviceToHost, s);
            cudaStreamSynchronize(s);
            if (g.h_scalars->done) break;
            record_body(g, p, ctl, s);
        }
        record_epilogue(g, ctl, s);
        direct = g.launch_count - c0;
    }
    cudaMemcpyAsync(g.h_scalars, g.d_scalars, sizeof(Scalars), cudaMemcpyDeviceToHost, s);
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        g.last_error = std::string("solve: ") + cudaGetErrorString(e);
        return 2;
    }
    fill_result(g, r);
    // bodies executed = iterations entered (the counter is advanced once per body)
    g.last_solve_launches = direct >= 0 ? direct : sg.prologue + (long long)g.h_scalars->iter * sg.body + sg.epilogue;
    r->launches = g.last_solve_launches;
    if (p.sync_stride <= 0) r->status = 0;
    return 0;
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
    g.bytes += cells * (3 * sizeof(double) + sizeof(float));
    return 0;
}

double read_norm(DevGrid& g, cudaStream_t s) {
    double v = 0;
    cudaMemcpyAsync(&v, g.d_norm, sizeof(double), cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    return v;
}
}  // namespace

int true_residual(DevGrid& g, const float* d_b, double* rel, cudaStream_t s) {
    int rc = ensure_fp64(g);
    if (rc) return rc;
    const size_t cells = (size_t)g.n * kTileCells;
    launch::norm64(g, nullptr, d_b, g.d_norm, s);
    const double bb = read_norm(g, s);
    if (!g.x64_valid) launch::widen(g, g.d_ch[kChX], g.d_x64, cells, s);
    launch::full_laplacian<double>(g, g.d_x64, g.d_ax64, nullptr, s);
    launch::residual64(g, d_b, g.d_ax64, g.d_r64, g.d_bsave, s);
    launch::norm64(g, g.d_r64, nullptr, g.d_norm, s);
    const double rr = read_norm(g, s);
    *rel = bb > 0 ? std::sqrt(rr / bb) : 0.0;
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

// FP64 defect correction: x64 accumulates FP32 PCG corrections e solving A e = r, with
// r = b - A x64 formed in FP64 on the device; stops when ||r||/||b|| < tol (FP64 true residual).
int mixed_solve(DevGrid& g, const SolveParams& p, cudaStream_t s, SolveResult* r) {
    int rc = ensure_fp64(g);
    if (rc) return rc;
    const size_t cells = (size_t)g.n * kTileCells;
    const long long own0 = g.launch_count;
    long long inner_recorded = 0, inner_executed = 0;
    cudaMemcpyAsync(g.d_bsave, g.d_ch[kChB], cells * sizeof(float), cudaMemcpyDeviceToDevice, s);
    if (p.warm_start) launch::widen(g, g.d_ch[kChX], g.d_x64, cells, s);
    else cudaMemsetAsync(g.d_x64, 0, cells * sizeof(double), s);
    launch::norm64(g, nullptr, g.d_bsave, g.d_norm, s);
    const double bb = read_norm(g, s);
    r->iters = 0;
    r->outer = 0;
    if (bb == 0.0) {
        cudaMemsetAsync(g.d_ch[kChX], 0, cells * sizeof(float), s);
        r->rel = 0;
        r->true_rel = 0;
        r->status = 0;
        r->launches = g.launch_count - own0;
        return cudaStreamSynchronize(s) == cudaSuccess ? 0 : 2;
    }
    double rel = 1.0;
    r->status = 5;
    for (int k = 0; k <= p.max_outer; k++) {
        launch::full_laplacian<double>(g, g.d_x64, g.d_ax64, nullptr, s);
        launch::residual64(g, g.d_bsave, g.d_ax64, g.d_r64, g.d_ch[kChB], s);
        launch::norm64(g, g.d_r64, nullptr, g.d_norm, s);
        rel = std::sqrt(read_norm(g, s) / bb);
        if (!(rel == rel)) { r->status = 6; break; }
        if (rel < p.tol) { r->status = 0; break; }
        if (k == p.max_outer) break;
        // each inner FP32 solve targets the defect that leaves the outer residual just under
        // tol, but never tighter than inner_tol (where FP32 stalls) nor looser than 0.1
        SolveParams ip = p;
        ip.precision = 0;
        double tau = 0.5 * p.tol / rel;
        tau = std::min(0.1, std::max(p.inner_tol, tau));
        ip.tol = tau;
        SolveResult ir;
        const long long a = g.launch_count;
        int e = pcg_solve(g, ip, s, &ir);
        if (e) return e;
        inner_recorded += g.launch_count - a;
        inner_executed += ir.launches;
        r->iters += ir.iters;
        r->outer++;
        launch::accumulate_correction(g, g.d_x64, g.d_ch[kChX], s);
    }
    launch::narrow(g, g.d_x64, g.d_ch[kChX], cells, s);
    g.x64_valid = true;
    r->launches = (g.launch_count - own0 - inner_recorded) + inner_executed;
    g.last_solve_launches = r->launches;
    // b channel ends as the last FP32 defect, mirroring "b channel will be modified"
    r->rel = rel;
    r->true_rel = rel;
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
