// solvers.cu -- chosen-form solver drivers: Sinkhorn (SinkhornKernel.jl:477-559),
// LAMP (MirrorProxKernel.jl:1019-1132) and annealed Sinkhorn (AnnealedSinkhorn.jl:65-177).
//
// A solve is one CUDA graph: a conditional WHILE node whose body holds U
// unrolled iterations (each a fixed sequence of pair passes) followed by a
// one-thread control kernel that keeps the loop running while ctl->stop == 0.
// Iteration counting, the check cadence, the tolerance test, itermax and tmax
// all live in the passes' device-side "finish" steps, so the host launches the
// graph once and synchronises once per solve (the reference synchronises after
// every launch, SinkhornKernel.jl:525 / MirrorProxKernel.jl:1049-1117).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <functional>
#include <vector>

#include "internal.h"
#include "small_kernels.cuh"

using namespace culamp_host;
using namespace culamp_dev;

#define CUDA_TRY(h, expr)                                                                       \
    do {                                                                                        \
        cudaError_t _e = (expr);                                                                \
        if (_e != cudaSuccess)                                                                  \
            return culamp_set_error((h), CULAMP_ERR_CUDA, "%s: %s (%s:%d)", #expr,             \
                                    cudaGetErrorString(_e), __FILE__, __LINE__);                \
    } while (0)

int culamp_plain_sinkhorn(culamp_handle h, const double *x, const double *y, int64_t n, int64_t m,
                          int32_t d, const double *r, const double *c, const culamp_args *args,
                          int64_t frequency, double p, const double *phi0, const double *psi0,
                          uint32_t flags, double *phi, double *psi, culamp_stats *stats,
                          culamp_log_row *log, int64_t log_cap, cudaStream_t st);
int culamp_plain_lamp(culamp_handle h, const double *x, const double *y, int64_t n, int64_t m,
                      int32_t d, const double *r, const double *c, const culamp_args *args,
                      int64_t frequency, double p, uint32_t flags, double *nu, double *phi,
                      double *psi, double *theta, culamp_stats *stats, culamp_log_row *log,
                      int64_t log_cap, cudaStream_t st);

namespace culamp_dev {

__global__ void set_start_kernel(Ctl *c) { c->t_start_ns = globaltimer_ns(); }

// Loop control of the WHILE node. Besides the finish steps' own itermax / tmax
// handling, the loop is bounded here independently: by the number of body
// executions (each body runs >= 1 iteration) and by tmax, so it always ends.
__global__ void loop_ctl_kernel(Ctl *c, cudaGraphConditionalHandle hnd) {
    c->loops += 1;
    if (!c->stop && (c->iter > c->itermax + 1 || c->loops > c->itermax + 2)) {
        c->stop = 1; c->stop_reason = 2; c->error = 1;
    }
    if (!c->stop && (double)(globaltimer_ns() - c->t_start_ns) * 1e-9 > c->tmax_s) {
        c->stop = 1; c->stop_reason = 3;
    }
    cudaGraphSetConditional(hnd, c->stop ? 0u : 1u);
}

}  // namespace culamp_dev

enum SolverKind { KIND_SK = 1, KIND_LAMP = 2, KIND_SYM = 3 };

// Everything a captured graph bakes into kernel parameters.
struct GraphKey {
    int kind = 0, n = 0, m = 0, d = 0, pm_iter = 0, pm_resid = 0, unroll = 0, feat = 0;
    int form = 0;         // 0 FP64 exponent, 1 FP32 exponent, 2 precision ladder
    long long freq = 0;   // check cadence the body is aligned to (0: gated checks)
    double p = 0, winf = 0, B = 0, eta_mu = 0;
    long long generation = -1;
    bool operator==(const GraphKey &o) const {
        return kind == o.kind && n == o.n && m == o.m && d == o.d && pm_iter == o.pm_iter && feat == o.feat &&
               form == o.form &&
               freq == o.freq &&
               pm_resid == o.pm_resid && unroll == o.unroll && generation == o.generation &&
               std::memcmp(&p, &o.p, sizeof(double)) == 0 && std::memcmp(&winf, &o.winf, sizeof(double)) == 0 &&
               std::memcmp(&B, &o.B, sizeof(double)) == 0 && std::memcmp(&eta_mu, &o.eta_mu, sizeof(double)) == 0;
    }
};

struct culamp_handle_s::Solver {
    int n = 0, m = 0, d = 0;
    long long generation = 0;
    DevBuf X, Y, r, c, phi, psi, res, cost, logz, aux, nu, nub, theta, thetab, eta_mu, tmp, ctl,
        logbuf, setup, ws_phi, ws_psi, prev_phi, prev_psi;
    DevBuf pers;               // persistent loop: per-CTA partials + grid barrier
    DevBuf hx, hy;             // host-variant staging (device side)
    // feature-cost path: both clouds as bf16 pieces in the MMA tile image + norms
    DevBuf fx, fy, fxn, fyn;
    int feat_np = 0;           // pieces reserved for (0: feature path off)
    int feat_kb = 0;           // K blocks of the packed clouds
    bool feat_active = false;  // the staged inputs are packed and the path is on
    Scratch scr;
    cudaStream_t cap_stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    struct Cached { GraphKey key; cudaGraphExec_t exec = nullptr; };
    std::vector<Cached> graphs;
    bool graph_pdl_failed = false;   // conditional bodies did not take programmatic edges

    void drop_graphs() {
        for (auto &g : graphs)
            if (g.exec) cudaGraphExecDestroy(g.exec);
        graphs.clear();
    }
    void release() {
        drop_graphs();
        DevBuf *all[] = {&X, &Y, &r, &c, &phi, &psi, &res, &cost, &logz, &aux, &nu, &nub, &theta,
                         &thetab, &eta_mu, &tmp, &ctl, &logbuf, &setup, &ws_phi, &ws_psi,
                         &prev_phi, &prev_psi, &pers, &hx, &hy, &fx, &fy, &fxn, &fyn};
        for (DevBuf *b : all) b->release();
        scr.release();
        if (cap_stream) cudaStreamDestroy(cap_stream);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        cap_stream = nullptr;
        ev0 = ev1 = nullptr;
    }
};

void culamp_solver_release(culamp_handle h) {
    if (h && h->solver) {
        h->solver->release();
        delete h->solver;
        h->solver = nullptr;
    }
}

namespace {

using Solver = culamp_handle_s::Solver;

// bf16 pieces per feature value for these inputs and flags (0: pair loops).
int feat_pieces(int d, uint32_t flags) {
    if (d < FEAT_MIN_D || (flags & CULAMP_FLAG_FEAT_FP64)) return 0;
    return (flags & CULAMP_FLAG_FEAT_X6) ? 3 : 2;
}

int ensure_solver(culamp_handle h, int n, int m, int d, int64_t log_cap, int feat_np = 0) {
    if (!h->solver) {
        h->solver = new (std::nothrow) Solver();
        if (!h->solver) return culamp_set_error(h, CULAMP_ERR_ALLOC, "solver state");
        if (cudaStreamCreateWithFlags(&h->solver->cap_stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreate(&h->solver->ev0) != cudaSuccess || cudaEventCreate(&h->solver->ev1) != cudaSuccess)
            return culamp_set_error(h, CULAMP_ERR_CUDA, "stream/event creation failed");
    }
    Solver &S = *h->solver;
    // + 2: the persistent loops copy column potentials in aligned pairs, which
    // may reach one element past the last column
    const size_t nm = (size_t)(n > m ? n : m) + 2;
    auto ptrs = [&S]() {
        return std::vector<void *>{S.X.ptr, S.Y.ptr, S.r.ptr, S.c.ptr, S.phi.ptr, S.psi.ptr,
                                   S.res.ptr, S.cost.ptr, S.logz.ptr, S.aux.ptr, S.nu.ptr,
                                   S.nub.ptr, S.theta.ptr, S.thetab.ptr, S.eta_mu.ptr, S.tmp.ptr,
                                   S.ctl.ptr, S.logbuf.ptr, S.scr.part.ptr, S.scr.tickets.ptr,
                                   S.scr.blk.ptr, S.fx.ptr, S.fy.ptr, S.fxn.ptr, S.fyn.ptr};
    };
    const std::vector<void *> before = ptrs();
    cudaError_t e = cudaSuccess;
    auto R = [&](DevBuf &b, size_t bytes, bool zero = false) {
        if (e == cudaSuccess) e = b.reserve(bytes, zero);
    };
    R(S.X, (size_t)n * d * sizeof(double));
    R(S.Y, (size_t)m * d * sizeof(double));
    R(S.r, nm * sizeof(double));
    R(S.c, nm * sizeof(double));
    R(S.phi, nm * sizeof(double));
    R(S.psi, nm * sizeof(double));
    R(S.res, nm * sizeof(double));
    R(S.cost, nm * sizeof(double));
    R(S.logz, nm * sizeof(double));
    R(S.aux, nm * sizeof(double));
    R(S.nu, nm * sizeof(double));
    R(S.nub, nm * sizeof(double));
    R(S.theta, nm * sizeof(double));
    R(S.thetab, nm * sizeof(double));
    R(S.eta_mu, nm * sizeof(double));
    R(S.tmp, nm * sizeof(double));
    R(S.ws_phi, nm * sizeof(double));
    R(S.ws_psi, nm * sizeof(double));
    R(S.prev_phi, nm * sizeof(double));
    R(S.prev_psi, nm * sizeof(double));
    R(S.ctl, sizeof(Ctl), true);
    R(S.setup, (8 + 2 * MAXD) * sizeof(double));
    R(S.logbuf, (size_t)(log_cap > 1 ? log_cap : 1) * sizeof(culamp_log_row));
    if (feat_np > 0) {
        R(S.fx, feat_piece_elems(n, d, feat_np) * sizeof(uint16_t));
        R(S.fy, feat_piece_elems(m, d, feat_np) * sizeof(uint16_t));
        R(S.fxn, (size_t)n * sizeof(double));
        R(S.fyn, (size_t)m * sizeof(double));
    }
    S.feat_np = feat_np;
    S.feat_active = false;
    // scratch for both pass orientations
    size_t pb = 0, nrb = 0;
    for (int mom = 0; mom < 2; ++mom)
        for (const LaunchShape &sh : {pass_shape(n, m, d, ACC_LSE, h->sm_count, mom),
                                      pass_shape(m, n, d, ACC_LSE, h->sm_count, mom),
                                      pass_shape(n, m, d, ACC_MAX, h->sm_count)}) {
            pb = sh.part_bytes > pb ? sh.part_bytes : pb;
            nrb = (size_t)sh.rb > nrb ? (size_t)sh.rb : nrb;
        }
    if (feat_np > 0)
        for (const FeatShape &fs : {feat_shape(n, m, h->sm_count, feat_np), feat_shape(m, n, h->sm_count, feat_np)}) {
            pb = fs.part_bytes > pb ? fs.part_bytes : pb;
            nrb = (size_t)fs.merge_rb > nrb ? (size_t)fs.merge_rb : nrb;
        }
    if (e == cudaSuccess) e = S.scr.reserve(pb, nrb);
    if (e != cudaSuccess) return culamp_set_error(h, CULAMP_ERR_ALLOC, "workspace: %s", cudaGetErrorString(e));
    if (before != ptrs()) {   // any pointer baked into a cached graph moved
        S.generation++;
        S.drop_graphs();
    }
    S.n = n;
    S.m = m;
    S.d = d;
    return CULAMP_OK;
}

// Iterations per graph body: about 200 us of work per body.
int pick_unroll(double pairs_per_iter) {
    const double t_us = pairs_per_iter / 1.0e6 + 6.0;   // ~1e12 pairs/s + launch gaps
    int u = (int)std::ceil(200.0 / t_us);
    if (u < 1) u = 1;
    if (u > 16) u = 16;
    return u;
}

// Build a WHILE graph whose body runs `body` `unroll` times.
cudaError_t build_while_graph(Solver &S, const GraphKey &key,
                              const std::function<cudaError_t(cudaStream_t)> &body, cudaGraphExec_t *out) {
    *out = nullptr;
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaGraphCreate(&g, 0);
    if (e != cudaSuccess) return e;
    cudaGraphConditionalHandle ch;
    e = cudaGraphConditionalHandleCreate(&ch, g, 1, cudaGraphCondAssignDefault);
    cudaGraphNodeParams np = {};
    cudaGraphNode_t node;
    if (e == cudaSuccess) {
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = ch;
        np.conditional.type = cudaGraphCondTypeWhile;
        np.conditional.size = 1;
        e = cudaGraphAddNode(&node, g, nullptr, 0, &np);
    }
    if (e == cudaSuccess) {
        cudaGraph_t bodyg = np.conditional.phGraph_out[0];
        e = cudaStreamBeginCaptureToGraph(S.cap_stream, bodyg, nullptr, nullptr, 0,
                                          cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            cudaError_t eb = cudaSuccess;
            for (int u = 0; u < key.unroll && eb == cudaSuccess; ++u) eb = body(S.cap_stream);
            if (eb == cudaSuccess) {
                loop_ctl_kernel<<<1, 1, 0, S.cap_stream>>>(S.ctl.as<Ctl>(), ch);
                eb = cudaGetLastError();
            }
            cudaGraph_t captured = nullptr;
            e = cudaStreamEndCapture(S.cap_stream, &captured);
            if (eb != cudaSuccess) e = eb;
            if (e != cudaSuccess && captured && captured != bodyg) cudaGraphDestroy(captured);
        }
    }
    cudaGraphExec_t exec = nullptr;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, g, 0);
    cudaGraphDestroy(g);
    *out = exec;
    return e;
}

// Build (or fetch) the WHILE graph of `key`. The passes are recorded with
// programmatic dependent launches; if the driver cannot keep those edges in a
// conditional body, the graph is recorded again with plain launches.
int get_graph(culamp_handle h, const GraphKey &key, const std::function<cudaError_t(cudaStream_t)> &body,
              cudaGraphExec_t *out, const std::function<void()> &reset = nullptr) {
    Solver &S = *h->solver;
    for (auto &g : S.graphs)
        if (g.key == key) { *out = g.exec; return CULAMP_OK; }
    cudaGraphExec_t exec = nullptr;
    cudaError_t e = cudaErrorNotSupported;
    if (!S.graph_pdl_failed) {
        if (reset) reset();
        e = build_while_graph(S, key, body, &exec);
        if (e != cudaSuccess) {
            cudaGetLastError();
            S.graph_pdl_failed = true;
        }
    }
    if (e != cudaSuccess) {
        PdlOff plain;
        if (reset) reset();
        e = build_while_graph(S, key, body, &exec);
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        return culamp_set_error(h, CULAMP_ERR_CUDA, "graph build: %s", cudaGetErrorString(e));
    }
    if (S.graphs.size() > 8) S.drop_graphs();
    S.graphs.push_back({key, exec});
    *out = exec;
    return CULAMP_OK;
}

int check_solver_args(culamp_handle h, const double *x, const double *y, int64_t n, int64_t m,
                      int32_t d, const double *r, const double *c, const culamp_args *args,
                      int64_t frequency, double p) {
    if (!h) return CULAMP_ERR_INVALID_ARG;
    if (!x || !y || !r || !c || !args)
        return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "null pointer argument");
    if (n < 1 || m < 1 || n > (1LL << 28) || m > (1LL << 28))
        return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "sizes out of range (n=%lld, m=%lld)",
                                (long long)n, (long long)m);
    if (d < 1 || d > MAXD)
        return culamp_set_error(h, d < 1 ? CULAMP_ERR_INVALID_ARG : CULAMP_ERR_UNSUPPORTED,
                                "d=%d outside [1, %d]", d, MAXD);
    if (!(p > 0.0)) return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "p must be > 0");
    if (frequency < 1) return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "frequency must be >= 1");
    if (args->itermax < 0) return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "itermax < 0");
    cudaSetDevice(h->device);
    return CULAMP_OK;
}

// Copy user inputs into the workspace and validate the marginals (positive,
// finite). Coordinates that are the same for every point of both clouds add
// exactly 0 to every cost (for p = 1, 2, Inf and any p > 0), so those
// dimensions are dropped: *d_eff receives the kept dimension count (>= 1).
int stage_inputs(culamp_handle h, const double *x, const double *y, int n, int m, int d,
                 const double *r, const double *c, cudaStream_t st, double *hr_out, int *d_eff) {
    Solver &S = *h->solver;
    CUDA_TRY(h, cudaMemcpyAsync(S.r.ptr, r, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    CUDA_TRY(h, cudaMemcpyAsync(S.c.ptr, c, (size_t)m * sizeof(double), cudaMemcpyDeviceToDevice, st));
    double *su = S.setup.as<double>();
    setup_reduce_kernel<<<1, 256, 0, st>>>(su, S.r.as<double>(), n);
    setup_reduce_kernel<<<1, 256, 0, st>>>(su + 3, S.c.as<double>(), m);
    dim_range_kernel<<<d, 256, 0, st>>>(su + 8, x, n, y, m, d);
    CUDA_TRY(h, cudaGetLastError());
    double hv[8 + 2 * MAXD];
    CUDA_TRY(h, cudaMemcpyAsync(hv, su, (8 + 2 * (size_t)d) * sizeof(double), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(h, cudaStreamSynchronize(st));
    if (!(hv[1] > 0.0) || !(hv[4] > 0.0) || !std::isfinite(hv[2]) || !std::isfinite(hv[5]))
        return culamp_set_error(h, CULAMP_ERR_INVALID_ARG,
                                "marginals must be positive and finite (min r=%g, min c=%g)", hv[1], hv[4]);
    DimKeep keep;
    int dk = 0;
    for (int k = 0; k < d; ++k) {
        const double lo = hv[8 + 2 * k], hi = hv[8 + 2 * k + 1];
        if (!std::isfinite(lo) || !std::isfinite(hi))
            return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "non-finite coordinate in dimension %d", k);
        if (hi > lo) keep.idx[dk++] = k;
    }
    if (dk == 0) keep.idx[dk++] = 0;
    if (dk == d) {
        CUDA_TRY(h, cudaMemcpyAsync(S.X.ptr, x, (size_t)n * d * sizeof(double), cudaMemcpyDeviceToDevice, st));
        CUDA_TRY(h, cudaMemcpyAsync(S.Y.ptr, y, (size_t)m * d * sizeof(double), cudaMemcpyDeviceToDevice, st));
    } else {
        gather_dims_kernel<<<(unsigned)(((long long)n * dk + 255) / 256), 256, 0, st>>>(S.X.as<double>(), x, n, d, dk, keep);
        gather_dims_kernel<<<(unsigned)(((long long)m * dk + 255) / 256), 256, 0, st>>>(S.Y.as<double>(), y, m, d, dk, keep);
        CUDA_TRY(h, cudaGetLastError());
    }
    if (hr_out) *hr_out = hv[0];
    *d_eff = dk;
    return CULAMP_OK;
}

// Pack the staged clouds for the tensor-core path when it was reserved and the
// kept dimension count still qualifies.
int prepare_features(culamp_handle h, int n, int m, int d_eff, cudaStream_t st) {
    Solver &S = *h->solver;
    S.feat_active = false;
    if (S.feat_np <= 0 || d_eff < FEAT_MIN_D) return CULAMP_OK;
    CUDA_TRY(h, feat_prepare(S.fx.as<uint16_t>(), S.fxn.as<double>(), S.X.as<double>(), n, d_eff, S.feat_np, st));
    CUDA_TRY(h, feat_prepare(S.fy.as<uint16_t>(), S.fyn.as<double>(), S.Y.as<double>(), m, d_eff, S.feat_np, st));
    S.feat_kb = feat_kblocks(d_eff);
    S.feat_active = true;
    return CULAMP_OK;
}

// Route a squared-Euclidean pass to the tensor-core feature path.
void apply_feat(const Solver &S, PassParams &P, bool rows_are_x) {
    if (!S.feat_active || pmode_of(P.pexp) != P_SQ) return;
    P.fx = rows_are_x ? S.fx.as<uint16_t>() : S.fy.as<uint16_t>();
    P.fy = rows_are_x ? S.fy.as<uint16_t>() : S.fx.as<uint16_t>();
    P.xn = rows_are_x ? S.fxn.as<double>() : S.fyn.as<double>();
    P.yn = rows_are_x ? S.fyn.as<double>() : S.fxn.as<double>();
    P.fkb = S.feat_kb;
    P.fpieces = S.feat_np;
}

PassParams mk(const double *X, const double *Y, int n, int m, int d, double p, Ctl *ctl) {
    PassParams P;
    std::memset(&P, 0, sizeof(P));
    P.X = X;
    P.Y = Y;
    P.n = n;
    P.m = m;
    P.d = d;
    P.pexp = p;
    P.ctl = ctl;
    return P;
}

// W_inf = max_ij C_ij with the solver's true p (MirrorProxKernel.jl:280-326).
int compute_winf(culamp_handle h, int n, int m, int d, double p, cudaStream_t st, double *winf) {
    Solver &S = *h->solver;
    double *dst = &h->pass_ctl.as<Ctl>()->winf;
    CUDA_TRY(h, cudaMemsetAsync(dst, 0, sizeof(double), st));
    CUDA_TRY(h, launch_max_cost(S.X.as<double>(), S.Y.as<double>(), n, m, d, p, dst, h->sm_count, st));
    CUDA_TRY(h, cudaMemcpyAsync(winf, dst, sizeof(double), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(h, cudaStreamSynchronize(st));
    return CULAMP_OK;
}

void fill_stats_common(culamp_stats *stats, const Ctl &c, float ms) {
    stats->iterations = c.iter;
    stats->num_iter = c.num_iter;
    stats->stopped = c.stop_reason;
    stats->elapsed_ms = ms;
    stats->log_rows = c.log_rows;
    stats->status = c.error ? CULAMP_ERR_DEVICE_TIMEOUT : CULAMP_OK;
}

int copy_log(culamp_handle h, const Ctl &c, culamp_log_row *log, int64_t log_cap, cudaStream_t st) {
    if (!log || log_cap <= 0 || c.log_rows <= 0) return CULAMP_OK;
    const long long rows = c.log_rows < log_cap ? c.log_rows : log_cap;
    CUDA_TRY(h, cudaMemcpyAsync(log, h->solver->logbuf.ptr, (size_t)rows * sizeof(culamp_log_row),
                                cudaMemcpyDeviceToHost, st));
    CUDA_TRY(h, cudaStreamSynchronize(st));
    return CULAMP_OK;
}

// ------------------------------------------------------------------ Sinkhorn

struct SkPlan {
    PassParams k1, k2, k3;
    PassParams k1f, k2f;   // precision ladder: the FP32-exponent row / column passes
    bool ladder = false;
    int pm_iter, pm_resid;
    LaunchShape s_rows, s_cols, s_rows_mom;
};

// Sinkhorn solves of at least this many pairs take the precision ladder unless
// CULAMP_FLAG_FORM_FP64 is set. Below it the default stays the FP64-exponent
// form, whose iterates follow the reference's step for step; the ladder there
// is CULAMP_FLAG_LADDER (in the persistent loop, where switching form costs
// nothing). At 4096^2 the graph-loop ladder took 86.7 ms against 83.9 ms in
// FP64, at 65536^2 2.87 s against 4.11 s (same 1e-6 FP64 check).
constexpr double LADDER_AUTO_PAIRS = 268435456.0;   // 16384^2

// The FP32-exponent forms (FORM_FP32, LADDER) exist for the packed p = 2 passes.
bool fp32_form_applies(const Solver &S, int d, int pm_iter) {
    return pm_iter == P_SQ && d <= MAXD_PACKED && !S.feat_active;
}

SkPlan make_sk_plan(culamp_handle h, int n, int m, int d, double p, uint32_t flags) {
    Solver &S = *h->solver;
    Ctl *ctl = S.ctl.as<Ctl>();
    SkPlan pl;
    const bool true_pinf = flags & CULAMP_FLAG_TRUE_PINF;
    // SinkhornKernel.jl:518-523 (iteration cost), :38-42 (residual cost)
    const double p_iter = (std::isinf(p) && !true_pinf) ? 2.0 : p;
    const double p_res = true_pinf ? p : (p == 1.0 ? 1.0 : 2.0);
    pl.pm_iter = pmode_of(p_iter);
    pl.pm_resid = pmode_of(p_res);
    double *X = S.X.as<double>(), *Y = S.Y.as<double>();
    // K1: phi = log r - LSE_j(-C/(eta W) + psi)
    pl.k1 = mk(X, Y, n, m, d, p_iter, ctl);
    pl.k1.ctr = X;
    pl.k1.epi = EPI_SK_ROW;
    pl.k1.coef_mode = COEF_SK;
    pl.k1.colpot = S.psi.as<double>();
    pl.k1.marg = S.r.as<double>();
    pl.k1.out = S.phi.as<double>();
    pl.k1.use_ref = 1;
    // K2: psi = log c - LSE_i(-C/(eta W) + phi); iteration bookkeeping
    pl.k2 = mk(Y, X, m, n, d, p_iter, ctl);
    pl.k2.ctr = X;
    pl.k2.epi = EPI_SK_ROW;
    pl.k2.coef_mode = COEF_SK;
    pl.k2.colpot = S.phi.as<double>();
    pl.k2.marg = S.c.as<double>();
    pl.k2.out = S.psi.as<double>();
    pl.k2.use_ref = 1;
    pl.k2.finish = FIN_SK_ITER;
    // K3 (check iterations): row residual + transport cost, tolerance test
    pl.k3 = mk(X, Y, n, m, d, p_res, ctl);
    pl.k3.ctr = X;
    pl.k3.epi = EPI_SK_RESID;
    pl.k3.coef_mode = COEF_SK;
    pl.k3.colpot = S.psi.as<double>();
    pl.k3.rowpot = S.phi.as<double>();
    pl.k3.marg = S.r.as<double>();
    pl.k3.out = S.res.as<double>();
    pl.k3.out2 = S.cost.as<double>();
    pl.k3.want_moment = 1;
    pl.k3.gate = GATE_CHECK;
    pl.k3.finish = FIN_SK_CHECK;
    apply_feat(S, pl.k1, true);
    apply_feat(S, pl.k2, false);
    apply_feat(S, pl.k3, true);
    if (fp32_form_applies(S, d, pl.pm_iter)) {
        if (flags & CULAMP_FLAG_FORM_FP32) {
            pl.k1.fp32 = 1;
            pl.k2.fp32 = 1;
        } else if ((flags & CULAMP_FLAG_LADDER) ||
                   (!(flags & CULAMP_FLAG_FORM_FP64) && (double)n * (double)m >= LADDER_AUTO_PAIRS)) {
            // FP32-exponent passes while ctl->fp32_phase holds, FP64 ones after
            pl.ladder = true;
            pl.k1f = pl.k1;
            pl.k2f = pl.k2;
            pl.k1f.fp32 = pl.k2f.fp32 = 1;
            pl.k1f.phase = pl.k2f.phase = PHASE_FP32;
            pl.k1.phase = pl.k2.phase = PHASE_FP64;
        }
    }
    pl.s_rows = pass_shape(n, m, d, ACC_LSE, h->sm_count);
    pl.s_cols = pass_shape(m, n, d, ACC_LSE, h->sm_count);
    pl.s_rows_mom = pass_shape(n, m, d, ACC_LSE, h->sm_count, true);
    return pl;
}

// Runs the Sinkhorn loop on the workspace (phi/psi hold the starting point).
int sinkhorn_loop(culamp_handle h, int n, int m, int d, double p, double eta, double winf,
                  const culamp_args *args, int64_t frequency, uint32_t flags, int64_t log_cap,
                  cudaStream_t st, Ctl *out_ctl, float *ms) {
    Solver &S = *h->solver;
    Ctl c;
    std::memset(&c, 0, sizeof(c));
    c.itermax = args->itermax;
    c.frequency = frequency;
    c.stop = args->itermax < 1;
    c.stop_reason = args->itermax < 1 ? 2 : 0;
    c.tmax_s = args->tmax;
    c.epsilon = args->epsilon;
    c.eta = eta;
    c.winf = winf;
    c.log = S.logbuf.as<culamp_log_row>();
    c.log_cap = log_cap;
    SkPlan pl = make_sk_plan(h, n, m, d, p, flags);
    // precision ladder: FP32-exponent iterations until a check's L1 residual is
    // within LADDER_FACTOR of the stopping threshold, then the FP64 form
    constexpr double LADDER_FACTOR = 32.0;
    c.fp32_phase = pl.ladder ? 1 : 0;
    c.ladder_switch = LADDER_FACTOR * args->epsilon / 6.0;
    c.ladder_prev = INFINITY;
    CUDA_TRY(h, cudaMemcpyAsync(S.ctl.ptr, &c, sizeof(Ctl), cudaMemcpyHostToDevice, st));
    set_start_kernel<<<1, 1, 0, st>>>(S.ctl.as<Ctl>());
    // Graph bodies hold whole multiples of `frequency` iterations when the
    // cadence is short: every body then starts at a check iteration
    // ((it - 1) % frequency == 0, SinkhornKernel.jl:527), so the residual pass
    // is recorded only where it runs instead of as a gated launch per iteration.
    const int base_unroll = pick_unroll((double)n * m * (frequency == 1 ? 3.0 : 2.0));
    const bool aligned = frequency <= 32;
    const int unroll = aligned ? (int)frequency * std::max(1, (int)std::lround((double)base_unroll / frequency))
                               : base_unroll;
    auto iteration = [&](cudaStream_t s, bool with_check) -> cudaError_t {
        cudaError_t e = cudaSuccess;
        if (pl.ladder) e = launch_pass(pl.k1f, pl.pm_iter, ACC_LSE, pl.s_rows, S.scr, s);
        if (e == cudaSuccess) e = launch_pass(pl.k1, pl.pm_iter, ACC_LSE, pl.s_rows, S.scr, s);
        if (e == cudaSuccess && pl.ladder) e = launch_pass(pl.k2f, pl.pm_iter, ACC_LSE, pl.s_cols, S.scr, s);
        if (e == cudaSuccess) e = launch_pass(pl.k2, pl.pm_iter, ACC_LSE, pl.s_cols, S.scr, s);
        if (e == cudaSuccess && with_check) e = launch_pass(pl.k3, pl.pm_resid, ACC_LSE, pl.s_rows_mom, S.scr, s);
        return e;
    };
    int body_pos = 0;   // iteration index inside the graph body being recorded
    auto body = [&](cudaStream_t s) -> cudaError_t {
        const bool with_check = !aligned || (body_pos % frequency) == 0;
        body_pos = (body_pos + 1) % unroll;
        return iteration(s, with_check);
    };
    const bool persist = !(flags & (CULAMP_FLAG_NO_GRAPH | CULAMP_FLAG_NO_PERSIST)) && !pl.k1.fp32 &&
                         !S.feat_active && d <= MAXD_PACKED;
    int pgrid = persist ? persist_grid(h->sm_count, d, pl.pm_iter) : 0;
    if (pgrid > 0 && !persist_eligible(n, m, d, pl.pm_iter, pl.pm_resid, pgrid)) pgrid = 0;
    if (pgrid > 0) CUDA_TRY(h, S.pers.reserve(persist_scratch_bytes(pgrid)));
    CUDA_TRY(h, cudaEventRecord(S.ev0, st));
    bool ran = false;
    if (pgrid > 0) {
        // the whole loop in one cooperative launch; a refused launch (e.g. the
        // CTAs cannot all be resident) falls back to the graph loop
        const cudaError_t e = launch_sk_persist(S.X.as<double>(), S.Y.as<double>(), S.r.as<double>(),
                                                S.c.as<double>(), S.phi.as<double>(), S.psi.as<double>(), n, m,
                                                d, pl.pm_iter, pl.k1.pexp, S.ctl.as<Ctl>(), S.pers.ptr, pgrid, st);
        if (e == cudaSuccess) ran = true;
        else cudaGetLastError();
    }
    if (ran) {
    } else if (flags & CULAMP_FLAG_NO_GRAPH) {
        // host-driven loop: check the stop flag after every iteration
        for (long long it = 0; it < args->itermax + 2; ++it) {
            CUDA_TRY(h, iteration(st, true));
            int stop = 0;
            CUDA_TRY(h, cudaMemcpyAsync(&stop, &S.ctl.as<Ctl>()->stop, sizeof(int), cudaMemcpyDeviceToHost, st));
            CUDA_TRY(h, cudaStreamSynchronize(st));
            if (stop) break;
        }
    } else {
        GraphKey key;
        key.kind = KIND_SK;
        key.n = n; key.m = m; key.d = d;
        key.pm_iter = pl.pm_iter; key.pm_resid = pl.pm_resid;
        key.p = p;
        key.feat = S.feat_active ? S.feat_np : 0;
        key.unroll = unroll;
        key.freq = aligned ? frequency : 0;
        key.generation = S.generation;
        key.form = pl.ladder ? 2 : (pl.k1.fp32 ? 1 : 0);
        cudaGraphExec_t ex = nullptr;
        int s = get_graph(h, key, body, &ex, [&body_pos]() { body_pos = 0; });
        if (s) return s;
        CUDA_TRY(h, cudaGraphLaunch(ex, st));
    }
    CUDA_TRY(h, cudaEventRecord(S.ev1, st));
    CUDA_TRY(h, cudaMemcpyAsync(out_ctl, S.ctl.ptr, sizeof(Ctl), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(h, cudaStreamSynchronize(st));
    CUDA_TRY(h, cudaEventElapsedTime(ms, S.ev0, S.ev1));
    if (out_ctl->error) return culamp_set_error(h, CULAMP_ERR_DEVICE_TIMEOUT, "loop control bound hit");
    return CULAMP_OK;
}

// Final residual_opt! pass (SinkhornKernel.jl:541-544): residual L1 and transport cost.
int sinkhorn_final(culamp_handle h, int n, int m, int d, double p, double eta, double winf,
                   uint32_t flags, cudaStream_t st, double *resid, double *obj) {
    Solver &S = *h->solver;
    SkPlan pl = make_sk_plan(h, n, m, d, p, flags);
    PassParams P = pl.k3;
    P.ctl = h->pass_ctl.as<Ctl>();
    P.gate = GATE_ALWAYS;
    P.coef_mode = COEF_FIXED;
    P.alpha = -1.0 / (eta * winf);
    P.beta = 1.0;
    P.finish = FIN_SUMS;
    CUDA_TRY(h, launch_pass(P, pl.pm_resid, ACC_LSE, pl.s_rows_mom, S.scr, st));
    double sums[4];
    CUDA_TRY(h, cudaMemcpyAsync(sums, h->pass_ctl.as<Ctl>()->sums, sizeof(sums), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(h, cudaStreamSynchronize(st));
    *resid = sums[0];
    *obj = sums[1];
    return CULAMP_OK;
}

}  // namespace

extern "C" int culamp_sinkhorn(culamp_handle h, const double *x, const double *y, int64_t n,
                               int64_t m, int32_t d, const double *r, const double *c,
                               const culamp_args *args, int64_t frequency, double p,
                               const double *phi0, const double *psi0, uint32_t flags,
                               double *phi, double *psi, culamp_stats *stats, culamp_log_row *log,
                               int64_t log_cap, void *stream) {
    int s = check_solver_args(h, x, y, n, m, d, r, c, args, frequency, p);
    if (s) return s;
    if (!phi || !psi) return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "null output pointer");
    if (!(args->eta_p > 0.0))
        return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "Sinkhorn needs eta_p > 0 (got %g)", args->eta_p);
    cudaStream_t st = (cudaStream_t)stream;
    if (flags & CULAMP_FLAG_FORM_PLAIN)
        return culamp_plain_sinkhorn(h, x, y, n, m, d, r, c, args, frequency, p, phi0, psi0, flags,
                                     phi, psi, stats, log, log_cap, st);
    s = ensure_solver(h, (int)n, (int)m, d, log ? log_cap : 0, feat_pieces(d, flags));
    if (s) return s;
    Solver &S = *h->solver;
    int dk = d;
    s = stage_inputs(h, x, y, (int)n, (int)m, d, r, c, st, nullptr, &dk);
    if (s) return s;
    d = dk;
    s = prepare_features(h, (int)n, (int)m, d, st);
    if (s) return s;
    if (phi0) CUDA_TRY(h, cudaMemcpyAsync(S.phi.ptr, phi0, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    else CUDA_TRY(h, cudaMemsetAsync(S.phi.ptr, 0, n * sizeof(double), st));
    if (psi0) CUDA_TRY(h, cudaMemcpyAsync(S.psi.ptr, psi0, m * sizeof(double), cudaMemcpyDeviceToDevice, st));
    else CUDA_TRY(h, cudaMemsetAsync(S.psi.ptr, 0, m * sizeof(double), st));
    double winf = 0.0;
    s = compute_winf(h, (int)n, (int)m, d, p, st, &winf);
    if (s) return s;
    Ctl hc;
    float ms = 0.f;
    s = sinkhorn_loop(h, (int)n, (int)m, d, p, args->eta_p, winf, args, frequency, flags,
                      log ? log_cap : 0, st, &hc, &ms);
    if (s) return s;
    double resid = 0, obj = 0;
    s = sinkhorn_final(h, (int)n, (int)m, d, p, args->eta_p, winf, flags, st, &resid, &obj);
    if (s) return s;
    CUDA_TRY(h, cudaMemcpyAsync(phi, S.phi.ptr, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    CUDA_TRY(h, cudaMemcpyAsync(psi, S.psi.ptr, m * sizeof(double), cudaMemcpyDeviceToDevice, st));
    s = copy_log(h, hc, log, log_cap, st);
    if (s) return s;
    CUDA_TRY(h, cudaStreamSynchronize(st));
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        fill_stats_common(stats, hc, ms);
        stats->residual = resid;
        stats->objective = obj;
        stats->winf = winf;
        stats->eta_t = NAN;
        stats->s_t = NAN;
    }
    return CULAMP_OK;
}

// -------------------------------------------------------- symmetric Sinkhorn

// Self-transport OT(a, a; x, x): the optimal plan is symmetric, so one
// potential f (P_ij = exp(f_i + f_j - C_ij/(eta_p W_inf))) solves it. Each
// iteration is ONE row pass, f <- (f + T(f))/2 with T(f) = log a - LSE_j(
// -C_ij/(eta_p W_inf) + f_j); its fixed point is the symmetric Sinkhorn
// solution and the averaged map converges in a few dozen passes where the
// alternating iteration needs hundreds. The same pass yields the L1 row
// residual at its input f, a_i |1 - exp(f_i - T(f)_i)| summed, so every
// iteration is checked. The two potential buffers alternate as input and output.
extern "C" int culamp_symmetric_sinkhorn(culamp_handle h, const double *x, int64_t n, int32_t d,
                                         const double *r, const culamp_args *args, int64_t frequency,
                                         double p, const double *f0, uint32_t flags, double *f,
                                         culamp_stats *stats, culamp_log_row *log, int64_t log_cap,
                                         void *stream) {
    int s = check_solver_args(h, x, x, n, n, d, r, r, args, frequency, p);
    if (s) return s;
    if (!f) return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "null output pointer");
    if (!(args->eta_p > 0.0))
        return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "Sinkhorn needs eta_p > 0 (got %g)", args->eta_p);
    if (flags & CULAMP_FLAG_FORM_PLAIN)
        return culamp_set_error(h, CULAMP_ERR_UNSUPPORTED, "symmetric solve has no plain form");
    cudaStream_t st = (cudaStream_t)stream;
    s = ensure_solver(h, (int)n, (int)n, d, log ? log_cap : 0, feat_pieces(d, flags));
    if (s) return s;
    Solver &S = *h->solver;
    int dk = d;
    s = stage_inputs(h, x, x, (int)n, (int)n, d, r, r, st, nullptr, &dk);
    if (s) return s;
    d = dk;
    s = prepare_features(h, (int)n, (int)n, d, st);
    if (s) return s;
    if (f0) CUDA_TRY(h, cudaMemcpyAsync(S.phi.ptr, f0, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    else CUDA_TRY(h, cudaMemsetAsync(S.phi.ptr, 0, n * sizeof(double), st));
    // all-ones bytes are a NaN: no fixed-reference hint before the first pass
    CUDA_TRY(h, cudaMemsetAsync(S.aux.ptr, 0xFF, n * sizeof(double), st));
    double winf = 0.0;
    s = compute_winf(h, (int)n, (int)n, d, p, st, &winf);
    if (s) return s;

    Ctl c;
    std::memset(&c, 0, sizeof(c));
    c.itermax = args->itermax;
    c.frequency = frequency;
    c.stop = args->itermax < 1;
    c.stop_reason = args->itermax < 1 ? 2 : 0;
    c.tmax_s = args->tmax;
    c.epsilon = args->epsilon;
    c.eta = args->eta_p;
    c.winf = winf;
    c.log = log ? S.logbuf.as<culamp_log_row>() : nullptr;
    c.log_cap = log ? log_cap : 0;
    CUDA_TRY(h, cudaMemcpyAsync(S.ctl.ptr, &c, sizeof(Ctl), cudaMemcpyHostToDevice, st));
    set_start_kernel<<<1, 1, 0, st>>>(S.ctl.as<Ctl>());

    const bool true_pinf = flags & CULAMP_FLAG_TRUE_PINF;
    const double p_iter = (std::isinf(p) && !true_pinf) ? 2.0 : p;   // as the Sinkhorn iteration
    const double p_res = true_pinf ? p : (p == 1.0 ? 1.0 : 2.0);      // as its residual pass
    const int pm = pmode_of(p_iter), pm_res = pmode_of(p_res);
    double *X = S.X.as<double>();
    PassParams pa = mk(X, X, (int)n, (int)n, d, p_iter, S.ctl.as<Ctl>());
    pa.ctr = X;
    pa.epi = EPI_SK_SYM;
    pa.coef_mode = COEF_SK;
    pa.marg = S.r.as<double>();
    pa.aux = S.aux.as<double>();
    pa.use_ref = 1;
    pa.finish = FIN_SK_SYM;
    apply_feat(S, pa, true);
    PassParams pb = pa;
    pa.colpot = pa.rowpot = S.phi.as<double>();
    pa.out = S.psi.as<double>();
    pb.colpot = pb.rowpot = S.psi.as<double>();
    pb.out = S.phi.as<double>();
    const LaunchShape sh = pass_shape((int)n, (int)n, d, ACC_LSE, h->sm_count);
    int unroll = pick_unroll((double)n * n);
    unroll += unroll & 1;   // every graph body starts on the phi -> psi pass
    int pos = 0;
    auto body = [&](cudaStream_t sx) -> cudaError_t {
        const PassParams &P = (pos & 1) ? pb : pa;
        pos += 1;
        return launch_pass(P, pm, ACC_LSE, sh, S.scr, sx);
    };
    CUDA_TRY(h, cudaEventRecord(S.ev0, st));
    if (flags & CULAMP_FLAG_NO_GRAPH) {
        for (long long it = 0; it < args->itermax + 2; ++it) {
            CUDA_TRY(h, body(st));
            int stop = 0;
            CUDA_TRY(h, cudaMemcpyAsync(&stop, &S.ctl.as<Ctl>()->stop, sizeof(int), cudaMemcpyDeviceToHost, st));
            CUDA_TRY(h, cudaStreamSynchronize(st));
            if (stop) break;
        }
    } else {
        GraphKey key;
        key.kind = KIND_SYM;
        key.n = key.m = (int)n;
        key.d = d;
        key.pm_iter = pm;
        key.p = p;
        key.feat = S.feat_active ? S.feat_np : 0;
        key.unroll = unroll;
        key.generation = S.generation;
        cudaGraphExec_t ex = nullptr;
        pos = 0;
        s = get_graph(h, key, body, &ex);
        if (s) return s;
        CUDA_TRY(h, cudaGraphLaunch(ex, st));
    }
    CUDA_TRY(h, cudaEventRecord(S.ev1, st));
    Ctl hc;
    CUDA_TRY(h, cudaMemcpyAsync(&hc, S.ctl.ptr, sizeof(Ctl), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(h, cudaStreamSynchronize(st));
    float ms = 0.f;
    CUDA_TRY(h, cudaEventElapsedTime(&ms, S.ev0, S.ev1));
    if (hc.error) return culamp_set_error(h, CULAMP_ERR_DEVICE_TIMEOUT, "loop control bound hit");
    // pass t reads buffer t % 2; iter = updates applied = the buffer holding the result
    const double *fres = (hc.iter & 1) ? S.psi.as<double>() : S.phi.as<double>();

    // residual and transport cost at the returned f (the Sinkhorn residual pass)
    PassParams pr = mk(X, X, (int)n, (int)n, d, p_res, h->pass_ctl.as<Ctl>());
    pr.ctr = X;
    pr.epi = EPI_SK_RESID;
    pr.coef_mode = COEF_FIXED;
    pr.alpha = -1.0 / (args->eta_p * winf);
    pr.beta = 1.0;
    pr.colpot = fres;
    pr.rowpot = fres;
    pr.marg = S.r.as<double>();
    pr.out = S.res.as<double>();
    pr.out2 = S.cost.as<double>();
    pr.want_moment = 1;
    pr.finish = FIN_SUMS;
    apply_feat(S, pr, true);
    CUDA_TRY(h, launch_pass(pr, pm_res, ACC_LSE, pass_shape((int)n, (int)n, d, ACC_LSE, h->sm_count, true),
                            S.scr, st));
    double sums[4];
    CUDA_TRY(h, cudaMemcpyAsync(sums, h->pass_ctl.as<Ctl>()->sums, sizeof(sums), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(h, cudaMemcpyAsync(f, fres, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    s = copy_log(h, hc, log, log_cap, st);
    if (s) return s;
    CUDA_TRY(h, cudaStreamSynchronize(st));
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        fill_stats_common(stats, hc, ms);
        stats->residual = sums[0];
        stats->objective = sums[1];
        stats->winf = winf;
        stats->eta_t = NAN;
        stats->s_t = NAN;
    }
    return CULAMP_OK;
}

// ---------------------------------------------------------------------- LAMP

namespace {

struct LampPlan {
    PassParams k1, k2, k2m, kd, k3, k4;
    PassParams k1f, k2f, k3f, k4f;   // precision ladder: FP32-exponent copies of k1 k2 k3 k4
    bool ladder = false;
    int pm;
    bool dual_min;
    LaunchShape s_rows, s_cols, s_rows_min, s_cols_mom;
};

LampPlan make_lamp_plan(culamp_handle h, int n, int m, int d, double p, double winf, double eta,
                        const culamp_args *args, uint32_t flags, bool checks) {
    Solver &S = *h->solver;
    Ctl *ctl = S.ctl.as<Ctl>();
    LampPlan pl;
    pl.pm = pmode_of(p);
    double *X = S.X.as<double>(), *Y = S.Y.as<double>();
    const double minv = std::tanh(-args->B / 2.0), maxv = std::tanh(args->B / 2.0);
    // K1: logZ_i = LSE_j(-(C s/(2W) + nu_j)/eta_t); phi_i = log r_i - logZ_i
    pl.k1 = mk(X, Y, n, m, d, p, ctl);
    pl.k1.ctr = X;
    pl.k1.epi = EPI_LOGZ;
    pl.k1.coef_mode = COEF_SPP_CUR;
    pl.k1.colpot = S.nu.as<double>();
    pl.k1.marg = S.r.as<double>();
    pl.k1.out = S.logz.as<double>();
    pl.k1.aux = S.aux.as<double>();
    pl.k1.use_ref = 1;
    pl.k1.finish = FIN_LAMP_Z;
    apply_feat(S, pl.k1, true);
    // K2: column residual at nu (+ cost on check iterations), fused theta_bar / nu_bar step
    pl.k2 = mk(Y, X, m, n, d, p, ctl);
    pl.k2.ctr = X;
    pl.k2.epi = EPI_SPP_COL;
    pl.k2.coef_mode = COEF_SPP_CUR;
    pl.k2.colpot = S.aux.as<double>();
    pl.k2.colpot_unit = 1;
    pl.k2.rowpot = S.nu.as<double>();
    pl.k2.cvec = S.c.as<double>();
    pl.k2.out = S.res.as<double>();
    pl.k2.out2 = S.cost.as<double>();
    pl.k2.want_moment = 0;
    pl.k2.use_ref = 1;
    pl.k2.gate = GATE_NOCHECK;
    pl.k2.lamp_step = LAMP_A;
    pl.k2.theta = S.theta.as<double>();
    pl.k2.thetab = S.thetab.as<double>();
    pl.k2.nu = S.nu.as<double>();
    pl.k2.nub = S.nub.as<double>();
    pl.k2.eta_mu_i = S.eta_mu.as<double>();
    pl.k2.eta_mu_exp = args->eta_mu;
    pl.k2.minv = minv;
    pl.k2.maxv = maxv;
    pl.k2.finish = FIN_LAMP_A;
    apply_feat(S, pl.k2, false);
    // the same pass with the cost moment, on check iterations only
    pl.k2m = pl.k2;
    pl.k2m.want_moment = 1;
    pl.k2m.use_ref = 0;
    pl.k2m.gate = GATE_CHECK;
    // Kd (check iterations): dual value at theta
    pl.dual_min = !(eta > 0.0);
    pl.kd = mk(X, Y, n, m, d, p, ctl);
    pl.kd.marg = S.r.as<double>();
    pl.kd.colpot = S.theta.as<double>();
    pl.kd.out = S.tmp.as<double>();
    pl.kd.gate = GATE_CHECK;
    pl.kd.finish = FIN_LAMP_DUAL;
    if (pl.dual_min) {
        pl.kd.epi = EPI_RAW;
        pl.kd.minmax_scale = 2.0 * winf;
    } else {
        pl.kd.ctr = X;
        pl.kd.epi = EPI_LOGZ;
        pl.kd.coef_mode = COEF_SPP_DUAL;
        pl.kd.use_ref = 1;
    }
    apply_feat(S, pl.kd, true);
    // K3: logZ at nu_bar with (eta_t', s')
    pl.k3 = pl.k1;
    pl.k3.coef_mode = COEF_SPP_NEXT;
    pl.k3.colpot = S.nub.as<double>();
    pl.k3.finish = FIN_NONE;
    // K4: column residual at nu_bar, fused theta / nu step, iteration bookkeeping
    pl.k4 = pl.k2;
    pl.k4.coef_mode = COEF_SPP_NEXT;
    pl.k4.rowpot = S.nub.as<double>();
    pl.k4.want_moment = 0;
    pl.k4.gate = GATE_ALWAYS;
    pl.k4.lamp_step = LAMP_B;
    pl.k4.finish = FIN_LAMP_B;
    // precision ladder (as for Sinkhorn), opt-in: FP32-exponent logZ and column
    // passes until a check's FP64 marginal residual is within 32x of the
    // tolerance or stops falling. It needs the checks (verbose or CHECK_ALWAYS)
    // and a tolerance; the check passes (cost moment, dual) stay FP64. Not the
    // default: LAMP's returned plan depends on the iteration it stops at (eta_t
    // follows the iteration count), and the FP32 phase moves that iteration, so
    // its transport cost leaves the reference's by ~1e-3 relative.
    if (fp32_form_applies(S, d, pl.pm) && checks && args->epsilon > 0.0 && (flags & CULAMP_FLAG_LADDER)) {
        pl.ladder = true;
        PassParams *fp[4] = {&pl.k1f, &pl.k2f, &pl.k3f, &pl.k4f};
        PassParams *dp[4] = {&pl.k1, &pl.k2, &pl.k3, &pl.k4};
        for (int q = 0; q < 4; ++q) {
            *fp[q] = *dp[q];
            fp[q]->fp32 = 1;
            fp[q]->phase = PHASE_FP32;
            dp[q]->phase = PHASE_FP64;
        }
    }
    pl.s_rows = pass_shape(n, m, d, ACC_LSE, h->sm_count);
    pl.s_cols = pass_shape(m, n, d, ACC_LSE, h->sm_count);
    pl.s_rows_min = pass_shape(n, m, d, ACC_MIN, h->sm_count);
    pl.s_cols_mom = pass_shape(m, n, d, ACC_LSE, h->sm_count, true);
    return pl;
}

}  // namespace

extern "C" int culamp_lamp(culamp_handle h, const double *x, const double *y, int64_t n, int64_t m,
                           int32_t d, const double *r, const double *c, const culamp_args *args,
                           int64_t frequency, double p, uint32_t flags, double *nu, double *phi,
                           double *psi, double *theta, culamp_stats *stats, culamp_log_row *log,
                           int64_t log_cap, void *stream) {
    int s = check_solver_args(h, x, y, n, m, d, r, c, args, frequency, p);
    if (s) return s;
    if (!(args->eta_p >= 0.0))
        return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "LAMP needs eta_p >= 0 (got %g)", args->eta_p);
    cudaStream_t st = (cudaStream_t)stream;
    if (flags & CULAMP_FLAG_FORM_PLAIN)
        return culamp_plain_lamp(h, x, y, n, m, d, r, c, args, frequency, p, flags, nu, phi, psi,
                                 theta, stats, log, log_cap, st);
    s = ensure_solver(h, (int)n, (int)m, d, log ? log_cap : 0, feat_pieces(d, flags));
    if (s) return s;
    Solver &S = *h->solver;
    double sum_rlogr = 0.0;
    int dk = d;
    s = stage_inputs(h, x, y, (int)n, (int)m, d, r, c, st, &sum_rlogr, &dk);
    if (s) return s;
    d = dk;
    s = prepare_features(h, (int)n, (int)m, d, st);
    if (s) return s;
    double winf = 0.0;
    s = compute_winf(h, (int)n, (int)m, d, p, st, &winf);
    if (s) return s;
    const double eta = args->eta_p / (2.0 * winf);
    CUDA_TRY(h, cudaMemsetAsync(S.theta.ptr, 0, m * sizeof(double), st));
    CUDA_TRY(h, cudaMemsetAsync(S.nu.ptr, 0, m * sizeof(double), st));
    CUDA_TRY(h, cudaMemsetAsync(S.thetab.ptr, 0, m * sizeof(double), st));
    CUDA_TRY(h, cudaMemsetAsync(S.nub.ptr, 0, m * sizeof(double), st));
    eta_mu_kernel<<<(unsigned)((m + 255) / 256), 256, 0, st>>>(S.eta_mu.as<double>(), S.c.as<double>(),
                                                               args->alpha / (double)n, args->tau_mu, m);
    CUDA_TRY(h, cudaGetLastError());
    Ctl hc0;
    std::memset(&hc0, 0, sizeof(hc0));
    hc0.itermax = args->itermax;
    hc0.frequency = frequency;
    hc0.stop = args->itermax < 1;
    hc0.stop_reason = args->itermax < 1 ? 2 : 0;
    hc0.check_enabled = args->verbose || (flags & CULAMP_FLAG_CHECK_ALWAYS);
    hc0.do_check = hc0.check_enabled;
    hc0.marginal_only = (flags & CULAMP_FLAG_MARGINAL_ONLY) ? 1 : 0;
    hc0.tmax_s = args->tmax;
    hc0.epsilon = args->epsilon;
    hc0.winf = winf;
    hc0.eta_lamp = eta;
    hc0.eta_t = INFINITY;
    hc0.s_t = 1.0;
    hc0.tau_p = 1.0;   // hard-coded in the reference (MirrorProxKernel.jl:1073)
    hc0.hr = eta * sum_rlogr;
    LampPlan pl = make_lamp_plan(h, (int)n, (int)m, d, p, winf, eta, args, flags, hc0.check_enabled != 0);
    hc0.fp32_phase = pl.ladder ? 1 : 0;
    hc0.ladder_switch = 32.0 * args->epsilon / 6.0;
    hc0.ladder_prev = INFINITY;
    hc0.log = S.logbuf.as<culamp_log_row>();
    hc0.log_cap = log ? log_cap : 0;
    CUDA_TRY(h, cudaMemcpyAsync(S.ctl.ptr, &hc0, sizeof(Ctl), cudaMemcpyHostToDevice, st));
    set_start_kernel<<<1, 1, 0, st>>>(S.ctl.as<Ctl>());
    auto body = [&](cudaStream_t cs) -> cudaError_t {
        cudaError_t e = cudaSuccess;
        if (pl.ladder) e = launch_pass(pl.k1f, pl.pm, ACC_LSE, pl.s_rows, S.scr, cs);
        if (e == cudaSuccess) e = launch_pass(pl.k1, pl.pm, ACC_LSE, pl.s_rows, S.scr, cs);
        if (e == cudaSuccess && pl.ladder) e = launch_pass(pl.k2f, pl.pm, ACC_LSE, pl.s_cols, S.scr, cs);
        if (e == cudaSuccess) e = launch_pass(pl.k2, pl.pm, ACC_LSE, pl.s_cols, S.scr, cs);
        if (e == cudaSuccess) e = launch_pass(pl.k2m, pl.pm, ACC_LSE, pl.s_cols_mom, S.scr, cs);
        if (e == cudaSuccess)
            e = launch_pass(pl.kd, pl.pm, pl.dual_min ? ACC_MIN : ACC_LSE,
                            pl.dual_min ? pl.s_rows_min : pl.s_rows, S.scr, cs);
        if (e == cudaSuccess && pl.ladder) e = launch_pass(pl.k3f, pl.pm, ACC_LSE, pl.s_rows, S.scr, cs);
        if (e == cudaSuccess) e = launch_pass(pl.k3, pl.pm, ACC_LSE, pl.s_rows, S.scr, cs);
        if (e == cudaSuccess && pl.ladder) e = launch_pass(pl.k4f, pl.pm, ACC_LSE, pl.s_cols, S.scr, cs);
        if (e == cudaSuccess) e = launch_pass(pl.k4, pl.pm, ACC_LSE, pl.s_cols, S.scr, cs);
        return e;
    };
    // small problems: the whole loop in one persistent cooperative launch
    const bool lpersist = !(flags & (CULAMP_FLAG_NO_GRAPH | CULAMP_FLAG_NO_PERSIST)) && !pl.ladder &&
                          !pl.dual_min && !S.feat_active && d <= MAXD_PACKED &&
                          (pl.pm == P_L1 || pl.pm == P_SQ || pl.pm == P_INF);
    int lgrid = lpersist ? lamp_persist_grid(h->sm_count, d, pl.pm) : 0;
    if (lgrid > 0 && !persist_eligible((int)n, (int)m, d, pl.pm, pl.pm, lgrid)) lgrid = 0;
    if (lgrid > 0) CUDA_TRY(h, S.pers.reserve(lamp_persist_scratch_bytes(lgrid)));
    CUDA_TRY(h, cudaEventRecord(S.ev0, st));
    bool lran = false;
    if (lgrid > 0) {
        LampPersistArgs la;
        la.X = S.X.as<double>(); la.Y = S.Y.as<double>(); la.r = S.r.as<double>(); la.c = S.c.as<double>();
        la.nu = S.nu.as<double>(); la.nub = S.nub.as<double>();
        la.theta = S.theta.as<double>(); la.thetab = S.thetab.as<double>();
        la.eta_mu = S.eta_mu.as<double>();
        la.logz = S.logz.as<double>(); la.aux = S.aux.as<double>();
        la.n = (int)n; la.m = (int)m; la.d = d; la.pm = pl.pm;
        la.pexp = p;
        la.eta_mu_exp = args->eta_mu;
        la.minv = std::tanh(-args->B / 2.0);
        la.maxv = std::tanh(args->B / 2.0);
        la.ctl = S.ctl.as<Ctl>();
        la.scratch = S.pers.ptr;
        // a refused cooperative launch falls back to the graph loop
        if (launch_lamp_persist(la, lgrid, st) == cudaSuccess) lran = true;
        else cudaGetLastError();
    }
    if (lran) {
    } else if (flags & CULAMP_FLAG_NO_GRAPH) {
        for (long long it = 0; it < args->itermax + 2; ++it) {
            CUDA_TRY(h, body(st));
            int stop = 0;
            CUDA_TRY(h, cudaMemcpyAsync(&stop, &S.ctl.as<Ctl>()->stop, sizeof(int), cudaMemcpyDeviceToHost, st));
            CUDA_TRY(h, cudaStreamSynchronize(st));
            if (stop) break;
        }
    } else {
        GraphKey key;
        key.kind = KIND_LAMP;
        key.form = pl.ladder ? 2 : 0;
        key.n = (int)n; key.m = (int)m; key.d = d;
        key.pm_iter = pl.pm;
        key.pm_resid = pl.dual_min ? 1 : 0;
        key.feat = S.feat_active ? S.feat_np : 0;
        key.unroll = pick_unroll((double)n * m * 4.0);
        key.generation = S.generation;
        key.p = p;
        key.winf = winf;
        key.B = args->B;
        key.eta_mu = args->eta_mu;
        cudaGraphExec_t ex = nullptr;
        s = get_graph(h, key, body, &ex);
        if (s) return s;
        CUDA_TRY(h, cudaGraphLaunch(ex, st));
    }
    CUDA_TRY(h, cudaEventRecord(S.ev1, st));
    Ctl hc;
    CUDA_TRY(h, cudaMemcpyAsync(&hc, S.ctl.ptr, sizeof(Ctl), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(h, cudaStreamSynchronize(st));
    float ms = 0.f;
    CUDA_TRY(h, cudaEventElapsedTime(&ms, S.ev0, S.ev1));
    if (hc.error) return culamp_set_error(h, CULAMP_ERR_DEVICE_TIMEOUT, "loop control bound hit");
    // post-loop (MirrorProxKernel.jl:1124-1129): logZ at (nu, eta_t, s), phi, psi;
    // then the column residual / cost of the returned state.
    {
        Ctl *pc = h->pass_ctl.as<Ctl>();
        PassParams a = pl.k1;
        a.ctl = pc;
        a.phase = PHASE_ANY;
        a.coef_mode = COEF_FIXED;
        const double c1 = hc.s_t / (2.0 * winf), invreg = 1.0 / hc.eta_t;
        a.alpha = -c1 * invreg;
        a.beta = -invreg;
        a.finish = FIN_NONE;
        CUDA_TRY(h, launch_pass(a, pl.pm, ACC_LSE, pl.s_rows, S.scr, st));
        PassParams b = pl.k2;
        b.ctl = pc;
        b.phase = PHASE_ANY;
        b.coef_mode = COEF_FIXED;
        b.alpha = a.alpha;
        b.beta = a.beta;
        b.lamp_step = LAMP_NONE;
        b.want_moment = 1;
        b.gate = GATE_ALWAYS;
        b.finish = FIN_SUMS;
        CUDA_TRY(h, launch_pass(b, pl.pm, ACC_LSE, pl.s_cols_mom, S.scr, st));
    }
    double sums[4];
    CUDA_TRY(h, cudaMemcpyAsync(sums, h->pass_ctl.as<Ctl>()->sums, sizeof(sums), cudaMemcpyDeviceToHost, st));
    if (phi) CUDA_TRY(h, cudaMemcpyAsync(phi, S.aux.ptr, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    if (nu) CUDA_TRY(h, cudaMemcpyAsync(nu, S.nu.ptr, m * sizeof(double), cudaMemcpyDeviceToDevice, st));
    if (theta) CUDA_TRY(h, cudaMemcpyAsync(theta, S.theta.ptr, m * sizeof(double), cudaMemcpyDeviceToDevice, st));
    if (psi) {
        // psi = -2 W_inf nu / eta_p (NaN / Inf when eta_p = 0, as in the reference)
        scale_kernel<<<(unsigned)((m + 255) / 256), 256, 0, st>>>(psi, S.nu.as<double>(),
                                                                  -2.0 * winf / args->eta_p, m);
        CUDA_TRY(h, cudaGetLastError());
    }
    s = copy_log(h, hc, log, log_cap, st);
    if (s) return s;
    CUDA_TRY(h, cudaStreamSynchronize(st));
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        fill_stats_common(stats, hc, ms);
        stats->num_iter = hc.iter;
        stats->residual = sums[0];
        stats->objective = sums[1];
        stats->winf = winf;
        stats->eta_t = hc.eta_t;
        stats->s_t = hc.s_t;
    }
    return CULAMP_OK;
}

// --------------------------------------------------------- annealed Sinkhorn

extern "C" int culamp_annealed_sinkhorn(culamp_handle h, const double *x, const double *y,
                                        int64_t n, int64_t m, int32_t d, const double *r,
                                        const double *c, const culamp_args *args,
                                        int64_t frequency, double p, uint32_t flags, double *phi,
                                        double *psi, culamp_stats *stats, culamp_log_row *log,
                                        int64_t log_cap, void *stream) {
    int s = check_solver_args(h, x, y, n, m, d, r, c, args, frequency, p);
    if (s) return s;
    if (!phi || !psi) return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "null output pointer");
    const double eta_final = args->epsilon;   // AnnealedSinkhorn.jl:78 (Q4)
    if (!(eta_final > 0.0))
        return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "annealed Sinkhorn needs epsilon > 0");
    if (!(args->anneal_mult > 0.0 && args->anneal_mult < 1.0) && args->eta_p > eta_final)
        return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "anneal_mult must be in (0, 1)");
    if (flags & CULAMP_FLAG_FORM_PLAIN)
        return culamp_set_error(h, CULAMP_ERR_UNSUPPORTED, "annealed Sinkhorn has no plain form");
    cudaStream_t st = (cudaStream_t)stream;
    s = ensure_solver(h, (int)n, (int)m, d, 0, feat_pieces(d, flags));
    if (s) return s;
    Solver &S = *h->solver;
    int dk = d;
    s = stage_inputs(h, x, y, (int)n, (int)m, d, r, c, st, nullptr, &dk);
    if (s) return s;
    d = dk;
    s = prepare_features(h, (int)n, (int)m, d, st);
    if (s) return s;
    double winf = 0.0;
    s = compute_winf(h, (int)n, (int)m, d, p, st, &winf);
    if (s) return s;
    // phi = log r, psi = log c; warm starts and previous values start there too
    const unsigned bn = (unsigned)((n + 255) / 256), bm = (unsigned)((m + 255) / 256);
    log_kernel<<<bn, 256, 0, st>>>(S.ws_phi.as<double>(), S.r.as<double>(), n);
    log_kernel<<<bm, 256, 0, st>>>(S.ws_psi.as<double>(), S.c.as<double>(), m);
    CUDA_TRY(h, cudaMemcpyAsync(S.prev_phi.ptr, S.ws_phi.ptr, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    CUDA_TRY(h, cudaMemcpyAsync(S.prev_psi.ptr, S.ws_psi.ptr, m * sizeof(double), cudaMemcpyDeviceToDevice, st));
    double eta = args->eta_p > eta_final ? args->eta_p : eta_final;
    double preveta = 1.0;
    const double q = args->anneal_mult;
    culamp_args a = *args;
    a.verbose = 0;
    long long total_iters = 0, stages = 0;
    float total_ms = 0.f;
    double resid = NAN, obj = NAN;
    int64_t rows = 0;
    Ctl hc;
    std::memset(&hc, 0, sizeof(hc));
    auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        a.eta_p = eta;
        CUDA_TRY(h, cudaMemcpyAsync(S.phi.ptr, S.ws_phi.ptr, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
        CUDA_TRY(h, cudaMemcpyAsync(S.psi.ptr, S.ws_psi.ptr, m * sizeof(double), cudaMemcpyDeviceToDevice, st));
        float ms = 0.f;
        s = sinkhorn_loop(h, (int)n, (int)m, d, p, eta, winf, &a, frequency, flags, 0, st, &hc, &ms);
        if (s) return s;
        s = sinkhorn_final(h, (int)n, (int)m, d, p, eta, winf, flags, st, &resid, &obj);
        if (s) return s;
        total_ms += ms;
        total_iters += hc.num_iter;
        stages += 1;
        const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        a.tmax = args->tmax - el;
        if (log && rows < log_cap) {
            culamp_log_row &lr = log[rows++];
            lr.time_s = el;
            lr.iter = (double)total_iters;
            lr.infeas = resid;
            lr.ot_objective = obj;
            lr.primal = NAN;
            lr.dual = eta;   // the reference prints eta in this column
        }
        if (eta == eta_final || el >= args->tmax) break;
        const double f = eta / preveta;
        extrapolate_kernel<<<bn, 256, 0, st>>>(S.ws_phi.as<double>(), S.prev_phi.as<double>(), S.phi.as<double>(), f, n);
        extrapolate_kernel<<<bm, 256, 0, st>>>(S.ws_psi.as<double>(), S.prev_psi.as<double>(), S.psi.as<double>(), f, m);
        CUDA_TRY(h, cudaGetLastError());
        preveta = eta;
        eta = q * eta > eta_final ? q * eta : eta_final;
    }
    CUDA_TRY(h, cudaMemcpyAsync(phi, S.phi.ptr, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    CUDA_TRY(h, cudaMemcpyAsync(psi, S.psi.ptr, m * sizeof(double), cudaMemcpyDeviceToDevice, st));
    CUDA_TRY(h, cudaStreamSynchronize(st));
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        stats->iterations = stages;
        stats->num_iter = total_iters;
        stats->residual = resid;
        stats->objective = obj;
        stats->winf = winf;
        stats->eta_t = eta;
        stats->s_t = NAN;
        stats->elapsed_ms = total_ms;
        stats->log_rows = rows;
        stats->stopped = hc.stop_reason;
        stats->status = CULAMP_OK;
    }
    return CULAMP_OK;
}

// ------------------------------------------------------------- host variants

namespace {
struct HostStage {
    culamp_handle h;
    std::vector<std::pair<void *, size_t>> allocs;
    ~HostStage() {
        for (auto &a : allocs) cudaFree(a.first);
    }
    double *put(const double *src, size_t count, cudaStream_t st, int *err) {
        void *p = nullptr;
        if (cudaMalloc(&p, count * sizeof(double) + 8) != cudaSuccess) { *err = CULAMP_ERR_ALLOC; return nullptr; }
        allocs.push_back({p, count});
        if (src && cudaMemcpyAsync(p, src, count * sizeof(double), cudaMemcpyHostToDevice, st) != cudaSuccess)
            *err = CULAMP_ERR_CUDA;
        return (double *)p;
    }
};
}  // namespace

extern "C" int culamp_sinkhorn_host(culamp_handle h, const double *x, const double *y, int64_t n,
                                    int64_t m, int32_t d, const double *r, const double *c,
                                    const culamp_args *args, int64_t frequency, double p,
                                    const double *phi0, const double *psi0, uint32_t flags,
                                    double *phi, double *psi, culamp_stats *stats,
                                    culamp_log_row *log, int64_t log_cap) {
    int s = check_solver_args(h, x, y, n, m, d, r, c, args, frequency, p);
    if (s) return s;
    if (!phi || !psi) return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "null output pointer");
    cudaStream_t st = nullptr;
    HostStage hs{h, {}};
    int err = 0;
    double *dx = hs.put(x, (size_t)n * d, st, &err), *dy = hs.put(y, (size_t)m * d, st, &err);
    double *dr = hs.put(r, n, st, &err), *dc = hs.put(c, m, st, &err);
    double *dphi0 = phi0 ? hs.put(phi0, n, st, &err) : nullptr;
    double *dpsi0 = psi0 ? hs.put(psi0, m, st, &err) : nullptr;
    double *dphi = hs.put(nullptr, n, st, &err), *dpsi = hs.put(nullptr, m, st, &err);
    if (err) return culamp_set_error(h, err, "host staging failed");
    s = culamp_sinkhorn(h, dx, dy, n, m, d, dr, dc, args, frequency, p, dphi0, dpsi0, flags, dphi,
                        dpsi, stats, log, log_cap, st);
    if (s) return s;
    CUDA_TRY(h, cudaMemcpyAsync(phi, dphi, n * sizeof(double), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(h, cudaMemcpyAsync(psi, dpsi, m * sizeof(double), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(h, cudaStreamSynchronize(st));
    return CULAMP_OK;
}

extern "C" int culamp_lamp_host(culamp_handle h, const double *x, const double *y, int64_t n,
                                int64_t m, int32_t d, const double *r, const double *c,
                                const culamp_args *args, int64_t frequency, double p,
                                uint32_t flags, double *nu, double *phi, double *psi,
                                double *theta, culamp_stats *stats, culamp_log_row *log,
                                int64_t log_cap) {
    int s = check_solver_args(h, x, y, n, m, d, r, c, args, frequency, p);
    if (s) return s;
    cudaStream_t st = nullptr;
    HostStage hs{h, {}};
    int err = 0;
    double *dx = hs.put(x, (size_t)n * d, st, &err), *dy = hs.put(y, (size_t)m * d, st, &err);
    double *dr = hs.put(r, n, st, &err), *dc = hs.put(c, m, st, &err);
    double *dnu = hs.put(nullptr, m, st, &err), *dphi = hs.put(nullptr, n, st, &err);
    double *dpsi = hs.put(nullptr, m, st, &err), *dth = hs.put(nullptr, m, st, &err);
    if (err) return culamp_set_error(h, err, "host staging failed");
    s = culamp_lamp(h, dx, dy, n, m, d, dr, dc, args, frequency, p, flags, dnu, dphi, dpsi, dth,
                    stats, log, log_cap, st);
    if (s) return s;
    if (nu) CUDA_TRY(h, cudaMemcpyAsync(nu, dnu, m * sizeof(double), cudaMemcpyDeviceToHost, st));
    if (phi) CUDA_TRY(h, cudaMemcpyAsync(phi, dphi, n * sizeof(double), cudaMemcpyDeviceToHost, st));
    if (psi) CUDA_TRY(h, cudaMemcpyAsync(psi, dpsi, m * sizeof(double), cudaMemcpyDeviceToHost, st));
    if (theta) CUDA_TRY(h, cudaMemcpyAsync(theta, dth, m * sizeof(double), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(h, cudaStreamSynchronize(st));
    return CULAMP_OK;
}
