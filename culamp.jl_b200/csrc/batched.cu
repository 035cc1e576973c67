// batched.cu -- many independent Sinkhorn problems of uneven size in one solve.
//
// Each instance runs sinkhorn_color_transfer (SinkhornKernel.jl:477-559) with
// its own control block (iteration counter, check cadence, stopping rule,
// W_inf), scratch and potentials, so its iterations and result are those of a
// culamp_sinkhorn call on it alone. What is shared is the launch: every
// half-step of every instance class is ONE kernel launch over all instances of
// the class (block / work-unit prefix tables map a CTA to its instance), and
// the loop over iterations runs in CUDA graphs with a device-side WHILE
// condition. A phase (one graph launch) lasts while the instances still running
// hold more than half of the pairs they held when it began; then the host
// re-plans the survivors -- finer column splits, since fewer instances must
// fill the GPU -- and launches the next phase. Within a phase, instances that
// stopped cost one early-exiting CTA per block.
//
// Classes: d <= 3 on the FP64-exponent pair loop (fixed-reference fast path),
// other d <= 256 on the FP64 generic pair loop, d >= 32 with p = 2 on the
// tensor-core feature path.
//
// Shapes. A single-instance pass splits its columns until the whole GPU is
// busy; in a batch the instances fill the GPU together, so each pair-pass CTA
// is sized to a common amount of work: (total pairs of the batch) /
// (target CTAs per SM x SMs), and each feature work unit to a number of
// 128-column tiles. Both knobs are chosen by timing candidates on the batch
// itself (three iterations each, from the same starting point, the better of
// two rounds), and the choice
// is cached on the handle for batches with the same signature; later phases
// keep the knobs and recompute the shapes for their smaller total work.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <vector>

#include "internal.h"

using namespace culamp_host;
using namespace culamp_dev;

#define BT_TRY(h, expr)                                                                         \
    do {                                                                                        \
        cudaError_t _e = (expr);                                                                \
        if (_e != cudaSuccess)                                                                  \
            return culamp_set_error((h), CULAMP_ERR_CUDA, "%s: %s (%s:%d)", #expr,             \
                                    cudaGetErrorString(_e), __FILE__, __LINE__);                \
    } while (0)

namespace {

__global__ void batch_start_kernel(Ctl *c, int count) {
    const unsigned long long t = globaltimer_ns();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
        c[i].t_start_ns = t;
}

// Loop control of the batched WHILE graph over the instances of this phase
// (active[0..na-1]): per instance the bounds of the single-instance loop
// control (iterations, body executions, tmax); the loop continues while the
// pairs of the instances still running exceed `min_pairs` (the phase ends when
// the running work has halved, so the host can re-plan finer shapes for the
// rest) and no device wait has given up.
__global__ void batch_loop_ctl_kernel(Ctl *cs, const int *active, int na, const double *pairs,
                                      double min_pairs, const int *err, cudaGraphConditionalHandle hnd) {
    __shared__ double run;
    if (threadIdx.x == 0) run = 0.0;
    __syncthreads();
    const unsigned long long now = globaltimer_ns();
    double mine = 0.0;
    for (int k = threadIdx.x; k < na; k += blockDim.x) {
        const int i = active[k];
        Ctl *c = cs + i;
        if (c->stop) continue;
        c->loops += 1;
        if (c->iter > c->itermax + 1 || c->loops > c->itermax + 2) {
            c->stop = 1; c->stop_reason = 2; c->error = 1;
        } else if ((double)(now - c->t_start_ns) * 1e-9 > c->tmax_s) {
            c->stop = 1; c->stop_reason = 3;
        } else {
            mine += pairs[i];
        }
    }
    if (mine > 0.0) atomicAdd(&run, mine);
    __syncthreads();
    if (threadIdx.x == 0) cudaGraphSetConditional(hnd, (run > min_pairs && !*err) ? 1u : 0u);
}

struct Inst {
    int n = 0, m = 0, d = 0;
    int cls = 0;                    // 1..3 packed d, 0 generic pair loop, -1 feature path
    size_t xo = 0, yo = 0;          // offsets of x / y in the coordinate buffers (doubles)
    size_t no = 0, mo = 0;          // offsets of the n- / m-vectors
    size_t fxo = 0, fyo = 0;        // offsets of the packed clouds (bf16 elements)
    size_t parto = 0, ticko = 0, blko = 0;
    size_t part_need = 0, tick_need = 0, blk_need = 0;
};

// One batched launch: instances of one class and one pass kind.
struct Group {
    int cls = 0;
    int pm = P_SQ;
    bool mom = false, fr = false;
    std::vector<int> members;       // instance indices
    size_t plist_off = 0;           // offset (entries) in the device parameter list
    size_t table_off = 0;           // offset (ints) of block_start / unit_start
    size_t table2_off = 0;          // feature: offset of the merge block_start table
    int total = 0;                  // CTAs (pair) or work units (feature)
    int total_merge = 0;            // feature merge CTAs
    size_t smem = 0;
};

struct Plan {
    std::vector<PassParams> params; // all groups' parameter entries, in group order
    std::vector<int> tables;
    std::vector<Group> k1, k2, k3, kf;   // row pass, column pass, check pass, final residual
};

}  // namespace

struct culamp_handle_s::Batch {
    DevBuf X, Y, r, c, phi, psi, ctl, ctl2, part, tickets, blk, fx, fy, fxn, fyn, plist, tables, err,
        pairs, active, mctab;
    std::vector<unsigned char> mctab_host;   // W_inf job table as uploaded
    cudaStream_t cap_stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::vector<unsigned long long> tuned_sig;
    int tuned_tpsm = 0, tuned_tpu = 0;

    void release() {
        DevBuf *all[] = {&X, &Y, &r, &c, &phi, &psi, &ctl, &ctl2, &part, &tickets, &blk, &fx, &fy,
                         &fxn, &fyn, &plist, &tables, &err, &pairs, &active, &mctab};
        for (DevBuf *b : all) b->release();
        if (cap_stream) cudaStreamDestroy(cap_stream);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        cap_stream = nullptr;
        ev0 = ev1 = nullptr;
    }
};

void culamp_batch_release(culamp_handle h) {
    if (h && h->batch) {
        h->batch->release();
        delete h->batch;
        h->batch = nullptr;
    }
}

namespace {

using Batch = culamp_handle_s::Batch;

// Pair-pass shape for one batch member: RPT rows per thread, columns split so
// one CTA handles about `work` pairs.
LaunchShape batch_pair_shape(int n, int m, int d, double work) {
    LaunchShape s{};
    const bool packed = d >= 1 && d <= MAXD_PACKED;
    s.R = RPT;
    s.rb = (n + ROWS - 1) / ROWS;
    const int ch = packed ? CHUNK : CHUNK_G;
    const double per_split = (double)ROWS * (double)m;
    int splits = (int)std::lround(per_split / std::max(work, 1.0));
    const int max_splits = (m + CHUNK - 1) / CHUNK;   // at least CHUNK columns per split
    splits = std::min(std::max(splits, 1), max_splits);
    int cps = (m + splits - 1) / splits;
    cps = ((cps + ch - 1) / ch) * ch;
    splits = (m + cps - 1) / cps;
    s.splits = splits;
    s.cols_per_split = cps;
    s.smem = (size_t)(packed ? CHUNK * 4 : CHUNK_G * (d + 1)) * sizeof(double);
    s.part_bytes = splits > 1 ? (size_t)splits * (size_t)n * 3 * sizeof(double) : 0;
    s.sms = 0;
    return s;
}

// Feature-pass shape for one batch member: work units of `tpu` column tiles.
FeatShape batch_feat_shape(int n, int m, int tpu, int pieces) {
    FeatShape fs{};
    fs.ncols = feat_tile_cols(pieces);
    fs.rtiles = (n + 127) / 128;
    fs.ctiles = (m + fs.ncols - 1) / fs.ncols;
    fs.rblk = feat_blocks(n);
    fs.cblk = feat_blocks(m);
    fs.tps = std::min(std::max(tpu, 1), fs.ctiles);
    fs.splits = (fs.ctiles + fs.tps - 1) / fs.tps;
    fs.units = fs.rtiles * fs.splits;
    fs.grid = 0;
    fs.merge_rb = (n + ROWS - 1) / ROWS;
    fs.part_bytes = (size_t)fs.splits * (size_t)n * 3 * sizeof(double);
    return fs;
}

struct Ctx {
    culamp_handle h;
    Batch *B;
    std::vector<Inst> in;
    int count = 0;
    int pm_iter = P_SQ, pm_res = P_SQ;
    double p_true = 2.0;
    int np = 0;                     // feature pieces (0: no feature members)
    uint32_t flags = 0;
    double total_pairs = 0.0;
};

// Parameter entry of instance i for one pass kind. `rows_x`: the pass reduces
// over columns for the rows of x (row pass) or the reverse (column pass).
PassParams entry(const Ctx &X, int i, bool rows_x, int kind) {
    const Inst &I = X.in[i];
    Batch &B = *X.B;
    PassParams P;
    std::memset(&P, 0, sizeof(P));
    double *xs = B.X.as<double>() + I.xo, *ys = B.Y.as<double>() + I.yo;
    double *phi = B.phi.as<double>() + I.no, *psi = B.psi.as<double>() + I.mo;
    double *r = B.r.as<double>() + I.no, *c = B.c.as<double>() + I.mo;
    Ctl *ctl = (kind == 4 ? B.ctl2.as<Ctl>() : B.ctl.as<Ctl>()) + i;
    P.X = rows_x ? xs : ys;
    P.Y = rows_x ? ys : xs;
    P.n = rows_x ? I.n : I.m;
    P.m = rows_x ? I.m : I.n;
    P.d = I.d;
    P.pexp = (kind == 3 || kind == 4) ? (X.pm_res == P_L1 ? 1.0 : 2.0) : (X.pm_iter == P_L1 ? 1.0 : 2.0);
    P.ctl = ctl;
    P.ctr = xs;
    P.coef_mode = COEF_SK;
    if (kind == 1) {            // phi = log r - LSE_j(-C/(eta W) + psi)
        P.epi = EPI_SK_ROW;
        P.colpot = psi;
        P.marg = r;
        P.out = phi;
        P.use_ref = 1;
    } else if (kind == 2) {     // psi = log c - LSE_i(-C/(eta W) + phi); iteration bookkeeping
        P.epi = EPI_SK_ROW;
        P.colpot = phi;
        P.marg = c;
        P.out = psi;
        P.use_ref = 1;
        P.finish = FIN_SK_ITER;
    } else {                    // 3: gated residual check; 4: final residual / cost
        P.epi = EPI_SK_RESID;
        P.colpot = psi;
        P.rowpot = phi;
        P.marg = r;
        P.want_moment = 1;
        P.gate = (kind == 3) ? GATE_CHECK : GATE_ALWAYS;
        P.finish = (kind == 3) ? FIN_SK_CHECK : FIN_SUMS;
    }
    P.part = B.part.as<double>() + I.parto;
    P.rb_ticket = B.tickets.as<unsigned>() + I.ticko;
    P.blk = B.blk.as<double>() + I.blko;
    if (I.cls < 0) {
        const uint16_t *fxs = B.fx.as<uint16_t>() + I.fxo, *fys = B.fy.as<uint16_t>() + I.fyo;
        const double *xn = B.fxn.as<double>() + I.no, *yn = B.fyn.as<double>() + I.mo;
        P.fx = rows_x ? fxs : fys;
        P.fy = rows_x ? fys : fxs;
        P.xn = rows_x ? xn : yn;
        P.yn = rows_x ? yn : xn;
        P.fkb = feat_kblocks(I.d);
        P.fpieces = X.np;
    }
    return P;
}

// Build the launch groups of every pass kind for shape knobs (tpsm, tpu) over
// the instances in `act` (pairs: their total pair count).
Plan make_plan(const Ctx &X, int tpsm, int tpu, int sms, const std::vector<int> &act, double pairs) {
    Plan pl;
    const double work = pairs / std::max(1.0, (double)tpsm * sms);
    const int kinds[4] = {1, 2, 3, 4};
    std::vector<Group> *dst[4] = {&pl.k1, &pl.k2, &pl.k3, &pl.kf};
    const int classes[5] = {1, 2, 3, 0, -1};
    for (int kk = 0; kk < 4; ++kk) {
        const int kind = kinds[kk];
        const bool rows_x = kind != 2;
        const bool mom = kind >= 3;
        for (int cls : classes) {
            Group g;
            g.cls = cls;
            g.mom = mom;
            g.fr = !mom && cls > 0;
            g.pm = mom ? X.pm_res : X.pm_iter;
            for (int i : act)
                if (X.in[i].cls == cls) g.members.push_back(i);
            if (g.members.empty()) continue;
            g.plist_off = pl.params.size();
            g.table_off = pl.tables.size();
            int acc = 0, acc2 = 0;
            std::vector<int> t1, t2;
            for (int i : g.members) {
                PassParams P = entry(X, i, rows_x, kind);
                t1.push_back(acc);
                if (cls >= 0) {
                    const LaunchShape sh = batch_pair_shape(P.n, P.m, P.d, work);
                    P.splits = sh.splits;
                    P.cols_per_split = sh.cols_per_split;
                    P.nrb = sh.rb;
                    P.grid_ticket = P.rb_ticket + sh.rb;
                    acc += sh.rb * sh.splits;
                    g.smem = std::max(g.smem, sh.smem);
                } else {
                    const FeatShape fs = batch_feat_shape(P.n, P.m, tpu, P.fpieces);
                    set_feat_geometry(P, fs);
                    P.grid_ticket = P.rb_ticket + fs.merge_rb;
                    t2.push_back(acc2);
                    acc += fs.units;
                    acc2 += fs.merge_rb;
                }
                pl.params.push_back(P);
            }
            t1.push_back(acc);
            g.total = acc;
            pl.tables.insert(pl.tables.end(), t1.begin(), t1.end());
            if (cls < 0) {
                t2.push_back(acc2);
                g.total_merge = acc2;
                g.table2_off = pl.tables.size();
                pl.tables.insert(pl.tables.end(), t2.begin(), t2.end());
            }
            dst[kk]->push_back(g);
        }
    }
    return pl;
}

// Scratch of instance i for any shape the batch may give it: pair passes up
// to one split per column tile, feature passes up to one slice per column
// tile, and the single-instance W_inf pass.
void scratch_need(Inst &I, int sms) {
    size_t part = 8, tick = 0, blk = 0;
    for (int o = 0; o < 2; ++o) {
        const int n = o ? I.m : I.n, m = o ? I.n : I.m;
        if (I.cls >= 0) {
            const LaunchShape sh = batch_pair_shape(n, m, I.d, 1.0);   // most splits
            part = std::max(part, sh.part_bytes);
            tick = std::max(tick, (size_t)sh.rb + 1);
            blk = std::max(blk, (size_t)sh.rb * 4);
        } else {
            const FeatShape fs = batch_feat_shape(n, m, 1, 3);   // narrowest tiles: most slices
            part = std::max(part, fs.part_bytes);
            tick = std::max(tick, (size_t)fs.merge_rb + 1);
            blk = std::max(blk, (size_t)fs.merge_rb * 4);
        }
    }
    const LaunchShape wsh = pass_shape(I.n, I.m, I.d, ACC_MAX, sms);
    part = std::max(part, wsh.part_bytes);
    tick = std::max(tick, (size_t)wsh.rb + 1);
    blk = std::max(blk, (size_t)wsh.rb * 4);
    I.part_need = (part + 7) / 8;     // doubles
    I.tick_need = tick;
    I.blk_need = blk;
}

cudaError_t launch_groups(const Ctx &X, const std::vector<Group> &gs, cudaStream_t st) {
    Batch &B = *X.B;
    const PassParams *pl = B.plist.as<PassParams>();
    const int *tb = B.tables.as<int>();
    for (const Group &g : gs) {
        cudaError_t e;
        if (g.cls >= 0)
            e = launch_pass_batched(pl + g.plist_off, tb + g.table_off, (int)g.members.size(), g.total, g.smem,
                                    g.pm, g.cls, ACC_LSE, g.mom, g.fr, st);
        else
            e = launch_feat_batched(X.np, ACC_LSE, g.mom, pl + g.plist_off, tb + g.table_off,
                                    tb + g.table2_off, (int)g.members.size(), g.total, g.total_merge,
                                    X.h->sm_count, B.err.as<int>(), st);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

int upload_plan(const Ctx &X, const Plan &pl, cudaStream_t st) {
    Batch &B = *X.B;
    culamp_handle h = X.h;
    if (B.plist.reserve(pl.params.size() * sizeof(PassParams)) != cudaSuccess ||
        B.tables.reserve(pl.tables.size() * sizeof(int)) != cudaSuccess)
        return culamp_set_error(h, CULAMP_ERR_ALLOC, "batch parameter tables");
    BT_TRY(h, cudaMemcpyAsync(B.plist.ptr, pl.params.data(), pl.params.size() * sizeof(PassParams),
                              cudaMemcpyHostToDevice, st));
    BT_TRY(h, cudaMemcpyAsync(B.tables.ptr, pl.tables.data(), pl.tables.size() * sizeof(int),
                              cudaMemcpyHostToDevice, st));
    BT_TRY(h, cudaStreamSynchronize(st));   // the host vectors go out of scope
    return CULAMP_OK;
}

// Control blocks of every instance (as culamp_sinkhorn's loop sets them up),
// potentials at zero, then W_inf of each instance into its control block.
int reset_state(const Ctx &X, const culamp_args *args, int64_t frequency, cudaStream_t st) {
    Batch &B = *X.B;
    culamp_handle h = X.h;
    std::vector<Ctl> cs(X.count);
    for (int i = 0; i < X.count; ++i) {
        Ctl &c = cs[i];
        std::memset(&c, 0, sizeof(c));
        c.itermax = args->itermax;
        c.frequency = frequency;
        c.stop = args->itermax < 1;
        c.stop_reason = args->itermax < 1 ? 2 : 0;
        c.tmax_s = args->tmax;
        c.epsilon = args->epsilon;
        c.eta = args->eta_p;
    }
    BT_TRY(h, cudaMemcpyAsync(B.ctl.ptr, cs.data(), cs.size() * sizeof(Ctl), cudaMemcpyHostToDevice, st));
    BT_TRY(h, cudaMemsetAsync(B.phi.ptr, 0, B.phi.bytes, st));
    BT_TRY(h, cudaMemsetAsync(B.psi.ptr, 0, B.psi.bytes, st));
    BT_TRY(h, cudaMemsetAsync(B.err.ptr, 0, sizeof(int), st));
    // W_inf of every instance in one launch (the control blocks hold winf = +0)
    std::vector<MaxCostInput> mc(X.count);
    for (int i = 0; i < X.count; ++i) {
        const Inst &I = X.in[i];
        mc[i] = {B.X.as<double>() + I.xo, B.Y.as<double>() + I.yo, I.n, I.m, I.d, &(B.ctl.as<Ctl>() + i)->winf};
    }
    BT_TRY(h, B.mctab.reserve(max_cost_table_bytes(X.count)));
    BT_TRY(h, launch_max_cost_batched(mc.data(), X.count, X.p_true, B.mctab.ptr, B.mctab_host, h->sm_count, st));
    batch_start_kernel<<<(X.count + 255) / 256, 256, 0, st>>>(B.ctl.as<Ctl>(), X.count);
    BT_TRY(h, cudaGetLastError());
    return CULAMP_OK;
}

// Device time of `iters` iterations (row + column passes, checks gated off by
// the cadence) of the plan, from the reset state.
int time_plan(const Ctx &X, const Plan &pl, const culamp_args *args, int iters, cudaStream_t st, float *ms) {
    Batch &B = *X.B;
    culamp_handle h = X.h;
    int s = upload_plan(X, pl, st);
    if (s) return s;
    culamp_args a = *args;
    a.itermax = iters + 2;
    a.epsilon = 0.0;
    s = reset_state(X, &a, 1 << 30, st);
    if (s) return s;
    // one warm-up iteration, then the timed ones
    BT_TRY(h, launch_groups(X, pl.k1, st));
    BT_TRY(h, launch_groups(X, pl.k2, st));
    BT_TRY(h, cudaEventRecord(B.ev0, st));
    for (int it = 0; it < iters; ++it) {
        BT_TRY(h, launch_groups(X, pl.k1, st));
        BT_TRY(h, launch_groups(X, pl.k2, st));
        BT_TRY(h, launch_groups(X, pl.k3, st));
    }
    BT_TRY(h, cudaEventRecord(B.ev1, st));
    BT_TRY(h, cudaEventSynchronize(B.ev1));
    BT_TRY(h, cudaEventElapsedTime(ms, B.ev0, B.ev1));
    return CULAMP_OK;
}

int build_graph(const Ctx &X, const Plan &pl, int unroll, int na, double min_pairs, cudaGraphExec_t *out) {
    Batch &B = *X.B;
    culamp_handle h = X.h;
    cudaGraph_t g = nullptr;
    BT_TRY(h, cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle ch;
    cudaError_t e = cudaGraphConditionalHandleCreate(&ch, g, 1, cudaGraphCondAssignDefault);
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
        e = cudaStreamBeginCaptureToGraph(B.cap_stream, bodyg, nullptr, nullptr, 0,
                                          cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            cudaError_t eb = cudaSuccess;
            for (int u = 0; u < unroll && eb == cudaSuccess; ++u) {
                eb = launch_groups(X, pl.k1, B.cap_stream);
                if (eb == cudaSuccess) eb = launch_groups(X, pl.k2, B.cap_stream);
                if (eb == cudaSuccess) eb = launch_groups(X, pl.k3, B.cap_stream);
            }
            if (eb == cudaSuccess) {
                batch_loop_ctl_kernel<<<1, 256, 0, B.cap_stream>>>(B.ctl.as<Ctl>(), B.active.as<int>(), na,
                                                                   B.pairs.as<double>(), min_pairs,
                                                                   B.err.as<int>(), ch);
                eb = cudaGetLastError();
            }
            cudaGraph_t captured = nullptr;
            e = cudaStreamEndCapture(B.cap_stream, &captured);
            if (eb != cudaSuccess) e = eb;
        }
    }
    cudaGraphExec_t exec = nullptr;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return culamp_set_error(h, CULAMP_ERR_CUDA, "batch graph build: %s", cudaGetErrorString(e));
    }
    *out = exec;
    return CULAMP_OK;
}

}  // namespace

extern "C" int culamp_batched_sinkhorn(culamp_handle h, const culamp_instance *inst, int32_t count,
                                       const culamp_args *args, int64_t frequency, double p,
                                       uint32_t flags, culamp_batch_stats *stats,
                                       culamp_batch_info *info, void *stream) {
    if (!h) return CULAMP_ERR_INVALID_ARG;
    if (!inst || !args || count < 1) return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "empty batch");
    if (frequency < 1) return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "frequency must be >= 1");
    if (args->itermax < 0) return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "itermax < 0");
    if (!(args->eta_p > 0.0))
        return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "Sinkhorn needs eta_p > 0 (got %g)", args->eta_p);
    if (flags & (CULAMP_FLAG_TRUE_PINF | CULAMP_FLAG_FORM_PLAIN))
        return culamp_set_error(h, CULAMP_ERR_UNSUPPORTED, "batched solves run the chosen form, reference p semantics");
    Ctx X;
    X.h = h;
    X.count = count;
    X.flags = flags;
    if (p == 1.0) { X.pm_iter = P_L1; X.pm_res = P_L1; }
    else if (p == 2.0 || std::isinf(p)) { X.pm_iter = P_SQ; X.pm_res = P_SQ; }   // SinkhornKernel.jl:518-520, :38-42
    else return culamp_set_error(h, CULAMP_ERR_UNSUPPORTED, "batched solves support p = 1, 2, Inf");
    X.p_true = p;
    cudaSetDevice(h->device);
    cudaStream_t st = (cudaStream_t)stream;
    if (!h->batch) {
        h->batch = new (std::nothrow) Batch();
        if (!h->batch) return culamp_set_error(h, CULAMP_ERR_ALLOC, "batch state");
        if (cudaStreamCreateWithFlags(&h->batch->cap_stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreate(&h->batch->ev0) != cudaSuccess || cudaEventCreate(&h->batch->ev1) != cudaSuccess)
            return culamp_set_error(h, CULAMP_ERR_CUDA, "stream/event creation failed");
    }
    Batch &B = *h->batch;
    X.B = &B;
    const int feat_np = (flags & CULAMP_FLAG_FEAT_FP64) ? 0 : ((flags & CULAMP_FLAG_FEAT_X6) ? 3 : 2);

    // ---- instances: class, offsets, signature
    X.in.resize(count);
    size_t xo = 0, yo = 0, no = 0, mo = 0, fxo = 0, fyo = 0;
    std::vector<unsigned long long> sig;
    sig.push_back((unsigned long long)count);
    sig.push_back(((unsigned long long)X.pm_iter << 8) | (unsigned long long)feat_np);
    for (int i = 0; i < count; ++i) {
        const culamp_instance &u = inst[i];
        if (!u.x || !u.y || !u.r || !u.c || !u.phi || !u.psi)
            return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "instance %d: null pointer", i);
        if (u.n < 1 || u.m < 1 || u.n > (1LL << 26) || u.m > (1LL << 26))
            return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "instance %d: sizes out of range", i);
        if (u.d < 1 || u.d > MAXD)
            return culamp_set_error(h, CULAMP_ERR_UNSUPPORTED, "instance %d: d=%d outside [1, %d]", i, u.d, MAXD);
        Inst &I = X.in[i];
        I.n = (int)u.n;
        I.m = (int)u.m;
        I.d = u.d;
        if (feat_np > 0 && I.d >= FEAT_MIN_D && X.pm_iter == P_SQ) I.cls = -1;
        else I.cls = (I.d <= MAXD_PACKED) ? I.d : 0;
        I.xo = xo; I.yo = yo; I.no = no; I.mo = mo;
        xo += (size_t)I.n * I.d;
        yo += (size_t)I.m * I.d;
        no += (size_t)I.n;
        mo += (size_t)I.m;
        if (I.cls < 0) {
            X.np = feat_np;
            I.fxo = fxo; I.fyo = fyo;
            fxo += feat_piece_elems(I.n, I.d, feat_np);
            fyo += feat_piece_elems(I.m, I.d, feat_np);
        }
        X.total_pairs += (double)I.n * (double)I.m;
        sig.push_back(((unsigned long long)I.n << 40) ^ ((unsigned long long)I.m << 12) ^ (unsigned long long)I.d);
    }
    const int sms = h->sm_count;
    const std::vector<int> tpsms = {2, 4, 8, 16, 32, 64};
    const std::vector<int> tpus = {4, 16};
    size_t parto = 0, ticko = 0, blko = 0;
    for (Inst &I : X.in) {
        scratch_need(I, sms);
        I.parto = parto; I.ticko = ticko; I.blko = blko;
        parto += I.part_need;
        ticko += I.tick_need;
        blko += I.blk_need;
    }

    // ---- workspace (grow-only)
    cudaError_t e = cudaSuccess;
    auto R = [&](DevBuf &b, size_t bytes, bool zero = false) {
        if (e == cudaSuccess) e = b.reserve(bytes > 0 ? bytes : 8, zero);
    };
    R(B.X, xo * sizeof(double));
    R(B.Y, yo * sizeof(double));
    R(B.r, no * sizeof(double));
    R(B.c, mo * sizeof(double));
    R(B.phi, no * sizeof(double));
    R(B.psi, mo * sizeof(double));
    R(B.ctl, (size_t)count * sizeof(Ctl));
    R(B.ctl2, (size_t)count * sizeof(Ctl));
    R(B.part, parto * sizeof(double));
    R(B.tickets, ticko * sizeof(unsigned), true);
    R(B.blk, blko * sizeof(double));
    R(B.err, 16, true);
    R(B.pairs, (size_t)count * sizeof(double));
    R(B.active, (size_t)count * sizeof(int));
    if (X.np > 0) {
        R(B.fx, fxo * sizeof(uint16_t));
        R(B.fy, fyo * sizeof(uint16_t));
        R(B.fxn, no * sizeof(double));
        R(B.fyn, mo * sizeof(double));
    }
    if (e != cudaSuccess) return culamp_set_error(h, CULAMP_ERR_ALLOC, "batch workspace: %s", cudaGetErrorString(e));
    // the tickets must start at zero for this batch's layout
    BT_TRY(h, cudaMemsetAsync(B.tickets.ptr, 0, ticko * sizeof(unsigned), st));
    std::vector<double> pairs(count);
    for (int i = 0; i < count; ++i) pairs[i] = (double)X.in[i].n * (double)X.in[i].m;
    BT_TRY(h, cudaMemcpyAsync(B.pairs.ptr, pairs.data(), count * sizeof(double), cudaMemcpyHostToDevice, st));

    // ---- stage inputs
    for (int i = 0; i < count; ++i) {
        const Inst &I = X.in[i];
        const culamp_instance &u = inst[i];
        BT_TRY(h, cudaMemcpyAsync(B.X.as<double>() + I.xo, u.x, (size_t)I.n * I.d * sizeof(double), cudaMemcpyDeviceToDevice, st));
        BT_TRY(h, cudaMemcpyAsync(B.Y.as<double>() + I.yo, u.y, (size_t)I.m * I.d * sizeof(double), cudaMemcpyDeviceToDevice, st));
        BT_TRY(h, cudaMemcpyAsync(B.r.as<double>() + I.no, u.r, (size_t)I.n * sizeof(double), cudaMemcpyDeviceToDevice, st));
        BT_TRY(h, cudaMemcpyAsync(B.c.as<double>() + I.mo, u.c, (size_t)I.m * sizeof(double), cudaMemcpyDeviceToDevice, st));
        if (I.cls < 0) {
            BT_TRY(h, feat_prepare(B.fx.as<uint16_t>() + I.fxo, B.fxn.as<double>() + I.no, B.X.as<double>() + I.xo, I.n, I.d, X.np, st));
            BT_TRY(h, feat_prepare(B.fy.as<uint16_t>() + I.fyo, B.fyn.as<double>() + I.mo, B.Y.as<double>() + I.yo, I.m, I.d, X.np, st));
        }
    }
    std::vector<int> all(count);
    for (int i = 0; i < count; ++i) all[i] = i;

    // ---- shape choice on the whole batch (cached per signature)
    double tune_ms = 0.0;
    int tpsm = B.tuned_tpsm, tpu = B.tuned_tpu;
    if (B.tuned_sig != sig || tpsm == 0) {
        float best = 1e30f;
        bool any_feat = X.np > 0, any_pair = false;
        for (const Inst &I : X.in) any_pair |= I.cls >= 0;
        const std::vector<int> c1 = any_pair ? tpsms : std::vector<int>{4};
        const std::vector<int> c2 = any_feat ? tpus : std::vector<int>{4};
        // two rounds over the candidates, each keeping its faster time: the
        // first round also brings the clocks up from idle, which would
        // otherwise favour whichever candidates come last
        std::vector<float> cand_ms(c1.size() * c2.size(), 1e30f);
        for (int round = 0; round < 2; ++round) {
            size_t k = 0;
            for (int a : c1)
                for (int b : c2) {
                    float ms = 0.f;
                    const Plan pl = make_plan(X, a, b, sms, all, X.total_pairs);
                    int s = time_plan(X, pl, args, 3, st, &ms);
                    if (s) return s;
                    tune_ms += ms;
                    cand_ms[k] = std::min(cand_ms[k], ms);
                    ++k;
                }
        }
        for (float ms : cand_ms) best = std::min(best, ms);
        // The timed iterations are the first ones, with every instance running;
        // later phases run fewer instances, and there more CTAs per SM keep the
        // GPU busier. Among candidates within TUNE_SLACK of the fastest, take
        // the one with the most CTAs per SM (measured on 512 uneven instances:
        // 2, 4, 8, 16, 32, 64 CTAs per SM -> 617, 605, 591-599, 574-581, 568,
        // 536 ms per solve, all within noise of each other in the tuning
        // iterations; 128 gave 535 ms for more tuning time).
        constexpr float TUNE_SLACK = 1.03f;
        float pick = 1e30f;
        tpsm = 0;
        tpu = 0;
        for (size_t i = 0; i < c1.size(); ++i)
            for (size_t j = 0; j < c2.size(); ++j) {
                const float ms = cand_ms[i * c2.size() + j];
                if (ms > best * TUNE_SLACK) continue;
                if (c1[i] > tpsm || (c1[i] == tpsm && ms < pick)) { tpsm = c1[i]; tpu = c2[j]; pick = ms; }
            }
        B.tuned_sig = sig;
        B.tuned_tpsm = tpsm;
        B.tuned_tpu = tpu;
    }
    // device time from here: W_inf passes, then the solve loop
    BT_TRY(h, cudaEventRecord(B.ev0, st));
    int s = reset_state(X, args, frequency, st);
    if (s) return s;

    // ---- the solve, in phases: each phase is one graph launch over the
    // instances still running, until their work has halved; the next phase
    // re-plans the survivors with finer column splits.
    std::vector<int> act = all;
    std::vector<Ctl> cs(count);
    int launches = 0, unroll = 1, phases = 0;
    while (!act.empty()) {
        double apairs = 0.0;
        for (int i : act) apairs += pairs[i];
        const Plan pl = make_plan(X, tpsm, tpu, sms, act, apairs);
        s = upload_plan(X, pl, st);
        if (s) return s;
        BT_TRY(h, cudaMemcpyAsync(B.active.ptr, act.data(), act.size() * sizeof(int), cudaMemcpyHostToDevice, st));
        int nl = 0;
        for (const auto *gs : {&pl.k1, &pl.k2, &pl.k3}) nl += (int)gs->size();
        launches = std::max(launches, nl);
        unroll = std::max(1, std::min(16, (int)std::ceil(200.0 / (apairs * 2.0 / 1.0e6 + 6.0 * nl))));
        const double min_pairs = act.size() > 1 ? 0.5 * apairs : 0.0;
        if (flags & CULAMP_FLAG_NO_GRAPH) {
            for (long long it = 0; it < args->itermax + 2; ++it) {
                BT_TRY(h, launch_groups(X, pl.k1, st));
                BT_TRY(h, launch_groups(X, pl.k2, st));
                BT_TRY(h, launch_groups(X, pl.k3, st));
                BT_TRY(h, cudaMemcpyAsync(cs.data(), B.ctl.ptr, (size_t)count * sizeof(Ctl), cudaMemcpyDeviceToHost, st));
                BT_TRY(h, cudaStreamSynchronize(st));
                double run = 0.0;
                for (int i : act) run += cs[i].stop ? 0.0 : pairs[i];
                if (run <= min_pairs) break;
            }
        } else {
            cudaGraphExec_t ex = nullptr;
            s = build_graph(X, pl, unroll, (int)act.size(), min_pairs, &ex);
            if (s) return s;
            const cudaError_t le = cudaGraphLaunch(ex, st);
            const cudaError_t se = cudaStreamSynchronize(st);
            cudaGraphExecDestroy(ex);
            BT_TRY(h, le);
            BT_TRY(h, se);
        }
        ++phases;
        BT_TRY(h, cudaMemcpyAsync(cs.data(), B.ctl.ptr, (size_t)count * sizeof(Ctl), cudaMemcpyDeviceToHost, st));
        int errv = 0;
        BT_TRY(h, cudaMemcpyAsync(&errv, B.err.ptr, sizeof(int), cudaMemcpyDeviceToHost, st));
        BT_TRY(h, cudaStreamSynchronize(st));
        std::vector<int> next;
        for (int i : act)
            if (!cs[i].stop) next.push_back(i);
        if (errv || next.size() == act.size()) break;   // a wait gave up, or no progress is possible
        act.swap(next);
    }
    BT_TRY(h, cudaEventRecord(B.ev1, st));

    // ---- final residual and transport cost of every instance (FIN_SUMS), on
    // fresh copies of the control blocks (the loop's are all stopped)
    BT_TRY(h, cudaMemcpyAsync(cs.data(), B.ctl.ptr, (size_t)count * sizeof(Ctl), cudaMemcpyDeviceToHost, st));
    BT_TRY(h, cudaStreamSynchronize(st));
    std::vector<Ctl> c2 = cs;
    for (Ctl &c : c2) { c.stop = 0; c.error = 0; c.log = nullptr; c.log_cap = 0; }
    BT_TRY(h, cudaMemcpyAsync(B.ctl2.ptr, c2.data(), (size_t)count * sizeof(Ctl), cudaMemcpyHostToDevice, st));
    {
        const Plan pf = make_plan(X, tpsm, tpu, sms, all, X.total_pairs);
        s = upload_plan(X, pf, st);
        if (s) return s;
        BT_TRY(h, launch_groups(X, pf.kf, st));
    }
    BT_TRY(h, cudaMemcpyAsync(c2.data(), B.ctl2.ptr, (size_t)count * sizeof(Ctl), cudaMemcpyDeviceToHost, st));
    int err = 0;
    BT_TRY(h, cudaMemcpyAsync(&err, B.err.ptr, sizeof(int), cudaMemcpyDeviceToHost, st));
    for (int i = 0; i < count; ++i) {
        const Inst &I = X.in[i];
        BT_TRY(h, cudaMemcpyAsync(inst[i].phi, B.phi.as<double>() + I.no, (size_t)I.n * sizeof(double), cudaMemcpyDeviceToDevice, st));
        BT_TRY(h, cudaMemcpyAsync(inst[i].psi, B.psi.as<double>() + I.mo, (size_t)I.m * sizeof(double), cudaMemcpyDeviceToDevice, st));
    }
    BT_TRY(h, cudaStreamSynchronize(st));
    float ms = 0.f;
    BT_TRY(h, cudaEventElapsedTime(&ms, B.ev0, B.ev1));
    bool bound_hit = false;
    if (stats) {
        for (int i = 0; i < count; ++i) {
            culamp_batch_stats &o = stats[i];
            std::memset(&o, 0, sizeof(o));
            o.iterations = cs[i].iter;
            o.num_iter = cs[i].num_iter;
            o.residual = c2[i].sums[0];
            o.objective = c2[i].sums[1];
            o.winf = cs[i].winf;
            o.stopped = cs[i].stop_reason;
            o.status = cs[i].error ? CULAMP_ERR_DEVICE_TIMEOUT : CULAMP_OK;
        }
    }
    for (const Ctl &c : cs) bound_hit |= c.error != 0;
    if (info) {
        std::memset(info, 0, sizeof(*info));
        info->elapsed_ms = ms;
        info->tune_ms = tune_ms;
        info->target_ctas_per_sm = tpsm;
        info->feat_tiles_per_unit = tpu;
        info->unroll = unroll;
        info->launches_per_iteration = launches;
        info->phases = phases;
    }
    if (err) return culamp_set_error(h, CULAMP_ERR_DEVICE_TIMEOUT, "a tensor-core pass gave up waiting");
    if (bound_hit) return culamp_set_error(h, CULAMP_ERR_DEVICE_TIMEOUT, "loop control bound hit");
    return CULAMP_OK;
}
