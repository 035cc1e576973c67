// engine.cuh -- the pair-reduction tile engine of libculamp_b200 (sm_100a).
//
// Every hot pass of CuLAMP.jl's kernelized solvers is one reduction over all
// (row o, column k) pairs of an on-the-fly cost C(x_o, y_k):
//
//   LSE_o  = log sum_k exp(alpha * C(x_o, y_k) + beta * pot_k)      (Sinkhorn / LAMP)
//   MAX_o  = max_k C(x_o, y_k)                                       (W_inf pre-pass)
//   MIN_o  = min_k C(x_o, y_k) + 2 W_inf theta_k                     (LAMP eta=0 dual)
//
// followed by a per-row epilogue (potential update, residual, LAMP mirror step)
// and optional FP64 scalar reductions feeding the solver's convergence control.
//
// Design (B200):
//  * A CTA owns ROWS = TPB*RPT output rows (RPT rows per thread, registers) and a
//    contiguous column slice; column points + their potentials are staged through
//    shared memory in CHUNK-column tiles (coalesced global loads, broadcast LDS).
//  * Precision ("chosen form"): the exponent alpha*C + beta*pot is formed in FP64.
//    For p=2 it uses C = |x|^2 + |y|^2 - 2 x.y with the column term folded into a
//    per-column constant, so a pair costs 3 DFMA (d=3). The running row max is
//    tracked in FP64 per KC-column sub-chunk; only the max-shifted exponent is
//    rounded to FP32 and exponentiated on the MUFU pipe (ex2), and the sum is
//    accumulated with compensated (Kahan) FP32 additions. Potentials, W_inf and
//    all scalar reductions are FP64.
//  * When one CTA row block would leave SMs idle, the column range is split over
//    `splits` CTAs; the last CTA of a row block (atomic ticket) merges the partial
//    (max, sum, moment) triples in a fixed order (deterministic) and runs the epilogue.
//  * The last epilogue CTA of the grid runs the "finish" step: ordered FP64 sums of
//    the block partials and the solver's iteration control (iteration counter,
//    check cadence, tolerance test, itermax / tmax), so a whole solve runs from a
//    CUDA graph with no host synchronisation per iteration.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "../../include/culamp.h"

namespace culamp_dev {

constexpr int TPB = 128;          // threads per CTA
constexpr int RPT = 1;            // output rows per thread, small-problem / generic variants
                                  // (measured: 1 row beats 2 by 14 % on a 4096^2 Sinkhorn solve --
                                  // twice the warps for these latency-bound passes)
constexpr int RPT_BIG = 8;        // output rows per thread, packed log-sum-exp, large n
constexpr int RPT_MID = 4;        // output rows per thread, packed log-sum-exp, mid-size n
constexpr int ROWS = TPB * RPT;   // output rows per CTA (RPT variant)
constexpr int CHUNK = 256;        // columns per shared-memory tile (d <= 3)
constexpr int KC = 4;             // columns per online-max sub-chunk
constexpr int MAXD_PACKED = 3;    // packed fast path: d <= 3
constexpr int MAXD = 256;         // generic path: d <= 256
constexpr int CHUNK_G = 32;       // columns per tile on the generic path
constexpr double LOG2E = 1.4426950408889634074;
constexpr double LN2 = 0.69314718055994530942;

enum PMode { P_L1 = 0, P_SQ = 1, P_INF = 2, P_GEN = 3 };
enum Acc { ACC_LSE = 0, ACC_MAX = 1, ACC_MIN = 2 };

// How alpha / beta of the exponent are obtained at kernel entry.
enum CoefMode {
    COEF_FIXED = 0,      // alpha, beta given by value
    COEF_SK = 1,         // alpha = -1/(ctl.eta * ctl.winf), beta = 1
    COEF_SPP_CUR = 2,    // eta_t, s = ctl.eta_t, ctl.s_t: alpha = -s/(2 W eta_t), beta = -1/eta_t
    COEF_SPP_NEXT = 3,   // same with ctl.eta_next, ctl.s_next
    COEF_SPP_DUAL = 4,   // reg = ctl.eta_lamp, s = 1
};

// Per-row epilogues.
enum Epi {
    EPI_SK_ROW = 0,      // out = log(marg) - L                          (a1)
    EPI_SK_RESID = 1,    // res = marg - exp(rowpot + L); cost = mass*E[C] (a3)
    EPI_LOGZ = 2,        // out = L; aux = log(marg) - L (if marg)       (a7)
    EPI_SPP_COL = 3,     // res = exp(-rowpot/eta_t + L); cost = res*E[C] (a8) [+ LAMP step]
    EPI_RAW = 4,         // out = value (max / min reductions)            (a6, a9)
    EPI_SK_SYM = 5,      // symmetric step: out = (f + log(marg) - L)/2; res at f; aux = L
};

enum LampStep { LAMP_NONE = 0, LAMP_A = 1, LAMP_B = 2 };

enum Finish {
    FIN_NONE = 0,
    FIN_SUMS = 1,        // just store the ordered scalar sums into ctl->sums
    FIN_SK_ITER = 2,     // Sinkhorn column pass: iteration bookkeeping
    FIN_SK_CHECK = 3,    // Sinkhorn residual pass: tolerance test
    FIN_LAMP_Z = 4,      // LAMP logZ(nu) pass: sum r.logZ
    FIN_LAMP_A = 5,      // LAMP column pass after infeas(nu)
    FIN_LAMP_DUAL = 6,   // LAMP dual pass: primal/dual, log, tolerance test
    FIN_LAMP_B = 7,      // LAMP column pass after infeas(nu_bar): commit eta_t, iteration
    FIN_MAXCOST = 8,     // W_inf = max of row maxima into ctl->winf
    FIN_SK_SYM = 9,      // symmetric Sinkhorn pass: tolerance test, iteration bookkeeping
};

// Precision ladder stall test: the FP32-exponent phase ends after this many
// consecutive checks without a new lowest residual (at the FP32 floor the
// residual wanders up and down; LAMP's also rises now and then early on).
constexpr int LADDER_PATIENCE = 3;

// One FP64 check of the FP32-exponent phase: ends the phase once the residual
// is within ladder_switch, or has not improved for LADDER_PATIENCE checks.
__device__ __forceinline__ void ladder_check(int &phase, double &best, int &bad, double l1, double sw) {
    if (!phase) return;
    if (l1 < best) { best = l1; bad = 0; }
    else bad += 1;
    if (l1 <= sw || bad >= LADDER_PATIENCE) phase = 0;
}

// Gate: when the kernel runs.
enum Gate { GATE_ALWAYS = 0, GATE_CHECK = 1, GATE_NOCHECK = 2 };

// Precision-ladder phase in which a pass runs (independent of the gate).
enum Phase {
    PHASE_ANY = 0,
    PHASE_FP32 = 1,      // runs while ctl->fp32_phase is set
    PHASE_FP64 = 2,      // runs once ctl->fp32_phase is cleared
};

// Device-resident solver state. All fields written by device code are read by
// later kernels only (stream order), never by concurrently running CTAs.
struct Ctl {
    long long iter;             // completed iterations
    long long itermax;
    long long frequency;
    long long num_iter;         // the reference's num_iter counter
    int stop;                   // kernels return immediately when set
    int stop_reason;            // 1 tolerance, 2 itermax, 3 tmax
    int do_check;               // the current iteration runs the check pass(es)
    int check_enabled;          // LAMP: verbose || CHECK_ALWAYS
    int marginal_only;          // LAMP: tolerance test ignores the gap
    int pending_stop;           // stop after this iteration's check (itermax/tmax)
    unsigned long long t_start_ns;
    double tmax_s;
    double epsilon;
    double eta;                 // Sinkhorn eta_p of the current stage
    double winf;
    double residual, objective, dualval;
    // LAMP
    double eta_lamp;            // eta = eta_p / (2 W_inf)
    double eta_t, s_t, eta_next, s_next, tau_p;
    double hr;                  // eta * sum(r log r)
    double sum_r_logz, sum_res_c, sum_cost, sum_res_nu, sum_r_dual, sum_c_theta;
    double primal, dual;
    // convergence log (device buffer)
    long long log_rows, log_cap;
    culamp_log_row *log;
    double sums[4];             // FIN_SUMS output
    int error;                  // device-side error code (bounded waits etc.)
    int fp32_phase;             // precision ladder: FP32-exponent iterations still active
    double ladder_switch;       // ... until a check's L1 residual falls to this
    double ladder_prev;         // the lowest check residual of the FP32 phase (stall test)
    int ladder_bad;             // checks since that lowest residual
    long long loops;            // WHILE-body executions (independent loop bound)
};

struct PassParams {
    const double *X;            // output-row points, point-major, ld = d
    const double *Y;            // column points
    int n, m, d;
    double pexp;                // exponent for P_GEN
    const double *ctr;          // centring point (d values) for the p=2 expansion; may be null
    int epi;                    // Epi
    int coef_mode;
    double alpha, beta;         // COEF_FIXED
    const double *colpot;       // beta * colpot_k enters the exponent; may be null
    int colpot_unit;            // colpot enters with coefficient 1 (beta then scales rowpot)
    const double *rowpot;       // per-row potential (EPI_SK_RESID: phi, EPI_SPP_COL: theta/nu)
    const double *marg;         // row marginal (EPI_SK_ROW / EPI_SK_RESID / EPI_LOGZ aux)
    double *out;                // EPI_SK_ROW / EPI_LOGZ / EPI_RAW / EPI_SPP_COL res / EPI_SK_RESID res
    double *out2;               // cost output (may be null)
    double *aux;                // EPI_LOGZ: log(marg) - L (may be null); EPI_SK_ROW: previous value backup
    double minmax_scale;        // ACC_MIN: multiplier of colpot (2 W_inf)
    // LAMP step fused into EPI_SPP_COL
    int lamp_step;
    double *theta, *thetab, *nu, *nub;
    const double *cvec, *eta_mu_i;
    double eta_mu_exp, minv, maxv;
    // moments
    int want_moment;            // 1: accumulate the softmax-weighted cost moment (MOM kernels)
    int use_ref;                // 1: fixed-reference fast path, reference = the row's previous LSE
    int fp32;                   // 1 (with use_ref, p = 2, d <= 3): its exponent in FP32 (FORM_FP32)
    // gating and control
    int gate;
    int phase;                  // Phase
    int finish;
    Ctl *ctl;
    // split-column scratch
    int splits;
    int cols_per_split;
    double *part;               // [splits][n][3] (max, sum, moment)
    unsigned int *rb_ticket;    // [row blocks]
    unsigned int *grid_ticket;  // [1]
    double *blk;                // [row blocks][4] block partial scalars
    // feature-cost path (p = 2, tensor cores): both clouds pre-split into bf16
    // pieces in the tile layout the MMA reads; null = the FP64 pair loops
    const uint16_t *fx;         // pieces of the output-row points
    const uint16_t *fy;         // pieces of the column points
    const double *xn, *yn;      // squared norms |x|^2, |y|^2 (FP64)
    int fkb;                    // 64-wide K blocks per point
    int fpieces;                // bf16 pieces per value: 2 (BF16x3) or 3 (BF16x6)
    // batched launches: this instance's row blocks (pair passes) and work-unit
    // geometry (feature passes: row tiles, column tiles, slices, tiles per slice)
    int nrb;
    int ft_rtiles, ft_ctiles, ft_splits, ft_tps;
    int ft_rblk, ft_cblk;       // packed 128-point blocks of the row / column clouds
};

// 2^x on the MUFU pipe (PTX ex2.approx.ftz.f32: relative error ~2^-22, results
// below 2^-126 flush to zero -- negligible next to the max-shifted term 1).
__device__ __forceinline__ float ex2_approx(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Exponent coefficients (natural-log units) for this launch.
__device__ __forceinline__ void resolve_coefs(const PassParams &P, double &alpha, double &beta) {
    const Ctl *c = P.ctl;
    switch (P.coef_mode) {
        case COEF_SK:
            alpha = -1.0 / (c->eta * c->winf);
            beta = 1.0;
            break;
        case COEF_SPP_CUR:
        case COEF_SPP_NEXT:
        case COEF_SPP_DUAL: {
            double et, st;
            if (P.coef_mode == COEF_SPP_CUR) { et = c->eta_t; st = c->s_t; }
            else if (P.coef_mode == COEF_SPP_NEXT) { et = c->eta_next; st = c->s_next; }
            else { et = c->eta_lamp; st = 1.0; }
            const double c1 = st / (2.0 * c->winf);
            const double invreg = 1.0 / et;
            alpha = -c1 * invreg;
            beta = -invreg;
            break;
        }
        default:
            alpha = P.alpha;
            beta = P.beta;
    }
}

template <int PM>
__device__ __forceinline__ double pair_cost_direct(const double *xr, const double *yk, int d, double pexp) {
    double acc = 0.0;
    if (PM == P_L1) {
        for (int k = 0; k < d; ++k) acc += fabs(xr[k] - yk[k]);
    } else if (PM == P_SQ) {
        for (int k = 0; k < d; ++k) { double t = xr[k] - yk[k]; acc = fma(t, t, acc); }
    } else if (PM == P_INF) {
        for (int k = 0; k < d; ++k) acc = fmax(acc, fabs(xr[k] - yk[k]));
    } else {
        for (int k = 0; k < d; ++k) acc += pow(fabs(xr[k] - yk[k]), pexp);
    }
    return acc;
}

// Kahan-compensated FP32 accumulation of exp terms.
struct KSum {
    float s, c;
    __device__ __forceinline__ void add(float v) {
        float y = v - c;
        float t = s + y;
        c = (t - s) - y;
        s = t;
    }
    __device__ __forceinline__ void scale(float f) { s *= f; c *= f; }
};

// ---------------------------------------------------------------------------
// Main tile loop. D > 0: packed compile-time dimension (<= 3); D == 0: generic.
// Produces per-row (M, S, MOM): LSE2 = M + log2(S) in log2 units of the shifted
// exponent, or the max/min value in M for ACC_MAX/ACC_MIN.
template <int PM, int D, int ACC, bool MOM>
__device__ __forceinline__ void tile_reduce(const PassParams &P, double alpha, double beta,
                                            int row_base, int cbeg, int cend, double *smem,
                                            double (&Mo)[RPT], double (&So)[RPT],
                                            double (&MOMo)[RPT], double (&Ho)[RPT]) {
    const int tid = threadIdx.x;
    const int d = (D > 0) ? D : P.d;
    const bool expand = (ACC == ACC_LSE) && (PM == P_SQ);
    const double a2 = alpha * LOG2E;          // log2-scaled cost multiplier
    const double b2 = beta * LOG2E;
    const int CH = (D > 0) ? CHUNK : CHUNK_G;
    const int LD = (D > 0) ? 4 : (P.d + 1);   // doubles per staged column

    double ctr[(D > 0) ? D : 1];
    if (D > 0) {
#pragma unroll
        for (int k = 0; k < (D > 0 ? D : 1); ++k) ctr[k] = P.ctr ? P.ctr[k] : 0.0;
    }

    // row state
    double xs[RPT][(D > 0) ? D : 1];          // centred row point (packed path)
    double xt[RPT][(D > 0) ? D : 1];          // -2 a2 (x - ctr) for the p=2 expansion
    int rows[RPT];
    bool rvalid[RPT];
    double M[RPT];
    KSum S[RPT];
    float MOMs[RPT];
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
        rows[r] = row_base + tid + r * TPB;
        rvalid[r] = rows[r] < P.n;
        M[r] = (ACC == ACC_MIN) ? INFINITY : -INFINITY;
        S[r].s = 0.f; S[r].c = 0.f;
        MOMs[r] = 0.f;
        Ho[r] = 0.0;
        if (D > 0) {
            double h = 0.0;
#pragma unroll
            for (int k = 0; k < (D > 0 ? D : 1); ++k) {
                double v = rvalid[r] ? (P.X[(size_t)rows[r] * D + k] - ctr[k]) : 0.0;
                xs[r][k] = v;
                xt[r][k] = -2.0 * a2 * v;
                h = fma(v, v, h);
            }
            Ho[r] = expand ? a2 * h : 0.0;
        }
    }

    for (int c0 = cbeg; c0 < cend; c0 += CH) {
        __syncthreads();
        // stage CH columns: (y - ctr)[d], g
        for (int q = tid; q < CH; q += TPB) {
            const int j = c0 + q;
            double *dst = smem + (size_t)q * LD;
            const bool ok = j < cend;
            double g;
            if (D > 0) {
                double yy = 0.0;
#pragma unroll
                for (int k = 0; k < (D > 0 ? D : 1); ++k) {
                    double v = ok ? (P.Y[(size_t)j * D + k] - ctr[k]) : 0.0;
                    dst[k] = v;
                    yy = fma(v, v, yy);
                }
#pragma unroll
                for (int k = (D > 0 ? D : 1); k < 3; ++k) dst[k] = 0.0;
                double pot = (ok && P.colpot) ? P.colpot[j] : 0.0;
                if (ACC == ACC_LSE) {
                    const double cb = P.colpot_unit ? LOG2E : b2;
                    g = (cb == 0.0) ? 0.0 : cb * pot;             // beta = 0 tolerates infinite pots
                    if (expand) g += a2 * yy;
                    if (!ok) g = -INFINITY;
                } else if (ACC == ACC_MIN) {
                    g = ok ? P.minmax_scale * pot : INFINITY;
                } else {
                    g = ok ? 0.0 : -INFINITY;
                }
                dst[3] = g;
            } else {
                for (int k = 0; k < d; ++k) dst[k] = ok ? P.Y[(size_t)j * d + k] : 0.0;
                double pot = (ok && P.colpot) ? P.colpot[j] : 0.0;
                const double cb = P.colpot_unit ? LOG2E : b2;
                if (ACC == ACC_LSE) g = ok ? ((cb == 0.0) ? 0.0 : cb * pot) : -INFINITY;
                else if (ACC == ACC_MIN) g = ok ? P.minmax_scale * pot : INFINITY;
                else g = ok ? 0.0 : -INFINITY;
                dst[d] = g;
            }
        }
        __syncthreads();
        const int ncols = min(CH, cend - c0);
        const int nsub = (ncols + KC - 1) / KC;
        for (int sc = 0; sc < nsub; ++sc) {
            double t[RPT][KC];
            float cst[RPT][KC];
#pragma unroll
            for (int kk = 0; kk < KC; ++kk) {
                const int q = sc * KC + kk;   // q < CH always (CH % KC == 0); padded cols carry g = +-inf
                const double *col = smem + (size_t)q * LD;
                if (D > 0) {
                    const double g = col[3];
                    double yv[(D > 0) ? D : 1];
#pragma unroll
                    for (int k = 0; k < (D > 0 ? D : 1); ++k) yv[k] = col[k];
#pragma unroll
                    for (int r = 0; r < RPT; ++r) {
                        double v;
                        float cf = 0.f;
                        if (expand) {
                            v = g;
#pragma unroll
                            for (int k = 0; k < (D > 0 ? D : 1); ++k) v = fma(xt[r][k], yv[k], v);
                            if (MOM) {
                                double cc = 0.0;
#pragma unroll
                                for (int k = 0; k < (D > 0 ? D : 1); ++k) { double df = xs[r][k] - yv[k]; cc = fma(df, df, cc); }
                                cf = (float)cc;
                            }
                        } else {
                            const double cc = pair_cost_direct<PM>(xs[r], yv, D, P.pexp);
                            if (ACC == ACC_LSE) v = fma(cc, a2, g);
                            else if (ACC == ACC_MIN) v = cc + g;
                            else v = cc + g;   // g = 0 or -inf (padding)
                            cf = (float)cc;
                        }
                        t[r][kk] = v;
                        cst[r][kk] = cf;
                    }
                } else {
                    const double g = col[d];
#pragma unroll
                    for (int r = 0; r < RPT; ++r) {
                        double v, cc = 0.0;
                        if (rvalid[r]) {
                            const double *xr = P.X + (size_t)rows[r] * d;
                            double acc = 0.0;
                            for (int k = 0; k < d; ++k) {
                                double df = xr[k] - col[k];
                                if (PM == P_L1) acc += fabs(df);
                                else if (PM == P_SQ) acc = fma(df, df, acc);
                                else if (PM == P_INF) acc = fmax(acc, fabs(df));
                                else acc += pow(fabs(df), P.pexp);
                            }
                            cc = acc;
                        }
                        if (ACC == ACC_LSE) v = fma(cc, a2, g);
                        else v = cc + g;
                        t[r][kk] = v;
                        cst[r][kk] = (float)cc;
                    }
                }
            }
#pragma unroll
            for (int r = 0; r < RPT; ++r) {
                if (ACC == ACC_LSE) {
                    double cm = t[r][0];
#pragma unroll
                    for (int kk = 1; kk < KC; ++kk) cm = fmax(cm, t[r][kk]);
                    if (cm == -INFINITY || cm != cm) continue;
                    if (cm > M[r]) {
                        const float f = ex2_approx((float)(M[r] - cm));
                        S[r].scale(f);
                        if (MOM) MOMs[r] *= f;
                        M[r] = cm;
                    }
#pragma unroll
                    for (int kk = 0; kk < KC; ++kk) {
                        const float e = ex2_approx((float)(t[r][kk] - M[r]));
                        S[r].add(e);
                        if (MOM) MOMs[r] = fmaf(e, cst[r][kk], MOMs[r]);
                    }
                } else if (ACC == ACC_MAX) {
#pragma unroll
                    for (int kk = 0; kk < KC; ++kk) M[r] = fmax(M[r], t[r][kk]);
                } else {
#pragma unroll
                    for (int kk = 0; kk < KC; ++kk) M[r] = fmin(M[r], t[r][kk]);
                }
            }
        }
    }
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
        Mo[r] = M[r];
        So[r] = (double)S[r].s + (double)(-S[r].c);
        MOMo[r] = (double)MOMs[r];
    }
}

// Merge (M, S, MOM) triples: value = 2^M * S (log2 units).
__device__ __forceinline__ void merge_lse(double &M, double &S, double &MOM, double M2, double S2,
                                          double MOM2) {
    if (M2 == -INFINITY || S2 == 0.0) return;
    if (M == -INFINITY || S == 0.0) { M = M2; S = S2; MOM = MOM2; return; }
    if (M2 == M) {   // fixed-reference partials share one max: exp2(0) = 1 exactly
        S += S2;
        MOM += MOM2;
        return;
    }
    if (M2 > M) {
        const double f = exp2(M - M2);
        S = S * f + S2;
        MOM = MOM * f + MOM2;
        M = M2;
    } else {
        const double f = exp2(M2 - M);
        S += S2 * f;
        MOM += MOM2 * f;
    }
}

// tanh mirror step of update_theta_residual (MirrorProx.jl:159-180) with W_inf = 1
// as the kernel driver calls it (MirrorProxKernel.jl:1104,1114).
__device__ __forceinline__ double theta_step(double th0, double res, double c, double emu,
                                             double eta_mu_exp, int adjust, double minv,
                                             double maxv, double winf) {
    const double difference = 2.0 * winf * (res - c) / emu;
    const double maxval = fmax(difference, -difference);
    const double expv = exp(difference - maxval) * pow((th0 + 1.0) / (1.0 - th0), 1.0 - eta_mu_exp);
    const double em = exp(-maxval);
    double t = (expv - em) / (expv + em);
    if (adjust) t = fmin(fmax(t, minv), maxv);
    return t;
}

// LAMP eta_t recursion eta_t <- 1/(tau_p + (1/eta_t)(1 - eta)) and s recursion,
// evaluated without contraction so it matches a plain IEEE evaluation.
__device__ __forceinline__ void lamp_next(double eta_t, double s_t, double tau_p, double eta,
                                          double &eta_n, double &s_n) {
    const double inv = __drcp_rn(eta_t);
    eta_n = __ddiv_rn(1.0, __dadd_rn(tau_p, __dmul_rn(inv, __dsub_rn(1.0, eta))));
    s_n = __dadd_rn(__dmul_rn(__dsub_rn(1.0, eta_n), s_t), eta_n);
}

__device__ __forceinline__ void put_log(Ctl *c, double it, double infeas, double obj, double primal,
                                        double dual) {
    if (!c->log || c->log_rows >= c->log_cap) return;
    culamp_log_row *r = &c->log[c->log_rows++];
    r->time_s = (double)(globaltimer_ns() - c->t_start_ns) * 1e-9;
    r->iter = it;
    r->infeas = infeas;
    r->ot_objective = obj;
    r->primal = primal;
    r->dual = dual;
}

// Iteration bookkeeping shared by the Sinkhorn and LAMP control steps.
__device__ __forceinline__ void end_of_iteration(Ctl *c) {
    c->iter += 1;
    if (c->iter >= c->itermax) c->pending_stop = 2;
    else if ((double)(globaltimer_ns() - c->t_start_ns) * 1e-9 > c->tmax_s) c->pending_stop = 3;
}

static __device__ __noinline__ void run_finish(const PassParams &P, const double (&tot)[4]) {
    Ctl *c = P.ctl;
    switch (P.finish) {
        case FIN_SUMS:
            for (int k = 0; k < 4; ++k) c->sums[k] = tot[k];
            break;
        case FIN_MAXCOST:
            c->winf = tot[0];
            break;
        case FIN_SK_ITER: {
            // after the psi update of iteration it = iter + 1; tot[0] = sum c.psi
            c->dualval = tot[0];
            end_of_iteration(c);
            c->do_check = ((c->iter - 1) % c->frequency) == 0;
            if (!c->do_check && c->pending_stop) { c->stop = 1; c->stop_reason = c->pending_stop; c->num_iter += 1; }
            else if (!c->do_check) c->num_iter += 1;
            break;
        }
        case FIN_SK_CHECK: {
            const double l1 = tot[0];
            c->residual = l1;
            c->objective = tot[1];
            // precision ladder: FP64 passes from here once the residual is near
            // the tolerance, or once the FP32-exponent iteration stops gaining
            // (its rounding floor lies above the tolerance)
            ladder_check(c->fp32_phase, c->ladder_prev, c->ladder_bad, l1, c->ladder_switch);
            put_log(c, (double)c->iter, l1, tot[1], nan(""), c->dualval + tot[2]);
            if (l1 <= c->epsilon / 6.0) { c->stop = 1; c->stop_reason = 1; }
            else {
                c->num_iter += 1;
                if (c->pending_stop) { c->stop = 1; c->stop_reason = c->pending_stop; }
            }
            break;
        }
        case FIN_SK_SYM: {
            // tot[0] = L1 row residual at the pass's input f, tot[2] = a.f. On
            // success f is final and iter counts the updates applied before it.
            const double l1 = tot[0];
            c->residual = l1;
            c->dualval = tot[2];
            if (c->log && (c->iter % c->frequency) == 0)
                put_log(c, (double)c->iter, l1, nan(""), nan(""), 2.0 * tot[2]);
            if (l1 <= c->epsilon / 6.0) { c->stop = 1; c->stop_reason = 1; }
            else {
                end_of_iteration(c);
                c->num_iter = c->iter;
                if (c->pending_stop) { c->stop = 1; c->stop_reason = c->pending_stop; }
            }
            break;
        }
        case FIN_LAMP_Z:
            c->sum_r_logz = tot[0];
            break;
        case FIN_LAMP_A: {
            c->sum_res_c = tot[0];
            c->sum_cost = tot[1];
            c->sum_res_nu = tot[2];
            double en, sn;
            lamp_next(c->eta_t, c->s_t, c->tau_p, c->eta_lamp, en, sn);
            c->eta_next = en;
            c->s_next = sn;
            break;
        }
        case FIN_LAMP_DUAL: {
            // MirrorProxKernel.jl:1084-1100
            const double q = c->eta_lamp / c->eta_t;
            const double primal = c->sum_cost * (1.0 - q) - q * c->sum_res_nu + q * c->sum_r_logz +
                                  2.0 * c->winf * c->sum_res_c;
            double dual;
            if (c->eta_lamp > 0) dual = -2.0 * c->eta_lamp * tot[0] - 2.0 * c->winf * c->sum_c_theta + 2.0 * c->hr;
            else dual = tot[0] - 2.0 * c->winf * c->sum_c_theta;
            c->primal = primal;
            c->dual = dual;
            c->residual = c->sum_res_c;
            // precision ladder, as in FIN_SK_CHECK, on the FP64 marginal residual
            ladder_check(c->fp32_phase, c->ladder_prev, c->ladder_bad, c->sum_res_c, c->ladder_switch);
            c->objective = c->sum_cost;
            put_log(c, (double)(c->iter + 1), c->sum_res_c, c->sum_cost, primal, dual);
            const bool gap_ok = c->marginal_only ? true : (primal - dual < c->epsilon / 6.0);
            if (gap_ok && c->sum_res_c < c->epsilon / 6.0) { c->stop = 1; c->stop_reason = 1; }
            break;
        }
        case FIN_LAMP_B: {
            c->eta_t = c->eta_next;
            c->s_t = c->s_next;
            end_of_iteration(c);
            c->num_iter = c->iter;
            c->do_check = c->check_enabled && ((c->iter % c->frequency) == 0);
            if (c->pending_stop) { c->stop = 1; c->stop_reason = c->pending_stop; }
            break;
        }
        default:
            break;
    }
}

// Block-wide FP64 sum of up to 4 values per thread; result valid in thread 0.
__device__ __forceinline__ void block_sum4(double (&v)[4], double *red) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        double x = v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        v[k] = x;
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0)
        for (int k = 0; k < 4; ++k) red[w * 4 + k] = v[k];
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 0; k < 4; ++k) {
            double s = 0.0;
            for (int ww = 0; ww < TPB / 32; ++ww) s += red[ww * 4 + k];
            v[k] = s;
        }
    }
}


// Block-wide FP64 max of one value; result valid in thread 0.
__device__ __forceinline__ double block_max1(double x, double *red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x = fmax(x, __shfl_down_sync(0xffffffffu, x, o));
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) red[w] = x;
    __syncthreads();
    if (threadIdx.x == 0)
        for (int ww = 1; ww < TPB / 32; ++ww) x = fmax(x, red[ww]);
    return x;
}

__device__ __forceinline__ void kahan_add(float &s, float &c, float v) {
    const float y = v - c;
    const float t = s + y;
    c = (t - s) - y;
    s = t;
}

// One column against R register-resident rows (packed d <= 3 log-sum-exp path).
// t = exponent in log2 units (FP64); f = t - M rounded to FP32; a new running
// max rescales the row's sums; e = 2^f on the MUFU pipe goes into an 8-term
// FP32 chunk sum (merged into a Kahan-compensated total every 8 columns).
template <int PM, int D, int R, bool MOM>
__device__ __forceinline__ void lse_step(const double4 col, const double (&xr)[R][D],
                                         const double (&xs)[(PM == P_SQ && MOM) ? R : 1][D],
                                         double a2, double pexp, double (&M)[R], float (&S)[R],
                                         float (&Cc)[R], float (&cs)[R], float (&mo)[R]) {
#pragma unroll
    for (int r = 0; r < R; ++r) {
        double t;
        float cf = 0.f;
        if (PM == P_SQ) {
            t = col.w;
            if (D >= 3) t = fma(xr[r][D >= 3 ? 2 : 0], col.z, t);
            if (D >= 2) t = fma(xr[r][D >= 2 ? 1 : 0], col.y, t);
            t = fma(xr[r][0], col.x, t);
            if (MOM) {
                const double yv[3] = {col.x, col.y, col.z};
                double cc = 0.0;
#pragma unroll
                for (int k = 0; k < D; ++k) {
                    const double df = xs[(PM == P_SQ && MOM) ? r : 0][k] - yv[k];
                    cc = fma(df, df, cc);
                }
                cf = (float)cc;
            }
        } else {
            const double yv[3] = {col.x, col.y, col.z};
            const double cc = pair_cost_direct<PM>(xr[r], yv, D, pexp);
            t = fma(cc, a2, col.w);
            if (MOM) cf = (float)cc;
        }
        float f = (float)(t - M[r]);
        if (f > 0.f) {
            const float sc = ex2_approx(-f);
            S[r] *= sc;
            Cc[r] *= sc;
            cs[r] *= sc;
            if (MOM) mo[r] *= sc;
            M[r] = t;
            f = 0.f;
        }
        const float e = ex2_approx(f);
        cs[r] += e;
        if (MOM) mo[r] = fmaf(e, cf, mo[r]);
    }
}

// ---------------------------------------------------------------------------
// Fixed-reference log-sum-exp (packed d <= 3, no moment).
//
// Each row carries a reference Mref (log2 units, the row's previous LSE). With
// x = t - Mref - 1, one DADD forms D = x + 1.5*2^20 (+2^-24 so the truncation
// below rounds). D's ulp is 2^-32, so for |x| < 2^19 its high word carries
// 2^19 + floor(x) in its low 20 bits and its low word is frac(x) * 2^32. Then
//   * k = floor(x) + FR_C0 is formed and clamped to [0, 126] by one integer
//     add + min-with-relu on the high word (IEEE bit patterns are monotone in
//     the value, so -inf and very negative x clamp to 0, +inf / NaN to 126);
//   * a funnel shift of the low word under 0x7F gives v = 1 + frac(x) (23 bits);
//   * ex2(v) lies in [2, 4) (exponent field 128); adding k to the exponent
//     field gives e = 2^(1 + frac(x) + k) = 2^(t - Mref) * 2^FR_C0: every term
//     is carried scaled by 2^FR_C0, exact for floor(x) in [-FR_C0, 126 - FR_C0],
//     one MUFU ex2 per pair.
// The terms of two rows (or, with one row per thread, of two columns) are
// summed with one packed FP32x2 add.
// No FP64->FP32 conversion, no FP64 min/max, no per-pair max test.
// A clamped-low term is carried as at most 4 (scaled), i.e. 2^(2 - FR_C0)
// relative to the reference. A column slice whose scaled partial sum exceeds
// 2^126 (a term clamped high, any term above the reference by >= 45, or a
// non-finite input) is recomputed by its CTA with tile_lse_packed; after the
// slices are merged, a row whose full LSE lies more than
// FR_C0 - 32 - log2(m) below its reference -- where the m clamped-low terms
// could reach 2^-30 of the row sum -- makes the merging CTA recompute its row
// block over all columns the same way.
constexpr int FR_C0 = 80;
constexpr double FR_UNSCALE = 0x1p-80;             // 2^-FR_C0
constexpr double FR_SUM_MAX = 0x1p126;             // largest accepted scaled partial sum
constexpr double FR_MAGIC = 1572864.0 + 0x1p-24;   // 1.5 * 2^20, plus the rounding half-ulp
constexpr int FR_H0 = 0x41380000;                  // high word of 1.5 * 2^20 (floor(x) = 0)
constexpr int FR_KOFF = FR_C0 - FR_H0;             // high word + FR_KOFF = floor(x) + FR_C0

__device__ __forceinline__ double fr_low_margin(int m) {
    return (double)FR_C0 - 32.0 - log2((double)(m > 1 ? m : 1));
}

// k = clamp(hi + FR_KOFF, 0, 126): one add and one min-with-relu.
__device__ __forceinline__ int fr_clamp_k(int hi) {
    int k;
    asm("{.reg .s32 t;\n\tadd.s32 t, %1, %2;\n\tmin.s32.relu %0, t, %3;}"
        : "=r"(k) : "r"(hi), "n"(FR_KOFF), "n"(126));
    return k;
}

// Packed FP32x2 add (sm_100): {a.lo + b.lo, a.hi + b.hi}.
__device__ __forceinline__ unsigned long long add_f32x2(unsigned long long a, unsigned long long b) {
    unsigned long long d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ unsigned long long pack_f32x2(float lo, float hi) {
    unsigned long long d;
    asm("mov.b64 %0, {%1, %2};" : "=l"(d) : "f"(lo), "f"(hi));
    return d;
}
__device__ __forceinline__ float lo_f32(unsigned long long v) { return __uint_as_float((unsigned)v); }
__device__ __forceinline__ float hi_f32(unsigned long long v) { return __uint_as_float((unsigned)(v >> 32)); }

// The row's previous log-sum-exp (natural log), read from the buffer the
// epilogue overwrites: phi -> log(marg) - phi, logZ -> logZ, column mass ->
// log(mass) - beta * rowpot.
__device__ __forceinline__ double row_reference(const PassParams &P, int o, double beta) {
    if (P.epi == EPI_SK_ROW) return log(P.marg[o]) - P.out[o];
    if (P.epi == EPI_LOGZ) return P.out[o];
    if (P.epi == EPI_SK_SYM) return P.aux ? P.aux[o] : NAN;
    if (P.epi == EPI_SPP_COL)
        return log(P.out[o]) - ((beta == 0.0 || !P.rowpot) ? 0.0 : beta * P.rowpot[o]);
    return NAN;
}

// Scaled terms e[r] = 2^(t - Mref_r) * 2^FR_C0 of one column against R rows.
template <int PM, int D, int R>
__device__ __forceinline__ void fr_terms(const double4 col, const double (&xr)[R][D], double a2,
                                         double pexp, const double (&K)[R], float (&e)[R]) {
#pragma unroll
    for (int r = 0; r < R; ++r) {
        double t;
        if (PM == P_SQ) {
            t = col.w;
            if (D >= 3) t = fma(xr[r][D >= 3 ? 2 : 0], col.z, t);
            if (D >= 2) t = fma(xr[r][D >= 2 ? 1 : 0], col.y, t);
            t = fma(xr[r][0], col.x, t);
        } else {
            const double yv[3] = {col.x, col.y, col.z};
            t = fma(pair_cost_direct<PM>(xr[r], yv, D, pexp), a2, col.w);
        }
        const double dv = t + K[r];
        const int k = fr_clamp_k(__double2hiint(dv));
        const float v = __int_as_float((int)__funnelshift_r((unsigned)__double2loint(dv), 0x7Fu, 9));
        e[r] = __int_as_float(__float_as_int(ex2_approx(v)) + (k << 23));
    }
}

// Packed accumulators: rows (2r, 2r+1) share one FP32x2 register; with one row
// per thread, even and odd columns do.
template <int R>
struct FrAcc {
    static constexpr int NP = (R + 1) / 2;
    unsigned long long cs[NP];
    __device__ __forceinline__ void zero() {
#pragma unroll
        for (int j = 0; j < NP; ++j) cs[j] = 0ull;
    }
    // R >= 2: one column's terms for all rows
    __device__ __forceinline__ void add_rows(const float (&e)[R]) {
#pragma unroll
        for (int j = 0; j < R / 2; ++j) cs[j] = add_f32x2(cs[j], pack_f32x2(e[2 * j], e[2 * j + 1]));
        if (R & 1) cs[NP - 1] = add_f32x2(cs[NP - 1], pack_f32x2(e[R - 1], 0.f));
    }
    // R == 1: the terms of two columns
    __device__ __forceinline__ void add_cols(float e0, float e1) { cs[0] = add_f32x2(cs[0], pack_f32x2(e0, e1)); }
    __device__ __forceinline__ float row(int r) const {
        if (R == 1) return lo_f32(cs[0]) + hi_f32(cs[0]);
        return (r & 1) ? hi_f32(cs[r >> 1]) : lo_f32(cs[r >> 1]);
    }
};

template <int PM, int D, int R>
__device__ __forceinline__ void fr_col(const double4 col, const double (&xr)[R][D], double a2,
                                       double pexp, const double (&K)[R], FrAcc<R> &acc) {
    float e[R];
    fr_terms<PM, D, R>(col, xr, a2, pexp, K, e);
    if constexpr (R == 1) acc.add_cols(e[0], 0.f);
    else acc.add_rows(e);
}

template <int PM, int D, int R>
__device__ __forceinline__ void fr_col2(const double4 c0, const double4 c1, const double (&xr)[R][D],
                                        double a2, double pexp, const double (&K)[R], FrAcc<R> &acc) {
    if constexpr (R == 1) {
        float e0[1], e1[1];
        fr_terms<PM, D, 1>(c0, xr, a2, pexp, K, e0);
        fr_terms<PM, D, 1>(c1, xr, a2, pexp, K, e1);
        acc.add_cols(e0[0], e1[0]);
    } else {
        fr_col<PM, D, R>(c0, xr, a2, pexp, K, acc);
        fr_col<PM, D, R>(c1, xr, a2, pexp, K, acc);
    }
}

// Returns false when a real row's partial sum overflowed the window (a term
// clamped high, or a non-finite input).
template <int PM, int D, int R>
__device__ __forceinline__ bool tile_lse_fixedref(const PassParams &P, double alpha, double beta,
                                                  int row_base, int cbeg, int cend, double *smem,
                                                  double (&Mo)[R], double (&So)[R],
                                                  double (&Ho)[R]) {
    constexpr bool SQ = (PM == P_SQ);
    const int tid = threadIdx.x;
    const double a2 = alpha * LOG2E;
    const double cb = P.colpot_unit ? LOG2E : beta * LOG2E;
    double ctr[D];
#pragma unroll
    for (int k = 0; k < D; ++k) ctr[k] = P.ctr ? P.ctr[k] : 0.0;
    double xr[R][D], K[R];
    float S[R], Cc[R];
    FrAcc<R> acc;
    acc.zero();
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int row = row_base + tid + r * TPB;
        const bool ok = row < P.n;
        double h = 0.0;
#pragma unroll
        for (int k = 0; k < D; ++k) {
            const double v = ok ? P.X[(size_t)row * D + k] - ctr[k] : 0.0;
            xr[r][k] = SQ ? -2.0 * a2 * v : v;
            h = fma(v, v, h);
        }
        const double m = (ok ? row_reference(P, row, beta) * LOG2E : 0.0) - (SQ ? a2 * h : 0.0);
        K[r] = FR_MAGIC - (m + 1.0);
        S[r] = 0.f; Cc[r] = 0.f;
    }
    double4 *tile = reinterpret_cast<double4 *>(smem);
    for (int c0 = cbeg; c0 < cend; c0 += CHUNK) {
        __syncthreads();
        for (int q = tid; q < CHUNK; q += TPB) {
            const int j = c0 + q;
            double4 v = make_double4(0.0, 0.0, 0.0, -INFINITY);
            if (j < cend) {
                double yy[3] = {0.0, 0.0, 0.0};
                double s2 = 0.0;
#pragma unroll
                for (int k = 0; k < D; ++k) {
                    yy[k] = P.Y[(size_t)j * D + k] - ctr[k];
                    s2 = fma(yy[k], yy[k], s2);
                }
                const double pot = P.colpot ? P.colpot[j] : 0.0;
                double g = (cb == 0.0) ? 0.0 : cb * pot;
                if (SQ) g += a2 * s2;
                v = make_double4(yy[0], yy[1], yy[2], g);
            }
            tile[q] = v;
        }
        __syncthreads();
        const int nc = min(CHUNK, cend - c0);
        int q = 0;
        // few rows per thread (small problems): unroll more columns so each warp
        // has enough independent pairs in flight to cover FP64 / MUFU latency.
        // 16 columns per FP32 chunk sum before the compensated merge: a 16-term
        // FP32 sum keeps a typical relative error near 2e-7 of the chunk
        constexpr int FR_UNROLL = (R > RPT) ? 1 : 4;
        for (; q + 16 <= nc; q += 16) {
#pragma unroll FR_UNROLL
            for (int u = 0; u < 16; u += 2)
                fr_col2<PM, D, R>(tile[q + u], tile[q + u + 1], xr, a2, P.pexp, K, acc);
#pragma unroll
            for (int r = 0; r < R; ++r) kahan_add(S[r], Cc[r], acc.row(r));
            acc.zero();
        }
        for (; q < nc; ++q) fr_col<PM, D, R>(tile[q], xr, a2, P.pexp, K, acc);
#pragma unroll
        for (int r = 0; r < R; ++r) kahan_add(S[r], Cc[r], acc.row(r));
        acc.zero();
    }
    bool good = true;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int row = row_base + tid + r * TPB;
        const bool real_row = row < P.n;
        double h = 0.0;
#pragma unroll
        for (int k = 0; k < D; ++k) {
            const double v = real_row ? P.X[(size_t)row * D + k] - ctr[k] : 0.0;
            h = fma(v, v, h);
        }
        Ho[r] = SQ ? a2 * h : 0.0;
        Mo[r] = (real_row ? row_reference(P, row, beta) * LOG2E : 0.0) - Ho[r];
        const double sv = (double)S[r] - (double)Cc[r];
        So[r] = sv * FR_UNSCALE;
        // this slice's partial sum must not hold a term clamped high; a small
        // partial is fine (the lower side is checked on the merged row)
        if (real_row && !(sv <= FR_SUM_MAX)) good = false;
    }
    return good;
}

// ---------------------------------------------------------------------------
// FP32-exponent fixed-reference tile (CULAMP_FLAG_FORM_FP32): the same tiling,
// reference and fallbacks as tile_lse_fixedref, but the exponent itself is
// formed in FP32 -- the column term g_j and the row term (reference and |x|^2
// part) are rounded to FP32 once, the d products are FP32 FMAs -- and 2^t goes
// straight to the MUFU ex2 (no clamp: ex2 saturates to +inf above 128, which
// the slice's sum check catches, and flushes to 0 below -126, which the
// merged-row check bounds). Two rows share each packed FP32x2 FMA and add.
// Per pair about 3.5 instructions and one MUFU op, against ~10 for the FP64
// exponent; the FP32 rounding of terms of size |g| + |K| (up to ~1e4 log2
// units at eta_p = 1e-3) limits each term to ~1e-4 relative, which is the
// precision the plain FP32 form has.
constexpr double FR32_LOW_MARGIN = 61.0;

__device__ __forceinline__ unsigned long long fma_f32x2(unsigned long long a, unsigned long long b,
                                                       unsigned long long c) {
    unsigned long long d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}

template <int PM, int D, int R>
__device__ __forceinline__ bool tile_lse_fr32(const PassParams &P, double alpha, double beta,
                                              int row_base, int cbeg, int cend, double *smem,
                                              double (&Mo)[R], double (&So)[R], double (&Ho)[R]) {
    static_assert(PM == P_SQ, "the FP32-exponent tile uses the |x|^2 + |y|^2 - 2 x.y expansion");
    constexpr int NP = (R + 1) / 2;
    const int tid = threadIdx.x;
    const double a2 = alpha * LOG2E;
    const double cb = P.colpot_unit ? LOG2E : beta * LOG2E;
    double ctr[D];
#pragma unroll
    for (int k = 0; k < D; ++k) ctr[k] = P.ctr ? P.ctr[k] : 0.0;
    unsigned long long xr2[NP][D], K2[NP];   // rows (2j, 2j+1) packed
    float S[R], Cc[R];
    unsigned long long acc[NP];
#pragma unroll
    for (int j = 0; j < NP; ++j) {
        float xv[2][D], kv[2];
#pragma unroll
        for (int h2 = 0; h2 < 2; ++h2) {
            const int r = 2 * j + h2;
            const int row = row_base + tid + r * TPB;
            const bool ok = r < R && row < P.n;
            double h = 0.0;
#pragma unroll
            for (int k = 0; k < D; ++k) {
                const double v = ok ? P.X[(size_t)row * D + k] - ctr[k] : 0.0;
                xv[h2][k] = (float)(-2.0 * a2 * v);
                h = fma(v, v, h);
            }
            // t - Mref = g_j + xr.y + (a2 |x|^2 - Mref)
            const double m = ok ? row_reference(P, row, beta) * LOG2E : 0.0;
            kv[h2] = ok ? (float)(a2 * h - m) : 0.f;
        }
#pragma unroll
        for (int k = 0; k < D; ++k) xr2[j][k] = pack_f32x2(xv[0][k], xv[1][k]);
        K2[j] = pack_f32x2(kv[0], kv[1]);
        acc[j] = 0ull;
    }
#pragma unroll
    for (int r = 0; r < R; ++r) { S[r] = 0.f; Cc[r] = 0.f; }
    float4 *tile = reinterpret_cast<float4 *>(smem);
    for (int c0 = cbeg; c0 < cend; c0 += CHUNK) {
        __syncthreads();
        for (int q = tid; q < CHUNK; q += TPB) {
            const int j = c0 + q;
            float4 v = make_float4(0.f, 0.f, 0.f, -INFINITY);
            if (j < cend) {
                double yy[3] = {0.0, 0.0, 0.0};
                double s2 = 0.0;
#pragma unroll
                for (int k = 0; k < D; ++k) {
                    yy[k] = P.Y[(size_t)j * D + k] - ctr[k];
                    s2 = fma(yy[k], yy[k], s2);
                }
                const double pot = P.colpot ? P.colpot[j] : 0.0;
                const double g = ((cb == 0.0) ? 0.0 : cb * pot) + a2 * s2;
                v = make_float4((float)yy[0], (float)yy[1], (float)yy[2], (float)g);
            }
            tile[q] = v;
        }
        __syncthreads();
        const int nc = min(CHUNK, cend - c0);
        for (int q0 = 0; q0 < nc; q0 += 16) {
            const int q1 = min(nc, q0 + 16);
#pragma unroll 4
            for (int q = q0; q < q1; ++q) {
                const float4 col = tile[q];
                const unsigned long long g2 = pack_f32x2(col.w, col.w);
                const unsigned long long y0 = pack_f32x2(col.x, col.x);
                const unsigned long long y1 = pack_f32x2(col.y, col.y);
                const unsigned long long y2 = pack_f32x2(col.z, col.z);
#pragma unroll
                for (int j = 0; j < NP; ++j) {
                    unsigned long long t = add_f32x2(g2, K2[j]);
                    if (D >= 3) t = fma_f32x2(xr2[j][D >= 3 ? 2 : 0], y2, t);
                    if (D >= 2) t = fma_f32x2(xr2[j][D >= 2 ? 1 : 0], y1, t);
                    t = fma_f32x2(xr2[j][0], y0, t);
                    const float e0 = ex2_approx(lo_f32(t));
                    const float e1 = (2 * j + 1 < R) ? ex2_approx(hi_f32(t)) : 0.f;
                    acc[j] = add_f32x2(acc[j], pack_f32x2(e0, e1));
                }
            }
#pragma unroll
            for (int j = 0; j < NP; ++j) {
                kahan_add(S[2 * j], Cc[2 * j], lo_f32(acc[j]));
                if (2 * j + 1 < R) kahan_add(S[2 * j + 1], Cc[2 * j + 1], hi_f32(acc[j]));
                acc[j] = 0ull;
            }
        }
    }
    bool good = true;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int row = row_base + tid + r * TPB;
        const bool real_row = row < P.n;
        double h = 0.0;
#pragma unroll
        for (int k = 0; k < D; ++k) {
            const double v = real_row ? P.X[(size_t)row * D + k] - ctr[k] : 0.0;
            h = fma(v, v, h);
        }
        Ho[r] = a2 * h;
        Mo[r] = (real_row ? row_reference(P, row, beta) * LOG2E : 0.0) - Ho[r];
        const double sv = (double)S[r] - (double)Cc[r];
        So[r] = sv;
        if (real_row && !(sv <= 0x1p64)) good = false;
    }
    return good;
}

// Packed (d <= 3) log-sum-exp tile: rows in registers, column tiles of CHUNK
// (y - ctr, g) double4 entries in shared memory, broadcast to the warp.
template <int PM, int D, int R, bool MOM, int UNROLL = 8>
__device__ __forceinline__ void tile_lse_packed(const PassParams &P, double alpha, double beta,
                                                int row_base, int cbeg, int cend, double *smem,
                                                double (&Mo)[R], double (&So)[R],
                                                double (&MOMo)[R], double (&Ho)[R]) {
    constexpr bool SQ = (PM == P_SQ);
    const int tid = threadIdx.x;
    const double a2 = alpha * LOG2E;
    const double cb = P.colpot_unit ? LOG2E : beta * LOG2E;
    double ctr[D];
#pragma unroll
    for (int k = 0; k < D; ++k) ctr[k] = P.ctr ? P.ctr[k] : 0.0;
    double xr[R][D];
    double xs[(SQ && MOM) ? R : 1][D];
    double M[R];
    float S[R], Cc[R], cs[R], mo[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int row = row_base + tid + r * TPB;
        const bool ok = row < P.n;
        double h = 0.0;
#pragma unroll
        for (int k = 0; k < D; ++k) {
            const double v = ok ? P.X[(size_t)row * D + k] - ctr[k] : 0.0;
            xr[r][k] = SQ ? -2.0 * a2 * v : v;
            if (SQ && MOM) xs[(SQ && MOM) ? r : 0][k] = v;
            h = fma(v, v, h);
        }
        Ho[r] = SQ ? a2 * h : 0.0;
        M[r] = -1e300;   // finite: an all -inf row keeps S = 0 without NaN
        S[r] = 0.f; Cc[r] = 0.f; cs[r] = 0.f; mo[r] = 0.f;
    }
    double4 *tile = reinterpret_cast<double4 *>(smem);
    for (int c0 = cbeg; c0 < cend; c0 += CHUNK) {
        __syncthreads();
        for (int q = tid; q < CHUNK; q += TPB) {
            const int j = c0 + q;
            double4 v = make_double4(0.0, 0.0, 0.0, -INFINITY);
            if (j < cend) {
                double yy[3] = {0.0, 0.0, 0.0};
                double s2 = 0.0;
#pragma unroll
                for (int k = 0; k < D; ++k) {
                    yy[k] = P.Y[(size_t)j * D + k] - ctr[k];
                    s2 = fma(yy[k], yy[k], s2);
                }
                const double pot = P.colpot ? P.colpot[j] : 0.0;
                double g = (cb == 0.0) ? 0.0 : cb * pot;
                if (SQ) g += a2 * s2;
                v = make_double4(yy[0], yy[1], yy[2], g);
            }
            tile[q] = v;
        }
        __syncthreads();
        const int nc = min(CHUNK, cend - c0);
        int q = 0;
        for (; q + 8 <= nc; q += 8) {
#pragma unroll UNROLL
            for (int u = 0; u < 8; ++u) lse_step<PM, D, R, MOM>(tile[q + u], xr, xs, a2, P.pexp, M, S, Cc, cs, mo);
#pragma unroll
            for (int r = 0; r < R; ++r) { kahan_add(S[r], Cc[r], cs[r]); cs[r] = 0.f; }
        }
        for (; q < nc; ++q) lse_step<PM, D, R, MOM>(tile[q], xr, xs, a2, P.pexp, M, S, Cc, cs, mo);
#pragma unroll
        for (int r = 0; r < R; ++r) { kahan_add(S[r], Cc[r], cs[r]); cs[r] = 0.f; }
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
        Mo[r] = M[r];
        So[r] = (double)S[r] - (double)Cc[r];
        MOMo[r] = (double)mo[r];
    }
}

// Per-row epilogue of a reduction pass (one thread per output row, R rows per
// thread) and the grid-level finish step run by the last CTA of the grid.
template <int ACC, int R>
__device__ __forceinline__ void row_epilogue(const PassParams &P, int rb, int row_base, double beta,
                                             const double (&Mv)[R], const double (&Sv)[R],
                                             const double (&MOMv)[R], const double (&Hv)[R],
                                             double *red, int &s_last, int nrb) {
    Ctl *ctl = P.ctl;
    double acc4[4] = {0.0, 0.0, 0.0, 0.0};
    double amax = -INFINITY;
    double en = 0.0;
    if (P.lamp_step == LAMP_A) { double sn; lamp_next(ctl->eta_t, ctl->s_t, ctl->tau_p, ctl->eta_lamp, en, sn); }
    else if (P.lamp_step == LAMP_B) en = ctl->eta_next;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int o = row_base + threadIdx.x + r * TPB;
        if (o >= P.n) continue;
        if (ACC != ACC_LSE) {
            if (P.out) P.out[o] = Mv[r];
            amax = fmax(amax, Mv[r]);
            if (P.marg) acc4[0] += P.marg[o] * Mv[r];
            continue;
        }
        // natural-log LSE of the row: ln2 * (H + M + log2 S)
        const double L = LN2 * (Hv[r] + Mv[r] + log2(Sv[r]));
        const double Ec = (Sv[r] > 0.0) ? MOMv[r] / Sv[r] : 0.0;   // softmax-weighted mean cost
        switch (P.epi) {
            case EPI_SK_ROW: {
                const double v = log(P.marg[o]) - L;
                P.out[o] = v;
                acc4[0] += P.marg[o] * v;
                break;
            }
            case EPI_SK_RESID: {
                const double mass = exp(P.rowpot[o] + L);
                const double res = P.marg[o] - mass;
                if (P.out) P.out[o] = res;
                if (P.out2) P.out2[o] = mass * Ec;
                acc4[0] += fabs(res);
                acc4[1] += mass * Ec;
                acc4[2] += P.marg[o] * P.rowpot[o];
                break;
            }
            case EPI_SK_SYM: {
                // f = rowpot = colpot (x against itself): T(f)_i = log a_i - L_i
                // and the row mass of P_ij = exp(f_i + f_j - C_ij/eps) is
                // a_i exp(f_i - T(f)_i); the next f is the average (f + T(f))/2
                const double f = P.rowpot[o];
                const double T = log(P.marg[o]) - L;
                const double mass = exp(f + L);
                P.out[o] = 0.5 * (f + T);
                if (P.aux) P.aux[o] = L;
                acc4[0] += fabs(P.marg[o] - mass);
                acc4[1] += mass * Ec;
                acc4[2] += P.marg[o] * f;
                break;
            }
            case EPI_LOGZ: {
                if (P.out) P.out[o] = L;
                if (P.marg) {
                    if (P.aux) P.aux[o] = log(P.marg[o]) - L;
                    acc4[0] += P.marg[o] * L;
                }
                break;
            }
            case EPI_SPP_COL: {
                const double rp = P.rowpot ? P.rowpot[o] : 0.0;
                const double res = exp(((beta == 0.0) ? 0.0 : beta * rp) + L);
                const double cst = res * Ec;
                if (P.out) P.out[o] = res;
                if (P.out2) P.out2[o] = cst;
                const double cj = P.cvec ? P.cvec[o] : 0.0;
                acc4[0] += fabs(res - cj);
                acc4[1] += cst;
                acc4[2] += res * rp;
                if (P.lamp_step == LAMP_A) {
                    const double th = P.theta[o];
                    acc4[3] += cj * th;
                    P.thetab[o] = theta_step(th, res, cj, P.eta_mu_i[o], P.eta_mu_exp, 0, P.minv, P.maxv, 1.0);
                    P.nub[o] = (1.0 - en) * P.nu[o] + en * th;
                } else if (P.lamp_step == LAMP_B) {
                    P.theta[o] = theta_step(P.theta[o], res, cj, P.eta_mu_i[o], P.eta_mu_exp, 1, P.minv, P.maxv, 1.0);
                    P.nu[o] = (1.0 - en) * P.nu[o] + en * P.thetab[o];
                }
                break;
            }
            default:
                if (P.out) P.out[o] = L;
                break;
        }
    }

    if (P.finish == FIN_NONE) return;
    if (ACC == ACC_MAX) {
        const double bm = block_max1(amax, red);
        acc4[0] = bm;
    } else {
        block_sum4(acc4, red);
    }
    if (threadIdx.x == 0) {
        for (int k = 0; k < 4; ++k) P.blk[rb * 4 + k] = acc4[k];
        __threadfence();
        const unsigned t = atomicAdd(P.grid_ticket, 1u);
        s_last = (t == (unsigned)nrb - 1u);
    }
    __syncthreads();
    if (s_last && threadIdx.x == 0) {
        __threadfence();
        double tot[4] = {0.0, 0.0, 0.0, 0.0};
        if (ACC == ACC_MAX) tot[0] = -INFINITY;
        for (int b = 0; b < nrb; ++b) {
            const volatile double *bb = P.blk + b * 4;
            if (ACC == ACC_MAX) tot[0] = fmax(tot[0], bb[0]);
            else for (int k = 0; k < 4; ++k) tot[k] += bb[k];
        }
        if (P.finish == FIN_LAMP_A) ctl->sum_c_theta = tot[3];
        run_finish(P, tot);
        *P.grid_ticket = 0u;
    }
}

// FR: this instantiation tries the fixed-reference loop first (P.use_ref must be
// set) and carries a compact online loop for its fallbacks; FR == false runs
// the online loop alone, fully unrolled.
// BAT == false: one pass, grid (row blocks, column splits), parameters P0.
// BAT == true: the same pass over many independent instances in one launch:
// CTA b belongs to the instance i with block_start[i] <= b < block_start[i+1]
// and is its local block b - block_start[i] = sp * nrb + rb. Each instance
// carries its own parameters (plist[i]), scratch, tickets and control block.
// F32: the fixed-reference loop forms the exponent in FP32 (tile_lse_fr32,
// CULAMP_FLAG_FORM_FP32); its fallbacks stay FP64.
template <int PM, int D, int ACC, int R, bool MOM, bool FR, bool BAT = false, bool F32 = false>
__global__ void __launch_bounds__(TPB, (R > RPT_MID) ? 3 : 4)
    pair_pass_kernel(const __grid_constant__ PassParams P0, const PassParams *plist,
                     const int *block_start, int count) {
    extern __shared__ __align__(16) double smem[];
    __shared__ double red[4 * (TPB / 32)];
    __shared__ int s_last;
    __shared__ int s_bat[3];                      // BAT: row block, split, row-block count
    __shared__ __align__(16) PassParams sP;       // BAT: this instance's parameters
    // Programmatic dependent launch: the launch may overlap the previous kernel
    // in the stream, so before reading anything that kernel may write (control
    // block, potentials, references, scratch) wait for it to complete. A no-op
    // for a launch without programmatic serialisation.
    asm volatile("griddepcontrol.wait;" ::: "memory");
    if constexpr (BAT) {
        if (threadIdx.x == 0) {
            int lo = 0, hi = count - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (block_start[mid] <= (int)blockIdx.x) lo = mid;
                else hi = mid - 1;
            }
            const int local = (int)blockIdx.x - block_start[lo];
            const int nrb = plist[lo].nrb;
            s_bat[0] = local % nrb;
            s_bat[1] = local / nrb;
            s_bat[2] = nrb;
            s_last = lo;
        }
        __syncthreads();
        const int *src = reinterpret_cast<const int *>(plist + s_last);
        int *dst = reinterpret_cast<int *>(&sP);
        for (int k = threadIdx.x; k < (int)(sizeof(PassParams) / sizeof(int)); k += TPB) dst[k] = src[k];
        __syncthreads();
    }
    const PassParams &P = *(BAT ? &sP : &P0);
#define CULAMP_RB (BAT ? s_bat[0] : (int)blockIdx.x)
#define CULAMP_SP (BAT ? s_bat[1] : (int)blockIdx.y)
#define CULAMP_NRB (BAT ? s_bat[2] : (int)gridDim.x)
    Ctl *ctl = P.ctl;
    if (ctl) {
        if (ctl->stop) return;
        if (P.gate == GATE_CHECK && !ctl->do_check) return;
        if (P.gate == GATE_NOCHECK && ctl->do_check) return;
        if (P.phase == PHASE_FP32 && !ctl->fp32_phase) return;
        if (P.phase == PHASE_FP64 && ctl->fp32_phase) return;
    }
    double alpha = 0.0, beta = 0.0;
    if (ACC == ACC_LSE) resolve_coefs(P, alpha, beta);

    const int row_base = CULAMP_RB * (TPB * R);
    const int cbeg = CULAMP_SP * P.cols_per_split;
    const int cend = min(P.m, cbeg + P.cols_per_split);

    double Mv[R], Sv[R], MOMv[R], Hv[R];
    bool fr_tried = false;   // the fixed-reference path ran for this row block
    if constexpr (ACC == ACC_LSE && D > 0) {
        bool done = false;
        if constexpr (FR && !MOM) {
            {
                // reference = the row's previous LSE, from the buffer the epilogue
                // is about to overwrite (read-only until every split has finished)
                bool ok = true;
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const int o = row_base + threadIdx.x + r * TPB;
                    if (o < P.n && !isfinite(row_reference(P, o, beta))) ok = false;
                }
                if (!__syncthreads_or(!ok)) {
                    fr_tried = true;
#pragma unroll
                    for (int r = 0; r < R; ++r) MOMv[r] = 0.0;
                    bool good;
                    if constexpr (F32 && PM == P_SQ)
                        good = tile_lse_fr32<PM, D, R>(P, alpha, beta, row_base, cbeg, cend, smem, Mv, Sv, Hv);
                    else
                        good = tile_lse_fixedref<PM, D, R>(P, alpha, beta, row_base, cbeg, cend, smem, Mv, Sv, Hv);
                    done = !__syncthreads_or(!good);
                }
            }
        }
        if (!done) {
            if constexpr (FR) tile_lse_packed<PM, D, R, MOM, 2>(P, alpha, beta, row_base, cbeg, cend, smem, Mv, Sv, MOMv, Hv);
            else tile_lse_packed<PM, D, R, MOM, 8>(P, alpha, beta, row_base, cbeg, cend, smem, Mv, Sv, MOMv, Hv);
        }
    } else {
        static_assert(R == RPT, "generic / min-max tiles use RPT rows per thread");
        tile_reduce<PM, D, ACC, MOM>(P, alpha, beta, row_base, cbeg, cend, smem, Mv, Sv, MOMv, Hv);
    }

    // the pair loop is done: let the next kernel in the stream start launching
    // (it waits for this grid's completion before it reads anything)
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");

    if (P.splits > 1) {
        // publish partials, take a ticket; the last CTA of this row block merges
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int row = row_base + threadIdx.x + r * TPB;
            if (row < P.n) {
                double *pp = P.part + ((size_t)CULAMP_SP * P.n + row) * 3;
                pp[0] = Mv[r]; pp[1] = Sv[r];
                if (MOM) pp[2] = MOMv[r];
            }
        }
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) {
            const unsigned t = atomicAdd(&P.rb_ticket[CULAMP_RB], 1u);
            s_last = (t == (unsigned)(P.splits - 1));
        }
        __syncthreads();
        if (!s_last) return;
        __threadfence();
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int row = row_base + threadIdx.x + r * TPB;
            if (row >= P.n) continue;
            double M = (ACC == ACC_MIN) ? INFINITY : -INFINITY, S = 0.0, MO = 0.0;
            // partials come from other CTAs: L2-coherent loads, issued 8 splits at a
            // time so their latencies overlap, then merged in split order
            for (int s0 = 0; s0 < P.splits; s0 += 8) {
                double m2[8], ss2[8], mo2[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    if (s0 + u < P.splits) {
                        const double *pp = P.part + ((size_t)(s0 + u) * P.n + row) * 3;
                        m2[u] = __ldcg(pp);
                        ss2[u] = __ldcg(pp + 1);
                        mo2[u] = MOM ? __ldcg(pp + 2) : 0.0;
                    }
                }
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    if (s0 + u >= P.splits) break;
                    if (ACC == ACC_LSE) merge_lse(M, S, MO, m2[u], ss2[u], mo2[u]);
                    else if (ACC == ACC_MAX) M = fmax(M, m2[u]);
                    else M = fmin(M, m2[u]);
                }
            }
            Mv[r] = M; Sv[r] = S; MOMv[r] = MO;
        }
        if (threadIdx.x == 0) P.rb_ticket[CULAMP_RB] = 0u;   // re-arm for the next launch
    }

    if constexpr (FR && ACC == ACC_LSE && D > 0 && !MOM) {
        // Lower side of the fixed-reference window, on the merged row: the full
        // LSE must be within fr_low_margin(m) of the reference, else clamped-low
        // terms could matter and the row block is recomputed over all columns.
        if (fr_tried) {
            const double a2 = alpha * LOG2E;
            const double margin = F32 ? FR32_LOW_MARGIN : fr_low_margin(P.m);
            bool bad = false;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int o = row_base + threadIdx.x + r * TPB;
                if (o >= P.n) continue;
                const double mref = row_reference(P, o, beta) * LOG2E - Hv[r];
                if (!(Sv[r] > 0.0) || Mv[r] + log2(Sv[r]) < mref - margin) bad = true;
            }
            (void)a2;
            if (__syncthreads_or(bad))
                tile_lse_packed<PM, D, R, false, 2>(P, alpha, beta, row_base, 0, P.m, smem, Mv, Sv, MOMv, Hv);
        }
    }

    row_epilogue<ACC, R>(P, CULAMP_RB, row_base, beta, Mv, Sv, MOMv, Hv, red, s_last, CULAMP_NRB);
#undef CULAMP_RB
#undef CULAMP_SP
#undef CULAMP_NRB
}

}  // namespace culamp_dev
