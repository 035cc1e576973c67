// persist.cu -- the whole Sinkhorn loop of a small problem in one persistent
// launch (SinkhornKernel.jl:477-559 with the passes of :341-444 and :9-81).
//
// At n, m of a few thousand points a pass is ~10 microseconds of pair work
// spread over 148 SMs, and a pass-per-launch loop pays for each pass a launch,
// a prologue that stages the rows, and a merge of column-split partials by the
// last CTA of each row block (a dependent round trip through L2). Here one
// cooperative launch of one CTA per SM runs every iteration:
//
//   * CTA b owns the output rows [b n / G, (b+1) n / G) of each half-step (G =
//     grid size), so a row's log-sum-exp is finished inside its CTA: no split
//     partials, no tickets. Its 16 warps spread the columns over their lanes,
//     four columns per thread in registers, and walk the CTA's rows (28 at a
//     time, two per packed FP32x2 accumulator, their data broadcast from a
//     shared-memory cache of the CTA's rows made at kernel entry). The
//     per-thread column sums are merged across each warp by a butterfly
//     reduce-scatter and across the warps in shared memory in a fixed order;
//     warp 0 finishes the group, one row per lane, with no further barrier.
//     The CTA is the only writer of its rows' potentials, so it keeps them and
//     each row's fixed-reference offset in that cache.
//   * Each term uses the fixed-reference exponent of the pass engine (DADD with
//     FR_MAGIC, funnel-shifted mantissa, one MUFU ex2, exponent-field add,
//     scaled by 2^FR_C0). Rows whose sums leave the window are shared out to
//     the CTA's warps and recomputed without a reference (a max pass, then a
//     sum pass of max-shifted terms).
//   * Half-steps are separated by a grid barrier (one monotonic arrival
//     counter in global memory). Every wait on it is bounded: after
//     PERSIST_WAIT_NS a waiting CTA adds the abort mark to the counter, sets
//     the control block's error flag and every CTA leaves the loop; the host
//     reports a device timeout.
//   * The control step of each iteration (iteration counter, check cadence,
//     itermax, tmax, the tolerance test of the check iterations) follows the
//     pass engine's FIN_SK_ITER / FIN_SK_CHECK. Decisions that every CTA needs
//     are computed by every CTA from the same data in the same order (the
//     tolerance test sums the per-CTA partials in a fixed order); the one
//     decision that reads the clock (tmax) is taken by CTA 0 and carried by its
//     arrival at the barrier. CTA 0 alone writes the control block and the log.
//
// The same machinery runs LAMP's loop (lamp_persist_kernel, further below).
//
// Potentials written by other CTAs are read with L2-coherent loads (ld.cg).

#include <algorithm>

#include "internal.h"

namespace culamp_dev {

constexpr int PTPB = 512;                  // threads per CTA (one CTA per SM)
constexpr int PWARPS = PTPB / 32;
constexpr int PRG = 28;                    // rows per group (warp 0 finishes one row per lane)
constexpr int PMAXR = 56;                  // rows per CTA and side (2 groups)
constexpr unsigned long long PERSIST_WAIT_NS = 2000000000ull;
constexpr int PERSIST_CARVEOUT = 10;       // percent of the unified L1 / shared memory

struct GridBar {
    // arrivals since the launch in the low 44 bits; + PERSIST_LATE once CTA 0
    // has found tmax passed, + PERSIST_ABORT once a CTA gave up waiting
    unsigned long long count;
    unsigned long long pad;
};
constexpr unsigned long long PERSIST_LATE = 1ull << 44;
constexpr unsigned long long PERSIST_ARRIVALS = PERSIST_LATE - 1ull;
constexpr unsigned long long PERSIST_ABORT = 1ull << 62;

struct PersistParams {
    const double *X, *Y;       // point clouds (n x d, m x d), read-only
    const double *r, *c;       // marginals
    double *phi, *psi;         // potentials, updated in place
    int n, m;
    double pexp;
    Ctl *ctl;
    double *blk;               // [G][4] per-CTA partial sums (fixed-order totals)
    GridBar *bar;              // zeroed before the launch
};

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void red_release_add_u64(unsigned long long *p, unsigned long long v) {
    asm volatile("red.release.gpu.global.add.u64 [%0], %1;" :: "l"(p), "l"(v) : "memory");
}

// Grid-wide barrier k (k = 0, 1, ... counted by `gen`) with a bounded wait.
// The arrival counter only grows: barrier k is complete once it reaches
// (k + 1) G. An arrival is one release-reduction (no round trip), the wait
// polls the counter with acquire loads; bar.sync before the arrival and after
// the wait extends both to the whole CTA. A CTA that gives up after
// PERSIST_WAIT_NS adds PERSIST_ABORT, which every waiter sees at once.
// The arrival can carry `extra` (CTA 0: PERSIST_LATE, its tmax decision);
// `*s_late` then tells every CTA, from the same counter read, whether it was
// added by the time the barrier completed -- CTA 0 adds it only at the barrier
// that ends an iteration, and stops after it, so every CTA sees the same.
// Returns false (in every thread of the CTA) when this CTA gave up or saw
// another CTA give up.
__device__ bool grid_sync(GridBar *gb, unsigned &gen, int *s_flag, unsigned long long extra = 0ull,
                          int *s_late = nullptr, unsigned long long limit_ns = PERSIST_WAIT_NS) {
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        red_release_add_u64(&gb->count, 1ull + extra);
        const unsigned long long target = (unsigned long long)(gen + 1u) * gridDim.x;
        unsigned long long t0 = 0;
        for (unsigned spins = 0;; ++spins) {
            const unsigned long long v = ld_acquire_u64(&gb->count);
            if (v >= PERSIST_ABORT) { ok = 0; break; }
            if ((v & PERSIST_ARRIVALS) >= target) {
                if (s_late) *s_late = (v & ~PERSIST_ARRIVALS) != 0ull;
                break;
            }
            if ((spins & 63u) == 63u) {
                const unsigned long long t = globaltimer_ns();
                if (t0 == 0) t0 = t;
                else if (t - t0 > limit_ns) {
                    red_release_add_u64(&gb->count, PERSIST_ABORT);
                    ok = 0;
                    break;
                }
            }
        }
        *s_flag = ok;
    }
    gen += 1u;
    __syncthreads();
    return *s_flag != 0;
}

// This CTA's rows of one side -- the points whose potential a half-step
// writes -- cached at kernel entry: constants, the row's potential (this CTA
// is its only writer) and the fixed-reference offset K of the row's next pass,
// K = FR_MAGIC - (M2 + 1) with M2 = (previous LSE) * log2(e) - H.
struct SideRows {
    double4 xr[PMAXR];         // p = 2: {-2 a2 v, K}; else {v, K}  (v = x - ctr)
    float4 vf[PMAXR];          // v in FP32 (p = 2 cost moment)
    float4 xf[PMAXR];          // p = 2, FP32-exponent passes: {-2 a2 v, -M2} in FP32
    double marg[PMAXR], logm[PMAXR];
    double H[PMAXR];           // a2 |v|^2 for p = 2, else 0
    double M2[PMAXR];          // the reference the row's K was made from
    double pot[PMAXR];
};

struct PShared {
    SideRows side[2];          // 0: the x points (phi), 1: the y points (psi)
    float red[PWARPS][32];
    float redm[PWARPS][32];
    double fl[32], fe[32];     // the group's rows recomputed by the fallback
    unsigned bad;              // rows of the group outside the window
    int flag;
    int late;                  // tmax passed (CTA 0's decision, via the barrier)
};

// One side of the problem as the rows of a half-step.
struct Side {
    const double *pts;         // points (n x D), read-only
    const double *marg;        // marginal
    double *pot;               // potential (global: other CTAs read it as columns)
    int n;
};

__device__ __forceinline__ int rows_lo(int n) { return (int)(((long long)blockIdx.x * n) / gridDim.x); }
__device__ __forceinline__ int rows_hi(int n) { return (int)(((long long)(blockIdx.x + 1) * n) / gridDim.x); }

// Butterfly reduce-scatter of 32 values over a warp: afterwards lane l holds in
// a[0] the warp total of value l (31 shuffles instead of 32 x 5).
__device__ __forceinline__ void warp_scatter32(float (&a)[32]) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 16, L = 32; o >= 1; o >>= 1, L >>= 1) {
        const bool up = (lane & o) != 0;
#pragma unroll
        for (int i = 0; i < L / 2; ++i) {
            const float send = up ? a[i] : a[i + L / 2];
            const float keep = up ? a[i + L / 2] : a[i];
            a[i] = keep + __shfl_xor_sync(0xffffffffu, send, o);
        }
    }
}

// One fixed-reference term from dv = t - Mref - 1 + FR_MAGIC (the pass
// engine's tile_lse_fixedref): 2^(t - Mref) * 2^C0 for t - Mref in
// [-C0, 126 - C0]. ZLOW: a term below the window becomes a subnormal (< 2^-126)
// instead of ~2..4, so it adds nothing to a moment -- the check pass's cost
// moment keeps terms down to 2^-C0 of the reference and no floor below them.
template <int C0, bool ZLOW>
__device__ __forceinline__ float fr_term(double dv) {
    const int hi = __double2hiint(dv);
    const float vm = __int_as_float((int)__funnelshift_r((unsigned)__double2loint(dv), 0x7Fu, 9));
    const int eb = __float_as_int(ex2_approx(vm));
    int k;
    if constexpr (!ZLOW) {
        asm("{.reg .s32 t;\n\tadd.s32 t, %1, %2;\n\tmin.s32.relu %0, t, %3;}"
            : "=r"(k) : "r"(hi), "n"(C0 - FR_H0), "n"(126));
        return __int_as_float(eb + (k << 23));
    } else {
        asm("{.reg .s32 t;\n\tadd.s32 t, %1, %2;\n\tmin.s32.relu %0, t, %3;}"
            : "=r"(k) : "r"(hi), "n"(C0 + 128 - FR_H0), "n"(254));
        return __int_as_float(eb + (k << 23) - (128 << 23));
    }
}

// Log-sum-exp of row o over all columns by one warp, without a reference: the
// recompute of a row whose fixed-reference sum left the window. Terms
// t_j = alpha C_oj + beta colpot_j (natural-log units) in FP64; first their
// maximum M, then 2^((t_j - M) log2 e) on the MUFU pipe (the online loop's
// term, |t_j - M| rounded to FP32) in Kahan-compensated FP32 sums per lane,
// merged in FP64. With MOM also the cost moment. Every lane returns L, E.
template <int PM, int D, bool MOM>
__device__ void row_lse_twopass(const double *rows, int o, const double *cols, int nc, const double *colpot,
                                double beta, double alpha, double inv_winf, double pexp, double &L, double &Ec) {
    const int lane = threadIdx.x & 31;
    double xv[D];
#pragma unroll
    for (int k = 0; k < D; ++k) xv[k] = rows[(size_t)o * D + k];
    double M = -INFINITY;
    for (int j = lane; j < nc; j += 32) {
        double yv[D];
#pragma unroll
        for (int k = 0; k < D; ++k) yv[k] = cols[(size_t)j * D + k];
        const double t = fma(alpha, pair_cost_direct<PM>(xv, yv, D, pexp), beta * __ldcg(colpot + j));
        M = fmax(M, t);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) M = fmax(M, __shfl_xor_sync(0xffffffffu, M, off));
    float S = 0.f, Sc = 0.f, MO = 0.f, MOc = 0.f;
    if (M > -INFINITY) {
        for (int j = lane; j < nc; j += 32) {
            double yv[D];
#pragma unroll
            for (int k = 0; k < D; ++k) yv[k] = cols[(size_t)j * D + k];
            const double cc = pair_cost_direct<PM>(xv, yv, D, pexp);
            const double t = fma(alpha, cc, beta * __ldcg(colpot + j));
            const float e = ex2_approx((float)((t - M) * LOG2E));
            kahan_add(S, Sc, e);
            if (MOM) kahan_add(MO, MOc, e * (float)(cc * inv_winf));
        }
    }
    double Sd = (double)S - (double)Sc, MOd = (double)MO - (double)MOc;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        Sd += __shfl_xor_sync(0xffffffffu, Sd, off);
        MOd += __shfl_xor_sync(0xffffffffu, MOd, off);
    }
    L = M + log(Sd);
    Ec = (MOM && Sd > 0.0) ? MOd / Sd / inv_winf : 0.0;
}

// Kernel-entry set-up of this CTA's rows of one side.
template <int PM, int D>
__device__ void cache_side(const Side &s, SideRows &R, const double (&ctr)[D], double a2) {
    constexpr bool SQ = (PM == P_SQ);
    const int lo = rows_lo(s.n), cnt = rows_hi(s.n) - lo;
    for (int i = threadIdx.x; i < PMAXR; i += PTPB) {
        const bool ok = i < cnt;
        const int o = lo + i;
        double v[3] = {0.0, 0.0, 0.0};
        double h = 0.0;
#pragma unroll
        for (int k = 0; k < D; ++k) {
            v[k] = ok ? s.pts[(size_t)o * D + k] - ctr[k] : 0.0;
            h = fma(v[k], v[k], h);
        }
        const double Hh = SQ ? a2 * h : 0.0;
        const double mg = ok ? s.marg[o] : 1.0;
        const double lm = log(mg);
        const double pot = ok ? __ldcg(s.pot + o) : 0.0;
        const double M2 = (lm - pot) * LOG2E - Hh;
        const double K = FR_MAGIC - (M2 + 1.0);
        R.xr[i] = SQ ? make_double4(-2.0 * a2 * v[0], -2.0 * a2 * v[1], -2.0 * a2 * v[2], K)
                     : make_double4(v[0], v[1], v[2], K);
        R.vf[i] = make_float4((float)v[0], (float)v[1], (float)v[2], 0.f);
        R.xf[i] = make_float4((float)(-2.0 * a2 * v[0]), (float)(-2.0 * a2 * v[1]), (float)(-2.0 * a2 * v[2]),
                              (float)(-M2));
        R.marg[i] = mg;
        R.logm[i] = lm;
        R.H[i] = Hh;
        R.M2[i] = M2;
        R.pot[i] = pot;
    }
}

// One half-step over this CTA's rows of side s (cached in R) against the
// columns `cols` (nc points, potential colpot entering with coefficient cb,
// log2 units), in groups of PRG rows; warp 0 finishes each group (lane r = row
// r) with the row's natural-log LSE L (and with MOM its softmax-weighted mean
// cost E) handed to the epilogue `epi`, whose four contributions per row are
// summed into part (valid in thread 0, in a fixed summation order).
template <int PM, int D, bool MOM, int CB, bool F32, class EPI, class SH>
__device__ void pass_rows(const Side &s, SideRows &R, const double *cols, int nc, const double *colpot,
                          double cb, const double (&ctr)[D], double a2, double inv_winf, double pexp,
                          const EPI &epi, SH &sh, double (&part)[4]) {
    constexpr bool SQ = (PM == P_SQ);
    // window exponent: the row update's LSE may move well above its reference
    // (FR_C0 leaves 46 above); the check's hardly moves, and its cost moment
    // wants the small terms
    constexpr int C0 = MOM ? 120 : FR_C0;
    constexpr int NP = PRG / 2;
    static_assert(CB == 2 || CB == 4, "columns per thread step");
    static_assert(!F32 || (SQ && !MOM), "the FP32-exponent pass is the p = 2 row update");
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int lo = rows_lo(s.n), cnt = rows_hi(s.n) - lo;
    const float invw_f = (float)inv_winf;
    part[0] = part[1] = part[2] = part[3] = 0.0;
    const double low_floor = 32.0 + log2((double)nc);   // lower side of the window on log2(S)
    for (int g0 = 0; g0 < cnt; g0 += PRG) {
        const int nrows = min(PRG, cnt - g0);
        unsigned long long acc[NP], mo[MOM ? NP : 1];
#pragma unroll
        for (int q = 0; q < NP; ++q) acc[q] = 0ull;
#pragma unroll
        for (int q = 0; q < (MOM ? NP : 1); ++q) mo[q] = 0ull;
        if constexpr (F32) {
            // the exponent in FP32 (the pass engine's tile_lse_fr32): t - Mref =
            // g_j - M2_i + xr_i . y_j with packed FP32x2 FMAs over the row pair,
            // 2^(t - Mref) by one MUFU ex2, no window clamp (a sum above 2^64 or
            // far below the reference takes the exact row)
            for (int jb = 0; jb < nc; jb += CB * PTPB) {
                unsigned long long gy[CB], y0[CB], y1[CB], y2[CB];
#pragma unroll
                for (int c = 0; c < CB; ++c) {
                    const int j = jb + c * PTPB + tid;
                    float yf[3] = {0.f, 0.f, 0.f};
                    float g = -INFINITY;
                    if (j < nc) {
                        double s2 = 0.0;
#pragma unroll
                        for (int k = 0; k < D; ++k) {
                            const double yy = cols[(size_t)j * D + k] - ctr[k];
                            s2 = fma(yy, yy, s2);
                            yf[k] = (float)yy;
                        }
                        g = (float)(cb * __ldcg(colpot + j) + a2 * s2);
                    }
                    gy[c] = pack_f32x2(g, g);
                    y0[c] = pack_f32x2(yf[0], yf[0]);
                    y1[c] = pack_f32x2(yf[1], yf[1]);
                    y2[c] = pack_f32x2(yf[2], yf[2]);
                }
#pragma unroll
                for (int q = 0; q < NP; ++q) {
                    const float4 fa = R.xf[g0 + 2 * q], fb = R.xf[g0 + 2 * q + 1];
                    const unsigned long long x0 = pack_f32x2(fa.x, fb.x), x1 = pack_f32x2(fa.y, fb.y);
                    const unsigned long long x2 = pack_f32x2(fa.z, fb.z), k2 = pack_f32x2(fa.w, fb.w);
#pragma unroll
                    for (int c = 0; c < CB; ++c) {
                        unsigned long long t = add_f32x2(gy[c], k2);
                        if (D >= 3) t = fma_f32x2(x2, y2[c], t);
                        if (D >= 2) t = fma_f32x2(x1, y1[c], t);
                        t = fma_f32x2(x0, y0[c], t);
                        acc[q] = add_f32x2(acc[q], pack_f32x2(ex2_approx(lo_f32(t)), ex2_approx(hi_f32(t))));
                    }
                }
            }
        } else
        for (int jb = 0; jb < nc; jb += CB * PTPB) {
            double4 col[CB];
            float cfy[(MOM && SQ) ? CB : 1][3];
#pragma unroll
            for (int c = 0; c < CB; ++c) {
                const int j = jb + c * PTPB + tid;
                double yy[3] = {0.0, 0.0, 0.0};
                double g = -INFINITY;
                if (j < nc) {
                    double s2 = 0.0;
#pragma unroll
                    for (int k = 0; k < D; ++k) {
                        yy[k] = cols[(size_t)j * D + k] - ctr[k];
                        s2 = fma(yy[k], yy[k], s2);
                    }
                    g = cb * __ldcg(colpot + j);
                    if (SQ) g += a2 * s2;
                }
                col[c] = make_double4(yy[0], yy[1], yy[2], g);
                if constexpr (MOM && SQ) {
#pragma unroll
                    for (int k = 0; k < 3; ++k) cfy[c][k] = (float)yy[k];
                }
            }
#pragma unroll
            for (int q = 0; q < NP; ++q) {
                const double4 ra = R.xr[g0 + 2 * q], rb = R.xr[g0 + 2 * q + 1];
                float ea[CB], eb[CB], ca[CB], cbw[CB];
#pragma unroll
                for (int c = 0; c < CB; ++c) {
                    double ta, tb;
                    ca[c] = cbw[c] = 0.f;
                    if (SQ) {
                        ta = col[c].w;
                        tb = col[c].w;
                        if (D >= 3) { ta = fma(ra.z, col[c].z, ta); tb = fma(rb.z, col[c].z, tb); }
                        if (D >= 2) { ta = fma(ra.y, col[c].y, ta); tb = fma(rb.y, col[c].y, tb); }
                        ta = fma(ra.x, col[c].x, ta);
                        tb = fma(rb.x, col[c].x, tb);
                    } else {
                        const double xa[3] = {ra.x, ra.y, ra.z}, xb[3] = {rb.x, rb.y, rb.z};
                        const double yv[3] = {col[c].x, col[c].y, col[c].z};
                        const double cca = pair_cost_direct<PM>(xa, yv, D, pexp);
                        const double ccb = pair_cost_direct<PM>(xb, yv, D, pexp);
                        ta = fma(cca, a2, col[c].w);
                        tb = fma(ccb, a2, col[c].w);
                        if (MOM) { ca[c] = (float)(cca * inv_winf); cbw[c] = (float)(ccb * inv_winf); }
                    }
                    ea[c] = fr_term<C0, MOM>(ta + ra.w);
                    eb[c] = fr_term<C0, MOM>(tb + rb.w);
                }
                if constexpr (MOM && SQ) {
                    const float4 fa = R.vf[g0 + 2 * q], fb = R.vf[g0 + 2 * q + 1];
#pragma unroll
                    for (int c = 0; c < CB; ++c) {
                        float d0 = fa.x - cfy[c][0], d1 = fa.y - cfy[c][1], d2 = fa.z - cfy[c][2];
                        ca[c] = fmaf(d2, d2, fmaf(d1, d1, d0 * d0)) * invw_f;
                        d0 = fb.x - cfy[c][0]; d1 = fb.y - cfy[c][1]; d2 = fb.z - cfy[c][2];
                        cbw[c] = fmaf(d2, d2, fmaf(d1, d1, d0 * d0)) * invw_f;
                    }
                }
#pragma unroll
                for (int c = 0; c < CB; ++c) acc[q] = add_f32x2(acc[q], pack_f32x2(ea[c], eb[c]));
                if constexpr (MOM) {
#pragma unroll
                    for (int c = 0; c < CB; ++c)
                        mo[q] = fma_f32x2(pack_f32x2(ea[c], eb[c]), pack_f32x2(ca[c], cbw[c]), mo[q]);
                }
            }
        }
        {
            float a[32];
#pragma unroll
            for (int q = 0; q < NP; ++q) { a[2 * q] = lo_f32(acc[q]); a[2 * q + 1] = hi_f32(acc[q]); }
#pragma unroll
            for (int i = PRG; i < 32; ++i) a[i] = 0.f;
            warp_scatter32(a);
            sh.red[warp][lane] = a[0];
        }
        if constexpr (MOM) {
            float a[32];
#pragma unroll
            for (int q = 0; q < NP; ++q) { a[2 * q] = lo_f32(mo[q]); a[2 * q + 1] = hi_f32(mo[q]); }
#pragma unroll
            for (int i = PRG; i < 32; ++i) a[i] = 0.f;
            warp_scatter32(a);
            sh.redm[warp][lane] = a[0];
        }
        __syncthreads();
        double L = 0.0, E = 0.0;
        const bool valid = lane < nrows;
        const int il = g0 + (valid ? lane : 0);
        if (warp == 0) {
            double S = 0.0, MOv = 0.0;
#pragma unroll
            for (int w = 0; w < PWARPS; ++w) {
                S += (double)sh.red[w][lane];
                if (MOM) MOv += (double)sh.redm[w][lane];
            }
            // the window: no term clamped high (S <= 2^126 scaled), and the full
            // sum within C0 - 32 - log2(nc) below the reference (the engine's
            // fr_low_margin), i.e. log2(S) >= 32 + log2(nc) = low_floor
            // FP32 exponents: unscaled terms, the engine's 2^64 / FR32_LOW_MARGIN window
            const bool good = F32 ? (S > 0.0 && S <= 0x1p64 && log2(S) >= -FR32_LOW_MARGIN)
                                  : (S > 0.0 && S <= FR_SUM_MAX && log2(S) >= low_floor);
            if (valid && good) {
                L = LN2 * (R.H[il] + R.M2[il] + (log2(S) - (F32 ? 0.0 : (double)C0)));
                E = MOM ? MOv / S / inv_winf : 0.0;
            }
            const unsigned bad = __ballot_sync(0xffffffffu, valid && !good);
            if (lane == 0) sh.bad = bad;
        }
        __syncthreads();
        if (sh.bad) {
            // rows outside the window (a reference far from the new LSE): the
            // warps share them, each row by the two-pass loop of row_lse_twopass
            for (int k = 0, seen = 0; k < 32; ++k) {
                if (!((sh.bad >> k) & 1u)) continue;
                if ((seen++ % PWARPS) == warp) {
                    double Lx, Ex;
                    row_lse_twopass<PM, D, MOM>(s.pts, lo + g0 + k, cols, nc, colpot, cb * LN2, a2 * LN2,
                                                inv_winf, pexp, Lx, Ex);
                    if (lane == 0) { sh.fl[k] = Lx; sh.fe[k] = Ex; }
                }
            }
            __syncthreads();
            if (warp == 0 && ((sh.bad >> lane) & 1u)) { L = sh.fl[lane]; E = sh.fe[lane]; }
        }
        if (warp == 0) {
            double cv[4] = {0.0, 0.0, 0.0, 0.0};
            if (valid) epi(s, R, il, lo + il, L, E, cv);
#pragma unroll
            for (int off = 16; off > 0; off >>= 1)
#pragma unroll
                for (int k = 0; k < EPI::kN; ++k) cv[k] += __shfl_down_sync(0xffffffffu, cv[k], off);
            if (lane == 0)
#pragma unroll
                for (int k = 0; k < EPI::kN; ++k) part[k] += cv[k];
        }
        if (g0 + PRG < cnt) __syncthreads();
    }
}

// Sinkhorn row update of warp_logsumexp_ct_fused! (EPI_SK_ROW): pot = log(marg)
// - L into the cache and s.pot, the row's next reference L; cv[0] = marg . pot.
struct EpiSkRow {
    static constexpr int kN = 1;   // contributions per row
    __device__ void operator()(const Side &s, SideRows &R, int il, int o, double L, double, double (&cv)[4]) const {
        const double v = R.logm[il] - L;
        s.pot[o] = v;
        R.pot[il] = v;
        const double M2 = L * LOG2E - R.H[il];
        R.M2[il] = M2;
        R.xr[il].w = FR_MAGIC - (M2 + 1.0);
        R.xf[il].w = (float)(-M2);
        cv[0] = R.marg[il] * v;
    }
};

// Sinkhorn row residual of residual_opt! (EPI_SK_RESID): cv = {|marg - mass|,
// mass E[C], marg . pot}.
struct EpiSkResid {
    static constexpr int kN = 3;
    __device__ void operator()(const Side &, SideRows &R, int il, int, double L, double E, double (&cv)[4]) const {
        const double f = R.pot[il];
        const double mass = exp(f + L);
        cv[0] = fabs(R.marg[il] - mass);
        cv[1] = mass * E;
        cv[2] = R.marg[il] * f;
    }
};

// Sum over CTAs of slot k of the per-CTA partials, in CTA order (the same
// value in every CTA).
__device__ __forceinline__ double cta_total(const double *blk, int k) {
    double s = 0.0;
    for (int b = 0; b < (int)gridDim.x; ++b) s += __ldcg(blk + b * 4 + k);
    return s;
}

// The NS slot totals over CTAs ([G][NS] partials) by one warp: lane l sums
// CTAs l, l + 32, ... in order, then a fixed butterfly -- the same values in
// every CTA, since every CTA runs the same steps on the same data. Valid in
// every lane.
template <int NS>
__device__ __forceinline__ void cta_totals(const double *blk, double (&tot)[NS]) {
    static_assert(NS % 2 == 0, "slots are read in pairs");
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < NS; ++k) tot[k] = 0.0;
    for (int b = lane; b < (int)gridDim.x; b += 32) {
#pragma unroll
        for (int k = 0; k < NS; k += 2) {
            const double2 v = __ldcg(reinterpret_cast<const double2 *>(blk + (size_t)b * NS + k));
            tot[k] += v.x;
            tot[k + 1] += v.y;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int k = 0; k < NS; ++k) tot[k] += __shfl_xor_sync(0xffffffffu, tot[k], o);
}
__device__ __forceinline__ void cta_totals4(const double *blk, double (&tot)[4]) { cta_totals<4>(blk, tot); }

// The Sinkhorn loop (SinkhornKernel.jl:477-559): row update, column update,
// and every `frequency` iterations the residual check, until the tolerance,
// itermax or tmax stops it; the control step of each iteration as in
// FIN_SK_ITER / FIN_SK_CHECK.
template <int PM, int D>
__global__ void __launch_bounds__(PTPB, 1) sk_persist_kernel(const __grid_constant__ PersistParams P) {
    __shared__ PShared sh;
    __shared__ double s_tot[4];
    __shared__ int s_stop;
    Ctl *ctl = P.ctl;
    if (ctl->stop) return;
    const double alpha = -1.0 / (ctl->eta * ctl->winf);
    const double a2 = alpha * LOG2E;
    const double inv_winf = 1.0 / ctl->winf;
    double ctr[D];
#pragma unroll
    for (int k = 0; k < D; ++k) ctr[k] = P.X[k];
    const Side sx{P.X, P.r, P.phi, P.n};
    const Side sy{P.Y, P.c, P.psi, P.m};
    cache_side<PM, D>(sx, sh.side[0], ctr, a2);
    cache_side<PM, D>(sy, sh.side[1], ctr, a2);
    __syncthreads();
    long long iter = ctl->iter, num_iter = ctl->num_iter;
    const long long itermax = ctl->itermax, freq = ctl->frequency;
    const double tol = ctl->epsilon / 6.0;
    const int b = blockIdx.x, tid = threadIdx.x;
    unsigned gen = 0;
    double part[4];
    int stop_reason = 0;
    bool checked = false, failed = false;
    double residual = 0.0, objective = 0.0;
    // precision ladder (p = 2): FP32-exponent row and column passes while the
    // phase lasts; it ends, the same way in every CTA, at the first check whose
    // FP64 residual is within ctl->ladder_switch or has not improved for
    // LADDER_PATIENCE checks
    int fp32_phase = (PM == P_SQ && ctl->fp32_phase) ? 1 : 0;
    double ladder_prev = ctl->ladder_prev;
    int ladder_bad = ctl->ladder_bad;
    const double ladder_switch = ctl->ladder_switch;
    for (;;) {
        if constexpr (PM == P_SQ) {
            if (fp32_phase) {
                pass_rows<PM, D, false, 4, true>(sx, sh.side[0], P.Y, P.m, P.psi, LOG2E, ctr, a2, inv_winf,
                                                 P.pexp, EpiSkRow{}, sh, part);
                if (!grid_sync(P.bar, gen, &sh.flag)) { failed = true; break; }
                pass_rows<PM, D, false, 4, true>(sy, sh.side[1], P.X, P.n, P.phi, LOG2E, ctr, a2, inv_winf,
                                                 P.pexp, EpiSkRow{}, sh, part);
            }
        }
        if (!fp32_phase) {
            pass_rows<PM, D, false, 4, false>(sx, sh.side[0], P.Y, P.m, P.psi, LOG2E, ctr, a2, inv_winf, P.pexp,
                                              EpiSkRow{}, sh, part);
            if (!grid_sync(P.bar, gen, &sh.flag)) { failed = true; break; }
            pass_rows<PM, D, false, 4, false>(sy, sh.side[1], P.X, P.n, P.phi, LOG2E, ctr, a2, inv_winf, P.pexp,
                                              EpiSkRow{}, sh, part);
        }
        unsigned long long late = 0ull;   // CTA 0's tmax decision, carried by its arrival
        if (tid == 0) {
            P.blk[b * 4 + 0] = part[0];
            if (b == 0 && (double)(globaltimer_ns() - ctl->t_start_ns) * 1e-9 > ctl->tmax_s) late = PERSIST_LATE;
        }
        if (!grid_sync(P.bar, gen, &sh.flag, late, &sh.late)) { failed = true; break; }
        // FIN_SK_ITER, the same in every CTA
        iter += 1;
        int pending = 0;
        if (iter >= itermax) pending = 2;
        else if (sh.late) pending = 3;
        const bool do_check = ((iter - 1) % freq) == 0;
        if (!do_check) {
            num_iter += 1;
            if (pending) { stop_reason = pending; break; }
            continue;
        }
        pass_rows<PM, D, true, 2, false>(sx, sh.side[0], P.Y, P.m, P.psi, LOG2E, ctr, a2, inv_winf, P.pexp,
                                             EpiSkResid{}, sh, part);
        if (tid == 0) {
            P.blk[b * 4 + 1] = part[0];
            P.blk[b * 4 + 2] = part[1];
            P.blk[b * 4 + 3] = part[2];
        }
        if (!grid_sync(P.bar, gen, &sh.flag)) { failed = true; break; }
        // FIN_SK_CHECK, the same in every CTA
        if (tid < 32) {
            double t4[4];
            cta_totals4(P.blk, t4);
            if (tid == 0)
                for (int k = 0; k < 4; ++k) s_tot[k] = t4[k];
        }
        if (tid == 0) {
            const double l1 = s_tot[1];
            int st = 0;
            if (l1 <= tol) st = 1;
            else if (pending) st = pending;
            if (b == 0) put_log(ctl, (double)iter, l1, s_tot[2], nan(""), s_tot[0] + s_tot[3]);
            s_stop = st;
        }
        __syncthreads();
        checked = true;
        residual = s_tot[1];
        objective = s_tot[2];
        ladder_check(fp32_phase, ladder_prev, ladder_bad, residual, ladder_switch);
        if (s_stop != 1) num_iter += 1;
        if (s_stop) { stop_reason = s_stop; break; }
    }
    if (tid != 0) return;
    if (failed) {
        ctl->error = 1;
        ctl->stop = 1;
        return;
    }
    if (b != 0) return;
    // CTA 0 writes the state the pass-per-launch loop leaves behind
    ctl->dualval = cta_total(P.blk, 0);
    ctl->iter = iter;
    ctl->num_iter = num_iter;
    ctl->stop = 1;
    ctl->stop_reason = stop_reason;
    ctl->pending_stop = (stop_reason >= 2) ? stop_reason : 0;
    ctl->fp32_phase = fp32_phase;
    ctl->ladder_prev = ladder_prev;
    ctl->ladder_bad = ladder_bad;
    if (checked) {
        ctl->residual = residual;
        ctl->objective = objective;
    }
}


// ---------------------------------------------------------------------------
// LAMP (MirrorProxKernel.jl:1019-1132) in one persistent launch, small problems.
//
// An iteration is four passes, each a pass_rows over one side's rows:
//   k1  logZ_i = LSE_j(alpha C_ij + beta nu_j) at (eta_t, s_t)          x rows
//   k2  column residual at nu and the theta_bar / nu_bar step            y rows
//       (with the cost moment on check iterations)
//   kd  (check iterations) the dual pass LSE_j(alpha_d C_ij + beta_d theta_j)
//       and the primal / dual / tolerance test                           x rows
//   k3  logZ at nu_bar with (eta_next, s_next)                           x rows
//   k4  column residual at nu_bar and the theta / nu step, the
//       iteration bookkeeping                                            y rows
// separated by grid barriers, as the pass engine's k1 k2 k2m kd k3 k4 with
// FIN_LAMP_Z / A / DUAL / B. The coefficients change every pass (eta_t falls
// ~1/t), so each pass first recomputes its rows' scaled coordinates and
// fixed-reference offsets from the cached centred points and the row's
// previous log-sum-exp (the dual pass keeps its own). The column state (nu,
// nu_bar, theta, theta_bar, eta_mu) of a CTA's y rows lives in its shared
// memory and is written through to HBM, where the x passes read it.

struct LampParams {
    const double *X, *Y, *r, *c;
    double *nu, *nub, *theta, *thetab;   // column state (global copies)
    const double *eta_mu;                 // per-column eta_mu_i
    double *logz, *aux;                   // x rows: logZ and aux = log r - logZ
    int n, m;
    double pexp;
    double eta_mu_exp, minv, maxv;
    Ctl *ctl;
    double *blk;                          // [G][LAMP_SLOTS] per-CTA partials
    GridBar *bar;
};
constexpr int LAMP_SLOTS = 6;   // k1: sum r logZ; k2: |res - c|, cost, res nu, c theta; kd: sum r L

struct LShared {
    SideRows side[2];
    double4 vv[2][PMAXR];      // centred point (v, |v|^2) of each cached row
    double ref[2][PMAXR];      // natural-log LSE of the row's previous pass
    double refd[PMAXR];        // x rows: of the previous dual pass
    double nu[PMAXR], nub[PMAXR], th[PMAXR], thb[PMAXR], emu[PMAXR];   // y rows
    float red[PWARPS][32];
    float redm[PWARPS][32];
    double fl[32], fe[32];     // the group's rows recomputed by the fallback
    unsigned bad;              // rows of the group outside the window
    int flag;
    int late;                  // tmax passed (CTA 0's decision, via the barrier)
};

// Rows of one side for a pass with exponent coefficient a2 (log2 units):
// scaled coordinates, H = a2 |v|^2 (p = 2), M2 = ref log2(e) - H and the
// fixed-reference offset K.
template <int PM>
__device__ void lamp_prep(SideRows &R, const double4 *vv, const double *ref, int cnt, double a2) {
    constexpr bool SQ = (PM == P_SQ);
    for (int i = threadIdx.x; i < PMAXR; i += PTPB) {
        if (i >= cnt) {   // unused slots: finite junk, never finished
            R.H[i] = 0.0;
            R.M2[i] = 0.0;
            R.xr[i] = make_double4(0.0, 0.0, 0.0, FR_MAGIC - 1.0);
            continue;
        }
        const double4 v = vv[i];
        const double H = SQ ? a2 * v.w : 0.0;
        const double M2 = ref[i] * LOG2E - H;
        R.H[i] = H;
        R.M2[i] = M2;
        R.xr[i] = SQ ? make_double4(-2.0 * a2 * v.x, -2.0 * a2 * v.y, -2.0 * a2 * v.z, FR_MAGIC - (M2 + 1.0))
                     : make_double4(v.x, v.y, v.z, FR_MAGIC - (M2 + 1.0));
    }
    __syncthreads();
}

// k1 / k3 (EPI_LOGZ with FIN_LAMP_Z): logZ and aux = log r - logZ; cv[0] = r logZ.
struct EpiLamZ {
    static constexpr int kN = 1;
    double *logz, *aux, *ref;
    __device__ void operator()(const Side &, SideRows &R, int il, int o, double L, double, double (&cv)[4]) const {
        logz[o] = L;
        aux[o] = R.logm[il] - L;
        ref[il] = L;
        cv[0] = R.marg[il] * L;
    }
};

// kd (EPI_LOGZ into the dual value): cv[0] = r L.
struct EpiLamDual {
    static constexpr int kN = 1;
    double *refd;
    __device__ void operator()(const Side &, SideRows &R, int il, int, double L, double, double (&cv)[4]) const {
        refd[il] = L;
        cv[0] = R.marg[il] * L;
    }
};

// k2 / k4 (EPI_SPP_COL with the fused theta steps, MirrorProxKernel.jl:1104-1115):
// res_j = exp(beta rowpot_j + L_j). STEP_A: theta_bar, nu_bar from theta, nu,
// cv = {|res - c|, res E[C], res nu, c theta}; STEP_B: theta, nu from
// theta_bar (adjusted into [minv, maxv]).
template <bool STEP_A>
struct EpiLamCol {
    static constexpr int kN = STEP_A ? 4 : 0;
    double beta, en, eta_mu_exp, minv, maxv;
    double *g_nu, *g_nub, *g_th, *g_thb;
    double *nu, *nub, *th, *thb, *emu, *ref;
    __device__ void operator()(const Side &, SideRows &R, int il, int o, double L, double E, double (&cv)[4]) const {
        const double cj = R.marg[il];
        ref[il] = L;
        if constexpr (STEP_A) {
            const double rp = nu[il];
            const double res = exp(beta * rp + L);
            const double t0 = th[il];
            cv[0] = fabs(res - cj);
            cv[1] = res * E;
            cv[2] = res * rp;
            cv[3] = cj * t0;
            const double tb = theta_step(t0, res, cj, emu[il], eta_mu_exp, 0, minv, maxv, 1.0);
            const double nb = (1.0 - en) * rp + en * t0;
            thb[il] = tb;
            nub[il] = nb;
            g_thb[o] = tb;
            g_nub[o] = nb;
        } else {
            const double res = exp(beta * nub[il] + L);
            const double t1 = theta_step(th[il], res, cj, emu[il], eta_mu_exp, 1, minv, maxv, 1.0);
            const double n1 = (1.0 - en) * nu[il] + en * thb[il];
            th[il] = t1;
            nu[il] = n1;
            g_th[o] = t1;
            g_nu[o] = n1;
        }
    }
};

template <int PM, int D>
__global__ void __launch_bounds__(PTPB, 1) lamp_persist_kernel(const __grid_constant__ LampParams P) {
    __shared__ LShared sh;
    __shared__ double s_tot[LAMP_SLOTS];
    __shared__ double s_chk[4];     // residual, cost, primal, dual of the last check
    __shared__ int s_stop;
    Ctl *ctl = P.ctl;
    if (ctl->stop) return;
    const double winf = ctl->winf, eta_l = ctl->eta_lamp, tau_p = ctl->tau_p, hr = ctl->hr;
    const double tol = ctl->epsilon / 6.0;
    const double inv_winf = 1.0 / winf;
    const int check_enabled = ctl->check_enabled, marginal_only = ctl->marginal_only;
    double ctr[D];
#pragma unroll
    for (int k = 0; k < D; ++k) ctr[k] = P.X[k];
    const Side sx{P.X, P.r, P.aux, P.n};
    const Side sy{P.Y, P.c, P.nu, P.m};
    const int b = blockIdx.x, tid = threadIdx.x;
    const int lx = rows_lo(P.n), cx = rows_hi(P.n) - lx;
    const int ly = rows_lo(P.m), cy = rows_hi(P.m) - ly;
    // row caches; the first pass of each kind has no reference yet (NaN: the
    // window test fails and the rows take the exact loop)
    for (int i = tid; i < PMAXR; i += PTPB) {
#pragma unroll
        for (int side = 0; side < 2; ++side) {
            const double *pts = side ? P.Y : P.X;
            const int o = (side ? ly : lx) + i;
            const bool ok = i < (side ? cy : cx);
            double v[3] = {0.0, 0.0, 0.0}, h = 0.0;
#pragma unroll
            for (int k = 0; k < D; ++k) {
                v[k] = ok ? pts[(size_t)o * D + k] - ctr[k] : 0.0;
                h = fma(v[k], v[k], h);
            }
            sh.vv[side][i] = make_double4(v[0], v[1], v[2], h);
            sh.side[side].vf[i] = make_float4((float)v[0], (float)v[1], (float)v[2], 0.f);
            const double mg = ok ? (side ? P.c[o] : P.r[o]) : 1.0;
            sh.side[side].marg[i] = mg;
            sh.side[side].logm[i] = log(mg);
            sh.ref[side][i] = NAN;
        }
        sh.refd[i] = NAN;
        const bool oky = i < cy;
        const int oy = ly + i;
        sh.nu[i] = oky ? P.nu[oy] : 0.0;
        sh.nub[i] = oky ? P.nub[oy] : 0.0;
        sh.th[i] = oky ? P.theta[oy] : 0.0;
        sh.thb[i] = oky ? P.thetab[oy] : 0.0;
        sh.emu[i] = oky ? P.eta_mu[oy] : 1.0;
    }
    if (tid < 4) s_chk[tid] = 0.0;
    __syncthreads();
    long long iter = ctl->iter;
    const long long itermax = ctl->itermax, freq = ctl->frequency;
    double eta_t = ctl->eta_t, s_t = ctl->s_t, eta_n = ctl->eta_next, s_n = ctl->s_next;
    int do_check = ctl->do_check;
    unsigned gen = 0;
    double part[4];
    int stop_reason = 0;
    bool failed = false, checked = false;
    for (;;) {
        // k1: logZ at (nu, eta_t, s_t)
        const double a2c = -s_t / (2.0 * winf * eta_t) * LOG2E;
        const double bc = -1.0 / eta_t;
        lamp_prep<PM>(sh.side[0], sh.vv[0], sh.ref[0], cx, a2c);
        pass_rows<PM, D, false, 4, false>(sx, sh.side[0], P.Y, P.m, P.nu, bc * LOG2E, ctr, a2c, inv_winf, P.pexp,
                                          EpiLamZ{P.logz, P.aux, sh.ref[0]}, sh, part);
        if (tid == 0) P.blk[b * LAMP_SLOTS + 0] = part[0];
        if (!grid_sync(P.bar, gen, &sh.flag)) { failed = true; break; }
        // k2 (k2m on check iterations): column residual at nu, theta_bar / nu_bar step
        lamp_next(eta_t, s_t, tau_p, eta_l, eta_n, s_n);
        lamp_prep<PM>(sh.side[1], sh.vv[1], sh.ref[1], cy, a2c);
        const EpiLamCol<true> ea{bc, eta_n, P.eta_mu_exp, P.minv, P.maxv, P.nu, P.nub, P.theta, P.thetab,
                                 sh.nu, sh.nub, sh.th, sh.thb, sh.emu, sh.ref[1]};
        if (do_check)
            pass_rows<PM, D, true, 2, false>(sy, sh.side[1], P.X, P.n, P.aux, LOG2E, ctr, a2c, inv_winf, P.pexp,
                                             ea, sh, part);
        else
            pass_rows<PM, D, false, 4, false>(sy, sh.side[1], P.X, P.n, P.aux, LOG2E, ctr, a2c, inv_winf, P.pexp,
                                              ea, sh, part);
        if (tid == 0)
            for (int k = 0; k < 4; ++k) P.blk[b * LAMP_SLOTS + 1 + k] = part[k];
        if (!grid_sync(P.bar, gen, &sh.flag)) { failed = true; break; }
        if (do_check) {
            // kd: the dual value at theta (eta_lamp, s = 1)
            const double a2d = -1.0 / (2.0 * winf * eta_l) * LOG2E;
            const double bd = -1.0 / eta_l;
            lamp_prep<PM>(sh.side[0], sh.vv[0], sh.refd, cx, a2d);
            pass_rows<PM, D, false, 4, false>(sx, sh.side[0], P.Y, P.m, P.theta, bd * LOG2E, ctr, a2d, inv_winf,
                                              P.pexp, EpiLamDual{sh.refd}, sh, part);
            if (tid == 0) P.blk[b * LAMP_SLOTS + 5] = part[0];
            if (!grid_sync(P.bar, gen, &sh.flag)) { failed = true; break; }
            // FIN_LAMP_A's sums and FIN_LAMP_DUAL (MirrorProxKernel.jl:1084-1100),
            // the same in every CTA
            if (tid < 32) {
                double t6[LAMP_SLOTS];
                cta_totals<LAMP_SLOTS>(P.blk, t6);
                if (tid == 0)
                    for (int k = 0; k < LAMP_SLOTS; ++k) s_tot[k] = t6[k];
            }
            if (tid == 0) {
                const double sum_r_logz = s_tot[0], sum_res_c = s_tot[1], sum_cost = s_tot[2];
                const double sum_res_nu = s_tot[3], sum_c_theta = s_tot[4];
                const double q = eta_l / eta_t;
                const double pr = sum_cost * (1.0 - q) - q * sum_res_nu + q * sum_r_logz + 2.0 * winf * sum_res_c;
                const double du = -2.0 * eta_l * s_tot[5] - 2.0 * winf * sum_c_theta + 2.0 * hr;
                if (b == 0) put_log(ctl, (double)(iter + 1), sum_res_c, sum_cost, pr, du);
                const bool gap_ok = marginal_only ? true : (pr - du < tol);
                s_stop = (gap_ok && sum_res_c < tol) ? 1 : 0;
                s_chk[0] = sum_res_c; s_chk[1] = sum_cost; s_chk[2] = pr; s_chk[3] = du;
            }
            __syncthreads();
            checked = true;
            if (s_stop) { stop_reason = 1; break; }
        }
        // k3: logZ at (nu_bar, eta_next, s_next)
        const double a2n = -s_n / (2.0 * winf * eta_n) * LOG2E;
        const double bn = -1.0 / eta_n;
        lamp_prep<PM>(sh.side[0], sh.vv[0], sh.ref[0], cx, a2n);
        pass_rows<PM, D, false, 4, false>(sx, sh.side[0], P.Y, P.m, P.nub, bn * LOG2E, ctr, a2n, inv_winf, P.pexp,
                                          EpiLamZ{P.logz, P.aux, sh.ref[0]}, sh, part);
        if (!grid_sync(P.bar, gen, &sh.flag)) { failed = true; break; }
        // k4: column residual at nu_bar, theta / nu step
        lamp_prep<PM>(sh.side[1], sh.vv[1], sh.ref[1], cy, a2n);
        const EpiLamCol<false> eb{bn, eta_n, P.eta_mu_exp, P.minv, P.maxv, P.nu, P.nub, P.theta, P.thetab,
                                  sh.nu, sh.nub, sh.th, sh.thb, sh.emu, sh.ref[1]};
        pass_rows<PM, D, false, 4, false>(sy, sh.side[1], P.X, P.n, P.aux, LOG2E, ctr, a2n, inv_winf, P.pexp,
                                          eb, sh, part);
        unsigned long long late = 0ull;
        if (tid == 0 && b == 0 && (double)(globaltimer_ns() - ctl->t_start_ns) * 1e-9 > ctl->tmax_s)
            late = PERSIST_LATE;
        if (!grid_sync(P.bar, gen, &sh.flag, late, &sh.late)) { failed = true; break; }
        // FIN_LAMP_B, the same in every CTA
        eta_t = eta_n;
        s_t = s_n;
        iter += 1;
        int pending = 0;
        if (iter >= itermax) pending = 2;
        else if (sh.late) pending = 3;
        do_check = check_enabled && (iter % freq) == 0;
        if (pending) { stop_reason = pending; break; }
    }
    if (tid != 0) return;
    if (failed) {
        ctl->error = 1;
        ctl->stop = 1;
        return;
    }
    if (b != 0) return;
    ctl->iter = iter;
    ctl->num_iter = iter;
    ctl->eta_t = eta_t;
    ctl->s_t = s_t;
    ctl->eta_next = eta_n;
    ctl->s_next = s_n;
    ctl->do_check = do_check;
    ctl->stop = 1;
    ctl->stop_reason = stop_reason;
    ctl->pending_stop = (stop_reason >= 2) ? stop_reason : 0;
    if (checked) {
        ctl->residual = s_chk[0];
        ctl->objective = s_chk[1];
        ctl->primal = s_chk[2];
        ctl->dual = s_chk[3];
    }
}

// The grid barrier on a barrier that one CTA never reaches: CTA 1 leaves at
// once, CTA 0 waits with the given limit. out = {CTA 0's wait gave up, the
// counter carries PERSIST_ABORT}.
__global__ void grid_wait_probe_kernel(GridBar *gb, unsigned long long limit_ns, int *out) {
    __shared__ int flag;
    if (blockIdx.x != 0) return;
    unsigned gen = 0;
    const bool ok = grid_sync(gb, gen, &flag, 0ull, nullptr, limit_ns);
    if (threadIdx.x == 0) {
        out[0] = ok ? 0 : 1;
        out[1] = (gb->count >= PERSIST_ABORT) ? 1 : 0;
    }
}

}  // namespace culamp_dev


namespace culamp_host {

using namespace culamp_dev;

bool persist_eligible(int n, int m, int d, int pm_iter, int pm_resid, int grid) {
    if (pm_iter != pm_resid) return false;
    if (pm_iter != P_L1 && pm_iter != P_SQ && pm_iter != P_INF) return false;
    if (d < 1 || d > MAXD_PACKED || grid < 1) return false;
    // each thread's FP32 partial of a row covers at most 16 terms
    if (n > PERSIST_MAX_POINTS || m > PERSIST_MAX_POINTS) return false;
    // every CTA's rows of both sides fit its shared-memory row cache
    return (std::max(n, m) + grid - 1) / grid <= PMAXR;
}

size_t persist_scratch_bytes(int grid) {
    return (size_t)grid * 4 * sizeof(double) + sizeof(GridBar);
}

namespace {

template <int PM>
cudaError_t launch_pm(int d, const cudaLaunchConfig_t &cfg, const PersistParams &P) {
    switch (d) {
        case 1: return cudaLaunchKernelEx(&cfg, sk_persist_kernel<PM, 1>, P);
        case 2: return cudaLaunchKernelEx(&cfg, sk_persist_kernel<PM, 2>, P);
        default: return cudaLaunchKernelEx(&cfg, sk_persist_kernel<PM, 3>, P);
    }
}

}  // namespace

// One CTA per SM, if the kernel fits; the shared-memory carveout is kept at
// the least the kernel needs (~20 KB) so the rest of the SM's 256 KB serves as
// L1 for the column loads.
template <class FN>
int persist_grid_of(FN fn, int sm_count) {
    int per_sm = 0;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, PERSIST_CARVEOUT);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, PTPB, 0);
    if (e != cudaSuccess || per_sm < 1) {
        cudaGetLastError();
        return 0;
    }
    return sm_count;
}

int persist_grid(int sm_count, int d, int pm) {
    if (pm == P_SQ)
        return persist_grid_of(d == 1 ? sk_persist_kernel<P_SQ, 1> : d == 2 ? sk_persist_kernel<P_SQ, 2>
                                                                          : sk_persist_kernel<P_SQ, 3>, sm_count);
    if (pm == P_L1)
        return persist_grid_of(d == 1 ? sk_persist_kernel<P_L1, 1> : d == 2 ? sk_persist_kernel<P_L1, 2>
                                                                          : sk_persist_kernel<P_L1, 3>, sm_count);
    return persist_grid_of(d == 1 ? sk_persist_kernel<P_INF, 1> : d == 2 ? sk_persist_kernel<P_INF, 2>
                                                                       : sk_persist_kernel<P_INF, 3>, sm_count);
}

namespace {

using LampFn = void (*)(LampParams);

LampFn lamp_fn(int d, int pm) {
    if (pm == P_SQ) return d == 1 ? lamp_persist_kernel<P_SQ, 1> : d == 2 ? lamp_persist_kernel<P_SQ, 2> : lamp_persist_kernel<P_SQ, 3>;
    if (pm == P_L1) return d == 1 ? lamp_persist_kernel<P_L1, 1> : d == 2 ? lamp_persist_kernel<P_L1, 2> : lamp_persist_kernel<P_L1, 3>;
    return d == 1 ? lamp_persist_kernel<P_INF, 1> : d == 2 ? lamp_persist_kernel<P_INF, 2> : lamp_persist_kernel<P_INF, 3>;
}

}  // namespace

int lamp_persist_grid(int sm_count, int d, int pm) { return persist_grid_of(lamp_fn(d, pm), sm_count); }

size_t lamp_persist_scratch_bytes(int grid) {
    return (size_t)grid * LAMP_SLOTS * sizeof(double) + sizeof(GridBar);
}

cudaError_t launch_lamp_persist(const LampPersistArgs &a, int grid, cudaStream_t st) {
    LampParams P;
    P.X = a.X; P.Y = a.Y; P.r = a.r; P.c = a.c;
    P.nu = a.nu; P.nub = a.nub; P.theta = a.theta; P.thetab = a.thetab;
    P.eta_mu = a.eta_mu;
    P.logz = a.logz; P.aux = a.aux;
    P.n = a.n; P.m = a.m; P.pexp = a.pexp;
    P.eta_mu_exp = a.eta_mu_exp; P.minv = a.minv; P.maxv = a.maxv;
    P.ctl = a.ctl;
    P.blk = reinterpret_cast<double *>(a.scratch);
    P.bar = reinterpret_cast<GridBar *>(P.blk + (size_t)grid * LAMP_SLOTS);
    cudaError_t e = cudaMemsetAsync(P.bar, 0, sizeof(GridBar), st);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(PTPB);
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, lamp_fn(a.d, a.pm), P);
}

cudaError_t launch_sk_persist(const double *X, const double *Y, const double *r, const double *c,
                              double *phi, double *psi, int n, int m, int d, int pm, double pexp,
                              Ctl *ctl, void *scratch, int grid, cudaStream_t st) {
    PersistParams P;
    P.X = X; P.Y = Y; P.r = r; P.c = c; P.phi = phi; P.psi = psi;
    P.n = n; P.m = m; P.pexp = pexp; P.ctl = ctl;
    P.blk = reinterpret_cast<double *>(scratch);
    P.bar = reinterpret_cast<GridBar *>(P.blk + (size_t)grid * 4);
    cudaError_t e = cudaMemsetAsync(P.bar, 0, sizeof(GridBar), st);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(PTPB);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;   // all CTAs co-resident, or the launch fails
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    if (pm == P_SQ) return launch_pm<P_SQ>(d, cfg, P);
    if (pm == P_L1) return launch_pm<P_L1>(d, cfg, P);
    return launch_pm<P_INF>(d, cfg, P);
}

}  // namespace culamp_host

extern "C" int culamp_probe_grid_wait(culamp_handle h, uint64_t limit_ns, void *stream) {
    using namespace culamp_dev;
    if (!h) return CULAMP_ERR_INVALID_ARG;
    if (limit_ns == 0 || limit_ns > 10000000000ull)
        return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "wait limit must be in (0, 10 s]");
    cudaSetDevice(h->device);
    cudaStream_t st = (cudaStream_t)stream;
    if (h->tmpA.reserve(sizeof(GridBar) + 2 * sizeof(int)) != cudaSuccess)
        return culamp_set_error(h, CULAMP_ERR_ALLOC, "probe buffer");
    GridBar *gb = h->tmpA.as<GridBar>();
    int *dev = reinterpret_cast<int *>(gb + 1);
    if (cudaMemsetAsync(h->tmpA.ptr, 0, sizeof(GridBar) + 2 * sizeof(int), st) != cudaSuccess)
        return culamp_set_error(h, CULAMP_ERR_CUDA, "probe set-up failed");
    // two co-resident CTAs, as the persistent loops launch theirs
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(2);
    cfg.blockDim = dim3(32);
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int out[2] = {-1, -1};
    if (cudaLaunchKernelEx(&cfg, grid_wait_probe_kernel, gb, (unsigned long long)limit_ns, dev) != cudaSuccess ||
        cudaMemcpyAsync(out, dev, sizeof(out), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return culamp_set_error(h, CULAMP_ERR_CUDA, "grid wait probe failed");
    if (out[0] == 1 && out[1] == 1)
        return culamp_set_error(h, CULAMP_ERR_DEVICE_TIMEOUT, "grid barrier wait gave up after %llu ns",
                                (unsigned long long)limit_ns);
    return culamp_set_error(h, CULAMP_ERR_CUDA, "grid barrier wait did not give up (%d, %d)", out[0], out[1]);
}
