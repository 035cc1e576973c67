// persist.cu -- the whole Sinkhorn loop of a small problem in ONE cooperative
// launch (p = 2, d <= 3, n and m up to SK_PERSIST_MAX = 6144 points).
//
// At n = m = 4096 a pair pass does ~17 M pair updates, a few microseconds of
// pipe time, but as a separate launch it costs ~21 us: launch and prologue,
// the per-split partials written to L2 and merged by a last CTA, the epilogue.
// Here one CTA per SM stays resident for the whole solve:
//   * a CTA owns groups of 32 output rows (one per lane); its 16 warps split
//     the columns, so a row's partial (max, sum, moment) triples meet in shared
//     memory and are merged by warp 0 -- nothing per pair or per split goes
//     through global memory;
//   * every pass stages the other cloud and its potential (y - ctr, g) for all
//     columns once into shared memory (max(n, m) x 32 B);
//   * passes are separated by a grid barrier (arrival counter + generation,
//     every wait bounded by 2 s of the global timer);
//   * the iteration control of the graph path (FIN_SK_ITER / FIN_SK_CHECK of
//     SinkhornKernel.jl:524-539 as restated in engine.cuh) runs redundantly in
//     every CTA on a shared-memory copy of the control block, from the same
//     per-CTA partial sums read in the same order and one time stamp taken by
//     CTA 0, so all CTAs take the same branch; CTA 0 writes the log and the
//     final control block.
// Per pair the arithmetic is the packed online loop's (lse_step: FP64
// exponent, FP32 ex2 and Kahan chunk sums), so results differ from the pass
// path only by the order of the partial merges.
#include <cuda_runtime.h>

#include <cstring>

#include "internal.h"

namespace culamp_dev {

constexpr int PS_THREADS = 512;
constexpr int PS_WARPS = PS_THREADS / 32;
constexpr int PS_ROWS = 32;
constexpr unsigned long long PS_WAIT_NS = 2000000000ull;

struct PersistArgs {
    const double *X, *Y;       // staged clouds, point-major, d = D
    int n, m;
    const double *r, *c;       // marginals
    double *phi, *psi;         // potentials (phi / psi hold the starting point)
    Ctl *ctl;                  // control block (initialised, t_start set)
    double *blk;               // [gridDim.x][4] per-CTA partial sums
    unsigned *bar;             // [0] arrivals, [1] generation (zero before the launch)
    unsigned long long *tstamp;// CTA 0's clock for the iteration's tmax test
    int *err;                  // set when a barrier wait gave up
};

// Grid barrier; false when the wait gave up (the error flag is then set).
__device__ __forceinline__ bool ps_sync(const PersistArgs &A, int *s_ok) {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned *gen = A.bar + 1;
        const unsigned g = *gen;
        __threadfence();
        const unsigned arrived = atomicAdd(A.bar, 1u);
        int ok = 1;
        if (arrived == gridDim.x - 1) {
            atomicExch(A.bar, 0u);
            __threadfence();
            atomicAdd(A.bar + 1, 1u);
        } else {
            const unsigned long long t0 = globaltimer_ns();
            while (*gen == g) {
                if (globaltimer_ns() - t0 > PS_WAIT_NS) { ok = 0; atomicExch(A.err, 1); break; }
                __nanosleep(32);
            }
        }
        __threadfence();
        *s_ok = ok && (*(volatile int *)A.err == 0);
    }
    __syncthreads();
    return *s_ok != 0;
}

enum { PS_ROW = 0, PS_RESID = 1 };

// One reduction pass: for every output row o of `Xr` (nr rows), the log-sum-exp
// over the nc columns of `Yc` of a2 |x_o - y_j|^2 + LOG2E colpot_j (log2 units,
// centred on ctr). PS_ROW: out_o = log(marg_o) - L_o, acc[0] = sum marg.out.
// PS_RESID (moment on): acc = (sum |marg - mass|, sum mass E[C], sum marg.rowpot)
// with mass_o = exp(rowpot_o + L_o). acc (thread 0) is this CTA's sum over its
// row groups.
template <int D, int MODE>
__device__ __forceinline__ void ps_pass(const double *Xr, int nr, const double *Yc, int nc,
                                        const double *colpot, const double *rowpot, const double *marg,
                                        double *out, const double (&ctr)[3], double a2, double4 *scol,
                                        double (*sM)[PS_ROWS], double (*sS)[PS_ROWS],
                                        double (*sMO)[PS_ROWS], double (&acc)[4]) {
    constexpr bool MOM = (MODE == PS_RESID);
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    // stage all columns: (y - ctr, LOG2E pot + a2 |y - ctr|^2); potentials were
    // written by other CTAs in the previous pass: L2 loads
    for (int q = tid; q < nc; q += PS_THREADS) {
        double yy[3] = {0.0, 0.0, 0.0};
        double s2 = 0.0;
#pragma unroll
        for (int k = 0; k < D; ++k) {
            yy[k] = Yc[(size_t)q * D + k] - ctr[k];
            s2 = fma(yy[k], yy[k], s2);
        }
        double g = LOG2E * __ldcg(colpot + q);
        g += a2 * s2;
        scol[q] = make_double4(yy[0], yy[1], yy[2], g);
    }
    const int per = (nc + PS_WARPS - 1) / PS_WARPS;
    const int cb = min(nc, w * per), ce = min(nc, cb + per);
    const int groups = (nr + PS_ROWS - 1) / PS_ROWS;
    for (int grp = blockIdx.x; grp < groups; grp += gridDim.x) {
        __syncthreads();   // staging done / previous group's merge has read sM
        const int o = grp * PS_ROWS + lane;
        const bool ok = o < nr;
        double xr[1][D];
        double xs[1][D];
        double h = 0.0;
#pragma unroll
        for (int k = 0; k < D; ++k) {
            const double v = ok ? Xr[(size_t)o * D + k] - ctr[k] : 0.0;
            xr[0][k] = -2.0 * a2 * v;
            xs[0][k] = v;
            h = fma(v, v, h);
        }
        double M[1] = {-1e300};
        float S[1] = {0.f}, Cc[1] = {0.f}, cs[1] = {0.f}, mo[1] = {0.f};
        int q = cb;
        for (; q + 8 <= ce; q += 8) {
#pragma unroll
            for (int u = 0; u < 8; ++u) lse_step<P_SQ, D, 1, MOM>(scol[q + u], xr, xs, a2, 2.0, M, S, Cc, cs, mo);
            kahan_add(S[0], Cc[0], cs[0]);
            cs[0] = 0.f;
        }
        for (; q < ce; ++q) lse_step<P_SQ, D, 1, MOM>(scol[q], xr, xs, a2, 2.0, M, S, Cc, cs, mo);
        kahan_add(S[0], Cc[0], cs[0]);
        sM[w][lane] = M[0];
        sS[w][lane] = (double)S[0] - (double)Cc[0];
        sMO[w][lane] = (double)mo[0];
        __syncthreads();
        if (w == 0) {
            double Mm = sM[0][lane], Sm = sS[0][lane], MOm = sMO[0][lane];
            for (int ww = 1; ww < PS_WARPS; ++ww) merge_lse(Mm, Sm, MOm, sM[ww][lane], sS[ww][lane], sMO[ww][lane]);
            double a0 = 0.0, a1 = 0.0, a2s = 0.0;
            if (ok) {
                const double L = LN2 * (a2 * h + Mm + log2(Sm));
                if (MODE == PS_ROW) {
                    const double v = log(marg[o]) - L;
                    out[o] = v;
                    a0 = marg[o] * v;
                } else {
                    const double rp = __ldcg(rowpot + o);
                    const double Ec = (Sm > 0.0) ? MOm / Sm : 0.0;
                    const double mass = exp(rp + L);
                    a0 = fabs(marg[o] - mass);
                    a1 = mass * Ec;
                    a2s = marg[o] * rp;
                }
            }
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                a0 += __shfl_down_sync(0xffffffffu, a0, off);
                a1 += __shfl_down_sync(0xffffffffu, a1, off);
                a2s += __shfl_down_sync(0xffffffffu, a2s, off);
            }
            if (lane == 0) { acc[0] += a0; acc[1] += a1; acc[2] += a2s; }
        }
    }
}

// Publish this CTA's sums, pass the barrier, and total every CTA's sums in CTA
// order (the same totals in every CTA).
__device__ __forceinline__ bool ps_totals(const PersistArgs &A, const double (&acc)[4], double (&tot)[4],
                                          int *s_ok) {
    if (threadIdx.x == 0)
        for (int k = 0; k < 4; ++k) A.blk[blockIdx.x * 4 + k] = acc[k];
    if (!ps_sync(A, s_ok)) return false;
    for (int k = 0; k < 4; ++k) tot[k] = 0.0;
    for (unsigned b = 0; b < gridDim.x; ++b)
        for (int k = 0; k < 4; ++k) tot[k] += __ldcg(A.blk + b * 4 + k);
    return true;
}

template <int D>
__global__ void __launch_bounds__(PS_THREADS, 1) sk_persistent_kernel(const __grid_constant__ PersistArgs A) {
    extern __shared__ double4 scol[];
    __shared__ double sM[PS_WARPS][PS_ROWS], sS[PS_WARPS][PS_ROWS], sMO[PS_WARPS][PS_ROWS];
    __shared__ Ctl sctl;
    __shared__ int s_ok;
    if (threadIdx.x == 0) {
        sctl = *A.ctl;
        if (blockIdx.x != 0) sctl.log = nullptr;   // CTA 0 writes the log
    }
    __syncthreads();
    double ctr[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int k = 0; k < D; ++k) ctr[k] = A.X[k];
    const double a2 = (-1.0 / (sctl.eta * sctl.winf)) * LOG2E;
    PassParams fin = {};
    fin.ctl = &sctl;
    fin.finish = FIN_SK_CHECK;
    bool alive = true;
    while (alive && !sctl.stop) {
        double acc[4] = {0.0, 0.0, 0.0, 0.0}, tot[4];
        // phi = log r - LSE_j(-C_ij/(eta W) + psi_j)
        ps_pass<D, PS_ROW>(A.X, A.n, A.Y, A.m, A.psi, nullptr, A.r, A.phi, ctr, a2, scol, sM, sS, sMO, acc);
        if (!(alive = ps_sync(A, &s_ok))) break;
        // psi = log c - LSE_i(-C_ij/(eta W) + phi_i); iteration bookkeeping
        acc[0] = 0.0;
        ps_pass<D, PS_ROW>(A.Y, A.m, A.X, A.n, A.phi, nullptr, A.c, A.psi, ctr, a2, scol, sM, sS, sMO, acc);
        if (blockIdx.x == 0 && threadIdx.x == 0) *(volatile unsigned long long *)A.tstamp = globaltimer_ns();
        if (!(alive = ps_totals(A, acc, tot, &s_ok))) break;
        if (threadIdx.x == 0) {
            Ctl *c = &sctl;
            const unsigned long long now = __ldcg(A.tstamp);
            c->dualval = tot[0];
            c->iter += 1;
            if (c->iter >= c->itermax) c->pending_stop = 2;
            else if ((double)(now - c->t_start_ns) * 1e-9 > c->tmax_s) c->pending_stop = 3;
            c->do_check = ((c->iter - 1) % c->frequency) == 0;
            if (!c->do_check && c->pending_stop) { c->stop = 1; c->stop_reason = c->pending_stop; c->num_iter += 1; }
            else if (!c->do_check) c->num_iter += 1;
            c->loops += 1;
        }
        __syncthreads();
        if (sctl.do_check && !sctl.stop) {
            // residual and transport cost at (phi, psi); tolerance test
            double acc2[4] = {0.0, 0.0, 0.0, 0.0};
            ps_pass<D, PS_RESID>(A.X, A.n, A.Y, A.m, A.psi, A.phi, A.r, nullptr, ctr, a2, scol, sM, sS, sMO, acc2);
            if (!(alive = ps_totals(A, acc2, tot, &s_ok))) break;
            if (threadIdx.x == 0) run_finish(fin, tot);
            __syncthreads();
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        if (*(volatile int *)A.err) sctl.error = 1;
        *A.ctl = sctl;
    }
}

}  // namespace culamp_dev

namespace culamp_host {

using culamp_dev::PersistArgs;

size_t sk_persistent_scratch_bytes(int sm_count) {
    return (size_t)sm_count * 4 * sizeof(double) + 64;
}

template <int D>
static cudaError_t launch_persist_d(const PersistArgs &A, int n, int m, int sm_count, cudaStream_t st,
                                    bool *used) {
    auto kern = culamp_dev::sk_persistent_kernel<D>;
    const size_t smem = (size_t)(n > m ? n : m) * sizeof(double4);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) { cudaGetLastError(); return cudaSuccess; }   // too large: pass path
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, culamp_dev::PS_THREADS, smem);
    if (e != cudaSuccess || per_sm < 1) { cudaGetLastError(); return cudaSuccess; }
    const int groups = ((n > m ? n : m) + culamp_dev::PS_ROWS - 1) / culamp_dev::PS_ROWS;
    int grid = sm_count;                           // one CTA per SM at most
    if (grid > groups) grid = groups;
    PersistArgs a = A;
    void *args[] = {&a};
    e = cudaLaunchCooperativeKernel((const void *)kern, dim3(grid), dim3(culamp_dev::PS_THREADS), args, smem, st);
    if (e != cudaSuccess) return e;
    *used = true;
    return cudaSuccess;
}

cudaError_t launch_sk_persistent(const double *X, const double *Y, int n, int m, int d, const double *r,
                                 const double *c, double *phi, double *psi, Ctl *ctl, void *scratch,
                                 int sm_count, cudaStream_t st, bool *used) {
    *used = false;
    if (d < 1 || d > 3 || n > SK_PERSIST_MAX || m > SK_PERSIST_MAX) return cudaSuccess;
    unsigned char *sb = reinterpret_cast<unsigned char *>(scratch);
    PersistArgs A;
    std::memset(&A, 0, sizeof(A));
    A.X = X; A.Y = Y; A.n = n; A.m = m; A.r = r; A.c = c; A.phi = phi; A.psi = psi; A.ctl = ctl;
    A.bar = reinterpret_cast<unsigned *>(sb);
    A.err = reinterpret_cast<int *>(sb + 8);
    A.tstamp = reinterpret_cast<unsigned long long *>(sb + 16);
    A.blk = reinterpret_cast<double *>(sb + 64);
    cudaError_t e = cudaMemsetAsync(sb, 0, 64, st);
    if (e != cudaSuccess) return e;
    switch (d) {
        case 1: return launch_persist_d<1>(A, n, m, sm_count, st, used);
        case 2: return launch_persist_d<2>(A, n, m, sm_count, st, used);
        default: return launch_persist_d<3>(A, n, m, sm_count, st, used);
    }
}

}  // namespace culamp_host
