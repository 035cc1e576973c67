// adjoint.cu -- the adjoint pass of the Sinkhorn transport cost.
//
// For the entropic OT value at optimal potentials, OT_eps = eps (a.phi + b.psi)
// with P_ij = exp(phi_i + psi_j - C_ij / eps), the envelope theorem gives
//     d OT_eps / d x_i = sum_j P_ij  grad_x C(x_i, y_j)       (eps held fixed)
// so one pass over all pairs, recomputing P_ij on the fly, yields the gradient
// with respect to every point without ever storing the n x m plan. The pass has
// the row-reduction shape of naive_findmaxindex_ct! (SinkhornKernel.jl:124-162):
// per row, a weighted sum over columns.
//
// Layout as the pair passes: a CTA owns 2 x 128 rows (registers), columns are
// staged through shared memory in tiles of 128 points + potential. The
// exponent is formed in FP64, the running row max is tracked in FP64, 2^u runs
// on the MUFU pipe, and the mass and gradient sums are FP64.
#include <cuda_runtime.h>

#include "internal.h"

namespace {

using namespace culamp_dev;

constexpr int ADJ_TPB = 128;
constexpr int ADJ_R = 2;
constexpr int ADJ_CHUNK = 128;

// d C(x, y) / d x_k for the reference's costs: p = 2 -> 2 (x - y); p = 1 ->
// sign(x - y); p = Inf -> sign(x - y) on the (first) maximising coordinate;
// other p -> p |x - y|^(p-1) sign(x - y).
template <int PM, int D>
__device__ __forceinline__ void cost_grad(const double (&df)[D], double p, double (&g)[D]) {
    if (PM == P_SQ) {
#pragma unroll
        for (int k = 0; k < D; ++k) g[k] = 2.0 * df[k];
    } else if (PM == P_L1) {
#pragma unroll
        for (int k = 0; k < D; ++k) g[k] = (df[k] > 0.0) - (df[k] < 0.0);
    } else if (PM == P_INF) {
        int kmax = 0;
        double vmax = -1.0;
#pragma unroll
        for (int k = 0; k < D; ++k) {
            const double a = fabs(df[k]);
            if (a > vmax) { vmax = a; kmax = k; }
        }
#pragma unroll
        for (int k = 0; k < D; ++k) g[k] = (k == kmax) ? (double)((df[k] > 0.0) - (df[k] < 0.0)) : 0.0;
    } else {
#pragma unroll
        for (int k = 0; k < D; ++k) {
            const double a = fabs(df[k]);
            g[k] = (a > 0.0) ? p * pow(a, p - 1.0) * ((df[k] > 0.0) - (df[k] < 0.0)) : 0.0;
        }
    }
}

template <int PM, int D>
__device__ __forceinline__ double cost_of(const double (&df)[D], double p) {
    double c = 0.0;
#pragma unroll
    for (int k = 0; k < D; ++k) {
        if (PM == P_SQ) c = fma(df[k], df[k], c);
        else if (PM == P_L1) c += fabs(df[k]);
        else if (PM == P_INF) c = fmax(c, fabs(df[k]));
        else c += pow(fabs(df[k]), p);
    }
    return c;
}

template <int PM, int D>
__global__ void __launch_bounds__(ADJ_TPB) adjoint_kernel(double *grad, double *mass,
                                                         const double *X, const double *Y, int n,
                                                         int m, const double *phi,
                                                         const double *psi, double k2,
                                                         double p) {
    __shared__ double ys[ADJ_CHUNK][D + 1];
    const int tid = threadIdx.x;
    double x[ADJ_R][D], ph[ADJ_R], M[ADJ_R], S[ADJ_R], G[ADJ_R][D];
    int rows[ADJ_R];
#pragma unroll
    for (int r = 0; r < ADJ_R; ++r) {
        rows[r] = blockIdx.x * ADJ_TPB * ADJ_R + tid + r * ADJ_TPB;
        const bool ok = rows[r] < n;
#pragma unroll
        for (int k = 0; k < D; ++k) {
            x[r][k] = ok ? X[(size_t)rows[r] * D + k] : 0.0;
            G[r][k] = 0.0;
        }
        ph[r] = ok ? phi[rows[r]] * LOG2E : 0.0;
        M[r] = -1e300;
        S[r] = 0.0;
    }
    for (int c0 = 0; c0 < m; c0 += ADJ_CHUNK) {
        __syncthreads();
        for (int q = tid; q < ADJ_CHUNK; q += ADJ_TPB) {
            const int j = c0 + q;
#pragma unroll
            for (int k = 0; k < D; ++k) ys[q][k] = (j < m) ? Y[(size_t)j * D + k] : 0.0;
            ys[q][D] = (j < m) ? psi[j] * LOG2E : -INFINITY;
        }
        __syncthreads();
        const int nc = min(ADJ_CHUNK, m - c0);
        for (int q = 0; q < nc; ++q) {
#pragma unroll
            for (int r = 0; r < ADJ_R; ++r) {
                double df[D];
#pragma unroll
                for (int k = 0; k < D; ++k) df[k] = x[r][k] - ys[q][k];
                // log2 of P_ij
                const double t = fma(cost_of<PM, D>(df, p), k2, ph[r] + ys[q][D]);
                if (t > M[r]) {
                    const double sc = exp2(M[r] - t);
                    S[r] *= sc;
#pragma unroll
                    for (int k = 0; k < D; ++k) G[r][k] *= sc;
                    M[r] = t;
                }
                const double e = (double)ex2_approx((float)(t - M[r]));
                double g[D];
                cost_grad<PM, D>(df, p, g);
                S[r] += e;
#pragma unroll
                for (int k = 0; k < D; ++k) G[r][k] = fma(e, g[k], G[r][k]);
            }
        }
    }
#pragma unroll
    for (int r = 0; r < ADJ_R; ++r) {
        if (rows[r] >= n) continue;
        const double scale = exp2(M[r]);
        if (mass) mass[rows[r]] = S[r] * scale;
#pragma unroll
        for (int k = 0; k < D; ++k) grad[(size_t)rows[r] * D + k] = G[r][k] * scale;
    }
}

template <int PM>
cudaError_t launch_adjoint_p(double *grad, double *mass, const double *x, const double *y, int n,
                             int m, int d, const double *phi, const double *psi, double k2,
                             double p, cudaStream_t st) {
    const unsigned blocks = (unsigned)((n + ADJ_TPB * ADJ_R - 1) / (ADJ_TPB * ADJ_R));
    switch (d) {
        case 1: adjoint_kernel<PM, 1><<<blocks, ADJ_TPB, 0, st>>>(grad, mass, x, y, n, m, phi, psi, k2, p); break;
        case 2: adjoint_kernel<PM, 2><<<blocks, ADJ_TPB, 0, st>>>(grad, mass, x, y, n, m, phi, psi, k2, p); break;
        case 3: adjoint_kernel<PM, 3><<<blocks, ADJ_TPB, 0, st>>>(grad, mass, x, y, n, m, phi, psi, k2, p); break;
        case 4: adjoint_kernel<PM, 4><<<blocks, ADJ_TPB, 0, st>>>(grad, mass, x, y, n, m, phi, psi, k2, p); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Fixed-reference adjoint (p = 2, d <= 3), the hot form for solved potentials.
//
// At solved potentials every row mass sum_j P_ij is its marginal a_i <= 1, so
// every term P_ij <= 1: the reference of the fixed-point exponent (the row
// log-sum-exp the pair passes use) is simply 0, known before the pass. Each
// pair then costs what a fixed-reference row pass costs -- d DFMA + 1 DADD for
// the exponent (|x|^2 + |y|^2 - 2 x.y with the column term in g_j and the row
// term in K_i), one integer clamp, one funnel shift, one MUFU ex2 and an
// exponent-field add -- plus d FP32 FMAs for Y_i = sum_j P_ij (y_j - c). The
// gradient is 2 (S_i (x_i - c) - Y_i) with S_i = sum_j P_ij, formed in FP64 at
// the end; the sums are 16-term FP32 chunks merged with Kahan compensation.
// Columns are split over CTAs (waves of resident CTAs, as the row passes) and
// the splits' (M, S, Y) partials merged by the last CTA of each row block. A
// slice whose sum leaves the window (a term above the reference, i.e. row mass
// well above 1) and a row whose total lies too far below it are recomputed
// with the FP64 online loop, so any potentials give the right result.
constexpr int AFR_TPB = 128;
constexpr int AFR_R = 4;
constexpr int AFR_CH = 256;
constexpr int AFR_NP = 5;   // partial record: M, S, Y_0..2

struct AdjFr {
    const double *X, *Y, *phi, *psi;
    int n, m;
    double k2;                 // -log2(e) / eps
    int splits, cols_per_split;
    double *part;              // [splits][n][AFR_NP] when splits > 1
    unsigned *tickets;         // [row blocks]
    double *grad, *mass;
};

// FP64 online loop over columns [cb, ce) for this thread's rows: M (log2 units),
// S = sum 2^(t - M), Yc_k = sum 2^(t - M) (y_k - c_k).
template <int D>
__device__ __forceinline__ void adj_online(const AdjFr &P, int row_base, int cb, int ce, double *smem,
                                           const double (&ctr)[D], double (&M)[AFR_R], double (&S)[AFR_R],
                                           double (&Yc)[AFR_R][3]) {
    const int tid = threadIdx.x;
    double xc[AFR_R][D], ph[AFR_R];
#pragma unroll
    for (int r = 0; r < AFR_R; ++r) {
        const int row = row_base + tid + r * AFR_TPB;
        const bool ok = row < P.n;
#pragma unroll
        for (int k = 0; k < D; ++k) xc[r][k] = ok ? P.X[(size_t)row * D + k] - ctr[k] : 0.0;
        ph[r] = ok ? P.phi[row] * LOG2E : 0.0;
        M[r] = -1e300;
        S[r] = 0.0;
        Yc[r][0] = Yc[r][1] = Yc[r][2] = 0.0;
    }
    double4 *tile = reinterpret_cast<double4 *>(smem);
    for (int c0 = cb; c0 < ce; c0 += AFR_CH) {
        __syncthreads();
        for (int q = tid; q < AFR_CH; q += AFR_TPB) {
            const int j = c0 + q;
            double v[3] = {0.0, 0.0, 0.0};
            if (j < ce)
#pragma unroll
                for (int k = 0; k < D; ++k) v[k] = P.Y[(size_t)j * D + k] - ctr[k];
            tile[q] = make_double4(v[0], v[1], v[2], j < ce ? P.psi[j] * LOG2E : -INFINITY);
        }
        __syncthreads();
        const int nc = min(AFR_CH, ce - c0);
        for (int q = 0; q < nc; ++q) {
            const double4 col = tile[q];
            const double yv[3] = {col.x, col.y, col.z};
#pragma unroll
            for (int r = 0; r < AFR_R; ++r) {
                double c = 0.0;
#pragma unroll
                for (int k = 0; k < D; ++k) { const double df = xc[r][k] - yv[k]; c = fma(df, df, c); }
                const double t = fma(c, P.k2, ph[r] + col.w);
                if (t > M[r]) {
                    const double sc = exp2(M[r] - t);
                    S[r] *= sc;
#pragma unroll
                    for (int k = 0; k < D; ++k) Yc[r][k] *= sc;
                    M[r] = t;
                }
                const double e = (double)ex2_approx((float)(t - M[r]));
                S[r] += e;
#pragma unroll
                for (int k = 0; k < D; ++k) Yc[r][k] = fma(e, yv[k], Yc[r][k]);
            }
        }
    }
}

// Fixed-reference loop over [cb, ce); returns false if a real row's sum left
// the window. M = 0 (the reference), S and Yc unscaled.
template <int D>
__device__ __forceinline__ bool adj_fixedref(const AdjFr &P, int row_base, int cb, int ce, double *smem,
                                             const double (&ctr)[D], double (&M)[AFR_R], double (&S)[AFR_R],
                                             double (&Yc)[AFR_R][3]) {
    const int tid = threadIdx.x;
    double xr[AFR_R][D], K[AFR_R];
    float St[AFR_R], Sc[AFR_R], Yt[AFR_R][3], Yq[AFR_R][3], cs[AFR_R], cy[AFR_R][3];
#pragma unroll
    for (int r = 0; r < AFR_R; ++r) {
        const int row = row_base + tid + r * AFR_TPB;
        const bool ok = row < P.n;
        double h = 0.0;
#pragma unroll
        for (int k = 0; k < D; ++k) {
            const double v = ok ? P.X[(size_t)row * D + k] - ctr[k] : 0.0;
            xr[r][k] = -2.0 * P.k2 * v;
            h = fma(v, v, h);
        }
        // full exponent T = g_j + xr.y + (phi_i log2 e + k2 |x - c|^2); reference 0
        const double rowterm = ok ? fma(P.k2, h, P.phi[row] * LOG2E) : 0.0;
        K[r] = FR_MAGIC - (1.0 - rowterm);
        St[r] = Sc[r] = cs[r] = 0.f;
#pragma unroll
        for (int k = 0; k < 3; ++k) Yt[r][k] = Yq[r][k] = cy[r][k] = 0.f;
    }
    double4 *tile = reinterpret_cast<double4 *>(smem);
    float4 *tf = reinterpret_cast<float4 *>(smem + 4 * AFR_CH);
    for (int c0 = cb; c0 < ce; c0 += AFR_CH) {
        __syncthreads();
        for (int q = tid; q < AFR_CH; q += AFR_TPB) {
            const int j = c0 + q;
            double v[3] = {0.0, 0.0, 0.0};
            double g = -INFINITY;
            if (j < ce) {
                double s2 = 0.0;
#pragma unroll
                for (int k = 0; k < D; ++k) {
                    v[k] = P.Y[(size_t)j * D + k] - ctr[k];
                    s2 = fma(v[k], v[k], s2);
                }
                g = fma(P.k2, s2, P.psi[j] * LOG2E);
            }
            tile[q] = make_double4(v[0], v[1], v[2], g);
            tf[q] = make_float4((float)v[0], (float)v[1], (float)v[2], 0.f);
        }
        __syncthreads();
        const int nc = min(AFR_CH, ce - c0);
        for (int q0 = 0; q0 < nc; q0 += 16) {
            const int q1 = min(nc, q0 + 16);
#pragma unroll 2
            for (int q = q0; q < q1; ++q) {
                const double4 col = tile[q];
                const float4 yf = tf[q];
                float e[AFR_R];
                fr_terms<P_SQ, D, AFR_R>(col, xr, 0.0, 0.0, K, e);
#pragma unroll
                for (int r = 0; r < AFR_R; ++r) {
                    cs[r] += e[r];
                    cy[r][0] = fmaf(e[r], yf.x, cy[r][0]);
                    if (D >= 2) cy[r][1] = fmaf(e[r], yf.y, cy[r][1]);
                    if (D >= 3) cy[r][2] = fmaf(e[r], yf.z, cy[r][2]);
                }
            }
#pragma unroll
            for (int r = 0; r < AFR_R; ++r) {
                kahan_add(St[r], Sc[r], cs[r]);
                cs[r] = 0.f;
#pragma unroll
                for (int k = 0; k < D; ++k) { kahan_add(Yt[r][k], Yq[r][k], cy[r][k]); cy[r][k] = 0.f; }
            }
        }
    }
    bool good = true;
#pragma unroll
    for (int r = 0; r < AFR_R; ++r) {
        const int row = row_base + tid + r * AFR_TPB;
        const double sv = (double)St[r] - (double)Sc[r];
        if (row < P.n && !(sv <= FR_SUM_MAX)) good = false;
        M[r] = 0.0;
        S[r] = sv * FR_UNSCALE;
#pragma unroll
        for (int k = 0; k < 3; ++k) Yc[r][k] = (k < D) ? ((double)Yt[r][k] - (double)Yq[r][k]) * FR_UNSCALE : 0.0;
    }
    return good;
}

__device__ __forceinline__ void adj_merge(double &M, double &S, double (&Y)[3], double M2, double S2,
                                          const double (&Y2)[3]) {
    if (!(S2 > 0.0)) return;
    if (!(S > 0.0)) { M = M2; S = S2; Y[0] = Y2[0]; Y[1] = Y2[1]; Y[2] = Y2[2]; return; }
    if (M2 == M) { S += S2; Y[0] += Y2[0]; Y[1] += Y2[1]; Y[2] += Y2[2]; return; }
    if (M2 > M) {
        const double f = exp2(M - M2);
        S = S * f + S2;
        for (int k = 0; k < 3; ++k) Y[k] = Y[k] * f + Y2[k];
        M = M2;
    } else {
        const double f = exp2(M2 - M);
        S += S2 * f;
        for (int k = 0; k < 3; ++k) Y[k] += Y2[k] * f;
    }
}

template <int D>
__global__ void __launch_bounds__(AFR_TPB, 3) adjoint_fr_kernel(const __grid_constant__ AdjFr P) {
    extern __shared__ __align__(16) double smem[];   // AFR_CH double4 + AFR_CH float4
    __shared__ int s_last;
    const int rb = blockIdx.x, sp = blockIdx.y;
    const int row_base = rb * AFR_TPB * AFR_R;
    const int cb = sp * P.cols_per_split;
    const int ce = min(P.m, cb + P.cols_per_split);
    double ctr[D];
#pragma unroll
    for (int k = 0; k < D; ++k) ctr[k] = P.X[k];   // centring point: the first row point
    double M[AFR_R], S[AFR_R], Yc[AFR_R][3];
    bool fr = adj_fixedref<D>(P, row_base, cb, ce, smem, ctr, M, S, Yc);
    if (__syncthreads_or(!fr)) adj_online<D>(P, row_base, cb, ce, smem, ctr, M, S, Yc);
    if (P.splits > 1) {
#pragma unroll
        for (int r = 0; r < AFR_R; ++r) {
            const int row = row_base + threadIdx.x + r * AFR_TPB;
            if (row >= P.n) continue;
            double *pp = P.part + ((size_t)sp * P.n + row) * AFR_NP;
            pp[0] = M[r]; pp[1] = S[r]; pp[2] = Yc[r][0]; pp[3] = Yc[r][1]; pp[4] = Yc[r][2];
        }
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) {
            const unsigned t = atomicAdd(&P.tickets[rb], 1u);
            s_last = (t == (unsigned)(P.splits - 1));
        }
        __syncthreads();
        if (!s_last) return;
        __threadfence();
        fr = true;
#pragma unroll
        for (int r = 0; r < AFR_R; ++r) {
            const int row = row_base + threadIdx.x + r * AFR_TPB;
            M[r] = -INFINITY; S[r] = 0.0; Yc[r][0] = Yc[r][1] = Yc[r][2] = 0.0;
            if (row >= P.n) continue;
            for (int s2 = 0; s2 < P.splits; ++s2) {
                const double *pp = P.part + ((size_t)s2 * P.n + row) * AFR_NP;
                const double y2[3] = {__ldcg(pp + 2), __ldcg(pp + 3), __ldcg(pp + 4)};
                const double m2 = __ldcg(pp);
                if (m2 != 0.0) fr = false;   // an online partial: the window check does not apply
                adj_merge(M[r], S[r], Yc[r], m2, __ldcg(pp + 1), y2);
            }
        }
        if (threadIdx.x == 0) P.tickets[rb] = 0u;
        fr = !__syncthreads_or(!fr);
    }
    if (fr) {
        // lower side of the window on the full row: clamped-low terms (each at most
        // 2^(2 - FR_C0) of the reference 1) must stay below 2^-30 of the row mass
        bool bad = false;
        const double margin = fr_low_margin(P.m);
#pragma unroll
        for (int r = 0; r < AFR_R; ++r) {
            const int row = row_base + threadIdx.x + r * AFR_TPB;
            if (row < P.n && (!(S[r] > 0.0) || log2(S[r]) < -margin)) bad = true;
        }
        if (__syncthreads_or(bad)) adj_online<D>(P, row_base, 0, P.m, smem, ctr, M, S, Yc);
    }
#pragma unroll
    for (int r = 0; r < AFR_R; ++r) {
        const int row = row_base + threadIdx.x + r * AFR_TPB;
        if (row >= P.n) continue;
        const double sc = exp2(M[r]);
        if (P.mass) P.mass[row] = S[r] * sc;
#pragma unroll
        for (int k = 0; k < D; ++k) {
            const double xc = P.X[(size_t)row * D + k] - ctr[k];
            P.grad[(size_t)row * D + k] = 2.0 * (xc * S[r] - Yc[r][k]) * sc;
        }
    }
}

}  // namespace

extern "C" int culamp_adjoint_sk(culamp_handle h, double *grad, double *mass, const double *x,
                                 const double *y, int64_t n, int64_t m, int32_t d,
                                 const double *phi, const double *psi, double reg, double winf,
                                 double p, void *stream) {
    if (!h) return CULAMP_ERR_INVALID_ARG;
    if (!grad || !x || !y || !phi || !psi || n < 1 || m < 1 || n > (1LL << 28) || m > (1LL << 28))
        return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "bad adjoint arguments");
    if (d < 1 || d > 4) return culamp_set_error(h, CULAMP_ERR_UNSUPPORTED, "adjoint supports 1 <= d <= 4");
    if (!(p > 0.0) || !(reg * winf > 0.0))
        return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "adjoint needs p > 0 and reg * winf > 0");
    cudaSetDevice(h->device);
    const double k2 = -LOG2E / (reg * winf);   // log2 units
    cudaError_t e;
    if (culamp_host::pmode_of(p) == P_SQ && d <= 3) {
        // fixed-reference form; columns split so the grid fills the resident slots
        const int rb = (int)((n + AFR_TPB * AFR_R - 1) / (AFR_TPB * AFR_R));
        const int slots = 3 * h->sm_count;
        int splits = (slots + rb - 1) / rb;
        const int max_splits = (int)((m + AFR_CH - 1) / AFR_CH);
        if (splits > max_splits) splits = max_splits;
        if (splits < 1) splits = 1;
        int cps = (int)((m + splits - 1) / splits);
        cps = ((cps + AFR_CH - 1) / AFR_CH) * AFR_CH;
        splits = (int)((m + cps - 1) / cps);
        if (splits > 1) {
            e = h->scratch.reserve((size_t)splits * (size_t)n * AFR_NP * sizeof(double), (size_t)rb);
            if (e != cudaSuccess)
                return culamp_set_error(h, CULAMP_ERR_ALLOC, "adjoint scratch: %s", cudaGetErrorString(e));
        }
        AdjFr P;
        P.X = x; P.Y = y; P.phi = phi; P.psi = psi;
        P.n = (int)n; P.m = (int)m; P.k2 = k2;
        P.splits = splits; P.cols_per_split = cps;
        P.part = h->scratch.part.as<double>();
        P.tickets = h->scratch.tickets.as<unsigned>();
        P.grad = grad; P.mass = mass;
        const size_t smem = AFR_CH * (4 * sizeof(double) + 4 * sizeof(float));
        const dim3 grid((unsigned)rb, (unsigned)splits);
        cudaStream_t st = (cudaStream_t)stream;
        switch (d) {
            case 1: adjoint_fr_kernel<1><<<grid, AFR_TPB, smem, st>>>(P); break;
            case 2: adjoint_fr_kernel<2><<<grid, AFR_TPB, smem, st>>>(P); break;
            default: adjoint_fr_kernel<3><<<grid, AFR_TPB, smem, st>>>(P); break;
        }
        e = cudaGetLastError();
        if (e != cudaSuccess)
            return culamp_set_error(h, CULAMP_ERR_CUDA, "adjoint launch: %s", cudaGetErrorString(e));
        return CULAMP_OK;
    }
    switch (culamp_host::pmode_of(p)) {
        case P_L1: e = launch_adjoint_p<P_L1>(grad, mass, x, y, (int)n, (int)m, d, phi, psi, k2, p, (cudaStream_t)stream); break;
        case P_SQ: e = launch_adjoint_p<P_SQ>(grad, mass, x, y, (int)n, (int)m, d, phi, psi, k2, p, (cudaStream_t)stream); break;
        case P_INF: e = launch_adjoint_p<P_INF>(grad, mass, x, y, (int)n, (int)m, d, phi, psi, k2, p, (cudaStream_t)stream); break;
        default: e = launch_adjoint_p<P_GEN>(grad, mass, x, y, (int)n, (int)m, d, phi, psi, k2, p, (cudaStream_t)stream); break;
    }
    if (e != cudaSuccess)
        return culamp_set_error(h, CULAMP_ERR_CUDA, "adjoint launch: %s", cudaGetErrorString(e));
    return CULAMP_OK;
}
