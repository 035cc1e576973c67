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
