// small_kernels.cuh -- elementwise / low-volume kernels (O(n) vectors and the
// non-hot FP64 certification and barycentric passes).
#pragma once

#include <cuda_runtime.h>
#include <math.h>

#include "engine.cuh"

namespace culamp_dev {

// phi_i = log(marg_i) - logz_i
static __global__ void log_minus_kernel(double *out, const double *marg, const double *logz, long long n) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) out[i] = log(marg[i]) - logz[i];
}

// Column potentials of a row-sharded Sinkhorn from the shards' column passes:
// shard g computed out_g,j = log c_j - LSE_{i in g}(...); the full column LSE
// is the log-sum-exp over shards, so psi_j = -log sum_g exp(-out_g,j) (FP64,
// max-shifted). parts: G rows of m.
static __global__ void lse_combine_kernel(double *psi, const double *parts, int G, long long m) {
    long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j >= m) return;
    double mx = -INFINITY;
    for (int g = 0; g < G; ++g) mx = fmax(mx, -parts[(size_t)g * m + j]);
    double s = 0.0;
    for (int g = 0; g < G; ++g) s += exp(-parts[(size_t)g * m + j] - mx);
    psi[j] = -(mx + log(s));
}

// update_theta_residual (MirrorProx.jl:159-180), elementwise.
static __global__ void theta_update_kernel(double *theta, const double *theta0, const double *residual,
                                    const double *c, const double *eta_mu_i, double eta_mu,
                                    int adjust, double minv, double maxv, double winf,
                                    long long m) {
    long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j < m)
        theta[j] = theta_step(theta0[j], residual[j], c[j], eta_mu_i[j], eta_mu, adjust, minv, maxv, winf);
}

template <typename F>
__device__ __forceinline__ double cost_generic(const double *xi, const double *yj, int d, double p) {
    double acc = 0.0;
    if (p == 1.0) {
        for (int k = 0; k < d; ++k) acc += fabs(xi[k] - yj[k]);
    } else if (p == 2.0) {
        for (int k = 0; k < d; ++k) { double t = xi[k] - yj[k]; acc = fma(t, t, acc); }
    } else if (isinf(p)) {
        for (int k = 0; k < d; ++k) acc = fmax(acc, fabs(xi[k] - yj[k]));
    } else {
        for (int k = 0; k < d; ++k) acc += pow(fabs(xi[k] - yj[k]), p);
    }
    return acc;
}

// |marg_i - sum_j exp(k C_ij + phi_i + psi_j)| summed over rows into *acc, all FP64
// (exp included). Warp per row; used once per solve to certify marginal errors.
static __global__ void marginal_fp64_kernel(double *acc, const double *x, const double *y, int n, int m,
                                     int d, const double *marg, const double *phi,
                                     const double *psi, double k, double p) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    double contrib = 0.0;
    if (warp < n) {
        const double *xi = x + (size_t)warp * d;
        double s = 0.0;
        for (int j = lane; j < m; j += 32) {
            const double cst = cost_generic<double>(xi, y + (size_t)j * d, d, p);
            s += exp(fma(cst, k, phi[warp]) + psi[j]);
        }
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) contrib = fabs(marg[warp] - s);
    }
    if (lane == 0 && contrib != 0.0) atomicAdd(acc, contrib);
}

// naive_findmaxindex_ct! (SinkhornKernel.jl:124-162) as a warp-per-row FP64 pass.
static __global__ void barycentric_sk_kernel(double *out, const double *x, const double *y, int n, int m,
                                      int d, const double *phi, const double *psi, double k,
                                      double p) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= n) return;
    const double *xi = x + (size_t)warp * d;
    double acc[MAXD_PACKED + 1] = {0.0, 0.0, 0.0, 0.0};
    double ps = 0.0;
    // generic d: accumulate per coordinate in a loop (d <= 64); packed buffer for d <= 3
    for (int kk = 0; kk < d; kk += MAXD_PACKED + 1) {
        for (int q = 0; q <= MAXD_PACKED; ++q) acc[q] = 0.0;
        ps = 0.0;
        for (int j = lane; j < m; j += 32) {
            const double cst = cost_generic<double>(xi, y + (size_t)j * d, d, p);
            const double prob = exp(cst * k + phi[warp] + psi[j]);
            ps += prob;
            for (int q = 0; q <= MAXD_PACKED && kk + q < d; ++q) acc[q] += y[(size_t)j * d + kk + q] * prob;
        }
        for (int o = 16; o > 0; o >>= 1) {
            ps += __shfl_down_sync(0xffffffffu, ps, o);
            for (int q = 0; q <= MAXD_PACKED; ++q) acc[q] += __shfl_down_sync(0xffffffffu, acc[q], o);
        }
        if (lane == 0)
            for (int q = 0; q <= MAXD_PACKED && kk + q < d; ++q) out[(size_t)warp * d + kk + q] = acc[q] / ps;
    }
}

// out = a*x + b*y elementwise (LAMP averaging outside the fused epilogue)
static __global__ void axpby_kernel(double *out, double a, const double *x, double b, const double *y,
                             long long n) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) out[i] = a * x[i] + b * y[i];
}

// out_i = scale * v_i
static __global__ void scale_kernel(double *out, const double *v, double scale, long long n) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) out[i] = scale * v[i];
}

// eta_mu_j = (c_j + alpha/n) / tau_mu (MirrorProxKernel.jl:1037)
static __global__ void eta_mu_kernel(double *out, const double *c, double alpha_over_n, double tau_mu,
                              long long m) {
    long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j < m) out[j] = (c[j] + alpha_over_n) / tau_mu;
}

// Annealing warm start: ws = v + f (v - prev); prev = v (AnnealedSinkhorn.jl:123-126)
static __global__ void extrapolate_kernel(double *ws, double *prev, const double *v, double f, long long n) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) {
        const double vi = v[i];
        ws[i] = vi + f * (vi - prev[i]);
        prev[i] = vi;
    }
}

// out_i = log(v_i)
static __global__ void log_kernel(double *out, const double *v, long long n) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) out[i] = log(v[i]);
}

// Single-block ordered FP64 reductions used at solve set-up:
// out[0] = sum v_i log v_i (v_i > 0), out[1] = min v_i, out[2] = sum v_i
static __global__ void setup_reduce_kernel(double *out, const double *v, long long n) {
    __shared__ double s0[256], s1[256], s2[256];
    double a = 0.0, mn = INFINITY, sm = 0.0;
    for (long long i = threadIdx.x; i < n; i += blockDim.x) {
        const double x = v[i];
        if (x > 0) a += x * log(x);
        mn = fmin(mn, x);
        sm += x;
    }
    s0[threadIdx.x] = a; s1[threadIdx.x] = mn; s2[threadIdx.x] = sm;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            s0[threadIdx.x] += s0[threadIdx.x + o];
            s1[threadIdx.x] = fmin(s1[threadIdx.x], s1[threadIdx.x + o]);
            s2[threadIdx.x] += s2[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) { out[0] = s0[0]; out[1] = s1[0]; out[2] = s2[0]; }
}

// Per-dimension [min, max] over the union of two point clouds: block k reduces
// dimension k. out[2k] = min, out[2k+1] = max.
static __global__ void dim_range_kernel(double *out, const double *x, long long n, const double *y,
                                        long long m, int d) {
    __shared__ double smn[256], smx[256];
    const int k = blockIdx.x;
    double mn = INFINITY, mx = -INFINITY;
    for (long long i = threadIdx.x; i < n + m; i += blockDim.x) {
        const double v = i < n ? x[i * d + k] : y[(i - n) * d + k];
        mn = fmin(mn, v);
        mx = fmax(mx, v);
    }
    smn[threadIdx.x] = mn;
    smx[threadIdx.x] = mx;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            smn[threadIdx.x] = fmin(smn[threadIdx.x], smn[threadIdx.x + o]);
            smx[threadIdx.x] = fmax(smx[threadIdx.x], smx[threadIdx.x + o]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) { out[2 * k] = smn[0]; out[2 * k + 1] = smx[0]; }
}

// out[i*dk + q] = in[i*d + keep[q]] for the kept dimensions (keep given by value).
struct DimKeep { int idx[64]; };
static __global__ void gather_dims_kernel(double *out, const double *in, long long n, int d, int dk,
                                          DimKeep keep) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= n * dk) return;
    const long long i = t / dk;
    const int q = (int)(t - i * dk);
    out[t] = in[i * d + keep.idx[q]];
}

}  // namespace culamp_dev
