// dense.cu -- the dense-cost GPU solvers of CuLAMP.jl: sinkhorn_log
// (src/solvers/Sinkhorn.jl:8-84) and the GPU LAMP (src/solvers/MirrorProx.jl:397-503),
// on a caller-supplied n x m cost matrix W (row-major FP64 device memory), as
// run_dot uses them for `--weights` matrices and the non-kernel grid costs
// (CmdLineUtils.jl:189-204: W read, divided by max |W|, moved to the GPU).
//
// Every pass streams W (or its transpose, built once per solve) from HBM once:
// the pair terms are not recomputed from coordinates, so these passes are
// HBM-bound (8 bytes per matrix element) -- the reference instead materialises
// broadcast temporaries (K .+ phi, exp.(...)) of the full matrix per update.
//
//  * dense_lse_kernel: one warp per matrix row; lanes stride over the row's
//    columns with coalesced loads; per lane an online log-sum-exp of
//    t_ij = a A_ij + gc g_j with the exponent and running max in FP64 and
//    2^(t - M) on the FP32 MUFU pipe (Kahan-compensated FP32 sums); the 32
//    lane partials merge with shuffles; one epilogue per row.
//  * dense_check_kernel: the convergence checks (every `frequency` iterations)
//    in exact FP64 (two passes over the row: max, then exp sums and moments).
//  * Row passes read W; column passes read W^T, so both are coalesced.
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "internal.h"

using namespace culamp_host;
using namespace culamp_dev;

namespace {

constexpr int DN_TPB = 256;            // 8 warps = 8 rows per CTA
constexpr int DN_ROWS = DN_TPB / 32;
constexpr int DN_CHECK = 8;            // doubles per row written by dense_check_kernel

enum DenseEpi {
    DN_SK = 0,     // out_i = log(marg_i) - L_i                (sinkhorn_log updates)
    DN_LOGZ = 1,   // out_i = L_i                              (LAMP logZ)
    DN_MASS = 2,   // out_i = exp(b * v_i + L_i)               (LAMP column mass, residual_c!)
};

struct DenseLse {
    const double *A;      // rows x cols, row-major
    long long rows, cols;
    double a2;            // LOG2E * a
    const double *g;      // column vector (cols) or null
    double gc2;           // LOG2E * gc
    int epi;
    const double *marg;   // DN_SK
    const double *v;      // DN_MASS
    double b;             // DN_MASS
    double *out;
};

__device__ __forceinline__ void lse_merge(double &M, double &S, double M2, double S2) {
    if (S2 == 0.0 || M2 == -INFINITY) return;
    if (S == 0.0 || M == -INFINITY) { M = M2; S = S2; return; }
    if (M2 > M) { S = S * exp2(M - M2) + S2; M = M2; }
    else S += S2 * exp2(M2 - M);
}

__global__ void __launch_bounds__(DN_TPB) dense_lse_kernel(const __grid_constant__ DenseLse P) {
    const int lane = threadIdx.x & 31;
    const long long row = (long long)blockIdx.x * DN_ROWS + (threadIdx.x >> 5);
    if (row >= P.rows) return;
    const double *Ar = P.A + row * P.cols;
    double M = -INFINITY;
    float S = 0.f, Cc = 0.f;
    long long j = lane;
    // four independent loads in flight per lane per step
    for (; j + 96 < P.cols; j += 128) {
        double w[4], t[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) w[u] = __ldcs(Ar + j + 32 * u);   // streamed once: evict first
#pragma unroll
        for (int u = 0; u < 4; ++u) t[u] = fma(P.a2, w[u], P.g ? P.gc2 * __ldg(P.g + j + 32 * u) : 0.0);
        double mx = fmax(fmax(t[0], t[1]), fmax(t[2], t[3]));
        if (mx > M) {
            const float f = (M == -INFINITY) ? 0.f : ex2_approx((float)(M - mx));
            S *= f;
            Cc *= f;
            M = mx;
        }
        if (M == -INFINITY) continue;
#pragma unroll
        for (int u = 0; u < 4; ++u) kahan_add(S, Cc, ex2_approx((float)(t[u] - M)));
    }
    for (; j < P.cols; j += 32) {
        const double t = fma(P.a2, __ldcs(Ar + j), P.g ? P.gc2 * __ldg(P.g + j) : 0.0);
        if (t > M) {
            const float f = (M == -INFINITY) ? 0.f : ex2_approx((float)(M - t));
            S *= f;
            Cc *= f;
            M = t;
        }
        if (M == -INFINITY) continue;
        kahan_add(S, Cc, ex2_approx((float)(t - M)));
    }
    double Md = M, Sd = (double)S - (double)Cc;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double M2 = __shfl_down_sync(0xffffffffu, Md, o);
        const double S2 = __shfl_down_sync(0xffffffffu, Sd, o);
        lse_merge(Md, Sd, M2, S2);
    }
    if (lane != 0) return;
    const double L = LN2 * (Md + log2(Sd));   // natural-log LSE of the row
    if (P.epi == DN_SK) P.out[row] = log(P.marg[row]) - L;
    else if (P.epi == DN_LOGZ) P.out[row] = L;
    else P.out[row] = exp(((P.b == 0.0) ? 0.0 : P.b * P.v[row]) + L);
}

// Exact FP64 row statistics for the convergence checks. With t_ij = a A_ij +
// gc g_j (g optional), e_ij = exp(t_ij - M_i), per row:
//   [0] M = max_j t   [1] S0 = sum e   [2] S1 = sum e A   [3] S2 = sum e (t - M)
//   [4] S3 = sum e w_j   [5] S4 = sum e w_j A   [6] S5 = sum A v_j
//   [7] MN = min_j (A + mc g_j)
struct DenseCheck {
    const double *A;
    long long rows, cols;
    double a, gc, mc;
    const double *g, *w, *v;
    double *out;
};

__global__ void __launch_bounds__(DN_TPB) dense_check_kernel(const __grid_constant__ DenseCheck P) {
    const int lane = threadIdx.x & 31;
    const long long row = (long long)blockIdx.x * DN_ROWS + (threadIdx.x >> 5);
    if (row >= P.rows) return;
    const double *Ar = P.A + row * P.cols;
    double M = -INFINITY, MN = INFINITY;
    for (long long j = lane; j < P.cols; j += 32) {
        const double A = Ar[j];
        const double gj = P.g ? P.g[j] : 0.0;
        M = fmax(M, fma(P.a, A, P.gc == 0.0 ? 0.0 : P.gc * gj));
        MN = fmin(MN, A + (P.mc == 0.0 ? 0.0 : P.mc * gj));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        M = fmax(M, __shfl_xor_sync(0xffffffffu, M, o));
        MN = fmin(MN, __shfl_xor_sync(0xffffffffu, MN, o));
    }
    double s[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (long long j = lane; j < P.cols; j += 32) {
        const double A = Ar[j];
        const double gj = P.g ? P.g[j] : 0.0;
        const double t = fma(P.a, A, P.gc == 0.0 ? 0.0 : P.gc * gj);
        const double e = exp(t - M);
        const double wj = P.w ? P.w[j] : 0.0;
        s[0] += e;
        s[1] += e * A;
        if (e > 0.0) s[2] += e * (t - M);
        s[3] += e * wj;
        s[4] += e * wj * A;
        if (P.v) s[5] += A * P.v[j];
    }
#pragma unroll
    for (int k = 0; k < 6; ++k)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s[k] += __shfl_xor_sync(0xffffffffu, s[k], o);
    if (lane != 0) return;
    double *o = P.out + row * DN_CHECK;
    o[0] = M;
    for (int k = 0; k < 6; ++k) o[1 + k] = s[k];
    o[7] = MN;
}

// out (m x n) = A^T (A: n x m), 32 x 32 tiles through shared memory.
__global__ void dense_transpose_kernel(double *out, const double *A, long long n, long long m) {
    __shared__ double tile[32][33];
    const long long c0 = (long long)blockIdx.x * 32, r0 = (long long)blockIdx.y * 32;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const long long r = r0 + k, c = c0 + threadIdx.x;
        if (r < n && c < m) tile[k][threadIdx.x] = A[r * m + c];
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const long long r = c0 + k, c = r0 + threadIdx.x;   // out row = A column
        if (r < m && c < n) out[r * n + c] = tile[threadIdx.x][k];
    }
}

// max |A| over all elements (W_inf of MirrorProx.jl:404, norm(W, Inf)); dst
// must hold +0 before the launch.
__global__ void dense_maxabs_kernel(const double *A, long long count, double *dst) {
    double mx = 0.0;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < count;
         k += (long long)gridDim.x * blockDim.x)
        mx = fmax(mx, fabs(A[k]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0)
        atomicMax(reinterpret_cast<unsigned long long *>(dst), (unsigned long long)__double_as_longlong(mx));
}

// LAMP elementwise steps (MirrorProx.jl:462-477) with update_theta_residual
// (:159-180, W_inf = 1 as the GPU LAMP passes it).
__device__ __forceinline__ double theta_res(double th0, double res, double c, double emu, double eta_mu) {
    const double difference = 2.0 * (res - c) / emu;
    const double maxval = fmax(difference, -difference);
    const double expv = exp(difference - maxval) * pow((th0 + 1.0) / (1.0 - th0), 1.0 - eta_mu);
    const double em = exp(-maxval);
    return (expv - em) / (expv + em);
}

// theta_bar = step(theta; tau_mu eta_mu); nu_bar = tau_p eta_t theta + (1 - tau_p eta_t) nu
__global__ void lamp_dense_step1(double *thb, double *nub, const double *theta, const double *nu,
                                 const double *res, const double *c, const double *emu, double eta_mu1,
                                 double te, long long m) {
    const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= m) return;
    thb[j] = theta_res(theta[j], res[j], c[j], emu[j], eta_mu1);
    nub[j] = te * theta[j] + (1.0 - te) * nu[j];
}

// theta = clamp(step(theta; eta_mu)); nu = (1 - tau_p eta_t) nu + tau_p eta_t theta_bar
__global__ void lamp_dense_step2(double *theta, double *nu, const double *thb, const double *res,
                                 const double *c, const double *emu, double eta_mu, double te,
                                 double minv, double maxv, long long m) {
    const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= m) return;
    const double t = theta_res(theta[j], res[j], c[j], emu[j], eta_mu);
    nu[j] = (1.0 - te) * nu[j] + te * thb[j];
    theta[j] = fmin(fmax(t, minv), maxv);
}

// plan_ij = exp(a W_ij + ga g_j + h_i)  (h row term, g column term)
__global__ void dense_plan_kernel(double *plan, const double *W, long long n, long long m, double a,
                                  const double *g, double ga, const double *h) {
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n * m) return;
    const long long i = k / m, j = k - i * m;
    plan[k] = exp(fma(a, W[k], ga * g[j]) + h[i]);
}

// h_i = log(r_i) - (M_i + log S0_i) from a check row (row normaliser of r .* softmax)
__global__ void dense_rownorm_kernel(double *h, const double *chk, const double *r, long long n) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    h[i] = log(r[i]) - (chk[i * DN_CHECK] + log(chk[i * DN_CHECK + 1]));
}

// g_i = log(r_i) - logz_i
__global__ void dense_sublog_kernel(double *g, const double *r, const double *logz, long long n) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    g[i] = log(r[i]) - logz[i];
}

unsigned grid_rows(long long rows) { return (unsigned)((rows + DN_ROWS - 1) / DN_ROWS); }
unsigned grid_lin(long long k) { return (unsigned)((k + 255) / 256); }

}  // namespace

// Workspace of the dense solvers, owned by the handle.
struct culamp_handle_s::Dense {
    DevBuf Wt, chk_r, chk_c, v1, v2, v3, v4, v5, v6, v7, v8, scal;
    void release() {
        DevBuf *all[] = {&Wt, &chk_r, &chk_c, &v1, &v2, &v3, &v4, &v5, &v6, &v7, &v8, &scal};
        for (DevBuf *b : all) b->release();
    }
};

void culamp_dense_release(culamp_handle h) {
    if (h && h->dense) {
        h->dense->release();
        delete h->dense;
        h->dense = nullptr;
    }
}

#define DN_TRY(h, expr)                                                                         \
    do {                                                                                        \
        cudaError_t _e = (expr);                                                                \
        if (_e != cudaSuccess)                                                                  \
            return culamp_set_error((h), CULAMP_ERR_CUDA, "%s: %s (%s:%d)", #expr,             \
                                    cudaGetErrorString(_e), __FILE__, __LINE__);                \
    } while (0)

namespace {

using Dense = culamp_handle_s::Dense;

cudaError_t lse_pass(const double *A, long long rows, long long cols, double a, const double *g, double gc,
                     int epi, const double *marg, const double *v, double b, double *out, cudaStream_t st) {
    DenseLse P;
    P.A = A; P.rows = rows; P.cols = cols;
    P.a2 = a * LOG2E;
    P.g = (gc == 0.0) ? nullptr : g;
    P.gc2 = gc * LOG2E;
    P.epi = epi; P.marg = marg; P.v = v; P.b = b; P.out = out;
    dense_lse_kernel<<<grid_rows(rows), DN_TPB, 0, st>>>(P);
    return cudaGetLastError();
}

cudaError_t check_pass(const double *A, long long rows, long long cols, double a, const double *g, double gc,
                       double mc, const double *w, const double *v, double *out, cudaStream_t st) {
    DenseCheck P;
    P.A = A; P.rows = rows; P.cols = cols;
    P.a = a; P.gc = gc; P.mc = mc;
    P.g = g; P.w = w; P.v = v; P.out = out;
    dense_check_kernel<<<grid_rows(rows), DN_TPB, 0, st>>>(P);
    return cudaGetLastError();
}

int check_dense_args(culamp_handle h, const double *W, int64_t n, int64_t m, const double *r,
                     const double *c, const culamp_args *args, int64_t frequency) {
    if (!h) return CULAMP_ERR_INVALID_ARG;
    if (!W || !r || !c || !args) return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "null pointer argument");
    if (n < 1 || m < 1 || n > 2000000 || m > 2000000 || (double)n * (double)m > 4.0e9)
        return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "sizes out of range (n=%lld, m=%lld)",
                                (long long)n, (long long)m);
    if (frequency < 1) return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "frequency must be >= 1");
    if (args->itermax < 0) return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "itermax < 0");
    cudaSetDevice(h->device);
    return CULAMP_OK;
}

int ensure_dense(culamp_handle h, int64_t n, int64_t m) {
    if (!h->dense) {
        h->dense = new (std::nothrow) Dense();
        if (!h->dense) return culamp_set_error(h, CULAMP_ERR_ALLOC, "dense workspace");
    }
    Dense &D = *h->dense;
    const size_t nm = (size_t)(n > m ? n : m);
    cudaError_t e = D.Wt.reserve((size_t)n * (size_t)m * sizeof(double));
    DevBuf *vecs[] = {&D.v1, &D.v2, &D.v3, &D.v4, &D.v5, &D.v6, &D.v7, &D.v8};
    for (DevBuf *b : vecs)
        if (e == cudaSuccess) e = b->reserve(nm * sizeof(double));
    if (e == cudaSuccess) e = D.chk_r.reserve((size_t)n * DN_CHECK * sizeof(double));
    if (e == cudaSuccess) e = D.chk_c.reserve((size_t)m * DN_CHECK * sizeof(double));
    if (e == cudaSuccess) e = D.scal.reserve(64);
    if (e != cudaSuccess) return culamp_set_error(h, CULAMP_ERR_ALLOC, "dense workspace: %s", cudaGetErrorString(e));
    return CULAMP_OK;
}

double host_s(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

void put_row(culamp_log_row *log, int64_t cap, int64_t &rows, double t, double it, double infeas, double obj,
             double primal, double dual) {
    if (log && rows < cap) log[rows] = culamp_log_row{t, it, infeas, obj, primal, dual};
    ++rows;
}

}  // namespace

/* sinkhorn_log (Sinkhorn.jl:8-84) on the GPU. */
extern "C" int culamp_sinkhorn_dense(culamp_handle h, const double *W, int64_t n, int64_t m,
                                     const double *r, const double *c, const culamp_args *args,
                                     int64_t frequency, const double *phi0, const double *psi0,
                                     double *phi, double *psi, double *plan, culamp_stats *stats,
                                     culamp_log_row *log, int64_t log_cap, void *stream) {
    int s = check_dense_args(h, W, n, m, r, c, args, frequency);
    if (s) return s;
    if (!phi || !psi || !stats) return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "null output");
    if (!(args->eta_p > 0.0)) return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "eta_p must be > 0");
    s = ensure_dense(h, n, m);
    if (s) return s;
    Dense &D = *h->dense;
    cudaStream_t st = (cudaStream_t)stream;
    std::memset(stats, 0, sizeof(*stats));
    cudaEvent_t e0, e1;
    DN_TRY(h, cudaEventCreate(&e0));
    DN_TRY(h, cudaEventCreate(&e1));
    DN_TRY(h, cudaEventRecord(e0, st));
    double *Wt = D.Wt.as<double>();
    dense_transpose_kernel<<<dim3((unsigned)((m + 31) / 32), (unsigned)((n + 31) / 32)), dim3(32, 8), 0, st>>>(
        Wt, W, n, m);
    DN_TRY(h, cudaGetLastError());
    if (phi0) DN_TRY(h, cudaMemcpyAsync(phi, phi0, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    else DN_TRY(h, cudaMemsetAsync(phi, 0, n * sizeof(double), st));
    if (psi0) DN_TRY(h, cudaMemcpyAsync(psi, psi0, m * sizeof(double), cudaMemcpyDeviceToDevice, st));
    else DN_TRY(h, cudaMemsetAsync(psi, 0, m * sizeof(double), st));
    const double eta = args->eta_p;
    const double a = -1.0 / eta;   // K = -W / eta_p
    // psi = log c - LSE_i(K_ij + phi_i) (over W^T rows); phi = log r - LSE_j(K_ij + psi_j)
    auto update = [&]() -> cudaError_t {
        cudaError_t e = lse_pass(Wt, m, n, a, phi, 1.0, DN_SK, c, nullptr, 0.0, psi, st);
        if (e == cudaSuccess) e = lse_pass(W, n, m, a, psi, 1.0, DN_SK, r, nullptr, 0.0, phi, st);
        return e;
    };
    std::vector<double> hr((size_t)n * DN_CHECK), hc((size_t)m * DN_CHECK), hphi(n), hpsi(m), hrv(n), hcv(m);
    DN_TRY(h, cudaMemcpyAsync(hrv.data(), r, n * sizeof(double), cudaMemcpyDeviceToHost, st));
    DN_TRY(h, cudaMemcpyAsync(hcv.data(), c, m * sizeof(double), cudaMemcpyDeviceToHost, st));
    // FP64 plan statistics at the current (phi, psi): (feas, obj, pobj, dobj)
    auto stats_now = [&](double out[4]) -> int {
        DN_TRY(h, check_pass(W, n, m, a, psi, 1.0, 0.0, nullptr, nullptr, D.chk_r.as<double>(), st));
        DN_TRY(h, check_pass(Wt, m, n, a, phi, 1.0, 0.0, nullptr, nullptr, D.chk_c.as<double>(), st));
        DN_TRY(h, cudaMemcpyAsync(hr.data(), D.chk_r.ptr, hr.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
        DN_TRY(h, cudaMemcpyAsync(hc.data(), D.chk_c.ptr, hc.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
        DN_TRY(h, cudaMemcpyAsync(hphi.data(), phi, n * sizeof(double), cudaMemcpyDeviceToHost, st));
        DN_TRY(h, cudaMemcpyAsync(hpsi.data(), psi, m * sizeof(double), cudaMemcpyDeviceToHost, st));
        DN_TRY(h, cudaStreamSynchronize(st));
        // p_ij = exp(phi_i + t_ij), t_ij = K_ij + psi_j = M_i + (t_ij - M_i)
        double feas = 0.0, obj = 0.0, ent = 0.0, tot = 0.0, lse_mx = -INFINITY;
        for (int64_t i = 0; i < n; ++i) lse_mx = std::fmax(lse_mx, hphi[i] + hr[i * DN_CHECK]);
        for (int64_t i = 0; i < n; ++i) {
            const double *q = &hr[i * DN_CHECK];
            const double sc = std::exp(hphi[i] + q[0]);
            const double rs = sc * q[1];
            feas += std::fabs(rs - hrv[i]);
            obj += sc * q[2];
            ent += sc * ((hphi[i] + q[0]) * q[1] + q[3]);    // sum_j p log p
            tot += std::exp(hphi[i] + q[0] - lse_mx) * q[1];
        }
        for (int64_t j = 0; j < m; ++j) {
            const double *q = &hc[j * DN_CHECK];
            feas += std::fabs(std::exp(hpsi[j] + q[0]) * q[1] - hcv[j]);
        }
        double cpsi = 0.0, rphi = 0.0;
        for (int64_t j = 0; j < m; ++j) cpsi += hcv[j] * hpsi[j];
        for (int64_t i = 0; i < n; ++i) rphi += hrv[i] * hphi[i];
        const double lse_all = std::log(tot) + lse_mx;
        out[0] = feas;
        out[1] = obj;                          // sum_ij p_ij W_ij
        out[2] = obj + eta * ent;
        out[3] = -eta * (-lse_all - cpsi - rphi);
        return CULAMP_OK;
    };
    const auto t0 = std::chrono::steady_clock::now();
    int64_t num_iter = 0, it = 0, rows = 0;
    int stopped = 0;
    double last[4] = {NAN, NAN, NAN, NAN};
    for (it = 1; it <= args->itermax; ++it) {
        DN_TRY(h, update());
        if (host_s(t0) > args->tmax) { stopped = 3; break; }
        if ((it - 1) % frequency == 0) {
            s = stats_now(last);
            if (s) return s;
            put_row(log, log_cap, rows, host_s(t0), (double)it, last[0], last[1], last[2], last[3]);
            if (last[2] - last[3] < args->epsilon / 6.0 && last[0] < args->epsilon / 6.0) { stopped = 1; break; }
        }
        ++num_iter;
    }
    if (it > args->itermax) { it = args->itermax; if (!stopped) stopped = 2; }
    DN_TRY(h, update());   // the final half-steps (Sinkhorn.jl:75-76)
    s = stats_now(last);
    if (s) return s;
    if (plan) {   // p = exp(K .+ phi .+ psi')
        dense_plan_kernel<<<grid_lin(n * m), 256, 0, st>>>(plan, W, n, m, a, psi, 1.0, phi);
        DN_TRY(h, cudaGetLastError());
    }
    DN_TRY(h, cudaEventRecord(e1, st));
    DN_TRY(h, cudaEventSynchronize(e1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    stats->iterations = it;
    stats->num_iter = num_iter;
    stats->residual = last[0];
    stats->objective = last[1];
    stats->winf = NAN;
    stats->eta_t = NAN;
    stats->s_t = NAN;
    stats->elapsed_ms = ms;
    stats->log_rows = rows < log_cap ? rows : log_cap;
    stats->stopped = stopped;
    stats->status = CULAMP_OK;
    return CULAMP_OK;
}

/* The GPU LAMP on a dense cost (MirrorProx.jl:397-503). */
extern "C" int culamp_lamp_dense(culamp_handle h, const double *W, int64_t n, int64_t m, const double *r,
                                 const double *c, const culamp_args *args, int64_t frequency,
                                 const double *theta0, double *theta, double *nu, double *plan,
                                 culamp_stats *stats, culamp_log_row *log, int64_t log_cap, void *stream) {
    int s = check_dense_args(h, W, n, m, r, c, args, frequency);
    if (s) return s;
    if (!theta || !nu || !stats) return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "null output");
    if (args->eta_p < 0.0) return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "eta_p must be >= 0");
    s = ensure_dense(h, n, m);
    if (s) return s;
    Dense &D = *h->dense;
    cudaStream_t st = (cudaStream_t)stream;
    std::memset(stats, 0, sizeof(*stats));
    cudaEvent_t e0, e1;
    DN_TRY(h, cudaEventCreate(&e0));
    DN_TRY(h, cudaEventCreate(&e1));
    DN_TRY(h, cudaEventRecord(e0, st));
    double *Wt = D.Wt.as<double>();
    dense_transpose_kernel<<<dim3((unsigned)((m + 31) / 32), (unsigned)((n + 31) / 32)), dim3(32, 8), 0, st>>>(
        Wt, W, n, m);
    DN_TRY(h, cudaGetLastError());
    // W_inf = norm(W, Inf) = max |W_ij| (MirrorProx.jl:404)
    double *winf_d = D.scal.as<double>();
    DN_TRY(h, cudaMemsetAsync(winf_d, 0, sizeof(double), st));
    dense_maxabs_kernel<<<1184, 256, 0, st>>>(W, n * m, winf_d);
    DN_TRY(h, cudaGetLastError());
    double winf = 0.0;
    DN_TRY(h, cudaMemcpyAsync(&winf, winf_d, sizeof(double), cudaMemcpyDeviceToHost, st));
    std::vector<double> hr(n), hc(m), hth(m);
    DN_TRY(h, cudaMemcpyAsync(hr.data(), r, n * sizeof(double), cudaMemcpyDeviceToHost, st));
    DN_TRY(h, cudaMemcpyAsync(hc.data(), c, m * sizeof(double), cudaMemcpyDeviceToHost, st));
    DN_TRY(h, cudaStreamSynchronize(st));
    if (!(winf > 0.0)) return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "W has no nonzero entry");
    const double etap = args->eta_p / 2.0 / winf;
    // theta (caller's start or 0); nu = nu_bar = theta_bar = copy(theta)
    if (theta0) DN_TRY(h, cudaMemcpyAsync(theta, theta0, m * sizeof(double), cudaMemcpyDeviceToDevice, st));
    else DN_TRY(h, cudaMemsetAsync(theta, 0, m * sizeof(double), st));
    double *thb = D.v1.as<double>(), *nub = D.v2.as<double>(), *res = D.v3.as<double>();
    double *logz = D.v4.as<double>(), *g = D.v5.as<double>(), *emu = D.v6.as<double>();
    double *ybuf = D.v7.as<double>(), *rnu = D.v8.as<double>();
    DN_TRY(h, cudaMemcpyAsync(nu, theta, m * sizeof(double), cudaMemcpyDeviceToDevice, st));
    {
        // eta_mu = (c + alpha / n) / tau_mu  (n = size(c) in the reference)
        std::vector<double> he(m);
        for (int64_t j = 0; j < m; ++j) he[j] = (hc[j] + args->alpha / (double)m) / args->tau_mu;
        DN_TRY(h, cudaMemcpyAsync(emu, he.data(), m * sizeof(double), cudaMemcpyHostToDevice, st));
        DN_TRY(h, cudaStreamSynchronize(st));
    }
    // infeas(theta, eta, s = 1) (MirrorProx.jl:427-430): logZ_i = LSE_j(-(W_ij/(2 W) + theta_j)/eta);
    // res_j = sum_i r_i exp(-(W_ij/(2 W) + theta_j)/eta - logZ_i), the second as a pass over
    // W^T: L_j = LSE_i(a W_ji + log r_i - logZ_i), res_j = exp(-theta_j / eta + L_j).
    // eta = Inf gives -(finite)/Inf = -0: uniform rows.
    auto coefs = [&](double eta_t, double &a, double &gc) {
        const bool inf = std::isinf(eta_t);
        a = inf ? 0.0 : -1.0 / (2.0 * eta_t * winf);
        gc = inf ? 0.0 : -1.0 / eta_t;
    };
    auto infeas = [&](const double *th, double eta_t) -> cudaError_t {
        double a, gc;
        coefs(eta_t, a, gc);
        cudaError_t e = lse_pass(W, n, m, a, th, gc, DN_LOGZ, nullptr, nullptr, 0.0, logz, st);
        if (e != cudaSuccess) return e;
        dense_sublog_kernel<<<grid_lin(n), 256, 0, st>>>(g, r, logz, n);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = lse_pass(Wt, m, n, a, g, 1.0, DN_MASS, nullptr, th, gc, res, st);
        return e;
    };
    std::vector<double> hA((size_t)n * DN_CHECK), hB((size_t)m * DN_CHECK), hC((size_t)n * DN_CHECK),
        hD((size_t)n * DN_CHECK), hnu(m);
    double hr_logr = 0.0;
    for (int64_t i = 0; i < n; ++i) hr_logr += hr[i] * std::log(hr[i]);
    double *chkA = D.chk_r.as<double>(), *chkB = D.chk_c.as<double>();
    // The convergence check of MirrorProx.jl:441-456 in FP64: P = row softmax of
    // -(W/(2 W) + nu')/eta_t; feas = |c - colsum(r .* P)|_1; obj = <W, round(r .* P, r, c)>
    // (Utilities.jl:158-165; its row factor min(r / rowsum, 1) is 1 up to rounding,
    // as the rows of r .* P sum to r); primalv (MirrorProx.jl:28-32) and dualv (:7-13).
    auto check = [&](double eta_t, double out[4]) -> int {
        double a, gc;
        coefs(eta_t, a, gc);
        DN_TRY(h, check_pass(W, n, m, a, nu, gc, 0.0, nullptr, nullptr, chkA, st));
        DN_TRY(h, cudaMemcpyAsync(hA.data(), chkA, hA.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
        dense_rownorm_kernel<<<grid_lin(n), 256, 0, st>>>(g, chkA, r, n);
        DN_TRY(h, cudaGetLastError());
        DN_TRY(h, check_pass(Wt, m, n, a, g, 1.0, 0.0, nullptr, nullptr, chkB, st));
        DN_TRY(h, cudaMemcpyAsync(hB.data(), chkB, hB.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
        DN_TRY(h, cudaMemcpyAsync(hnu.data(), nu, m * sizeof(double), cudaMemcpyDeviceToHost, st));
        DN_TRY(h, cudaMemcpyAsync(hth.data(), theta, m * sizeof(double), cudaMemcpyDeviceToHost, st));
        DN_TRY(h, cudaStreamSynchronize(st));
        std::vector<double> colsum(m), y(m), rnu_h(m);
        double feas = 0.0;
        for (int64_t j = 0; j < m; ++j) {
            const double *q = &hB[j * DN_CHECK];
            colsum[j] = std::exp(gc * hnu[j] + q[0]) * q[1];
            feas += std::fabs(hc[j] - colsum[j]);
            y[j] = std::fmin(hc[j] / colsum[j], 1.0);
            rnu_h[j] = hc[j] - y[j] * colsum[j];
        }
        DN_TRY(h, cudaMemcpyAsync(ybuf, y.data(), m * sizeof(double), cudaMemcpyHostToDevice, st));
        DN_TRY(h, cudaMemcpyAsync(rnu, rnu_h.data(), m * sizeof(double), cudaMemcpyHostToDevice, st));
        DN_TRY(h, check_pass(W, n, m, a, nu, gc, 0.0, ybuf, rnu, chkA, st));
        DN_TRY(h, cudaMemcpyAsync(hC.data(), chkA, hC.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
        if (etap > 0.0)
            DN_TRY(h, check_pass(W, n, m, -0.5 / etap, theta, -winf / etap, 0.0, nullptr, nullptr, chkA, st));
        else
            DN_TRY(h, check_pass(W, n, m, 0.0, theta, 0.0, 2.0 * winf, nullptr, nullptr, chkA, st));
        DN_TRY(h, cudaMemcpyAsync(hD.data(), chkA, hD.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
        DN_TRY(h, cudaStreamSynchronize(st));
        double pw = 0.0, ent = 0.0, wpp = 0.0, rmu1 = 0.0, corr = 0.0;
        for (int64_t i = 0; i < n; ++i) {
            const double *qa = &hA[i * DN_CHECK], *qc = &hC[i * DN_CHECK];
            pw += hr[i] * qa[2] / qa[1];                          // <W, r .* P>
            ent += hr[i] * (qa[3] / qa[1] - std::log(qa[1]));      // r . neg_entropy(P, rows)
            wpp += hr[i] * qc[5] / qc[1];                          // <W, gamma++>
            const double rmu = hr[i] - hr[i] * qc[4] / qc[1];
            rmu1 += std::fabs(rmu);
            corr += rmu * qc[6];                                   // r_mu' W r_nu
        }
        double cdev = 0.0, cth = 0.0, dterm = 0.0;
        for (int64_t j = 0; j < m; ++j) {
            cdev += std::fabs(colsum[j] - hc[j]);
            cth += hc[j] * hth[j];
        }
        for (int64_t i = 0; i < n; ++i) {
            const double *qd = &hD[i * DN_CHECK];
            dterm += hr[i] * ((etap > 0.0) ? qd[0] + std::log(qd[1]) : qd[7]);
        }
        out[0] = feas;
        out[1] = wpp + corr / rmu1;
        out[2] = 2.0 * (0.5 * pw + winf * cdev + etap * ent + etap * hr_logr);
        out[3] = (etap > 0.0) ? 2.0 * ((-winf * cth - etap * dterm) + etap * hr_logr)
                              : -2.0 * winf * cth + dterm;
        return CULAMP_OK;
    };
    const auto t0 = std::chrono::steady_clock::now();
    const double tau_p = args->tau_p;
    const double minv = std::tanh(-args->B / 2.0), maxv = std::tanh(args->B / 2.0);
    double eta_t = INFINITY;
    DN_TRY(h, infeas(nu, eta_t));
    int64_t it = 0, rows = 0;
    int stopped = 0;
    double last[4] = {NAN, NAN, NAN, NAN};
    for (it = 1; it <= args->itermax; ++it) {
        if (host_s(t0) > args->tmax) { stopped = 3; --it; break; }
        if ((it - 1) % frequency == 0) {
            s = check(eta_t, last);
            if (s) return s;
            put_row(log, log_cap, rows, host_s(t0), (double)it, last[0], last[1], last[2], last[3]);
            if (last[0] < args->epsilon / 2.0 && last[2] - last[3] < args->epsilon / 2.0) { stopped = 1; break; }
        }
        eta_t = 1.0 / (tau_p + (1.0 / eta_t) * (1.0 - etap));
        const double te = tau_p * eta_t;
        lamp_dense_step1<<<grid_lin(m), 256, 0, st>>>(thb, nub, theta, nu, res, c, emu,
                                                     args->tau_mu * args->eta_mu, te, m);
        DN_TRY(h, cudaGetLastError());
        DN_TRY(h, infeas(nub, eta_t));
        lamp_dense_step2<<<grid_lin(m), 256, 0, st>>>(theta, nu, thb, res, c, emu, args->eta_mu, te, minv,
                                                     maxv, m);
        DN_TRY(h, cudaGetLastError());
        DN_TRY(h, infeas(nu, eta_t));
    }
    if (it > args->itermax) { it = args->itermax; if (!stopped) stopped = 2; }
    if (!stopped) stopped = 2;
    // the returned state: r .* softmax(-(W/(2 W) + nu')/eta_t) and its statistics
    s = check(eta_t, last);
    if (s) return s;
    if (plan) {
        double a, gc;
        coefs(eta_t, a, gc);
        DN_TRY(h, check_pass(W, n, m, a, nu, gc, 0.0, nullptr, nullptr, chkA, st));
        dense_rownorm_kernel<<<grid_lin(n), 256, 0, st>>>(g, chkA, r, n);
        dense_plan_kernel<<<grid_lin(n * m), 256, 0, st>>>(plan, W, n, m, a, nu, gc, g);
        DN_TRY(h, cudaGetLastError());
    }
    DN_TRY(h, cudaEventRecord(e1, st));
    DN_TRY(h, cudaEventSynchronize(e1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    stats->iterations = it;
    stats->num_iter = it;
    stats->residual = last[0];
    stats->objective = last[1];
    stats->winf = winf;
    stats->eta_t = eta_t;
    stats->s_t = 1.0;
    stats->elapsed_ms = ms;
    stats->log_rows = rows < log_cap ? rows : log_cap;
    stats->stopped = stopped;
    stats->status = CULAMP_OK;
    return CULAMP_OK;
}
