// plain.cu -- the "plain FP32 form": CuLAMP.jl's kernels restated one-to-one in
// FP32 CUDA C++ (warp per output row, lanes striding the columns, per-element
// online log-sum-exp with a branch, 5-step shuffle merge; 256 threads and
// ceil(N/8) blocks) driven by a host loop that synchronises after every
// iteration, exactly like SinkhornKernel.jl:513-540 and MirrorProxKernel.jl:1076-1120.
// Potentials, coordinates and reductions are FP32. It is the baseline the chosen
// form is measured against (CULAMP_FLAG_FORM_PLAIN).
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "internal.h"

#define CUDA_TRY(h, expr)                                                                       \
    do {                                                                                        \
        cudaError_t _e = (expr);                                                                \
        if (_e != cudaSuccess)                                                                  \
            return culamp_set_error((h), CULAMP_ERR_CUDA, "%s: %s (%s:%d)", #expr,             \
                                    cudaGetErrorString(_e), __FILE__, __LINE__);                \
    } while (0)

namespace plain {

constexpr int THREADS = 256;

__device__ __forceinline__ float pcost(float dr, float dg, float db, int pm, float p) {
    if (pm == 0) return fabsf(dr) + fabsf(dg) + fabsf(db);
    if (pm == 1) return fmaf(dr, dr, fmaf(dg, dg, db * db));
    if (pm == 2) return fmaxf(fabsf(dr), fmaxf(fabsf(dg), fabsf(db)));
    return powf(fabsf(dr), p) + powf(fabsf(dg), p) + powf(fabsf(db), p);
}

__device__ __forceinline__ void lse_combine(float &m, float &s, float m2, float s2) {
    const float mm = m > m2 ? m : m2;
    s = s * expf(m - mm) + s2 * expf(m2 - mm);
    if (!(s == s)) s = 0.f;
    m = mm;
}

__device__ __forceinline__ void warp_lse(float &m, float &s) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const float m2 = __shfl_down_sync(0xffffffffu, m, o);
        const float s2 = __shfl_down_sync(0xffffffffu, s, o);
        if (m2 == -INFINITY) continue;
        if (m == -INFINITY) { m = m2; s = s2; continue; }
        lse_combine(m, s, m2, s2);
    }
}

// Row LSE of v_ij = C_ij * a + b * pot_j (warp_logsumexp_ct_fused!, SinkhornKernel.jl:341-444,
// and warp_logsumexp_spp_ct_fused!, MirrorProxKernel.jl:833-938). mode 0: out = log(marg) - LSE;
// mode 1: out = LSE.
__global__ void lse_rows(float *out, const float *X, const float *Y, int n, int m, const float *marg,
                         const float *pot, float a, float b, int pm, float p, int mode) {
    const int nwarps = (gridDim.x * blockDim.x) / 32;
    int row = (blockIdx.x * blockDim.x + threadIdx.x) / 32;
    const int lane = threadIdx.x & 31;
    for (; row < n; row += nwarps) {
        const float xr = X[row * 3], xg = X[row * 3 + 1], xb = X[row * 3 + 2];
        float ml = -INFINITY, sl = 0.f;
        for (int j = lane; j < m; j += 32) {
            const float c = pcost(xr - Y[j * 3], xg - Y[j * 3 + 1], xb - Y[j * 3 + 2], pm, p);
            const float v = fmaf(c, a, b == 0.f ? 0.f : b * pot[j]);
            if (v <= ml) sl += expf(v - ml);
            else { sl = sl * expf(ml - v) + 1.f; ml = v; }
        }
        warp_lse(ml, sl);
        if (lane == 0) {
            const float L = logf(sl) + ml;
            out[row] = mode == 0 ? logf(marg[row]) - L : L;
        }
    }
}

// residual_opt! (SinkhornKernel.jl:9-81): res = marg - sum_j exp(C a + phi_i + psi_j), cost.
__global__ void sk_residual(float *res, float *cost, const float *X, const float *Y, int n, int m,
                            const float *marg, const float *phi, const float *psi, float a, int pm,
                            float p) {
    const int nwarps = (gridDim.x * blockDim.x) / 32;
    int row = (blockIdx.x * blockDim.x + threadIdx.x) / 32;
    const int lane = threadIdx.x & 31;
    for (; row < n; row += nwarps) {
        const float xr = X[row * 3], xg = X[row * 3 + 1], xb = X[row * 3 + 2];
        float acc = 0.f, cacc = 0.f;
        for (int j = lane; j < m; j += 32) {
            const float c = pcost(xr - Y[j * 3], xg - Y[j * 3 + 1], xb - Y[j * 3 + 2], pm, p);
            const float e = expf(fmaf(c, a, phi[row]) + psi[j]);
            acc += e;
            cacc += e * c;
        }
        for (int o = 16; o > 0; o >>= 1) {
            acc += __shfl_down_sync(0xffffffffu, acc, o);
            cacc += __shfl_down_sync(0xffffffffu, cacc, o);
        }
        if (lane == 0) { res[row] = marg[row] - acc; cost[row] = cacc; }
    }
}

// residual_spp_c! (MirrorProxKernel.jl:7-94), warp per column j.
__global__ void spp_col(float *res, float *cost, const float *X, const float *Y, int n, int m,
                        const float *marg1, const float *theta, const float *logz, float c1,
                        float invreg, int pm, float p) {
    const int nwarps = (gridDim.x * blockDim.x) / 32;
    int col = (blockIdx.x * blockDim.x + threadIdx.x) / 32;
    const int lane = threadIdx.x & 31;
    for (; col < m; col += nwarps) {
        const float yr = Y[col * 3], yg = Y[col * 3 + 1], yb = Y[col * 3 + 2];
        const float th = theta[col];
        float acc = 0.f, cacc = 0.f;
        for (int i = lane; i < n; i += 32) {
            const float c = pcost(yr - X[i * 3], yg - X[i * 3 + 1], yb - X[i * 3 + 2], pm, p);
            const float v = fmaf(fmaf(c, c1, th), -invreg, -logz[i]);
            const float e = expf(v) * marg1[i];
            acc += e;
            cacc += e * c;
        }
        for (int o = 16; o > 0; o >>= 1) {
            acc += __shfl_down_sync(0xffffffffu, acc, o);
            cacc += __shfl_down_sync(0xffffffffu, cacc, o);
        }
        if (lane == 0) { res[col] = acc; cost[col] = cacc; }
    }
}

// max / min reductions (max_logsumexp_spp_ct!, warp_min_reduce!)
__global__ void minmax_rows(float *out, const float *X, const float *Y, int n, int m,
                            const float *pot, float scale, int pm, float p, int is_min) {
    const int nwarps = (gridDim.x * blockDim.x) / 32;
    int row = (blockIdx.x * blockDim.x + threadIdx.x) / 32;
    const int lane = threadIdx.x & 31;
    for (; row < n; row += nwarps) {
        const float xr = X[row * 3], xg = X[row * 3 + 1], xb = X[row * 3 + 2];
        float v = is_min ? INFINITY : -INFINITY;
        for (int j = lane; j < m; j += 32) {
            float c = pcost(xr - Y[j * 3], xg - Y[j * 3 + 1], xb - Y[j * 3 + 2], pm, p);
            if (is_min) v = fminf(v, fmaf(pot[j], scale, c));
            else v = fmaxf(v, c);
        }
        for (int o = 16; o > 0; o >>= 1) {
            const float w = __shfl_down_sync(0xffffffffu, v, o);
            v = is_min ? fminf(v, w) : fmaxf(v, w);
        }
        if (lane == 0) out[row] = v;
    }
}

__global__ void theta_update(float *theta, const float *theta0, const float *res, const float *c,
                             const float *emu, float eta_mu, int adjust, float minv, float maxv, int m) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= m) return;
    const float difference = 2.f * (res[j] - c[j]) / emu[j];
    const float maxval = fmaxf(difference, -difference);
    const float th = theta0[j];
    const float expv = expf(difference - maxval) * powf((th + 1.f) / (1.f - th), 1.f - eta_mu);
    const float em = expf(-maxval);
    float t = (expv - em) / (expv + em);
    if (adjust) t = fminf(fmaxf(t, minv), maxv);
    theta[j] = t;
}

__global__ void axpby(float *out, float a, const float *x, float b, const float *y, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = a * x[i] + b * y[i];
}

// FP32 sums: out[0] = sum |v - w| (w may be null), out[1] = sum u (may be null),
// out[2] = sum v*t (t may be null)
__global__ void sums(float *out, const float *v, const float *w, const float *u, const float *t, int n) {
    __shared__ float s0[THREADS], s1[THREADS], s2[THREADS];
    float a = 0.f, b = 0.f, cc = 0.f;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        a += fabsf(v[i] - (w ? w[i] : 0.f));
        if (u) b += u[i];
        if (t) cc += v[i] * t[i];
    }
    s0[threadIdx.x] = a; s1[threadIdx.x] = b; s2[threadIdx.x] = cc;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            s0[threadIdx.x] += s0[threadIdx.x + o];
            s1[threadIdx.x] += s1[threadIdx.x + o];
            s2[threadIdx.x] += s2[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) { out[0] = s0[0]; out[1] = s1[0]; out[2] = s2[0]; }
}

// FP64 point-major (d <= 3) -> FP32 padded to 3 coordinates
__global__ void to_f32_pts(float *out, const double *in, int n, int d) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int k = 0; k < 3; ++k) out[i * 3 + k] = k < d ? (float)in[(size_t)i * d + k] : 0.f;
}
__global__ void to_f32(float *out, const double *in, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (float)in[i];
}
__global__ void to_f64(double *out, const float *in, int n, double scale) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = scale * (double)in[i];
}
__global__ void log_minus(float *out, const float *marg, const float *logz, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = logf(marg[i]) - logz[i];
}

struct Buf {
    std::vector<void *> ptrs;
    ~Buf() { for (void *p : ptrs) cudaFree(p); }
    float *f(size_t n) {
        void *p = nullptr;
        if (cudaMalloc(&p, (n + 4) * sizeof(float)) != cudaSuccess) return nullptr;
        ptrs.push_back(p);
        cudaMemset(p, 0, (n + 4) * sizeof(float));
        return (float *)p;
    }
};

inline unsigned warp_blocks(int n) { return (unsigned)((n + 7) / 8); }
inline unsigned lin_blocks(int n) { return (unsigned)((n + THREADS - 1) / THREADS); }
inline int pm_of(double p) { return p == 1.0 ? 0 : (p == 2.0 ? 1 : (std::isinf(p) ? 2 : 3)); }

}  // namespace plain

using namespace plain;

int culamp_plain_sinkhorn(culamp_handle h, const double *x, const double *y, int64_t n64, int64_t m64,
                          int32_t d, const double *r, const double *c, const culamp_args *args,
                          int64_t frequency, double p, const double *phi0, const double *psi0,
                          uint32_t flags, double *phi, double *psi, culamp_stats *stats,
                          culamp_log_row *log, int64_t log_cap, cudaStream_t st) {
    if (d > 3) return culamp_set_error(h, CULAMP_ERR_UNSUPPORTED, "plain form supports d <= 3");
    const int n = (int)n64, m = (int)m64;
    Buf B;
    float *X = B.f((size_t)n * 3), *Y = B.f((size_t)m * 3), *fr = B.f(n), *fc = B.f(m);
    float *fphi = B.f(n), *fpsi = B.f(m), *res = B.f(n), *cost = B.f(n), *rm = B.f(n), *sm = B.f(4);
    if (!X || !Y || !fr || !fc || !fphi || !fpsi || !res || !cost || !rm || !sm)
        return culamp_set_error(h, CULAMP_ERR_ALLOC, "plain workspace");
    to_f32_pts<<<lin_blocks(n), THREADS, 0, st>>>(X, x, n, d);
    to_f32_pts<<<lin_blocks(m), THREADS, 0, st>>>(Y, y, m, d);
    to_f32<<<lin_blocks(n), THREADS, 0, st>>>(fr, r, n);
    to_f32<<<lin_blocks(m), THREADS, 0, st>>>(fc, c, m);
    if (phi0) to_f32<<<lin_blocks(n), THREADS, 0, st>>>(fphi, phi0, n);
    if (psi0) to_f32<<<lin_blocks(m), THREADS, 0, st>>>(fpsi, psi0, m);
    const bool tp = flags & CULAMP_FLAG_TRUE_PINF;
    const int pm_iter = pm_of((std::isinf(p) && !tp) ? 2.0 : p);
    const int pm_res = tp ? pm_of(p) : (p == 1.0 ? 0 : 1);
    // W_inf (max_logsumexp_spp_ct! + host maximum)
    minmax_rows<<<warp_blocks(n), THREADS, 0, st>>>(rm, X, Y, n, m, nullptr, 0.f, pm_of(p), (float)p, 0);
    std::vector<float> hrm(n);
    CUDA_TRY(h, cudaMemcpyAsync(hrm.data(), rm, n * sizeof(float), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(h, cudaStreamSynchronize(st));
    float winf = -INFINITY;
    for (float v : hrm) winf = v > winf ? v : winf;
    const float a = (float)(-1.0 / (args->eta_p * (double)winf));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, st);
    auto t0 = std::chrono::steady_clock::now();
    long long it = 0, num_iter = 0, rows = 0;
    int stopped = 0;
    float hs[3] = {0, 0, 0};
    for (it = 1; it <= args->itermax; ++it) {
        const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (el > args->tmax) { stopped = 3; it -= 1; break; }
        lse_rows<<<warp_blocks(n), THREADS, 0, st>>>(fphi, X, Y, n, m, fr, fpsi, a, 1.f, pm_iter, (float)p, 0);
        lse_rows<<<warp_blocks(m), THREADS, 0, st>>>(fpsi, Y, X, m, n, fc, fphi, a, 1.f, pm_iter, (float)p, 0);
        CUDA_TRY(h, cudaStreamSynchronize(st));
        if ((it - 1) % frequency == 0) {
            sk_residual<<<warp_blocks(n), THREADS, 0, st>>>(res, cost, X, Y, n, m, fr, fphi, fpsi, a, pm_res, (float)p);
            sums<<<1, THREADS, 0, st>>>(sm, res, nullptr, cost, nullptr, n);
            CUDA_TRY(h, cudaMemcpyAsync(hs, sm, 3 * sizeof(float), cudaMemcpyDeviceToHost, st));
            CUDA_TRY(h, cudaStreamSynchronize(st));
            if (log && rows < log_cap) {
                culamp_log_row &lr = log[rows++];
                lr.time_s = el;
                lr.iter = (double)it;
                lr.infeas = hs[0];
                lr.ot_objective = hs[1];
                lr.primal = NAN;
                lr.dual = NAN;
            }
            if (hs[0] <= args->epsilon / 6.0) { stopped = 1; break; }
        }
        num_iter += 1;
    }
    if (it > args->itermax) { it = args->itermax; if (!stopped) stopped = 2; }
    cudaEventRecord(e1, st);
    sk_residual<<<warp_blocks(n), THREADS, 0, st>>>(res, cost, X, Y, n, m, fr, fphi, fpsi, a, pm_res, (float)p);
    sums<<<1, THREADS, 0, st>>>(sm, res, nullptr, cost, nullptr, n);
    CUDA_TRY(h, cudaMemcpyAsync(hs, sm, 3 * sizeof(float), cudaMemcpyDeviceToHost, st));
    to_f64<<<lin_blocks(n), THREADS, 0, st>>>(phi, fphi, n, 1.0);
    to_f64<<<lin_blocks(m), THREADS, 0, st>>>(psi, fpsi, m, 1.0);
    CUDA_TRY(h, cudaStreamSynchronize(st));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        stats->iterations = it;
        stats->num_iter = num_iter;
        stats->residual = hs[0];
        stats->objective = hs[1];
        stats->winf = winf;
        stats->eta_t = NAN;
        stats->s_t = NAN;
        stats->elapsed_ms = ms;
        stats->log_rows = rows;
        stats->stopped = stopped;
    }
    return CULAMP_OK;
}

int culamp_plain_lamp(culamp_handle h, const double *x, const double *y, int64_t n64, int64_t m64,
                      int32_t d, const double *r, const double *c, const culamp_args *args,
                      int64_t frequency, double p, uint32_t flags, double *nu, double *phi,
                      double *psi, double *theta, culamp_stats *stats, culamp_log_row *log,
                      int64_t log_cap, cudaStream_t st) {
    if (d > 3) return culamp_set_error(h, CULAMP_ERR_UNSUPPORTED, "plain form supports d <= 3");
    const int n = (int)n64, m = (int)m64;
    Buf B;
    float *X = B.f((size_t)n * 3), *Y = B.f((size_t)m * 3), *fr = B.f(n), *fc = B.f(m);
    float *th = B.f(m), *thb = B.f(m), *fnu = B.f(m), *fnub = B.f(m), *res = B.f(m), *cost = B.f(m);
    float *logz = B.f(n), *emu = B.f(m), *tmp = B.f(n), *sm = B.f(4), *rm = B.f(n);
    if (!X || !Y || !fr || !fc || !th || !thb || !fnu || !fnub || !res || !cost || !logz || !emu || !tmp || !sm || !rm)
        return culamp_set_error(h, CULAMP_ERR_ALLOC, "plain workspace");
    to_f32_pts<<<lin_blocks(n), THREADS, 0, st>>>(X, x, n, d);
    to_f32_pts<<<lin_blocks(m), THREADS, 0, st>>>(Y, y, m, d);
    to_f32<<<lin_blocks(n), THREADS, 0, st>>>(fr, r, n);
    to_f32<<<lin_blocks(m), THREADS, 0, st>>>(fc, c, m);
    const int pm = pm_of(p);
    minmax_rows<<<warp_blocks(n), THREADS, 0, st>>>(rm, X, Y, n, m, nullptr, 0.f, pm, (float)p, 0);
    std::vector<float> hv(n > m ? n : m);
    CUDA_TRY(h, cudaMemcpyAsync(hv.data(), rm, n * sizeof(float), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(h, cudaStreamSynchronize(st));
    float winf = -INFINITY;
    for (int i = 0; i < n; ++i) winf = hv[i] > winf ? hv[i] : winf;
    const double eta = args->eta_p / (2.0 * winf);
    std::vector<float> hc(m), hr(n);
    CUDA_TRY(h, cudaMemcpy(hc.data(), fc, m * sizeof(float), cudaMemcpyDeviceToHost));
    CUDA_TRY(h, cudaMemcpy(hr.data(), fr, n * sizeof(float), cudaMemcpyDeviceToHost));
    for (int j = 0; j < m; ++j) hv[j] = (float)((hc[j] + args->alpha / n) / args->tau_mu);
    CUDA_TRY(h, cudaMemcpy(emu, hv.data(), m * sizeof(float), cudaMemcpyHostToDevice));
    double hrr = 0.0;
    for (int i = 0; i < n; ++i) if (hr[i] > 0) hrr += hr[i] * std::log((double)hr[i]);
    hrr *= eta;
    double eta_t = INFINITY, s_t = 1.0;
    const double tau_p = 1.0;
    const float minv = (float)std::tanh(-args->B / 2.0), maxv = (float)std::tanh(args->B / 2.0);
    const bool check = args->verbose || (flags & CULAMP_FLAG_CHECK_ALWAYS);
    float hs[3] = {0, 0, 0};
    auto infeas = [&](const float *thv, double et, double s) {
        const float invreg = (float)(1.0 / et), c1 = (float)(s / (2.0 * winf));
        lse_rows<<<warp_blocks(n), THREADS, 0, st>>>(logz, X, Y, n, m, nullptr, thv, -c1 * invreg, -invreg, pm, (float)p, 1);
        cudaStreamSynchronize(st);
        spp_col<<<warp_blocks(m), THREADS, 0, st>>>(res, cost, X, Y, n, m, fr, thv, logz, c1, invreg, pm, (float)p);
        cudaStreamSynchronize(st);
    };
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, st);
    auto t0 = std::chrono::steady_clock::now();
    long long it = 0, rows = 0, done = 0;
    int stopped = 0;
    for (it = 1; it <= args->itermax; ++it) {
        const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (el > args->tmax) { stopped = 3; break; }
        if (check && (it - 1) % frequency == 0) {
            infeas(fnu, eta_t, s_t);
            sums<<<1, THREADS, 0, st>>>(sm, res, fc, cost, fnu, m);
            CUDA_TRY(h, cudaMemcpyAsync(hs, sm, 3 * sizeof(float), cudaMemcpyDeviceToHost, st));
            float rl = 0.f;
            sums<<<1, THREADS, 0, st>>>(sm + 3, fr, nullptr, nullptr, logz, n);
            CUDA_TRY(h, cudaMemcpyAsync(&rl, sm + 3 + 2, sizeof(float), cudaMemcpyDeviceToHost, st));
            CUDA_TRY(h, cudaStreamSynchronize(st));
            const double q = eta / eta_t;
            const double primal = hs[1] * (1.0 - q) - q * hs[2] + q * rl + 2.0 * winf * hs[0];
            double dual;
            float dv[3] = {0, 0, 0};
            if (eta > 0) {
                lse_rows<<<warp_blocks(n), THREADS, 0, st>>>(tmp, X, Y, n, m, nullptr, th,
                                                             (float)(-1.0 / (2.0 * winf) / eta),
                                                             (float)(-1.0 / eta), pm, (float)p, 1);
            } else {
                minmax_rows<<<warp_blocks(n), THREADS, 0, st>>>(tmp, X, Y, n, m, th, 2.f * winf, pm, (float)p, 1);
            }
            sums<<<1, THREADS, 0, st>>>(sm, fr, nullptr, nullptr, tmp, n);
            CUDA_TRY(h, cudaMemcpyAsync(dv, sm, 3 * sizeof(float), cudaMemcpyDeviceToHost, st));
            float ct = 0.f;
            sums<<<1, THREADS, 0, st>>>(sm + 3, fc, nullptr, nullptr, th, m);
            CUDA_TRY(h, cudaMemcpyAsync(&ct, sm + 3 + 2, sizeof(float), cudaMemcpyDeviceToHost, st));
            CUDA_TRY(h, cudaStreamSynchronize(st));
            if (eta > 0) dual = -2.0 * eta * dv[2] - 2.0 * winf * ct + 2.0 * hrr;
            else dual = dv[2] - 2.0 * winf * ct;
            if (log && rows < log_cap) {
                culamp_log_row &lr = log[rows++];
                lr.time_s = el; lr.iter = (double)it; lr.infeas = hs[0]; lr.ot_objective = hs[1];
                lr.primal = primal; lr.dual = dual;
            }
            const bool gap_ok = (flags & CULAMP_FLAG_MARGINAL_ONLY) ? true : (primal - dual < args->epsilon / 6.0);
            if (gap_ok && hs[0] < args->epsilon / 6.0) { stopped = 1; break; }
        }
        infeas(fnu, eta_t, s_t);
        theta_update<<<lin_blocks(m), THREADS, 0, st>>>(thb, th, res, fc, emu, (float)args->eta_mu, 0, minv, maxv, m);
        eta_t = 1.0 / (tau_p + (1.0 / eta_t) * (1.0 - eta));
        axpby<<<lin_blocks(m), THREADS, 0, st>>>(fnub, (float)(1.0 - eta_t), fnu, (float)eta_t, th, m);
        cudaStreamSynchronize(st);
        s_t = (1.0 - eta_t) * s_t + eta_t;
        infeas(fnub, eta_t, s_t);
        theta_update<<<lin_blocks(m), THREADS, 0, st>>>(th, th, res, fc, emu, (float)args->eta_mu, 1, minv, maxv, m);
        axpby<<<lin_blocks(m), THREADS, 0, st>>>(fnu, (float)(1.0 - eta_t), fnu, (float)eta_t, thb, m);
        CUDA_TRY(h, cudaStreamSynchronize(st));
        done = it;
    }
    if (!stopped) stopped = 2;
    cudaEventRecord(e1, st);
    infeas(fnu, eta_t, s_t);
    sums<<<1, THREADS, 0, st>>>(sm, res, fc, cost, nullptr, m);
    CUDA_TRY(h, cudaMemcpyAsync(hs, sm, 3 * sizeof(float), cudaMemcpyDeviceToHost, st));
    log_minus<<<lin_blocks(n), THREADS, 0, st>>>(tmp, fr, logz, n);
    if (phi) to_f64<<<lin_blocks(n), THREADS, 0, st>>>(phi, tmp, n, 1.0);
    if (nu) to_f64<<<lin_blocks(m), THREADS, 0, st>>>(nu, fnu, m, 1.0);
    if (theta) to_f64<<<lin_blocks(m), THREADS, 0, st>>>(theta, th, m, 1.0);
    if (psi) to_f64<<<lin_blocks(m), THREADS, 0, st>>>(psi, fnu, m, -2.0 * winf / args->eta_p);
    CUDA_TRY(h, cudaStreamSynchronize(st));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        stats->iterations = done;
        stats->num_iter = done;
        stats->residual = hs[0];
        stats->objective = hs[1];
        stats->winf = winf;
        stats->eta_t = eta_t;
        stats->s_t = s_t;
        stats->elapsed_ms = ms;
        stats->log_rows = rows;
        stats->stopped = stopped;
    }
    return CULAMP_OK;
}
