// capi.cu -- handle management, EOTArgs / JSON settings and the pass-level C ABI.
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>

#include "internal.h"
#include "small_kernels.cuh"

using namespace culamp_host;
using namespace culamp_dev;

int culamp_set_error(culamp_handle h, int code, const char *fmt, ...) {
    if (h) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof(buf), fmt, ap);
        va_end(ap);
        h->err = buf;
    }
    return code;
}

#define CUDA_TRY(h, expr)                                                                       \
    do {                                                                                        \
        cudaError_t _e = (expr);                                                                \
        if (_e != cudaSuccess)                                                                  \
            return culamp_set_error((h), CULAMP_ERR_CUDA, "%s: %s (%s:%d)", #expr,             \
                                    cudaGetErrorString(_e), __FILE__, __LINE__);                \
    } while (0)

extern "C" int culamp_version(void) { return CULAMP_VERSION; }

extern "C" const char *culamp_status_string(int s) {
    switch (s) {
        case CULAMP_OK: return "ok";
        case CULAMP_ERR_INVALID_ARG: return "invalid argument";
        case CULAMP_ERR_CUDA: return "CUDA error";
        case CULAMP_ERR_ALLOC: return "allocation failed";
        case CULAMP_ERR_UNSUPPORTED: return "unsupported";
        case CULAMP_ERR_IO: return "I/O error";
        case CULAMP_ERR_DEVICE_TIMEOUT: return "device-side wait timed out";
        default: return "unknown status";
    }
}

extern "C" const char *culamp_last_error(culamp_handle h) { return h ? h->err.c_str() : "null handle"; }

extern "C" int culamp_create(culamp_handle *out, int device) {
    if (!out) return CULAMP_ERR_INVALID_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) return CULAMP_ERR_CUDA;
    if (device < 0 || device >= ndev) return CULAMP_ERR_INVALID_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return CULAMP_ERR_CUDA;
    culamp_handle h = new (std::nothrow) culamp_handle_s();
    if (!h) return CULAMP_ERR_ALLOC;
    h->device = device;
    cudaDeviceGetAttribute(&h->sm_count, cudaDevAttrMultiProcessorCount, device);
    if (h->pass_ctl.reserve(sizeof(Ctl), true) != cudaSuccess) {
        delete h;
        return CULAMP_ERR_ALLOC;
    }
    *out = h;
    return CULAMP_OK;
}

void culamp_solver_release(culamp_handle h);   // solvers.cu
void culamp_batch_release(culamp_handle h);    // batched.cu
void culamp_dense_release(culamp_handle h);    // dense.cu

extern "C" int culamp_destroy(culamp_handle h) {
    if (!h) return CULAMP_ERR_INVALID_ARG;
    cudaSetDevice(h->device);
    culamp_solver_release(h);
    culamp_batch_release(h);
    culamp_dense_release(h);
    h->scratch.release();
    h->pass_ctl.release();
    h->tmpA.release();
    h->tmpB.release();
    delete h;
    return CULAMP_OK;
}

// ----------------------------------------------------------------- settings

extern "C" int culamp_args_default(culamp_args *a) {
    if (!a) return CULAMP_ERR_INVALID_ARG;
    // EOTArgs defaults, src/Utilities.jl:18-31
    a->eta_p = 0.0;
    a->eta_mu = 0.0;
    a->tau_p = 1.0;
    a->tau_mu = 1.0;
    a->alpha = 0.01;
    a->B = 1.0;
    a->epsilon = 1e-4;
    a->anneal_mult = 0.95;
    a->itermax = 10000;
    a->inner_iter = 10;
    a->tmax = INFINITY;
    a->verbose = 1;
    a->_pad = 0;
    return CULAMP_OK;
}

namespace {
// Minimal reader for a flat JSON object of numbers / booleans (the EOTArgs files
// under configurations/ and test.json). Nested values are skipped.
struct JsonReader {
    std::string buf;
    const char *s;
    size_t i = 0, n;
    explicit JsonReader(std::string str) : buf(std::move(str)), s(buf.c_str()), n(buf.size()) {}
    void ws() { while (i < n && std::isspace((unsigned char)s[i])) ++i; }
    bool lit(char c) { ws(); if (i < n && s[i] == c) { ++i; return true; } return false; }
    bool str(std::string &out) {
        ws();
        if (i >= n || s[i] != '"') return false;
        ++i;
        out.clear();
        while (i < n && s[i] != '"') {
            if (s[i] == '\\' && i + 1 < n) ++i;
            out.push_back(s[i++]);
        }
        if (i >= n) return false;
        ++i;
        return true;
    }
    bool skip_value() {
        ws();
        if (i >= n) return false;
        char c = s[i];
        if (c == '"') { std::string t; return str(t); }
        if (c == '{' || c == '[') {
            char open = c, close = (c == '{') ? '}' : ']';
            int depth = 0;
            while (i < n) {
                if (s[i] == '"') { std::string t; if (!str(t)) return false; continue; }
                if (s[i] == open) ++depth;
                if (s[i] == close && --depth == 0) { ++i; return true; }
                ++i;
            }
            return false;
        }
        while (i < n && s[i] != ',' && s[i] != '}' && !std::isspace((unsigned char)s[i])) ++i;
        return true;
    }
    // number, true/false, Infinity / NaN tokens
    bool scalar(double &v) {
        ws();
        if (i >= n) return false;
        if (!std::strncmp(s + i, "true", 4)) { i += 4; v = 1.0; return true; }
        if (!std::strncmp(s + i, "false", 5)) { i += 5; v = 0.0; return true; }
        if (!std::strncmp(s + i, "Infinity", 8)) { i += 8; v = INFINITY; return true; }
        if (!std::strncmp(s + i, "-Infinity", 9)) { i += 9; v = -INFINITY; return true; }
        char *end = nullptr;
        v = std::strtod(s + i, &end);
        if (end == s + i) return false;
        i = (size_t)(end - s);
        return true;
    }
};
}  // namespace

extern "C" int culamp_args_from_json_string(const char *json, culamp_args *a) {
    if (!json || !a) return CULAMP_ERR_INVALID_ARG;
    culamp_args_default(a);
    JsonReader r(json);
    if (!r.lit('{')) return CULAMP_ERR_INVALID_ARG;
    if (r.lit('}')) return CULAMP_OK;
    for (;;) {
        std::string key;
        if (!r.str(key) || !r.lit(':')) return CULAMP_ERR_INVALID_ARG;
        r.ws();
        const bool is_scalar = r.i < r.n && r.s[r.i] != '"' && r.s[r.i] != '{' && r.s[r.i] != '[';
        double v = 0.0;
        if (is_scalar) {
            if (!r.scalar(v)) return CULAMP_ERR_INVALID_ARG;
            if (key == "eta_p") a->eta_p = v;
            else if (key == "eta_mu") a->eta_mu = v;
            else if (key == "tau_p") a->tau_p = v;
            else if (key == "tau_mu") a->tau_mu = v;
            else if (key == "alpha") a->alpha = v;
            else if (key == "B") a->B = v;
            else if (key == "epsilon") a->epsilon = v;
            else if (key == "anneal_mult") a->anneal_mult = v;
            else if (key == "itermax") {
                if (v != std::floor(v)) return CULAMP_ERR_INVALID_ARG;   // Int field
                a->itermax = (int64_t)v;
            } else if (key == "inner_iter") {
                if (v != std::floor(v)) return CULAMP_ERR_INVALID_ARG;
                a->inner_iter = (int64_t)v;
            } else if (key == "tmax") a->tmax = v;
            else if (key == "verbose") a->verbose = v != 0.0;
        } else if (!r.skip_value()) {
            return CULAMP_ERR_INVALID_ARG;
        }
        if (r.lit(',')) continue;
        if (r.lit('}')) break;
        return CULAMP_ERR_INVALID_ARG;
    }
    return CULAMP_OK;
}

extern "C" int culamp_args_from_json(const char *path, culamp_args *a) {
    if (!path || !a) return CULAMP_ERR_INVALID_ARG;
    std::ifstream f(path);
    if (!f) return CULAMP_ERR_IO;
    std::stringstream ss;
    ss << f.rdbuf();
    return culamp_args_from_json_string(ss.str().c_str(), a);
}

// ------------------------------------------------------------ pass level

namespace {

int check_common(culamp_handle h, const void *x, const void *y, int64_t n, int64_t m, int32_t d,
                 double p) {
    if (!h) return CULAMP_ERR_INVALID_ARG;
    if (n < 1 || m < 1 || n > (int64_t)INT32_MAX / 4 || m > (int64_t)INT32_MAX / 4)
        return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "sizes out of range (n=%lld, m=%lld)",
                                (long long)n, (long long)m);
    if (d < 1 || d > MAXD)
        return culamp_set_error(h, d < 1 ? CULAMP_ERR_INVALID_ARG : CULAMP_ERR_UNSUPPORTED,
                                "d=%d outside [1, %d]", d, MAXD);
    if (!(p > 0.0)) return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "p must be > 0 (got %g)", p);
    if (!x || !y) return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "null coordinate pointer");
    cudaSetDevice(h->device);
    return CULAMP_OK;
}

PassParams base_params(const double *X, const double *Y, int n, int m, int d, double p) {
    PassParams P;
    std::memset(&P, 0, sizeof(P));
    P.X = X;
    P.Y = Y;
    P.n = n;
    P.m = m;
    P.d = d;
    P.pexp = p;
    P.coef_mode = COEF_FIXED;
    return P;
}

int run_pass(culamp_handle h, PassParams P, int pm, int acc, cudaStream_t st) {
    LaunchShape sh = pass_shape(P.n, P.m, P.d, acc, h->sm_count, P.want_moment != 0);
    cudaError_t e = h->scratch.reserve(sh.part_bytes, (size_t)sh.rb);
    if (e != cudaSuccess)
        return culamp_set_error(h, CULAMP_ERR_ALLOC, "scratch: %s", cudaGetErrorString(e));
    e = launch_pass(P, pm, acc, sh, h->scratch, st);
    if (e != cudaSuccess)
        return culamp_set_error(h, CULAMP_ERR_CUDA, "pair pass launch: %s", cudaGetErrorString(e));
    return CULAMP_OK;
}

}  // namespace

extern "C" int culamp_max_cost(culamp_handle h, const double *x, const double *y, int64_t n,
                               int64_t m, int32_t d, double p, double *rowmax, double *winf_host,
                               void *stream) {
    int s = check_common(h, x, y, n, m, d, p);
    if (s) return s;
    cudaStream_t st = (cudaStream_t)stream;
    if (!rowmax) {
        // W_inf alone: the register-tiled maximum (same per-pair costs)
        double *dst = &h->pass_ctl.as<Ctl>()->winf;
        CUDA_TRY(h, cudaMemsetAsync(dst, 0, sizeof(double), st));
        CUDA_TRY(h, launch_max_cost(x, y, (int)n, (int)m, d, p, dst, h->sm_count, st));
    } else {
        PassParams P = base_params(x, y, (int)n, (int)m, d, p);
        P.epi = EPI_RAW;
        P.out = rowmax;
        P.ctl = h->pass_ctl.as<Ctl>();
        P.finish = FIN_MAXCOST;
        s = run_pass(h, P, pmode_of(p), ACC_MAX, st);
        if (s) return s;
    }
    if (winf_host) {
        CUDA_TRY(h, cudaMemcpyAsync(winf_host, &h->pass_ctl.as<Ctl>()->winf, sizeof(double),
                                    cudaMemcpyDeviceToHost, st));
        CUDA_TRY(h, cudaStreamSynchronize(st));
    }
    return CULAMP_OK;
}

extern "C" int culamp_lse_rows_sk(culamp_handle h, double *out, const double *x, const double *y,
                                  int64_t n, int64_t m, int32_t d, const double *marg,
                                  const double *pot, double reg, double winf, double p,
                                  void *stream) {
    int s = check_common(h, x, y, n, m, d, p);
    if (s) return s;
    if (!out || !marg || !pot) return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "null pointer");
    PassParams P = base_params(x, y, (int)n, (int)m, d, p);
    P.ctr = x;
    P.epi = EPI_SK_ROW;
    P.alpha = -1.0 / (reg * winf);
    P.beta = 1.0;
    P.colpot = pot;
    P.marg = marg;
    P.out = out;
    P.use_ref = 1;   // out's previous content (the last phi) is the reference hint
    return run_pass(h, P, pmode_of(p), ACC_LSE, (cudaStream_t)stream);
}

extern "C" int culamp_lse_rows_sk_form(culamp_handle h, double *out, const double *x, const double *y,
                                       int64_t n, int64_t m, int32_t d, const double *marg,
                                       const double *pot, double reg, double winf, double p,
                                       uint32_t flags, void *stream) {
    if (!(flags & CULAMP_FLAG_FORM_FP32))
        return culamp_lse_rows_sk(h, out, x, y, n, m, d, marg, pot, reg, winf, p, stream);
    int s = check_common(h, x, y, n, m, d, p);
    if (s) return s;
    if (!out || !marg || !pot) return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "null pointer");
    if (pmode_of(p) != P_SQ || d > MAXD_PACKED)
        return culamp_set_error(h, CULAMP_ERR_UNSUPPORTED,
                                "the FP32-exponent form needs p = 2 and d <= %d (got p = %g, d = %d)",
                                MAXD_PACKED, p, (int)d);
    PassParams P = base_params(x, y, (int)n, (int)m, d, p);
    P.ctr = x;
    P.epi = EPI_SK_ROW;
    P.alpha = -1.0 / (reg * winf);
    P.beta = 1.0;
    P.colpot = pot;
    P.marg = marg;
    P.out = out;
    P.use_ref = 1;
    P.fp32 = 1;
    return run_pass(h, P, P_SQ, ACC_LSE, (cudaStream_t)stream);
}

extern "C" int culamp_residual_sk(culamp_handle h, double *res, double *cost, const double *x,
                                  const double *y, int64_t n, int64_t m, int32_t d,
                                  const double *marg, const double *phi, const double *psi,
                                  double reg, double winf, double p, void *stream) {
    int s = check_common(h, x, y, n, m, d, p);
    if (s) return s;
    if (!res || !marg || !phi || !psi) return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "null pointer");
    PassParams P = base_params(x, y, (int)n, (int)m, d, p);
    P.ctr = x;
    P.epi = EPI_SK_RESID;
    P.alpha = -1.0 / (reg * winf);
    P.beta = 1.0;
    P.colpot = psi;
    P.rowpot = phi;
    P.marg = marg;
    P.out = res;
    P.out2 = cost;
    P.want_moment = cost ? 1 : 0;
    return run_pass(h, P, pmode_of(p), ACC_LSE, (cudaStream_t)stream);
}

extern "C" int culamp_lse_rows_spp(culamp_handle h, double *out, const double *x, const double *y,
                                   int64_t n, int64_t m, int32_t d, const double *theta,
                                   double reg, double st, double winf, double p, void *stream) {
    int s = check_common(h, x, y, n, m, d, p);
    if (s) return s;
    if (!out || !theta) return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "null pointer");
    PassParams P = base_params(x, y, (int)n, (int)m, d, p);
    P.ctr = x;
    P.epi = EPI_LOGZ;
    const double invreg = 1.0 / reg;
    P.alpha = -(st / (2.0 * winf)) * invreg;
    P.beta = -invreg;
    P.colpot = theta;
    P.out = out;
    P.use_ref = 1;   // out's previous content (the last logZ) is the reference hint
    return run_pass(h, P, pmode_of(p), ACC_LSE, (cudaStream_t)stream);
}

extern "C" int culamp_col_residual_spp(culamp_handle h, double *res, double *cost, const double *x,
                                       const double *y, int64_t n, int64_t m, int32_t d,
                                       const double *marg1, const double *theta,
                                       const double *logz, double reg, double st, double winf,
                                       double p, void *stream) {
    int s = check_common(h, x, y, n, m, d, p);
    if (s) return s;
    if (!res || !marg1 || !theta || !logz)
        return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "null pointer");
    cudaStream_t cs = (cudaStream_t)stream;
    if (h->tmpA.reserve((size_t)n * sizeof(double)) != cudaSuccess)
        return culamp_set_error(h, CULAMP_ERR_ALLOC, "temporary");
    double *phi = h->tmpA.as<double>();
    log_minus_kernel<<<(unsigned)((n + 255) / 256), 256, 0, cs>>>(phi, marg1, logz, n);
    CUDA_TRY(h, cudaGetLastError());
    // rows of this pass = problem columns (y), columns = problem rows (x)
    PassParams P = base_params(y, x, (int)m, (int)n, d, p);
    P.ctr = y;
    P.epi = EPI_SPP_COL;
    const double invreg = 1.0 / reg;
    P.alpha = -(st / (2.0 * winf)) * invreg;
    P.beta = -invreg;
    P.colpot = phi;
    P.colpot_unit = 1;
    P.rowpot = theta;
    P.out = res;
    P.out2 = cost;
    P.want_moment = cost ? 1 : 0;
    return run_pass(h, P, pmode_of(p), ACC_LSE, cs);
}

extern "C" int culamp_min_reduce(culamp_handle h, double *out, const double *x, const double *y,
                                 int64_t n, int64_t m, int32_t d, const double *theta, double winf,
                                 double p, void *stream) {
    int s = check_common(h, x, y, n, m, d, p);
    if (s) return s;
    if (!out || !theta) return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "null pointer");
    PassParams P = base_params(x, y, (int)n, (int)m, d, p);
    P.epi = EPI_RAW;
    P.colpot = theta;
    P.minmax_scale = 2.0 * winf;
    P.out = out;
    return run_pass(h, P, pmode_of(p), ACC_MIN, (cudaStream_t)stream);
}

extern "C" int culamp_lse_combine(culamp_handle h, double *psi, const double *parts, int32_t shards,
                                  int64_t m, void *stream) {
    if (!h) return CULAMP_ERR_INVALID_ARG;
    if (!psi || !parts || shards < 1 || m < 1)
        return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "bad lse_combine arguments");
    cudaSetDevice(h->device);
    lse_combine_kernel<<<(unsigned)((m + 255) / 256), 256, 0, (cudaStream_t)stream>>>(psi, parts, shards, m);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return culamp_set_error(h, CULAMP_ERR_CUDA, "lse_combine: %s", cudaGetErrorString(e));
    return CULAMP_OK;
}

extern "C" int culamp_theta_update(culamp_handle h, double *theta, const double *theta0,
                                   const double *residual, const double *c,
                                   const double *eta_mu_i, double eta_mu, int32_t adjust,
                                   double minv, double maxv, double winf, int64_t m,
                                   void *stream) {
    if (!h) return CULAMP_ERR_INVALID_ARG;
    if (m < 1 || !theta || !theta0 || !residual || !c || !eta_mu_i)
        return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "bad theta_update arguments");
    cudaSetDevice(h->device);
    theta_update_kernel<<<(unsigned)((m + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
        theta, theta0, residual, c, eta_mu_i, eta_mu, adjust, minv, maxv, winf, m);
    CUDA_TRY(h, cudaGetLastError());
    return CULAMP_OK;
}

extern "C" int culamp_barycentric_sk(culamp_handle h, double *out, const double *x,
                                     const double *y, int64_t n, int64_t m, int32_t d,
                                     const double *phi, const double *psi, double reg,
                                     double winf, double p, void *stream) {
    int s = check_common(h, x, y, n, m, d, p);
    if (s) return s;
    if (!out || !phi || !psi) return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "null pointer");
    const unsigned blocks = (unsigned)((n + 7) / 8);
    barycentric_sk_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(out, x, y, (int)n, (int)m, d,
                                                                       phi, psi,
                                                                       -1.0 / (reg * winf), p);
    CUDA_TRY(h, cudaGetLastError());
    return CULAMP_OK;
}

extern "C" int culamp_marginal_error_fp64(culamp_handle h, const double *x, const double *y,
                                          int64_t n, int64_t m, int32_t d, const double *r,
                                          const double *c, const double *phi, const double *psi,
                                          double reg, double winf, double p, double *row_l1,
                                          double *col_l1, void *stream) {
    int s = check_common(h, x, y, n, m, d, p);
    if (s) return s;
    if (!r || !c || !phi || !psi) return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "null pointer");
    cudaStream_t st = (cudaStream_t)stream;
    if (h->tmpB.reserve(4 * sizeof(double)) != cudaSuccess)
        return culamp_set_error(h, CULAMP_ERR_ALLOC, "temporary");
    double *acc = h->tmpB.as<double>();
    CUDA_TRY(h, cudaMemsetAsync(acc, 0, 2 * sizeof(double), st));
    const double k = -1.0 / (reg * winf);
    marginal_fp64_kernel<<<(unsigned)((n + 7) / 8), 256, 0, st>>>(acc, x, y, (int)n, (int)m, d, r,
                                                                     phi, psi, k, p);
    marginal_fp64_kernel<<<(unsigned)((m + 7) / 8), 256, 0, st>>>(acc + 1, y, x, (int)m, (int)n, d,
                                                                     c, psi, phi, k, p);
    CUDA_TRY(h, cudaGetLastError());
    double hv[2];
    CUDA_TRY(h, cudaMemcpyAsync(hv, acc, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(h, cudaStreamSynchronize(st));
    if (row_l1) *row_l1 = hv[0];
    if (col_l1) *col_l1 = hv[1];
    return CULAMP_OK;
}
