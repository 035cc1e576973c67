/*
 * culamp_oracle.c -- FP64 CPU restatement of CuLAMP.jl's kernelized entropic-OT
 * path (OpenMP over output rows). TEST INFRASTRUCTURE ONLY: used by tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline / reference arm as the
 * checker and the CPU baseline, never by the product library.
 *
 * Parity status: partially pinned (see culamp_oracle.h for what pins it).
 *
 * Every function cites the reference file:line it restates (paths relative to
 * the CuLAMP.jl project root). Reductions are two-pass (max, then sum of
 * exp(v - max)) in FP64; the reference's single-pass online merge
 * (MirrorProx.jl:229-235) is the same sum up to FP64 rounding.
 */
#include "culamp_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static double now_s(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

int or_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void or_set_num_threads(int t) {
#ifdef _OPENMP
    if (t > 0) omp_set_num_threads(t);
#else
    (void)t;
#endif
}

/* Pair cost, SinkhornKernel.jl:375-384 / MirrorProxKernel.jl:43-51:
 * p==1 -> sum|d|, p==2 -> sum d^2 (squared, no root), p==Inf -> max|d|,
 * otherwise sum |d|^p (no root). */
double or_cost(const double *xi, const double *yj, int d, double p) {
    double acc = 0.0;
    if (p == 1.0) {
        for (int k = 0; k < d; ++k) acc += fabs(xi[k] - yj[k]);
    } else if (p == 2.0) {
        for (int k = 0; k < d; ++k) {
            double t = xi[k] - yj[k];
            acc = fma(t, t, acc);
        }
    } else if (isinf(p)) {
        for (int k = 0; k < d; ++k) {
            double t = fabs(xi[k] - yj[k]);
            acc = t > acc ? t : acc;
        }
    } else {
        for (int k = 0; k < d; ++k) acc += pow(fabs(xi[k] - yj[k]), p);
    }
    return acc;
}

/* max_logsumexp_spp_ct! (MirrorProxKernel.jl:280-326): rowmax_i = max_j C_ij. */
void or_max_cost_rows(const double *x, const double *y, int64_t n, int64_t m, int d,
                      double p, double *rowmax) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        double mx = -INFINITY;
        for (int64_t j = 0; j < m; ++j) {
            double cst = or_cost(x + i * d, y + j * d, d, p);
            mx = cst > mx ? cst : mx;
        }
        rowmax[i] = mx;
    }
}

/* W_inf = maximum(rowmax) (SinkhornKernel.jl:500-502, MirrorProxKernel.jl:1032-1034). */
double or_max_cost(const double *x, const double *y, int64_t n, int64_t m, int d, double p) {
    double *rm = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    or_max_cost_rows(x, y, n, m, d, p, rm);
    double w = -INFINITY;
    for (int64_t i = 0; i < n; ++i) w = rm[i] > w ? rm[i] : w;
    free(rm);
    return w;
}

/* warp_logsumexp_ct_fused! / _opt! (SinkhornKernel.jl:341-444, 230-338):
 * out_i = log(marg_i) - LSE_j(C_ij * (-1/(reg*W_inf)) + pot_j). */
void or_sk_lse(double *out, const double *x, const double *y, int64_t n, int64_t m, int d,
               const double *marg, const double *pot, double reg, double winf, double cost_p) {
    const double invreg = -1.0 / (reg * winf);
#pragma omp parallel
    {
        double *v = (double *)malloc(sizeof(double) * (size_t)(m > 0 ? m : 1));
#pragma omp for schedule(static)
        for (int64_t i = 0; i < n; ++i) {
            double mx = -INFINITY;
            for (int64_t j = 0; j < m; ++j) {
                double cst = or_cost(x + i * d, y + j * d, d, cost_p);
                v[j] = fma(cst, invreg, pot[j]);
                mx = v[j] > mx ? v[j] : mx;
            }
            double s = 0.0;
            for (int64_t j = 0; j < m; ++j) s += exp(v[j] - mx);
            out[i] = log(marg[i]) - (log(s) + mx);
        }
        free(v);
    }
}

/* residual_opt! (SinkhornKernel.jl:9-81): res_i = marg_i - sum_j exp(v_ij),
 * cost_i = sum_j exp(v_ij) * C_ij with v_ij = C_ij*(-1/(reg W_inf)) + phi_i + psi_j. */
void or_sk_residual(double *res, double *cost, const double *x, const double *y, int64_t n,
                    int64_t m, int d, const double *marg, const double *phi, const double *psi,
                    double reg, double winf, double cost_p) {
    const double invreg = -1.0 / (reg * winf);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        double acc = 0.0, cacc = 0.0;
        for (int64_t j = 0; j < m; ++j) {
            double cst = or_cost(x + i * d, y + j * d, d, cost_p);
            double e = exp(fma(cst, invreg, phi[i]) + psi[j]);
            acc += e;
            cacc += e * cst;
        }
        res[i] = marg[i] - acc;
        cost[i] = cacc;
    }
}

/* warp_logsumexp_spp_ct_fused! / _opt! (MirrorProxKernel.jl:833-938, 702-829):
 * out_i = LSE_j(-(C_ij * st/(2 W_inf) + theta_j) / reg). */
void or_spp_lse(double *out, const double *x, const double *y, int64_t n, int64_t m, int d,
                const double *theta, double reg, double st, double winf, double p) {
    const double c1 = st / (2.0 * winf);
    const double invreg = 1.0 / reg;
#pragma omp parallel
    {
        double *v = (double *)malloc(sizeof(double) * (size_t)(m > 0 ? m : 1));
#pragma omp for schedule(static)
        for (int64_t i = 0; i < n; ++i) {
            double mx = -INFINITY;
            for (int64_t j = 0; j < m; ++j) {
                double cst = or_cost(x + i * d, y + j * d, d, p);
                v[j] = -(fma(cst, c1, theta[j])) * invreg;
                mx = v[j] > mx ? v[j] : mx;
            }
            double s = 0.0;
            for (int64_t j = 0; j < m; ++j) s += exp(v[j] - mx);
            out[i] = log(s) + mx;
        }
        free(v);
    }
}

/* residual_spp_c! (MirrorProxKernel.jl:7-94), one output per column j:
 * res_j  = sum_i marg1_i * exp(-(C_ij c1 + theta_j)/reg - logZ_i)
 * cost_j = sum_i marg1_i * exp(...) * C_ij. */
void or_spp_col_residual(double *res, double *cost, const double *x, const double *y,
                         int64_t n, int64_t m, int d, const double *marg1, const double *theta,
                         const double *logz, double reg, double st, double winf, double p) {
    const double c1 = st / (2.0 * winf);
    const double invreg = 1.0 / reg;
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < m; ++j) {
        double acc = 0.0, cacc = 0.0;
        for (int64_t i = 0; i < n; ++i) {
            double cst = or_cost(y + j * d, x + i * d, d, p);
            double value = fma(fma(cst, c1, theta[j]), -invreg, -logz[i]);
            double e = exp(value);
            acc += e * marg1[i];
            cacc += e * cst * marg1[i];
        }
        res[j] = acc;
        cost[j] = cacc;
    }
}

/* warp_min_reduce! (MirrorProxKernel.jl:941-1016): out_i = min_j (C_ij + 2 W_inf theta_j). */
void or_min_reduce(double *out, const double *x, const double *y, int64_t n, int64_t m, int d,
                   const double *theta, double winf, double p) {
    const double c1 = 2.0 * winf;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        double mn = INFINITY;
        for (int64_t j = 0; j < m; ++j) {
            double v = fma(theta[j], c1, or_cost(x + i * d, y + j * d, d, p));
            mn = v < mn ? v : mn;
        }
        out[i] = mn;
    }
}

/* update_theta_residual (MirrorProx.jl:159-180): stable tanh mirror step
 * theta_j <- tanh(W_inf (res_j - c_j)/eta_mu_j + (1-eta_mu)/2 log((1+theta0)/(1-theta0))). */
void or_theta_update(double *theta, const double *theta0, const double *residual,
                     const double *c, const double *eta_mu_i, double eta_mu, int adjust,
                     double minv, double maxv, double winf, int64_t m) {
    for (int64_t j = 0; j < m; ++j) {
        double difference = 2.0 * winf * (residual[j] - c[j]) / eta_mu_i[j];
        double thetav = theta0[j];
        double maxval = difference > -difference ? difference : -difference;
        double expv = exp(difference - maxval) * pow((thetav + 1.0) / (1.0 - thetav), 1.0 - eta_mu);
        double t = (expv - exp(-maxval)) / (expv + exp(-maxval));
        if (adjust) t = t < minv ? minv : (t > maxv ? maxv : t);
        theta[j] = t;
    }
}

/* naive_findmaxindex_ct! (SinkhornKernel.jl:124-162): barycentric image
 * out_i = sum_j y_j P_ij / sum_j P_ij with P_ij = exp(-C_ij/(reg W_inf) + phi_i + psi_j). */
void or_barycentric_sk(double *out, const double *x, const double *y, int64_t n, int64_t m,
                       int d, const double *phi, const double *psi, double reg, double winf,
                       double cost_p) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        double acc[16] = {0};
        double ps = 0.0;
        for (int64_t j = 0; j < m; ++j) {
            double cst = or_cost(x + i * d, y + j * d, d, cost_p);
            double prob = exp(-cst / (reg * winf) + phi[i] + psi[j]);
            ps += prob;
            for (int k = 0; k < d && k < 16; ++k) acc[k] += y[j * d + k] * prob;
        }
        for (int k = 0; k < d && k < 16; ++k) out[i * d + k] = acc[k] / ps;
    }
}

/* Envelope gradient sum_j P_ij grad_x C(x_i, y_j), all FP64 (the cost
 * derivative of the reference's costs: p=2 -> 2 d, p=1 -> sign d, p=Inf ->
 * sign d on the first maximising coordinate, other p -> p |d|^(p-1) sign d). */
void or_envelope_grad(double *grad, double *mass, const double *x, const double *y, int64_t n,
                      int64_t m, int d, const double *phi, const double *psi, double reg,
                      double winf, double p, const int64_t *rows, int64_t nrows) {
    if (!rows) nrows = n;
    const double k = -1.0 / (reg * winf);
#pragma omp parallel for schedule(static)
    for (int64_t q = 0; q < nrows; ++q) {
        const int64_t i = rows ? rows[q] : q;
        double g[64] = {0};
        double s = 0.0;
        for (int64_t j = 0; j < m; ++j) {
            const double *xi = x + i * d, *yj = y + j * d;
            const double pij = exp(or_cost(xi, yj, d, p) * k + phi[i] + psi[j]);
            s += pij;
            int kmax = 0;
            double vmax = -1.0;
            for (int kk = 0; kk < d; ++kk) {
                double a = fabs(xi[kk] - yj[kk]);
                if (a > vmax) { vmax = a; kmax = kk; }
            }
            for (int kk = 0; kk < d && kk < 64; ++kk) {
                const double df = xi[kk] - yj[kk];
                const double sg = (df > 0) - (df < 0);
                double dc;
                if (p == 2.0) dc = 2.0 * df;
                else if (p == 1.0) dc = sg;
                else if (isinf(p)) dc = (kk == kmax) ? sg : 0.0;
                else dc = fabs(df) > 0 ? p * pow(fabs(df), p - 1.0) * sg : 0.0;
                g[kk] += pij * dc;
            }
        }
        for (int kk = 0; kk < d && kk < 64; ++kk) grad[q * d + kk] = g[kk];
        if (mass) mass[q] = s;
    }
}

static double l1_norm(const double *v, int64_t n) {
    double s = 0.0;
    for (int64_t i = 0; i < n; ++i) s += fabs(v[i]);
    return s;
}
static double vsum(const double *v, int64_t n) {
    double s = 0.0;
    for (int64_t i = 0; i < n; ++i) s += v[i];
    return s;
}
static double vdot(const double *a, const double *b, int64_t n) {
    double s = 0.0;
    for (int64_t i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}

static void put_log(or_log_row *lb, int64_t cap, or_stats *st, double t, double it,
                    double infeas, double obj, double primal, double dual) {
    if (!lb || st->log_rows >= cap) return;
    or_log_row *r = &lb[st->log_rows++];
    r->time_s = t;
    r->iter = it;
    r->infeas = infeas;
    r->ot_objective = obj;
    r->primal = primal;
    r->dual = dual;
}

/* Cost p used by the Sinkhorn passes. Reference behaviour (SinkhornKernel.jl:518-523
 * with the _opt kernel's p==1 ? L1 : squared branch, :259-263): p=Inf iterates on the
 * squared-Euclidean cost while W_inf stays the Chebyshev max. The residual kernel
 * (SinkhornKernel.jl:38-42) uses p==1 ? L1 : squared for every p. */
static double sk_iter_p(double p, int flags) {
    if (isinf(p) && !(flags & OR_TRUE_PINF)) return 2.0;
    return p;
}
static double sk_resid_p(double p, int flags) {
    if (flags & OR_TRUE_PINF) return p;
    return p == 1.0 ? 1.0 : 2.0;
}

/* sinkhorn_color_transfer (SinkhornKernel.jl:477-559) with return_assignments=false. */
int or_sinkhorn_kernel(const double *x, const double *y, int64_t n, int64_t m, int d,
                       const double *r, const double *c, const or_args *args, int64_t frequency,
                       double p, const double *phi0, const double *psi0, int flags,
                       double *phi, double *psi, or_stats *st, or_log_row *logbuf, int64_t log_cap) {
    memset(st, 0, sizeof(*st));
    if (frequency < 1) frequency = 1;
    for (int64_t i = 0; i < n; ++i) phi[i] = phi0 ? phi0[i] : 0.0;
    for (int64_t j = 0; j < m; ++j) psi[j] = psi0 ? psi0[j] : 0.0;
    double *res = (double *)calloc((size_t)(n + 1), sizeof(double));
    double *cost = (double *)calloc((size_t)(n + 1), sizeof(double));
    const double t0 = now_s();
    const double eta = args->eta_p;
    const double winf = or_max_cost(x, y, n, m, d, p);
    const double ip = sk_iter_p(p, flags), rp = sk_resid_p(p, flags);
    st->winf = winf;
    int64_t num_iter = 0, it;
    for (it = 1; it <= args->itermax; ++it) {
        double el = now_s() - t0;
        if (el > args->tmax) break;
        or_sk_lse(phi, x, y, n, m, d, r, psi, eta, winf, ip);
        or_sk_lse(psi, y, x, m, n, d, c, phi, eta, winf, ip);
        st->iterations = it;
        if ((it - 1) % frequency == 0) {
            or_sk_residual(res, cost, x, y, n, m, d, r, phi, psi, eta, winf, rp);
            double res_r = l1_norm(res, n);
            double obj = vsum(cost, n);
            double dual = vdot(psi, c, m) + vdot(phi, r, n);
            put_log(logbuf, log_cap, st, el, (double)it, res_r, obj, NAN, dual);
            if (res_r <= args->epsilon / 6.0) {
                st->stopped = 1;
                break;
            }
        }
        num_iter += 1;
    }
    or_sk_residual(res, cost, x, y, n, m, d, r, phi, psi, eta, winf, rp);
    st->residual = l1_norm(res, n);
    st->objective = vsum(cost, n);
    st->num_iter = num_iter;
    free(res);
    free(cost);
    return 0;
}

static double neg_entropy_vec(const double *v, int64_t n) {
    double s = 0.0;
    for (int64_t i = 0; i < n; ++i)
        if (v[i] > 0.0) s += v[i] * log(v[i]);
    return s;
}

/* extragradient_color_transfer (MirrorProxKernel.jl:1019-1132), without the
 * barycentric maps. Outputs nu (the averaged dual, M), phi = log r - logZ (N),
 * psi = -2 W_inf nu / eta_p (M) and theta (M). */
int or_lamp_kernel(const double *x, const double *y, int64_t n, int64_t m, int d,
                   const double *r, const double *c, const or_args *args, int64_t frequency,
                   double p, int flags, double *nu, double *phi, double *psi, double *theta,
                   or_stats *st, or_log_row *logbuf, int64_t log_cap) {
    memset(st, 0, sizeof(*st));
    if (frequency < 1) frequency = 1;
    double *thb = (double *)calloc((size_t)m, sizeof(double));
    double *nub = (double *)calloc((size_t)m, sizeof(double));
    double *res = (double *)calloc((size_t)m, sizeof(double));
    double *cost = (double *)calloc((size_t)m, sizeof(double));
    double *sumvals = (double *)calloc((size_t)n, sizeof(double));
    double *eta_mu = (double *)calloc((size_t)m, sizeof(double));
    double *tmp = (double *)calloc((size_t)(n > m ? n : m), sizeof(double));
    for (int64_t j = 0; j < m; ++j) {
        theta[j] = 0.0;
        nu[j] = 0.0;
    }
    const double winf = or_max_cost(x, y, n, m, d, p);
    const double eta = args->eta_p / (2.0 * winf);
    for (int64_t j = 0; j < m; ++j) eta_mu[j] = (c[j] + args->alpha / (double)n) / args->tau_mu;
    const double t0 = now_s();
    const double hr = eta * neg_entropy_vec(r, n);
    double s_t = 1.0, eta_t = INFINITY;
    const double tau_p = 1.0; /* hard-coded in the reference (MirrorProxKernel.jl:1073) */
    const double minv = tanh(-args->B / 2.0), maxv = tanh(args->B / 2.0);
    const int check = args->verbose || (flags & OR_CHECK_ALWAYS);
    st->winf = winf;
    for (int64_t it = 1; it <= args->itermax; ++it) {
        double el = now_s() - t0;
        if (el > args->tmax) break;
        st->iterations = it;
        if (check && (it - 1) % frequency == 0) {
            or_spp_lse(sumvals, x, y, n, m, d, nu, eta_t, s_t, winf, p);
            or_spp_col_residual(res, cost, x, y, n, m, d, r, nu, sumvals, eta_t, s_t, winf, p);
            double residual_value = 0.0;
            for (int64_t j = 0; j < m; ++j) residual_value += fabs(res[j] - c[j]);
            double objective = vsum(cost, m);
            double q = eta / eta_t;
            double primal = vsum(cost, m) * (1.0 - q) - q * vdot(res, nu, m) +
                            q * vdot(r, sumvals, n) + 2.0 * winf * residual_value;
            double dual;
            if (eta > 0) {
                or_spp_lse(tmp, x, y, n, m, d, theta, eta, 1.0, winf, p);
                dual = -2.0 * eta * vdot(r, tmp, n) - 2.0 * winf * vdot(c, theta, m) + 2.0 * hr;
            } else {
                or_min_reduce(tmp, x, y, n, m, d, theta, winf, p);
                dual = vdot(r, tmp, n) - 2.0 * winf * vdot(c, theta, m);
            }
            put_log(logbuf, log_cap, st, el, (double)it, residual_value, objective, primal, dual);
            int gap_ok = (flags & OR_MARGINAL_ONLY) ? 1 : (primal - dual < args->epsilon / 6.0);
            if (gap_ok && residual_value < args->epsilon / 6.0) {
                st->stopped = 1;
                break;
            }
        }
        /* infeas(nu, eta_t, s_t) (MirrorProxKernel.jl:1042-1065) */
        or_spp_lse(sumvals, x, y, n, m, d, nu, eta_t, s_t, winf, p);
        or_spp_col_residual(res, cost, x, y, n, m, d, r, nu, sumvals, eta_t, s_t, winf, p);
        or_theta_update(thb, theta, res, c, eta_mu, args->eta_mu, 0, minv, maxv, 1.0, m);
        eta_t = 1.0 / (tau_p + (1.0 / eta_t) * (1.0 - eta));
        for (int64_t j = 0; j < m; ++j) nub[j] = (1.0 - eta_t) * nu[j] + eta_t * theta[j];
        s_t = (1.0 - eta_t) * s_t + eta_t;
        or_spp_lse(sumvals, x, y, n, m, d, nub, eta_t, s_t, winf, p);
        or_spp_col_residual(res, cost, x, y, n, m, d, r, nub, sumvals, eta_t, s_t, winf, p);
        or_theta_update(theta, theta, res, c, eta_mu, args->eta_mu, 1, minv, maxv, 1.0, m);
        for (int64_t j = 0; j < m; ++j) nu[j] = (1.0 - eta_t) * nu[j] + eta_t * thb[j];
    }
    /* post-loop (MirrorProxKernel.jl:1124-1129) */
    or_spp_lse(sumvals, x, y, n, m, d, nu, eta_t, s_t, winf, p);
    for (int64_t i = 0; i < n; ++i) phi[i] = log(r[i]) - sumvals[i];
    for (int64_t j = 0; j < m; ++j) psi[j] = -2.0 * winf * nu[j] / args->eta_p;
    /* final residual of the returned state (reported, not part of the reference's return) */
    or_spp_col_residual(res, cost, x, y, n, m, d, r, nu, sumvals, eta_t, s_t, winf, p);
    double rv = 0.0;
    for (int64_t j = 0; j < m; ++j) rv += fabs(res[j] - c[j]);
    st->residual = rv;
    st->objective = vsum(cost, m);
    st->eta_t = eta_t;
    st->s_t = s_t;
    st->num_iter = st->iterations;
    free(thb); free(nub); free(res); free(cost); free(sumvals); free(eta_mu); free(tmp);
    return 0;
}

/* annealed_sinkhorn_euclidean (AnnealedSinkhorn.jl:65-177), potentials only. */
int or_annealed_sinkhorn_kernel(const double *x, const double *y, int64_t n, int64_t m, int d,
                                const double *r, const double *c, const or_args *args,
                                int64_t frequency, double p, int flags, double *phi, double *psi,
                                or_stats *st, or_log_row *logbuf, int64_t log_cap) {
    memset(st, 0, sizeof(*st));
    or_args a = *args;
    const double eta_final = args->epsilon;
    double eta = args->eta_p > eta_final ? args->eta_p : eta_final;
    double *phiws = (double *)malloc(sizeof(double) * (size_t)n);
    double *psiws = (double *)malloc(sizeof(double) * (size_t)m);
    double *phiprev = (double *)malloc(sizeof(double) * (size_t)n);
    double *psiprev = (double *)malloc(sizeof(double) * (size_t)m);
    for (int64_t i = 0; i < n; ++i) phi[i] = phiws[i] = phiprev[i] = log(r[i]);
    for (int64_t j = 0; j < m; ++j) psi[j] = psiws[j] = psiprev[j] = log(c[j]);
    const double q = args->anneal_mult;
    double preveta = 1.0;
    const double tmax = args->tmax;
    a.verbose = 0;
    int64_t total_iters = 0;
    const double t0 = now_s();
    or_stats inner;
    for (;;) {
        a.eta_p = eta;
        or_sinkhorn_kernel(x, y, n, m, d, r, c, &a, frequency, p, phiws, psiws, flags, phi, psi,
                           &inner, NULL, 0);
        st->iterations += 1; /* stages run */
        total_iters += inner.num_iter;
        double el = now_s() - t0;
        a.tmax = tmax - el;
        put_log(logbuf, log_cap, st, el, (double)total_iters, inner.residual, inner.objective, NAN,
                eta);
        st->residual = inner.residual;
        st->objective = inner.objective;
        st->winf = inner.winf;
        if (eta == eta_final || el >= tmax) break;
        for (int64_t i = 0; i < n; ++i) phiws[i] = phi[i] + (eta / preveta) * (phi[i] - phiprev[i]);
        for (int64_t j = 0; j < m; ++j) psiws[j] = psi[j] + (eta / preveta) * (psi[j] - psiprev[j]);
        memcpy(phiprev, phi, sizeof(double) * (size_t)n);
        memcpy(psiprev, psi, sizeof(double) * (size_t)m);
        preveta = eta;
        eta = q * eta > eta_final ? q * eta : eta_final;
    }
    st->num_iter = total_iters;
    free(phiws); free(psiws); free(phiprev); free(psiprev);
    return 0;
}

/* ---------------- dense CPU solvers (config-1 baseline) ---------------- */

static double row_lse(const double *v, int64_t m, double *mx_out) {
    double mx = -INFINITY;
    for (int64_t j = 0; j < m; ++j) mx = v[j] > mx ? v[j] : mx;
    double s = 0.0;
    for (int64_t j = 0; j < m; ++j) s += exp(v[j] - mx);
    if (mx_out) *mx_out = mx;
    return log(s) + mx;
}

/* sinkhorn_log (Sinkhorn.jl:8-84) on a dense, already W_inf-normalised W. */
int or_sinkhorn_dense(const double *W, int64_t n, const double *r, const double *c,
                      const or_args *args, int64_t frequency, double *phi, double *psi,
                      or_stats *st, or_log_row *logbuf, int64_t log_cap) {
    memset(st, 0, sizeof(*st));
    if (frequency < 1) frequency = 1;
    const double ep = args->eta_p;
    for (int64_t i = 0; i < n; ++i) phi[i] = psi[i] = 0.0;
    const double t0 = now_s();
    int64_t num_iter = 0;
    for (int64_t it = 1; it <= args->itermax; ++it) {
        st->iterations = it;
        /* psi = log c - logsumexp(K .+ phi, 1)' (column LSE) */
#pragma omp parallel
        {
            double *v = (double *)malloc(sizeof(double) * (size_t)n);
#pragma omp for schedule(static)
            for (int64_t j = 0; j < n; ++j) {
                for (int64_t i = 0; i < n; ++i) v[i] = -W[i * n + j] / ep + phi[i];
                psi[j] = log(c[j]) - row_lse(v, n, NULL);
            }
#pragma omp for schedule(static)
            for (int64_t i = 0; i < n; ++i) {
                for (int64_t j = 0; j < n; ++j) v[j] = -W[i * n + j] / ep + psi[j];
                phi[i] = log(r[i]) - row_lse(v, n, NULL);
            }
            free(v);
        }
        double el = now_s() - t0;
        if (el > args->tmax) break;
        if ((it - 1) % frequency == 0) {
            double feas_r = 0.0, obj = 0.0, ent = 0.0, lse_mx = -INFINITY, lse_s = 0.0;
            double *colsum = (double *)calloc((size_t)n, sizeof(double));
            for (int64_t i = 0; i < n; ++i) {
                double rs = 0.0;
                for (int64_t j = 0; j < n; ++j) {
                    double a = -W[i * n + j] / ep + phi[i] + psi[j];
                    lse_mx = a > lse_mx ? a : lse_mx;
                }
                for (int64_t j = 0; j < n; ++j) {
                    double pij = exp(-W[i * n + j] / ep + phi[i] + psi[j]);
                    rs += pij;
                    colsum[j] += pij;
                    obj += pij * W[i * n + j];
                    if (pij > 0) ent += pij * log(pij);
                }
                feas_r += fabs(rs - r[i]);
            }
            for (int64_t i = 0; i < n; ++i)
                for (int64_t j = 0; j < n; ++j) lse_s += exp(-W[i * n + j] / ep + phi[i] + psi[j] - lse_mx);
            double feas = feas_r;
            for (int64_t j = 0; j < n; ++j) feas += fabs(colsum[j] - c[j]);
            free(colsum);
            double pobj = obj + ep * ent;
            double lse_all = log(lse_s) + lse_mx;
            double dobj = -ep * (-lse_all - vdot(c, psi, n) - vdot(r, phi, n));
            put_log(logbuf, log_cap, st, el, (double)it, feas, obj, pobj, dobj);
            st->residual = feas;
            st->objective = obj;
            if (pobj - dobj < args->epsilon / 6.0 && feas < args->epsilon / 6.0) {
                st->stopped = 1;
                break;
            }
        }
        num_iter += 1;
    }
    /* final half-steps (Sinkhorn.jl:75-76) */
    {
        double *v = (double *)malloc(sizeof(double) * (size_t)n);
        for (int64_t j = 0; j < n; ++j) {
            for (int64_t i = 0; i < n; ++i) v[i] = -W[i * n + j] / ep + phi[i];
            psi[j] = log(c[j]) - row_lse(v, n, NULL);
        }
        for (int64_t i = 0; i < n; ++i) {
            for (int64_t j = 0; j < n; ++j) v[j] = -W[i * n + j] / ep + psi[j];
            phi[i] = log(r[i]) - row_lse(v, n, NULL);
        }
        free(v);
    }
    double feas = 0.0, obj = 0.0;
    double *colsum = (double *)calloc((size_t)n, sizeof(double));
    for (int64_t i = 0; i < n; ++i) {
        double rs = 0.0;
        for (int64_t j = 0; j < n; ++j) {
            double pij = exp(-W[i * n + j] / ep + phi[i] + psi[j]);
            rs += pij;
            colsum[j] += pij;
            obj += pij * W[i * n + j];
        }
        feas += fabs(rs - r[i]);
    }
    for (int64_t j = 0; j < n; ++j) feas += fabs(colsum[j] - c[j]);
    free(colsum);
    st->residual = feas;
    st->objective = obj;
    st->num_iter = num_iter;
    return 0;
}

/* softmax(-(W/2W_inf .+ th')/eta_t, rows) into P (n x n) */
static void lamp_rows_softmax(double *P, const double *W, int64_t n, double winf,
                              const double *th, double eta_t) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        double *row = P + i * n;
        double mx = -INFINITY;
        for (int64_t j = 0; j < n; ++j) {
            row[j] = -(W[i * n + j] / (2.0 * winf) + th[j]) / eta_t;
            mx = row[j] > mx ? row[j] : mx;
        }
        double s = 0.0;
        for (int64_t j = 0; j < n; ++j) {
            row[j] = exp(row[j] - mx);
            s += row[j];
        }
        for (int64_t j = 0; j < n; ++j) row[j] /= s;
    }
}

/* primalv(p, W, W_inf, eta_p, r, c) (MirrorProx.jl:28-32) */
static double lamp_primalv(const double *P, const double *W, int64_t n, double winf, double etap,
                           const double *r, const double *c) {
    double a = 0.0, ent = 0.0, rlr = 0.0, feas = 0.0;
    double *col = (double *)calloc((size_t)n, sizeof(double));
    for (int64_t i = 0; i < n; ++i) {
        double rowent = 0.0;
        for (int64_t j = 0; j < n; ++j) {
            double pij = P[i * n + j];
            a += W[i * n + j] * r[i] * pij;
            col[j] += r[i] * pij;
            if (pij > 0) rowent += pij * log(pij);
        }
        ent += r[i] * rowent;
        if (r[i] > 0) rlr += r[i] * log(r[i]);
    }
    for (int64_t j = 0; j < n; ++j) feas += winf * fabs(col[j] - c[j]);
    free(col);
    return 2.0 * (0.5 * a + feas + etap * ent + etap * rlr);
}

/* dualv(theta, W, W_inf, eta_p, r, c) (MirrorProx.jl:7-13) */
static double lamp_dualv(const double *th, const double *W, int64_t n, double winf, double etap,
                         const double *r, const double *c) {
    if (etap == 0.0) {
        double s = -vdot(c, th, n) * 2.0 * winf;
        for (int64_t i = 0; i < n; ++i) {
            double mn = INFINITY;
            for (int64_t j = 0; j < n; ++j) {
                double v = W[i * n + j] + 2.0 * winf * th[j];
                mn = v < mn ? v : mn;
            }
            s += r[i] * mn;
        }
        return s;
    }
    double *v = (double *)malloc(sizeof(double) * (size_t)n);
    double rl = 0.0, rlr = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        for (int64_t j = 0; j < n; ++j) v[j] = -(0.5 * W[i * n + j] + winf * th[j]) / etap;
        rl += r[i] * row_lse(v, n, NULL);
        rlr += r[i] * log(r[i]);
    }
    free(v);
    return 2.0 * ((-winf * vdot(c, th, n) - etap * rl) + etap * rlr);
}

/* round(gamma, mu, nu) (Utilities.jl:158-165), then dot with W. */
static double rounded_objective(const double *PR, const double *W, int64_t n, const double *mu,
                                const double *nuv) {
    double *g = (double *)malloc(sizeof(double) * (size_t)(n * n));
    double *col = (double *)calloc((size_t)n, sizeof(double));
    double *rmu = (double *)malloc(sizeof(double) * (size_t)n);
    double *rnu = (double *)malloc(sizeof(double) * (size_t)n);
    for (int64_t i = 0; i < n; ++i) {
        double rs = 0.0;
        for (int64_t j = 0; j < n; ++j) rs += PR[i * n + j];
        double f = mu[i] / rs;
        f = f < 1.0 ? f : 1.0;
        for (int64_t j = 0; j < n; ++j) {
            g[i * n + j] = PR[i * n + j] * f;
            col[j] += g[i * n + j];
        }
    }
    for (int64_t j = 0; j < n; ++j) {
        double f = nuv[j] / col[j];
        col[j] = f < 1.0 ? f : 1.0;
    }
    for (int64_t j = 0; j < n; ++j) rnu[j] = nuv[j];
    double nr = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        double rs = 0.0;
        for (int64_t j = 0; j < n; ++j) {
            g[i * n + j] *= col[j];
            rs += g[i * n + j];
            rnu[j] -= g[i * n + j];
        }
        rmu[i] = mu[i] - rs;
        nr += fabs(rmu[i]);
    }
    double obj = 0.0;
    for (int64_t i = 0; i < n; ++i)
        for (int64_t j = 0; j < n; ++j) obj += (g[i * n + j] + rmu[i] * rnu[j] / nr) * W[i * n + j];
    free(g); free(col); free(rmu); free(rnu);
    return obj;
}

/* LAMP on the CPU (MirrorProx.jl:506-575) on a dense W. `plan` (n x n) receives
 * r .* softmax(...) at the end (may be NULL). */
int or_lamp_dense(const double *W, int64_t n, const double *r, const double *c,
                  const or_args *args, int64_t frequency, double *theta, double *nu,
                  double *plan, or_stats *st, or_log_row *logbuf, int64_t log_cap) {
    memset(st, 0, sizeof(*st));
    if (frequency < 1) frequency = 1;
    double winf = 0.0;
    for (int64_t k = 0; k < n * n; ++k) winf = fabs(W[k]) > winf ? fabs(W[k]) : winf;
    const double etap = args->eta_p / (2.0 * winf);
    double *thb = (double *)calloc((size_t)n, sizeof(double));
    double *nub = (double *)calloc((size_t)n, sizeof(double));
    double *gam = (double *)calloc((size_t)n, sizeof(double));
    double *res = (double *)calloc((size_t)n, sizeof(double));
    double *eta_mu = (double *)malloc(sizeof(double) * (size_t)n);
    double *P = (double *)malloc(sizeof(double) * (size_t)(n * n));
    for (int64_t j = 0; j < n; ++j) {
        theta[j] = nu[j] = 0.0;
        eta_mu[j] = (c[j] + args->alpha / (double)n) / args->tau_mu;
    }
    double eta_t = INFINITY;
    const double tau_p = args->tau_p;
    const double t0 = now_s();
    const double half_k = 0.5 * (1.0 - args->tau_mu * args->eta_mu);
    const double lo = tanh(-args->B / 2.0), hi = tanh(args->B / 2.0);
    st->winf = winf;
    for (int64_t it = 1; it <= args->itermax; ++it) {
        double el = now_s() - t0;
        if (el > args->tmax) break;
        st->iterations = it;
        if ((it - 1) % frequency == 0) {
            lamp_rows_softmax(P, W, n, winf, nu, eta_t);
            double feas = 0.0;
            double *col = (double *)calloc((size_t)n, sizeof(double));
            for (int64_t i = 0; i < n; ++i)
                for (int64_t j = 0; j < n; ++j) col[j] += r[i] * P[i * n + j];
            for (int64_t j = 0; j < n; ++j) feas += fabs(col[j] - c[j]);
            free(col);
            for (int64_t i = 0; i < n; ++i)
                for (int64_t j = 0; j < n; ++j) P[i * n + j] *= r[i];
            double obj = rounded_objective(P, W, n, r, c);
            for (int64_t i = 0; i < n; ++i)
                for (int64_t j = 0; j < n; ++j) P[i * n + j] /= r[i];
            double pobj = lamp_primalv(P, W, n, winf, etap, r, c);
            double dobj = lamp_dualv(gam, W, n, winf, etap, r, c);
            put_log(logbuf, log_cap, st, el, (double)it, feas, obj, pobj, dobj);
            st->residual = feas;
            st->objective = obj;
            if ((pobj - dobj) < args->epsilon / 6.0 && feas < args->epsilon / 6.0) {
                st->stopped = 1;
                break;
            }
        }
        /* infeas(nu, eta_t) (MirrorProx.jl:532-538): column sums of the row-softmax plan */
        lamp_rows_softmax(P, W, n, winf, nu, eta_t);
        for (int64_t j = 0; j < n; ++j) res[j] = 0.0;
        for (int64_t i = 0; i < n; ++i)
            for (int64_t j = 0; j < n; ++j) res[j] += r[i] * P[i * n + j];
        for (int64_t j = 0; j < n; ++j)
            thb[j] = tanh((res[j] - c[j]) / eta_mu[j] + half_k * log((theta[j] + 1.0) / (1.0 - theta[j])));
        eta_t = 1.0 / (tau_p + (1.0 / eta_t) * (1.0 - etap));
        for (int64_t j = 0; j < n; ++j) nub[j] = nu[j] + tau_p * eta_t * (theta[j] - nu[j]);
        lamp_rows_softmax(P, W, n, winf, nub, eta_t);
        for (int64_t j = 0; j < n; ++j) res[j] = 0.0;
        for (int64_t i = 0; i < n; ++i)
            for (int64_t j = 0; j < n; ++j) res[j] += r[i] * P[i * n + j];
        for (int64_t j = 0; j < n; ++j)
            theta[j] = tanh((res[j] - c[j]) / eta_mu[j] + half_k * log((theta[j] + 1.0) / (1.0 - theta[j])));
        for (int64_t j = 0; j < n; ++j) gam[j] = theta[j] + tau_p * eta_t * (theta[j] - gam[j]);
        for (int64_t j = 0; j < n; ++j) theta[j] = theta[j] < lo ? lo : (theta[j] > hi ? hi : theta[j]);
        for (int64_t j = 0; j < n; ++j) nu[j] = nu[j] + tau_p * eta_t * (thb[j] - nu[j]);
    }
    lamp_rows_softmax(P, W, n, winf, nu, eta_t);
    {
        double feas = 0.0;
        double *col = (double *)calloc((size_t)n, sizeof(double));
        for (int64_t i = 0; i < n; ++i)
            for (int64_t j = 0; j < n; ++j) col[j] += r[i] * P[i * n + j];
        for (int64_t j = 0; j < n; ++j) feas += fabs(col[j] - c[j]);
        free(col);
        st->residual = feas;
    }
    if (plan)
        for (int64_t i = 0; i < n; ++i)
            for (int64_t j = 0; j < n; ++j) plan[i * n + j] = r[i] * P[i * n + j];
    st->eta_t = eta_t;
    st->num_iter = st->iterations;
    free(thb); free(nub); free(gam); free(res); free(eta_mu); free(P);
    return 0;
}
