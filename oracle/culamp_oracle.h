/*
 * culamp_oracle.h -- FP64 CPU restatement of CuLAMP.jl's kernelized entropic-OT
 * path. TEST INFRASTRUCTURE ONLY: the checker for the CUDA library and the
 * timed CPU baseline. Nothing in the product links or calls this code.
 *
 * Parity status: partially pinned. The reference (Julia + CUDA.jl) cannot run
 * in this environment and its own tests are broken (MirrorProx.jl:335-388 uses
 * undefined names), so the only golden values available from the reference
 * itself are the archived max-cost normalisers W_inf of its integer 64x64 grid
 * (data_archive/data/updated_pnorm.csv column `maxval`: 126 for p=1, 7938 for
 * p=2, 63 for p=Inf). Everything else is pinned by (a) a second, independent
 * numpy restatement (oracle/oracle.py), (b) closed forms (eta_t=Inf gives
 * uniform rows), (c) self-consistency (exact column marginals right after a
 * column update) and (d) an exact-LP optimum (scipy HiGHS) as eta -> 0.
 *
 * Layout: coordinates are point-major, x[i*d + k] -- the reference's 3xN
 * column-major CuArray (img[k, i], CmdLineUtils.jl:208-212) has exactly this
 * memory layout.
 */
#ifndef CULAMP_ORACLE_H
#define CULAMP_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* EOTArgs (src/Utilities.jl:18-31). */
typedef struct {
    double eta_p, eta_mu, tau_p, tau_mu, alpha, B, epsilon, anneal_mult;
    int64_t itermax, inner_iter;
    double tmax;
    int32_t verbose;
    int32_t _pad;
} or_args;

/* One convergence-log row, the columns the reference prints
 * (SinkhornKernel.jl:533, MirrorProxKernel.jl:1097). Unused fields are NaN. */
typedef struct {
    double time_s, iter, infeas, ot_objective, primal, dual;
} or_log_row;

typedef struct {
    int64_t iterations;     /* iterations run (loop index reached)          */
    int64_t num_iter;       /* the reference's `num_iter` counter           */
    double residual;        /* final L1 marginal residual                   */
    double objective;       /* final sum of the cost cache                  */
    double winf;            /* max-cost normaliser                          */
    double eta_t, s_t;      /* LAMP final eta_t and s                       */
    int64_t log_rows;       /* rows written to the log buffer               */
    int32_t stopped;        /* 1 = stopped on the tolerance test            */
    int32_t _pad;
} or_stats;

/* Solver option bits (not in the reference; 0 = reference behaviour). */
#define OR_TRUE_PINF        1  /* Sinkhorn p=Inf uses true L-inf cost (reference quirk off) */
#define OR_CHECK_ALWAYS     2  /* LAMP: run the check block even when !verbose              */
#define OR_MARGINAL_ONLY    4  /* LAMP: stop on the marginal test alone (no gap test)       */

double or_cost(const double *xi, const double *yj, int d, double p);
void or_max_cost_rows(const double *x, const double *y, int64_t n, int64_t m, int d,
                      double p, double *rowmax);
double or_max_cost(const double *x, const double *y, int64_t n, int64_t m, int d, double p);

/* Sinkhorn row pass (a1/a2). cost_p is the p used for the cost (the caller
 * passes the quirk-adjusted value). */
void or_sk_lse(double *out, const double *x, const double *y, int64_t n, int64_t m, int d,
               const double *marg, const double *pot, double reg, double winf, double cost_p);
void or_sk_residual(double *res, double *cost, const double *x, const double *y, int64_t n,
                    int64_t m, int d, const double *marg, const double *phi, const double *psi,
                    double reg, double winf, double cost_p);
void or_spp_lse(double *out, const double *x, const double *y, int64_t n, int64_t m, int d,
                const double *theta, double reg, double st, double winf, double p);
void or_spp_col_residual(double *res, double *cost, const double *x, const double *y,
                         int64_t n, int64_t m, int d, const double *marg1, const double *theta,
                         const double *logz, double reg, double st, double winf, double p);
void or_min_reduce(double *out, const double *x, const double *y, int64_t n, int64_t m, int d,
                   const double *theta, double winf, double p);
void or_theta_update(double *theta, const double *theta0, const double *residual,
                     const double *c, const double *eta_mu_i, double eta_mu, int adjust,
                     double minv, double maxv, double winf, int64_t m);
void or_barycentric_sk(double *out, const double *x, const double *y, int64_t n, int64_t m,
                       int d, const double *phi, const double *psi, double reg, double winf,
                       double cost_p);

/* FP64 envelope gradient of the Sinkhorn transport cost (checker for the
 * adjoint pass): grad[i*d+k] = sum_j P_ij dC/dx_ik, mass[i] = sum_j P_ij,
 * P_ij = exp(phi_i + psi_j - C_ij/(reg W_inf)). Rows listed in `rows` (count
 * nrows) only; rows == NULL means all n. Output rows are compact (nrows x d). */
void or_envelope_grad(double *grad, double *mass, const double *x, const double *y, int64_t n,
                      int64_t m, int d, const double *phi, const double *psi, double reg,
                      double winf, double p, const int64_t *rows, int64_t nrows);

/* Solver drivers. phi0/psi0 may be NULL. log may be NULL. */
int or_sinkhorn_kernel(const double *x, const double *y, int64_t n, int64_t m, int d,
                       const double *r, const double *c, const or_args *args, int64_t frequency,
                       double p, const double *phi0, const double *psi0, int flags,
                       double *phi, double *psi, or_stats *st, or_log_row *logbuf, int64_t log_cap);
int or_lamp_kernel(const double *x, const double *y, int64_t n, int64_t m, int d,
                   const double *r, const double *c, const or_args *args, int64_t frequency,
                   double p, int flags, double *nu, double *phi, double *psi, double *theta,
                   or_stats *st, or_log_row *logbuf, int64_t log_cap);
int or_annealed_sinkhorn_kernel(const double *x, const double *y, int64_t n, int64_t m, int d,
                                const double *r, const double *c, const or_args *args,
                                int64_t frequency, double p, int flags, double *phi, double *psi,
                                or_stats *st, or_log_row *logbuf, int64_t log_cap);

/* Dense CPU solvers on a caller-normalised cost matrix W (n x m, row-major). */
int or_sinkhorn_dense(const double *W, int64_t n, const double *r, const double *c,
                      const or_args *args, int64_t frequency, double *phi, double *psi,
                      or_stats *st, or_log_row *logbuf, int64_t log_cap);
int or_lamp_dense(const double *W, int64_t n, const double *r, const double *c,
                  const or_args *args, int64_t frequency, double *theta, double *nu,
                  double *plan, or_stats *st, or_log_row *logbuf, int64_t log_cap);

int or_num_threads(void);
void or_set_num_threads(int t);

#ifdef __cplusplus
}
#endif
#endif
