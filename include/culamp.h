/*
 * culamp.h -- C ABI of libculamp_b200, a B200-native (sm_100a) implementation of
 * CuLAMP.jl's kernelized entropic optimal-transport path: the fused on-the-fly
 * cost plus online log-sum-exp row / column reductions behind the `lamp`,
 * `sinkhorn` and `annealed_sinkhorn` `--kernel` solvers.
 *
 * Conventions
 *  - Every entry point returns an int status (CULAMP_OK = 0) and never throws.
 *    culamp_last_error() gives a one-line reason for the last failure on a handle.
 *  - Arrays are FP64, as in every shipped reference run (CmdLineUtils.jl:208 builds
 *    Float64 coordinates). Coordinates are point-major: x[i*d + k]. The reference's
 *    3 x N column-major CuArray (img[k, i]) has exactly this memory layout, so a
 *    Julia caller passes pointer(img) unchanged.
 *  - "Device" entry points take device pointers in caller-owned memory and a CUDA
 *    stream (cudaStream_t passed as void*, NULL = legacy default stream); they are
 *    asynchronous unless stated. "_host" entry points take host pointers, copy in,
 *    solve and copy out synchronously.
 *  - Cost C(x, y) is the reference's: p = 1 -> sum|d|, p = 2 -> sum d^2 (squared,
 *    no root), p = Inf -> max|d|, any other p > 0 -> sum |d|^p (no root).
 *  - A handle owns its workspace and CUDA graphs; use one handle per host thread.
 */
#ifndef CULAMP_H
#define CULAMP_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CULAMP_VERSION 100

/* status codes */
#define CULAMP_OK                 0
#define CULAMP_ERR_INVALID_ARG    1   /* bad size, pointer, p, eta, marginal ...     */
#define CULAMP_ERR_CUDA           2   /* a CUDA runtime call failed                  */
#define CULAMP_ERR_ALLOC          3   /* device or host allocation failed            */
#define CULAMP_ERR_UNSUPPORTED    4   /* valid but not implemented (e.g. d > 16)     */
#define CULAMP_ERR_IO             5   /* settings / potential file could not be read */
#define CULAMP_ERR_DEVICE_TIMEOUT 6   /* a bounded device-side wait gave up          */

/* Solver option bits. 0 reproduces the reference's behaviour. */
#define CULAMP_FLAG_TRUE_PINF      1u  /* Sinkhorn p=Inf iterates on the true L-inf cost.
                                          Default follows SinkhornKernel.jl:518-520, whose
                                          _opt kernel evaluates squared-Euclidean for p=Inf. */
#define CULAMP_FLAG_CHECK_ALWAYS   2u  /* LAMP: run the convergence check every `frequency`
                                          iterations even when args.verbose == 0
                                          (MirrorProxKernel.jl:1081 checks only when verbose) */
#define CULAMP_FLAG_MARGINAL_ONLY  4u  /* LAMP: stop on the marginal test alone           */
#define CULAMP_FLAG_FORM_PLAIN     8u  /* plain FP32 form: the reference's kernel shape
                                          (warp per row, FP32 potentials, host-synchronised
                                          loop). Default is the chosen form.               */
#define CULAMP_FLAG_NO_GRAPH      16u  /* chosen form without CUDA graphs (debugging)      */
#define CULAMP_FLAG_FEAT_X6       32u  /* feature clouds (d >= 32, squared cost): BF16x6
                                          split products (3 bf16 pieces, ~24-bit products)
                                          instead of the default BF16x3 (2 pieces)          */
#define CULAMP_FLAG_FORM_FP32    128u  /* Sinkhorn, p = 2, d <= 3: the chosen form's engine with the
                                          exponent formed in FP32 (same tiling, reference,
                                          graph loop; ~1e-4 relative per term)               */
#define CULAMP_FLAG_LADDER       256u  /* Sinkhorn and LAMP, p = 2, d <= 3: FP32-exponent passes
                                          until a check's FP64 L1 residual falls to
                                          32 x epsilon/6 or stops falling (no new lowest
                                          residual in 3 checks), then the FP64-exponent form
                                          to the tolerance. The check passes are FP64 in every
                                          form. LAMP needs its checks (verbose or
                                          CHECK_ALWAYS) and epsilon > 0.                    */
#define CULAMP_FLAG_FORM_FP64    512u  /* Sinkhorn: FP64-exponent passes throughout. Without
                                          it (and without FORM_FP32) Sinkhorn solves of
                                          n m >= 16384^2 pairs with p = 2 (or the p = Inf
                                          quirk) and d <= 3 take the precision ladder. LAMP
                                          takes the ladder only with FLAG_LADDER.           */
#define CULAMP_FLAG_NO_PERSIST  1024u  /* Sinkhorn: one launch per pass (CUDA graph) instead of the
                                          whole loop in one persistent launch, which small
                                          problems (n, m <= 8192, d <= 3, p = 1, 2 or Inf)
                                          take by default                                   */
#define CULAMP_FLAG_FEAT_FP64     64u  /* feature clouds on the FP64 pair loops instead of
                                          the tensor cores (exact inner products, slow)     */

/* EOTArgs (src/Utilities.jl:18-31), same field names and defaults. */
typedef struct culamp_args {
    double eta_p, eta_mu, tau_p, tau_mu, alpha, B, epsilon, anneal_mult;
    int64_t itermax, inner_iter;
    double tmax;
    int32_t verbose;
    int32_t _pad;
} culamp_args;

/* One row of the convergence log the reference prints:
 * time(s),iter,infeas,ot_objective,primal,dual (SinkhornKernel.jl:533,
 * MirrorProxKernel.jl:1097). Fields a solver does not print are NaN
 * (annealed Sinkhorn stores eta in `dual`). */
typedef struct culamp_log_row {
    double time_s, iter, infeas, ot_objective, primal, dual;
} culamp_log_row;

typedef struct culamp_stats {
    int64_t iterations;   /* loop index reached (iterations whose updates ran)        */
    int64_t num_iter;     /* the reference's num_iter counter (SinkhornKernel.jl:539) */
    double residual;      /* final L1 marginal residual                               */
    double objective;     /* final transport cost sum(P .* C) (sum of the cost cache) */
    double winf;          /* max-cost normaliser W_inf                                 */
    double eta_t, s_t;    /* LAMP: final eta_t and s                                   */
    double elapsed_ms;    /* device time of the solve                                  */
    int64_t log_rows;     /* rows written to the caller's log buffer                   */
    int32_t stopped;      /* 1 = tolerance met, 2 = itermax, 3 = tmax                  */
    int32_t status;
} culamp_stats;

typedef struct culamp_handle_s *culamp_handle;

/* ---------------------------------------------------------------- handle */
int culamp_version(void);
int culamp_create(culamp_handle *out, int device);
int culamp_destroy(culamp_handle h);
const char *culamp_status_string(int status);
const char *culamp_last_error(culamp_handle h);

/* ---------------------------------------------------------------- settings */
/* Defaults of EOTArgs (Utilities.jl:18-31). */
int culamp_args_default(culamp_args *out);
/* read_args_json (Utilities.jl:88-92): JSON object with any subset of the EOTArgs
 * keys; missing keys keep their defaults, unknown keys are ignored. */
int culamp_args_from_json(const char *path, culamp_args *out);
int culamp_args_from_json_string(const char *json, culamp_args *out);

/* ------------------------------------------------------ pass-level kernels
 * Device pointers, asynchronous on `stream`. Scratch comes from the handle. */

/* max_logsumexp_spp_ct! (MirrorProxKernel.jl:280-326): rowmax[i] = max_j C(x_i, y_j)
 * (rowmax may be NULL); *winf_host (may be NULL) receives max_i rowmax[i]
 * (SinkhornKernel.jl:500-502) -- this one call synchronises the stream. With
 * rowmax NULL only W_inf is formed, by a register-tiled pass over 64 x 64 pair
 * tiles (same value bit for bit). */
int culamp_max_cost(culamp_handle h, const double *x, const double *y, int64_t n, int64_t m,
                    int32_t d, double p, double *rowmax, double *winf_host, void *stream);

/* warp_logsumexp_ct_fused! (SinkhornKernel.jl:341-444):
 * out[i] = log(marg[i]) - LSE_j(-C(x_i,y_j)/(reg*winf) + pot[j]).
 * out is overwritten in place, as the reference updates phi; its previous
 * content (e.g. the last iteration's phi) is read as a hint that enables the
 * fixed-reference fast path. Any previous content is valid: a missing, stale or
 * non-finite hint only makes the kernel fall back to its online loop. */
int culamp_lse_rows_sk(culamp_handle h, double *out, const double *x, const double *y,
                       int64_t n, int64_t m, int32_t d, const double *marg, const double *pot,
                       double reg, double winf, double p, void *stream);

/* culamp_lse_rows_sk with a form: flags = CULAMP_FLAG_FORM_FP32 runs the
 * FP32-exponent pass (p = 2, d <= 3; CULAMP_ERR_UNSUPPORTED otherwise), 0 the
 * default pass. The pass the precision ladder runs first; no reference
 * counterpart (the reference kernel forms its exponents in FP32 throughout). */
int culamp_lse_rows_sk_form(culamp_handle h, double *out, const double *x, const double *y,
                            int64_t n, int64_t m, int32_t d, const double *marg, const double *pot,
                            double reg, double winf, double p, uint32_t flags, void *stream);

/* residual_opt! (SinkhornKernel.jl:9-81): res[i] = marg[i] - sum_j P_ij,
 * cost[i] = sum_j P_ij C_ij with P_ij = exp(-C_ij/(reg*winf) + phi[i] + psi[j]).
 * The reference evaluates C here as p==1 ? L1 : squared (SinkhornKernel.jl:38-42);
 * pass that p to reproduce it. */
int culamp_residual_sk(culamp_handle h, double *res, double *cost, const double *x,
                       const double *y, int64_t n, int64_t m, int32_t d, const double *marg,
                       const double *phi, const double *psi, double reg, double winf, double p,
                       void *stream);

/* warp_logsumexp_spp_ct_fused! (MirrorProxKernel.jl:833-938):
 * out[i] = LSE_j(-(C_ij * st/(2 winf) + theta[j]) / reg). reg = +Inf is allowed.
 * out's previous content (the last logZ) is a hint, as for culamp_lse_rows_sk. */
int culamp_lse_rows_spp(culamp_handle h, double *out, const double *x, const double *y,
                        int64_t n, int64_t m, int32_t d, const double *theta, double reg,
                        double st, double winf, double p, void *stream);

/* residual_spp_c! (MirrorProxKernel.jl:7-94), one output per column j:
 * res[j] = sum_i marg1[i] exp(-(C_ij st/(2 winf) + theta[j])/reg - logz[i]),
 * cost[j] = sum_i marg1[i] exp(...) C_ij. */
int culamp_col_residual_spp(culamp_handle h, double *res, double *cost, const double *x,
                            const double *y, int64_t n, int64_t m, int32_t d,
                            const double *marg1, const double *theta, const double *logz,
                            double reg, double st, double winf, double p, void *stream);

/* warp_min_reduce! (MirrorProxKernel.jl:941-1016): out[i] = min_j (C_ij + 2 winf theta[j]). */
int culamp_min_reduce(culamp_handle h, double *out, const double *x, const double *y,
                      int64_t n, int64_t m, int32_t d, const double *theta, double winf,
                      double p, void *stream);

/* update_theta_residual (MirrorProx.jl:159-180), elementwise over m entries;
 * theta may alias theta0. */
int culamp_theta_update(culamp_handle h, double *theta, const double *theta0,
                        const double *residual, const double *c, const double *eta_mu_i,
                        double eta_mu, int32_t adjust, double minv, double maxv, double winf,
                        int64_t m, void *stream);

/* naive_findmaxindex_ct! (SinkhornKernel.jl:124-162): barycentric image
 * out[i*d+k] = sum_j y[j*d+k] P_ij / sum_j P_ij, P_ij = exp(-C_ij/(reg winf) + phi[i] + psi[j]). */
int culamp_barycentric_sk(culamp_handle h, double *out, const double *x, const double *y,
                          int64_t n, int64_t m, int32_t d, const double *phi, const double *psi,
                          double reg, double winf, double p, void *stream);

/* Adjoint of the Sinkhorn transport cost. No direct counterpart in the
 * reference; it has the row-reduction shape of naive_findmaxindex_ct!
 * (SinkhornKernel.jl:124-162). With P_ij = exp(phi[i] + psi[j] - C_ij/(reg*winf)):
 *   grad[i*d+k] = sum_j P_ij dC(x_i, y_j)/dx_ik,   mass[i] = sum_j P_ij (may be NULL).
 * At optimal potentials grad is d OT_eps / d x_i (envelope theorem, eps = reg*winf
 * held fixed), computed without storing the n x m plan. 1 <= d <= 4. */
int culamp_adjoint_sk(culamp_handle h, double *grad, double *mass, const double *x,
                      const double *y, int64_t n, int64_t m, int32_t d, const double *phi,
                      const double *psi, double reg, double winf, double p, void *stream);

/* --------------------------------------------------------- solver level
 * Device pointers; the call returns when the solve has finished (it reads the
 * convergence state back once per batch of graph-launched iterations).
 * `log` (host memory, may be NULL) receives up to log_cap rows. */

/* sinkhorn_color_transfer with return_assignments=false (SinkhornKernel.jl:477-559):
 * phi (n), psi (m) in the reference's units (P_ij = exp(phi_i + psi_j - C_ij/(eta_p W_inf))).
 * phi0 / psi0 (device, may be NULL) are warm starts. */
int culamp_sinkhorn(culamp_handle h, const double *x, const double *y, int64_t n, int64_t m,
                    int32_t d, const double *r, const double *c, const culamp_args *args,
                    int64_t frequency, double p, const double *phi0, const double *psi0,
                    uint32_t flags, double *phi, double *psi, culamp_stats *stats,
                    culamp_log_row *log, int64_t log_cap, void *stream);

/* extragradient_color_transfer without the barycentric maps (MirrorProxKernel.jl:1019-1132):
 * nu, psi, theta (m), phi (n); psi = -2 W_inf nu / eta_p, phi = log r - logZ(nu). */
int culamp_lamp(culamp_handle h, const double *x, const double *y, int64_t n, int64_t m,
                int32_t d, const double *r, const double *c, const culamp_args *args,
                int64_t frequency, double p, uint32_t flags, double *nu, double *phi,
                double *psi, double *theta, culamp_stats *stats, culamp_log_row *log,
                int64_t log_cap, void *stream);

/* annealed_sinkhorn_euclidean, potentials only (AnnealedSinkhorn.jl:65-177):
 * eta_p -> max(anneal_mult * eta, epsilon) stages with extrapolated warm starts;
 * epsilon is both the final eta and the inner tolerance, as in the reference. */
int culamp_annealed_sinkhorn(culamp_handle h, const double *x, const double *y, int64_t n,
                             int64_t m, int32_t d, const double *r, const double *c,
                             const culamp_args *args, int64_t frequency, double p,
                             uint32_t flags, double *phi, double *psi, culamp_stats *stats,
                             culamp_log_row *log, int64_t log_cap, void *stream);

/* Self-transport OT(r, r; x, x), the two symmetric terms of the Sinkhorn
 * divergence. No counterpart in the reference. The plan is symmetric, so one
 * potential f solves it (P_ij = exp(f_i + f_j - C_ij/(eta_p W_inf)), W_inf of x
 * against itself); each iteration is one row pass f <- (f + T(f))/2 with T the
 * row update of SinkhornKernel.jl:518-520, checked every pass against the L1
 * row residual at its input (stop at residual <= epsilon/6, as culamp_sinkhorn).
 * stats: iterations = averaged updates applied; residual / objective from the
 * Sinkhorn residual pass at the returned f. f0 (device, may be NULL) warm-starts;
 * `frequency` only paces the log. flags: FEAT_X6 / FEAT_FP64 / NO_GRAPH /
 * TRUE_PINF. */
int culamp_symmetric_sinkhorn(culamp_handle h, const double *x, int64_t n, int32_t d,
                              const double *r, const culamp_args *args, int64_t frequency,
                              double p, const double *f0, uint32_t flags, double *f,
                              culamp_stats *stats, culamp_log_row *log, int64_t log_cap,
                              void *stream);

/* Row-sharded Sinkhorn (several GPUs, or several row blocks on one): shard g's
 * column pass (culamp_lse_rows_sk over its rows) gives out_g = log c - LSE over
 * its rows; the column potential is the log-sum-exp over shards,
 * psi_j = -log sum_g exp(-out_g,j). parts: `shards` device rows of m values
 * (e.g. an all-gather of the shards' outputs). No counterpart in the reference
 * (it runs on one GPU); replaces the column LSE of SinkhornKernel.jl:520-523
 * when the rows are split. */
int culamp_lse_combine(culamp_handle h, double *psi, const double *parts, int32_t shards, int64_t m,
                       void *stream);

/* ---------------------------------------------------------------- batched solves */
/* Many independent Sinkhorn problems of uneven n, m and d solved together. No
 * counterpart in the reference (its drivers solve one problem per call); each
 * instance follows sinkhorn_color_transfer (SinkhornKernel.jl:477-559) exactly as
 * culamp_sinkhorn would -- same iterations, checks and stopping rule -- with its
 * own control state. Every half-step of every class of instance (d <= 3, other
 * d on the FP64 pair loops, d >= 32 with p = 2 on the tensor cores) is one
 * launch over all instances, and the loop over iterations runs in CUDA graphs
 * with a device-side loop condition: one graph launch per phase, a phase ending
 * when the work of the instances still running has halved, after which the
 * survivors are re-planned with finer column splits. Tile shapes are chosen by
 * timing candidates on the batch itself (cached per batch signature). */
typedef struct culamp_instance {
    const double *x;      /* n x d points (device)                                     */
    const double *y;      /* m x d points (device)                                     */
    const double *r;      /* n row marginal (device)                                   */
    const double *c;      /* m column marginal (device)                                */
    double *phi;          /* n output potential (device)                               */
    double *psi;          /* m output potential (device)                               */
    int64_t n, m;
    int32_t d;
    int32_t reserved;
} culamp_instance;

typedef struct culamp_batch_stats {
    int64_t iterations;   /* as culamp_stats.iterations                                */
    int64_t num_iter;
    double residual;      /* final L1 row residual (FP64 sums)                         */
    double objective;     /* final transport cost                                      */
    double winf;
    int32_t stopped;      /* 1 tolerance, 2 itermax, 3 tmax                            */
    int32_t status;
} culamp_batch_stats;

typedef struct culamp_batch_info {
    double elapsed_ms;    /* device time of the W_inf passes and the solve loop        */
    double tune_ms;       /* device time spent timing shape candidates (0 when cached) */
    int32_t target_ctas_per_sm;   /* chosen pair-pass shape: CTAs per SM over the batch */
    int32_t feat_tiles_per_unit;  /* chosen feature-pass work-unit size (column tiles)  */
    int32_t unroll;       /* iterations per graph body (last phase)                    */
    int32_t launches_per_iteration;
    int32_t phases;       /* graph launches: the loop re-plans when the running work halves */
    int32_t reserved;
} culamp_batch_info;

/* p = 1 or 2 (p = Inf follows the reference and iterates on the squared cost).
 * flags: CULAMP_FLAG_FEAT_X6 / CULAMP_FLAG_FEAT_FP64 / CULAMP_FLAG_NO_GRAPH.
 * stats: count entries (may be NULL); info may be NULL. */
int culamp_batched_sinkhorn(culamp_handle h, const culamp_instance *inst, int32_t count,
                            const culamp_args *args, int64_t frequency, double p, uint32_t flags,
                            culamp_batch_stats *stats, culamp_batch_info *info, void *stream);

/* Host-buffer variants: same arguments with host pointers; copies in, solves and
 * copies out (the end-to-end path a Julia Array caller uses). */
int culamp_sinkhorn_host(culamp_handle h, const double *x, const double *y, int64_t n,
                         int64_t m, int32_t d, const double *r, const double *c,
                         const culamp_args *args, int64_t frequency, double p,
                         const double *phi0, const double *psi0, uint32_t flags, double *phi,
                         double *psi, culamp_stats *stats, culamp_log_row *log,
                         int64_t log_cap);
int culamp_lamp_host(culamp_handle h, const double *x, const double *y, int64_t n, int64_t m,
                     int32_t d, const double *r, const double *c, const culamp_args *args,
                     int64_t frequency, double p, uint32_t flags, double *nu, double *phi,
                     double *psi, double *theta, culamp_stats *stats, culamp_log_row *log,
                     int64_t log_cap);

/* ------------------------------------------------------------ dense costs
 * The GPU solvers of run_dot without --kernel (CmdLineUtils.jl:189-204): a
 * caller-supplied cost matrix W (n x m, row-major FP64 device memory, e.g. a
 * --weights CSV divided by max |W| as run_dot does). Every pass streams W or its
 * transpose (built once per call in the handle's workspace) from HBM.
 *
 * sinkhorn_log (Sinkhorn.jl:8-84): psi = log c - LSE_i(-W_ij/eta_p + phi_i),
 * phi = log r - LSE_j(-W_ij/eta_p + psi_j) per iteration; every `frequency`
 * iterations an FP64 check of the plan p = exp(-W/eta_p + phi + psi'): log row
 * (time, iter, feas = |rowsum - r|_1 + |colsum - c|_1, <p, W>, primal, dual), stop
 * when primal - dual < epsilon/6 and feas < epsilon/6; then the final two
 * half-steps. phi0 / psi0 may be NULL (zeros). plan (n x m) may be NULL.
 * Synchronous at check iterations. */
int culamp_sinkhorn_dense(culamp_handle h, const double *W, int64_t n, int64_t m,
                          const double *r, const double *c, const culamp_args *args,
                          int64_t frequency, const double *phi0, const double *psi0,
                          double *phi, double *psi, double *plan, culamp_stats *stats,
                          culamp_log_row *log, int64_t log_cap, void *stream);

/* The GPU LAMP on a dense cost (MirrorProx.jl:397-503): W_inf = max |W_ij|,
 * eta = eta_p / (2 W_inf); per iteration the extragradient step with
 * infeas(theta, eta_t) = (logZ_i = LSE_j(-(W_ij/(2 W_inf) + theta_j)/eta_t), column mass
 * res_j = sum_i r_i exp(... - logZ_i)); every `frequency` iterations an FP64 check:
 * feas = |c - colsum(r .* P)|_1, objective <W, round(r .* P, r, c)> (Utilities.jl:158-165),
 * primalv / dualv (MirrorProx.jl:7-32); stop when feas < epsilon/2 and
 * primal - dual < epsilon/2. Outputs theta, nu (m) and optionally the plan
 * r .* softmax(-(W/(2 W_inf) .+ nu')/eta_t) (n x m, may be NULL). theta0 may be NULL. */
int culamp_lamp_dense(culamp_handle h, const double *W, int64_t n, int64_t m, const double *r,
                      const double *c, const culamp_args *args, int64_t frequency,
                      const double *theta0, double *theta, double *nu, double *plan,
                      culamp_stats *stats, culamp_log_row *log, int64_t log_cap, void *stream);

/* FP64 re-evaluation of a Sinkhorn-form plan's L1 marginal errors, exp in FP64
 * (used to certify "1e-6 L1, FP64-checked"). Device pointers; synchronous. */
int culamp_marginal_error_fp64(culamp_handle h, const double *x, const double *y, int64_t n,
                               int64_t m, int32_t d, const double *r, const double *c,
                               const double *phi, const double *psi, double reg, double winf,
                               double p, double *row_l1, double *col_l1, void *stream);

/* Scratch-free variant of culamp_lse_rows_sk, for callers that cannot let the
 * library allocate device memory when they call it: hosts that own all device
 * memory through their own pool or budget and forbid third-party cudaMalloc.
 * No counterpart in the reference (its kernels allocate nothing, but its
 * solvers allocate their caches with CuArray).
 * Same arguments and result as culamp_lse_rows_sk, without a handle. Its scratch
 * is fixed file-scope device memory (3 MiB of split partials + 256 KiB of
 * tickets, held on every GPU that loads the library until exit); n is limited
 * to 8,388,608 rows for every d (CULAMP_ERR_UNSUPPORTED beyond, before any
 * launch). The first call on a device resolves that memory's address and may
 * load the module: make it before any stream capture; a failed set-up
 * (CULAMP_ERR_CUDA) is retried by the next call. All calls share the scratch,
 * so calls that overlap on the GPU race; serialise them. Calls no cudaMalloc /
 * cudaFree. */
int culamp_lse_rows_sk_noalloc(double *out, const double *x, const double *y, int64_t n,
                               int64_t m, int32_t d, const double *marg, const double *pot,
                               double reg, double winf, double p, void *stream);

/* ------------------------------------------------------------ diagnostics
 * No counterpart in the reference. Measures, on the running GPU, the sustained
 * instruction rates that bound the pair passes: out[0] = DFMA/s, out[1] = MUFU
 * ex2/s, out[2] = FP64->FP32 conversions/s, out[3] = SM count. Synchronous. */
int culamp_probe_pipes(culamp_handle h, double *out, void *stream);

/* No counterpart in the reference. Runs the tensor-core path's bounded
 * mbarrier wait (the one every role of the feature pass uses) on a barrier
 * phase that nothing completes, with the given limit in ns (at most 10 s).
 * Returns CULAMP_ERR_DEVICE_TIMEOUT when the wait gave up and reported it, as
 * it must; the device context stays usable. Synchronous. */
int culamp_probe_wait(culamp_handle h, uint64_t limit_ns, void *stream);

/* No counterpart in the reference. Runs the persistent loops' grid barrier
 * (two co-resident CTAs, one of which never arrives) with the given wait limit
 * in ns (at most 10 s). Returns CULAMP_ERR_DEVICE_TIMEOUT when the waiting CTA
 * gave up and published the abort, as it must; the device context stays
 * usable. Synchronous. */
int culamp_probe_grid_wait(culamp_handle h, uint64_t limit_ns, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* CULAMP_H */
