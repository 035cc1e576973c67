"""Oracle for the kernelized entropic-OT path: TEST INFRASTRUCTURE ONLY.

Two independent FP64 restatements of CuLAMP.jl's algorithms:

* ``C``   -- ctypes bindings to oracle/culamp_oracle.c (OpenMP, any size the CPU
  finishes), built by oracle/Makefile into oracle/_build/.
* ``np_*`` -- a vectorised numpy restatement for small sizes, written separately
  so the two can check each other.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
arm may import this module. Parity status: partially pinned -- the reference
cannot run here; its archived W_inf values (126 / 7938 / 63 for p = 1 / 2 / Inf
on its integer 64x64 grid, data_archive/data/updated_pnorm.csv) are the only
values taken from reference outputs.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libculamp_oracle.so")

TRUE_PINF = 1
CHECK_ALWAYS = 2
MARGINAL_ONLY = 4


class OrArgs(C.Structure):
    _fields_ = [("eta_p", C.c_double), ("eta_mu", C.c_double), ("tau_p", C.c_double),
                ("tau_mu", C.c_double), ("alpha", C.c_double), ("B", C.c_double),
                ("epsilon", C.c_double), ("anneal_mult", C.c_double),
                ("itermax", C.c_int64), ("inner_iter", C.c_int64), ("tmax", C.c_double),
                ("verbose", C.c_int32), ("_pad", C.c_int32)]


class OrLogRow(C.Structure):
    _fields_ = [("time_s", C.c_double), ("iter", C.c_double), ("infeas", C.c_double),
                ("ot_objective", C.c_double), ("primal", C.c_double), ("dual", C.c_double)]


class OrStats(C.Structure):
    _fields_ = [("iterations", C.c_int64), ("num_iter", C.c_int64), ("residual", C.c_double),
                ("objective", C.c_double), ("winf", C.c_double), ("eta_t", C.c_double),
                ("s_t", C.c_double), ("log_rows", C.c_int64), ("stopped", C.c_int32),
                ("_pad", C.c_int32)]


def build() -> str:
    """Compile the C oracle (make) if missing; returns the library path."""
    if not os.path.exists(LIB_PATH) or (
            os.path.getmtime(LIB_PATH) < os.path.getmtime(os.path.join(HERE, "culamp_oracle.c"))):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(LIB_PATH)
        P = C.POINTER(C.c_double)
        i64 = C.c_int64
        _lib.or_max_cost.restype = C.c_double
        _lib.or_max_cost.argtypes = [P, P, i64, i64, C.c_int, C.c_double]
        _lib.or_cost.restype = C.c_double
        for name in ("or_sinkhorn_kernel", "or_lamp_kernel", "or_annealed_sinkhorn_kernel",
                     "or_sinkhorn_dense", "or_lamp_dense"):
            getattr(_lib, name).restype = C.c_int
    return _lib


def _p(a):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _c64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


@dataclass
class Args:
    """EOTArgs with the reference defaults (src/Utilities.jl:18-31)."""
    eta_p: float = 0.0
    eta_mu: float = 0.0
    tau_p: float = 1.0
    tau_mu: float = 1.0
    alpha: float = 0.01
    B: float = 1.0
    epsilon: float = 1e-4
    anneal_mult: float = 0.95
    itermax: int = 10_000
    inner_iter: int = 10
    tmax: float = math.inf
    verbose: bool = True

    def c(self) -> OrArgs:
        return OrArgs(self.eta_p, self.eta_mu, self.tau_p, self.tau_mu, self.alpha, self.B,
                      self.epsilon, self.anneal_mult, int(self.itermax), int(self.inner_iter),
                      self.tmax, int(bool(self.verbose)), 0)


def set_threads(t: int) -> None:
    lib().or_set_num_threads(C.c_int(t))


def num_threads() -> int:
    return int(lib().or_num_threads())


def _logs(buf, st):
    rows = []
    for k in range(st.log_rows):
        r = buf[k]
        rows.append((r.time_s, int(r.iter), r.infeas, r.ot_objective, r.primal, r.dual))
    return rows


# ---------------------------------------------------------------- C bindings

def max_cost(x, y, p):
    x, y = _c64(x), _c64(y)
    return lib().or_max_cost(_p(x), _p(y), x.shape[0], y.shape[0], x.shape[1], float(p))


def max_cost_rows(x, y, p):
    x, y = _c64(x), _c64(y)
    out = np.empty(x.shape[0])
    lib().or_max_cost_rows(_p(x), _p(y), C.c_int64(x.shape[0]), C.c_int64(y.shape[0]),
                           C.c_int(x.shape[1]), C.c_double(p), _p(out))
    return out


def sk_lse(x, y, marg, pot, reg, winf, cost_p):
    x, y, marg, pot = map(_c64, (x, y, marg, pot))
    out = np.empty(x.shape[0])
    lib().or_sk_lse(_p(out), _p(x), _p(y), C.c_int64(x.shape[0]), C.c_int64(y.shape[0]),
                    C.c_int(x.shape[1]), _p(marg), _p(pot), C.c_double(reg), C.c_double(winf),
                    C.c_double(cost_p))
    return out


def sk_residual(x, y, marg, phi, psi, reg, winf, cost_p):
    x, y, marg, phi, psi = map(_c64, (x, y, marg, phi, psi))
    res = np.empty(x.shape[0])
    cost = np.empty(x.shape[0])
    lib().or_sk_residual(_p(res), _p(cost), _p(x), _p(y), C.c_int64(x.shape[0]),
                         C.c_int64(y.shape[0]), C.c_int(x.shape[1]), _p(marg), _p(phi),
                         _p(psi), C.c_double(reg), C.c_double(winf), C.c_double(cost_p))
    return res, cost


def spp_lse(x, y, theta, reg, st, winf, p):
    x, y, theta = map(_c64, (x, y, theta))
    out = np.empty(x.shape[0])
    lib().or_spp_lse(_p(out), _p(x), _p(y), C.c_int64(x.shape[0]), C.c_int64(y.shape[0]),
                     C.c_int(x.shape[1]), _p(theta), C.c_double(reg), C.c_double(st),
                     C.c_double(winf), C.c_double(p))
    return out


def spp_col_residual(x, y, marg1, theta, logz, reg, st, winf, p):
    x, y, marg1, theta, logz = map(_c64, (x, y, marg1, theta, logz))
    res = np.empty(y.shape[0])
    cost = np.empty(y.shape[0])
    lib().or_spp_col_residual(_p(res), _p(cost), _p(x), _p(y), C.c_int64(x.shape[0]),
                              C.c_int64(y.shape[0]), C.c_int(x.shape[1]), _p(marg1), _p(theta),
                              _p(logz), C.c_double(reg), C.c_double(st), C.c_double(winf),
                              C.c_double(p))
    return res, cost


def min_reduce(x, y, theta, winf, p):
    x, y, theta = map(_c64, (x, y, theta))
    out = np.empty(x.shape[0])
    lib().or_min_reduce(_p(out), _p(x), _p(y), C.c_int64(x.shape[0]), C.c_int64(y.shape[0]),
                        C.c_int(x.shape[1]), _p(theta), C.c_double(winf), C.c_double(p))
    return out


def theta_update(theta0, residual, c, eta_mu_i, eta_mu, adjust, minv, maxv, winf=1.0):
    theta0, residual, c, eta_mu_i = map(_c64, (theta0, residual, c, eta_mu_i))
    out = np.empty_like(theta0)
    lib().or_theta_update(_p(out), _p(theta0), _p(residual), _p(c), _p(eta_mu_i),
                          C.c_double(eta_mu), C.c_int(int(adjust)), C.c_double(minv),
                          C.c_double(maxv), C.c_double(winf), C.c_int64(theta0.shape[0]))
    return out


def barycentric_sk(x, y, phi, psi, reg, winf, cost_p):
    x, y, phi, psi = map(_c64, (x, y, phi, psi))
    out = np.empty_like(x)
    lib().or_barycentric_sk(_p(out), _p(x), _p(y), C.c_int64(x.shape[0]),
                            C.c_int64(y.shape[0]), C.c_int(x.shape[1]), _p(phi), _p(psi),
                            C.c_double(reg), C.c_double(winf), C.c_double(cost_p))
    return out


def envelope_grad(x, y, phi, psi, reg, winf, p, rows=None):
    """FP64 sum_j P_ij grad_x C(x_i, y_j) and sum_j P_ij for the listed rows."""
    x, y, phi, psi = map(_c64, (x, y, phi, psi))
    d = x.shape[1]
    ridx = None if rows is None else np.ascontiguousarray(rows, dtype=np.int64)
    k = x.shape[0] if ridx is None else ridx.shape[0]
    grad = np.empty((k, d))
    mass = np.empty(k)
    lib().or_envelope_grad(_p(grad), _p(mass), _p(x), _p(y), C.c_int64(x.shape[0]),
                           C.c_int64(y.shape[0]), C.c_int(d), _p(phi), _p(psi), C.c_double(reg),
                           C.c_double(winf), C.c_double(p),
                           ridx.ctypes.data_as(C.POINTER(C.c_int64)) if ridx is not None else None,
                           C.c_int64(k))
    return grad, mass


def sinkhorn_kernel(x, y, r, c, args: Args, frequency=100, p=2.0, phi0=None, psi0=None,
                    flags=0, log_cap=100000):
    x, y, r, c = map(_c64, (x, y, r, c))
    n, m = x.shape[0], y.shape[0]
    phi = np.empty(n)
    psi = np.empty(m)
    st = OrStats()
    buf = (OrLogRow * log_cap)()
    a = args.c()
    lib().or_sinkhorn_kernel(_p(x), _p(y), C.c_int64(n), C.c_int64(m), C.c_int(x.shape[1]),
                             _p(r), _p(c), C.byref(a), C.c_int64(frequency), C.c_double(p),
                             _p(_c64(phi0)) if phi0 is not None else None,
                             _p(_c64(psi0)) if psi0 is not None else None,
                             C.c_int(flags), _p(phi), _p(psi), C.byref(st), buf,
                             C.c_int64(log_cap))
    return phi, psi, st, _logs(buf, st)


def lamp_kernel(x, y, r, c, args: Args, frequency=100, p=2.0, flags=0, log_cap=100000):
    x, y, r, c = map(_c64, (x, y, r, c))
    n, m = x.shape[0], y.shape[0]
    nu, phi, psi, theta = np.empty(m), np.empty(n), np.empty(m), np.empty(m)
    st = OrStats()
    buf = (OrLogRow * log_cap)()
    a = args.c()
    lib().or_lamp_kernel(_p(x), _p(y), C.c_int64(n), C.c_int64(m), C.c_int(x.shape[1]),
                         _p(r), _p(c), C.byref(a), C.c_int64(frequency), C.c_double(p),
                         C.c_int(flags), _p(nu), _p(phi), _p(psi), _p(theta), C.byref(st), buf,
                         C.c_int64(log_cap))
    return nu, phi, psi, theta, st, _logs(buf, st)


def annealed_sinkhorn_kernel(x, y, r, c, args: Args, frequency=10, p=2.0, flags=0,
                             log_cap=10000):
    x, y, r, c = map(_c64, (x, y, r, c))
    n, m = x.shape[0], y.shape[0]
    phi, psi = np.empty(n), np.empty(m)
    st = OrStats()
    buf = (OrLogRow * log_cap)()
    a = args.c()
    lib().or_annealed_sinkhorn_kernel(_p(x), _p(y), C.c_int64(n), C.c_int64(m),
                                      C.c_int(x.shape[1]), _p(r), _p(c), C.byref(a),
                                      C.c_int64(frequency), C.c_double(p), C.c_int(flags),
                                      _p(phi), _p(psi), C.byref(st), buf, C.c_int64(log_cap))
    return phi, psi, st, _logs(buf, st)


def sinkhorn_dense(W, r, c, args: Args, frequency=50, log_cap=100000):
    W, r, c = map(_c64, (W, r, c))
    n = r.shape[0]
    phi, psi = np.empty(n), np.empty(n)
    st = OrStats()
    buf = (OrLogRow * log_cap)()
    a = args.c()
    lib().or_sinkhorn_dense(_p(W), C.c_int64(n), _p(r), _p(c), C.byref(a),
                            C.c_int64(frequency), _p(phi), _p(psi), C.byref(st), buf,
                            C.c_int64(log_cap))
    return phi, psi, st, _logs(buf, st)


def lamp_dense(W, r, c, args: Args, frequency=50, log_cap=100000, want_plan=False):
    W, r, c = map(_c64, (W, r, c))
    n = r.shape[0]
    theta, nu = np.empty(n), np.empty(n)
    plan = np.empty((n, n)) if want_plan else None
    st = OrStats()
    buf = (OrLogRow * log_cap)()
    a = args.c()
    lib().or_lamp_dense(_p(W), C.c_int64(n), _p(r), _p(c), C.byref(a), C.c_int64(frequency),
                        _p(theta), _p(nu), _p(plan), C.byref(st), buf, C.c_int64(log_cap))
    return theta, nu, plan, st, _logs(buf, st)


# ------------------------------------------------- independent numpy mirror

def np_cost(x, y, p):
    """Dense pair cost (small sizes). Same convention as the reference's
    kernels: p=2 squared, p=Inf Chebyshev, other p sum |d|^p (no root)."""
    diff = np.abs(np.asarray(x, np.float64)[:, None, :] - np.asarray(y, np.float64)[None, :, :])
    if p == 1:
        return diff.sum(-1)
    if p == 2:
        return (diff ** 2).sum(-1)
    if math.isinf(p):
        return diff.max(-1)
    return (diff ** p).sum(-1)


def np_lse(a, axis):
    mx = a.max(axis=axis, keepdims=True)
    return (np.log(np.exp(a - mx).sum(axis=axis, keepdims=True)) + mx).squeeze(axis)


def bf16_rn(a):
    """Nearest bf16 value (ties to even) of each FP64 entry, as FP64: keep 7 of
    the 52 stored mantissa bits, rounding on the bit pattern."""
    b = np.ascontiguousarray(a, np.float64).copy().view(np.uint64)
    b = (b + np.uint64((1 << 44) - 1) + ((b >> np.uint64(45)) & np.uint64(1))) & ~np.uint64((1 << 45) - 1)
    return b.view(np.float64)


def bf16_pieces(a, pieces):
    """a = a_0 + a_1 + ... + rest: a_k is the bf16 rounding of what a_0..a_{k-1} leave."""
    out, rest = [], np.asarray(a, np.float64).copy()
    for _ in range(pieces):
        h = bf16_rn(rest)
        out.append(h)
        rest = rest - h
    return out


def split_dot(x, y, pieces):
    """<x_i, y_j> from bf16 pieces with FP64 sums: pieces=2 is BF16x3
    (x0y0 + x0y1 + x1y0), pieces=3 is BF16x6 (+ x0y2 + x1y1 + x2y0)."""
    xs, ys = bf16_pieces(x, pieces), bf16_pieces(y, pieces)
    dot = np.zeros((len(x), len(y)))
    for a in range(pieces):
        for b in range(pieces - a):
            dot += xs[a] @ ys[b].T
    return dot


def feature_cost(x, y, pieces=None):
    """Squared Euclidean cost |x|^2 + |y|^2 - 2<x, y> with exact FP64 norms and
    the inner products exact (pieces=None) or from bf16 split products."""
    x, y = np.asarray(x, np.float64), np.asarray(y, np.float64)
    dot = x @ y.T if pieces is None else split_dot(x, y, pieces)
    return (x * x).sum(1)[:, None] + (y * y).sum(1)[None, :] - 2.0 * dot


def np_sinkhorn_kernel(x, y, r, c, eta_p, itermax, frequency=1, epsilon=0.0, p=2.0,
                       true_pinf=False, phi0=None, psi0=None, cost=None, winf=None):
    """Sinkhorn of SinkhornKernel.jl:477-559 restated with dense numpy arrays.
    `cost` replaces the pair cost of the iterations and the residual (p = 2
    only), `winf` the normaliser max_ij C_ij."""
    if winf is None:
        winf = np_cost(x, y, p).max()
    ip = 2.0 if (math.isinf(p) and not true_pinf) else p
    rp = p if true_pinf else (1.0 if p == 1 else 2.0)
    Ci = np_cost(x, y, ip) if cost is None else cost
    Cr = np_cost(x, y, rp) if cost is None else cost
    phi = np.zeros(len(r)) if phi0 is None else np.array(phi0, np.float64)
    psi = np.zeros(len(c)) if psi0 is None else np.array(psi0, np.float64)
    k = -1.0 / (eta_p * winf)
    it_done = 0
    for it in range(1, itermax + 1):
        phi = np.log(r) - np_lse(Ci * k + psi[None, :], 1)
        psi = np.log(c) - np_lse(Ci.T * k + phi[None, :], 1)
        it_done = it
        if (it - 1) % frequency == 0:
            P = np.exp(Cr * k + phi[:, None] + psi[None, :])
            if np.abs(r - P.sum(1)).sum() <= epsilon / 6:
                break
    P = np.exp(Cr * k + phi[:, None] + psi[None, :])
    return phi, psi, np.abs(r - P.sum(1)).sum(), (P * Cr).sum(), it_done, winf


def np_symmetric_sinkhorn(x, r, eta_p, itermax, epsilon=0.0, p=2.0, f0=None, cost=None, winf=None):
    """Self-transport OT(r, r; x, x) by the averaged symmetric iteration
    f <- (f + T(f))/2, T(f) = log r - LSE_j(-C_ij/(eta_p W) + f_j): the row
    update of SinkhornKernel.jl:518-520 with both potentials equal. No
    counterpart in the reference; its fixed point is the Sinkhorn solution with
    phi = psi. Every iteration first tests the L1 row residual at its input f
    (residual <= epsilon/6 stops before updating). Returns (f, residual at f,
    transport cost at f, updates applied, W)."""
    ip = 2.0 if math.isinf(p) else p
    rp = 1.0 if p == 1 else 2.0
    Ci = np_cost(x, x, ip) if cost is None else cost
    Cr = np_cost(x, x, rp) if cost is None else cost
    winf = np_cost(x, x, p).max() if winf is None else winf
    k = -1.0 / (eta_p * winf)
    f = np.zeros(len(r)) if f0 is None else np.array(f0, np.float64)
    done = 0
    while True:
        L = np_lse(Ci * k + f[None, :], 1)
        res = np.abs(r - np.exp(f + L)).sum()
        if res <= epsilon / 6 or done >= itermax:
            break
        f = 0.5 * (f + np.log(r) - L)
        done += 1
    P = np.exp(Cr * k + f[:, None] + f[None, :])
    return f, np.abs(r - P.sum(1)).sum(), (P * Cr).sum(), done, winf


def np_theta_update(theta0, res, c, eta_mu_i, eta_mu, adjust, minv, maxv):
    t = np.tanh((res - c) / eta_mu_i + 0.5 * (1 - eta_mu) * np.log((1 + theta0) / (1 - theta0)))
    return np.clip(t, minv, maxv) if adjust else t


def np_lamp_kernel(x, y, r, c, eta_p, itermax, p=2.0, alpha=0.01, tau_mu=1.0, eta_mu=0.0,
                   B=1.0, cost=None, winf=None):
    """LAMP of MirrorProxKernel.jl:1019-1132 (non-verbose: runs itermax).
    `cost` / `winf` as in np_sinkhorn_kernel."""
    C_ = np_cost(x, y, p) if cost is None else cost
    winf = C_.max() if winf is None else winf
    n, m = C_.shape
    eta = eta_p / (2 * winf)
    emu = (c + alpha / n) / tau_mu
    theta = np.zeros(m)
    nu = np.zeros(m)
    s_t, eta_t = 1.0, math.inf
    minv, maxv = math.tanh(-B / 2), math.tanh(B / 2)

    def infeas(th, et, s):
        if math.isinf(et):
            A = np.zeros_like(C_)
        else:
            A = -(C_ * (s / (2 * winf)) + th[None, :]) / et
        logz = np_lse(A, 1)
        P = np.exp(A - logz[:, None]) * r[:, None]
        return logz, P.sum(0), (P * C_).sum(0)

    for _ in range(itermax):
        _, res, _ = infeas(nu, eta_t, s_t)
        thb = np_theta_update(theta, res, c, emu, eta_mu, False, minv, maxv)
        eta_t = 1.0 / (1.0 + (1.0 / eta_t) * (1.0 - eta))
        nub = (1 - eta_t) * nu + eta_t * theta
        s_t = (1 - eta_t) * s_t + eta_t
        _, res, _ = infeas(nub, eta_t, s_t)
        theta = np_theta_update(theta, res, c, emu, eta_mu, True, minv, maxv)
        nu = (1 - eta_t) * nu + eta_t * thb
    logz, res, cost = infeas(nu, eta_t, s_t)
    phi = np.log(r) - logz
    psi = -2 * winf * nu / eta_p if eta_p != 0 else np.full(m, np.nan)
    return nu, phi, psi, theta, np.abs(res - c).sum(), cost.sum(), eta_t


def fp64_marginal_error_sk(x, y, r, c, phi, psi, eta_p, winf, p):
    """FP64 re-evaluation of the L1 marginal errors of a Sinkhorn-form plan
    P_ij = exp(phi_i + psi_j - C_ij/(eta_p W_inf)) via the C oracle:
    returns (row L1, column L1)."""
    res_r, _ = sk_residual(x, y, r, phi, psi, eta_p, winf, p)
    res_c, _ = sk_residual(y, x, c, psi, phi, eta_p, winf, p)
    return float(np.abs(res_r).sum()), float(np.abs(res_c).sum())


# ------------------------------------------------ dense-cost GPU solvers (numpy)

def np_neg_entropy_rows(P):
    """neg_entropy(P, dims=2) (Utilities.jl:137-143): sum_j P_ij log P_ij over P > 0."""
    with np.errstate(divide="ignore", invalid="ignore"):
        return np.where(P > 0, P * np.log(np.where(P > 0, P, 1.0)), 0.0).sum(1)


def np_round(g, mu, nu):
    """round (Utilities.jl:158-165): rows scaled to <= mu, columns to <= nu, then
    the rank-one correction of the remaining row / column deficits."""
    g1 = g * np.minimum(mu / g.sum(1), 1.0)[:, None]
    g2 = g1 * np.minimum(nu / g1.sum(0), 1.0)[None, :]
    rmu = mu - g2.sum(1)
    rnu = nu - g2.sum(0)
    return g2 + np.outer(rmu, rnu) / np.abs(rmu).sum()


def np_primalv(P, W, winf, etap, r, c):
    """primalv(p, W, W_inf, eta_p, r, c) (MirrorProx.jl:28-32)."""
    rP = r[:, None] * P
    return 2 * (0.5 * (W * rP).sum() + (winf * np.abs(rP.sum(0) - c)).sum()
                + etap * np.dot(r, np_neg_entropy_rows(P)) + etap * np.dot(r, np.log(r)))


def np_dualv(theta, W, winf, etap, r, c):
    """dualv(theta, W, W_inf, eta_p, r, c) (MirrorProx.jl:7-13)."""
    if etap == 0:
        return -np.dot(c, 2 * winf * theta) + np.dot(r, (W + 2 * winf * theta[None, :]).min(1))
    lse = np_lse(-(0.5 * W + winf * theta[None, :]) / etap, 1)
    return 2 * ((-winf * np.dot(c, theta) - etap * np.dot(r, lse)) + etap * np.dot(r, np.log(r)))


def np_theta_res(theta0, res, c, eta_mu_i, eta_mu):
    """update_theta_residual (MirrorProx.jl:159-180) with W_inf = 1, no clamp:
    tanh(d/2 + (1 - eta_mu)/2 log((1+theta)/(1-theta))), d = 2 (res - c) / eta_mu_i."""
    return np.tanh((res - c) / eta_mu_i + 0.5 * (1 - eta_mu) * np.log((1 + theta0) / (1 - theta0)))


def np_lamp_dense_gpu(W, r, c, eta_p, itermax, frequency=50, epsilon=1e-4, eta_mu=0.0, tau_p=1.0,
                      tau_mu=1.0, alpha=0.01, B=1.0):
    """The GPU LAMP of MirrorProx.jl:397-503 on a dense W (n x m; r: n, c: m).
    Returns (r .* P, theta, nu, log rows (iter, feas, obj, primal, dual), iterations,
    eta_t, stopped)."""
    n, m = W.shape
    winf = np.abs(W).max()
    theta = np.zeros(m)
    etap = eta_p / 2 / winf
    nu = theta.copy()
    emu = (c + alpha / m) / tau_mu
    minv, maxv = math.tanh(-B / 2), math.tanh(B / 2)

    def softmax_rows(th, eta_t):
        A = np.zeros_like(W) if math.isinf(eta_t) else -(W / (2 * winf) + th[None, :]) / eta_t
        return np.exp(A - np_lse(A, 1)[:, None])

    def infeas(th, eta_t):
        return (r[:, None] * softmax_rows(th, eta_t)).sum(0)

    eta_t = math.inf
    res = infeas(nu, eta_t)
    log = []
    stopped, it = 2, 0
    for it in range(1, itermax + 1):
        if (it - 1) % frequency == 0:
            P = softmax_rows(nu, eta_t)
            rP = r[:, None] * P
            obj = (W * np_round(rP, r, c)).sum()
            primal = np_primalv(P, W, winf, etap, r, c)
            dual = np_dualv(theta, W, winf, etap, r, c)
            feas = np.abs(c - rP.sum(0)).sum()
            log.append((it, feas, obj, primal, dual))
            if feas < epsilon / 2 and primal - dual < epsilon / 2:
                stopped = 1
                break
        thb = np_theta_res(theta, res, c, emu, tau_mu * eta_mu)
        eta_t = 1 / (tau_p + (1 / eta_t) * (1 - etap))
        nub = tau_p * eta_t * theta + (1 - tau_p * eta_t) * nu
        res = infeas(nub, eta_t)
        theta = np_theta_res(theta, res, c, emu, eta_mu)
        nu = (1 - tau_p * eta_t) * nu + tau_p * eta_t * thb
        theta = np.clip(theta, minv, maxv)
        res = infeas(nu, eta_t)
    plan = r[:, None] * softmax_rows(nu, eta_t)
    return plan, theta, nu, log, it, eta_t, stopped


def np_sinkhorn_dense(W, r, c, eta_p, itermax, frequency=50, epsilon=1e-4):
    """sinkhorn_log (Sinkhorn.jl:8-84) for any n x m W. Returns (p, phi, psi, log
    rows (iter, feas, obj, pobj, dobj), iterations, num_iter, stopped)."""
    n, m = W.shape
    K = -W / eta_p
    phi, psi = np.zeros(n), np.zeros(m)
    log, num_iter, stopped, it = [], 0, 2, 0
    for it in range(1, itermax + 1):
        psi = np.log(c) - np_lse(K + phi[:, None], 0)
        phi = np.log(r) - np_lse(K + psi[None, :], 1)
        if (it - 1) % frequency == 0:
            p = np.exp(K + phi[:, None] + psi[None, :])
            feas = np.abs(p.sum(0) - c).sum() + np.abs(p.sum(1) - r).sum()
            obj = (p * W).sum()
            with np.errstate(divide="ignore", invalid="ignore"):
                ent = np.where(p > 0, p * np.log(np.where(p > 0, p, 1.0)), 0.0).sum()
            pobj = obj + eta_p * ent
            X = K + phi[:, None] + psi[None, :]
            lse_all = np.log(np.exp(X - X.max()).sum()) + X.max()
            dobj = -eta_p * (-lse_all - np.dot(c, psi) - np.dot(r, phi))
            log.append((it, feas, obj, pobj, dobj))
            if pobj - dobj < epsilon / 6 and feas < epsilon / 6:
                stopped = 1
                break
        num_iter += 1
    psi = np.log(c) - np_lse(K + phi[:, None], 0)
    phi = np.log(r) - np_lse(K + psi[None, :], 1)
    return np.exp(K + phi[:, None] + psi[None, :]), phi, psi, log, it, num_iter, stopped


# ------------------------------------------------ cell-similarity feature costs

def np_cell_cost(data, metric, normalize_features=True):
    """feature_cost(kernel, i, j) of CellUtilities.jl:127-172 for all row pairs
    of one data matrix (rows = points), with CellCostKernel's statistics
    (:69-112): row sums s_i (0 -> 1, or all 1 when not normalising), squared
    norms, means and centred squared norms of the raw rows, metric scale
    l1: 2, l2: sqrt(2), cosine / correlation: 2."""
    a = np.asarray(data, dtype=np.float64)
    n, d = a.shape
    s = a.sum(1) if normalize_features else np.ones(n)
    if normalize_features:
        s = np.where(s > 0, s, 1.0)
    sq = (a * a).sum(1)
    mean = a.mean(1)
    csq = ((a - mean[:, None]) ** 2).sum(1)
    metric = "correlation" if metric == "pearson" else metric
    scale = {"l1": 2.0, "l2": math.sqrt(2.0), "cosine": 2.0, "correlation": 2.0}[metric]
    if metric == "l1":
        u = a / s[:, None]
        return np.abs(u[:, None, :] - u[None, :, :]).sum(-1) / scale
    dot = (a @ a.T) / (s[:, None] * s[None, :])
    nrm = sq / s ** 2
    if metric == "l2":
        return np.sqrt(np.maximum(nrm[:, None] + nrm[None, :] - 2 * dot, 0.0)) / scale
    if metric == "cosine":
        den = np.sqrt(nrm[:, None] * nrm[None, :])
        with np.errstate(divide="ignore", invalid="ignore"):
            sim = np.clip(dot / den, -1.0, 1.0)
        return np.where(den > 0, (1.0 - sim) / scale, 0.0)
    mu = mean / s
    cen = csq / s ** 2
    den = np.sqrt(cen[:, None] * cen[None, :])
    with np.errstate(divide="ignore", invalid="ignore"):
        corr = np.clip((dot - d * mu[:, None] * mu[None, :]) / den, -1.0, 1.0)
    special = np.where(np.abs(mu[:, None] - mu[None, :]) <= math.sqrt(np.finfo(float).eps), 0.0, 1.0 / scale)
    return np.where(den > 0, (1.0 - corr) / scale, special)
