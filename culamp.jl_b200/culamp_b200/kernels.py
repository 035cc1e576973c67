"""Pass-level kernels, named after the CuLAMP.jl device kernels they replace.

All arguments are float64 CUDA tensors; point clouds are (N, d). Each call is
one asynchronous launch on the current torch stream (max_logsumexp_spp_ct also
returns W_inf, which synchronises).
"""
from __future__ import annotations

import ctypes as C

import torch

from .solvers import _dev, _stream, get_handle


def _h(t):
    return get_handle(t.device.index)


def _empty(n, like):
    return torch.empty(n, dtype=torch.float64, device=like.device)


def max_logsumexp_spp_ct(x, y, p, rows: bool = True):
    """MirrorProxKernel.jl:280-326 + `maximum` (SinkhornKernel.jl:500-502):
    returns (rowmax, W_inf); with rows=False only W_inf is formed (rowmax None)."""
    n, d = x.shape
    m = y.shape[0]
    out = _empty(n, x) if rows else None
    w = C.c_double()
    h = _h(x)
    h.check(h._lib.culamp_max_cost(h.ptr, _dev(x, "x"), _dev(y, "y"), n, m, d, float(p),
                                   C.c_void_p(out.data_ptr()) if rows else None, C.byref(w),
                                   _stream()),
            "culamp_max_cost")
    return out, w.value


def warp_logsumexp_ct_fused(x, y, marginal, pot, reg, winf, p, out=None, flags=0):
    """SinkhornKernel.jl:341-444: log(marg_i) - LSE_j(-C_ij/(reg W) + pot_j).
    With `out` given the result overwrites it in place, and its previous
    content (the last phi of an iteration) serves as the kernel's reference.
    flags = FLAG_FORM_FP32 runs the FP32-exponent pass (p = 2, d <= 3)."""
    n, d = x.shape
    m = y.shape[0]
    out = _empty(n, x) if out is None else out
    h = _h(x)
    if flags:
        h.check(h._lib.culamp_lse_rows_sk_form(h.ptr, C.c_void_p(out.data_ptr()), _dev(x, "x"),
                                               _dev(y, "y"), n, m, d, _dev(marginal, "marginal", n),
                                               _dev(pot, "pot", m), float(reg), float(winf), float(p),
                                               int(flags), _stream()), "culamp_lse_rows_sk_form")
        return out
    h.check(h._lib.culamp_lse_rows_sk(h.ptr, C.c_void_p(out.data_ptr()), _dev(x, "x"),
                                      _dev(y, "y"), n, m, d, _dev(marginal, "marginal", n),
                                      _dev(pot, "pot", m), float(reg), float(winf), float(p),
                                      _stream()), "culamp_lse_rows_sk")
    return out


def residual_opt(x, y, marginal, phi, psi, reg, winf, p):
    """SinkhornKernel.jl:9-81: (marg_i - sum_j P_ij, sum_j P_ij C_ij)."""
    n, d = x.shape
    m = y.shape[0]
    res, cost = _empty(n, x), _empty(n, x)
    h = _h(x)
    h.check(h._lib.culamp_residual_sk(h.ptr, C.c_void_p(res.data_ptr()),
                                      C.c_void_p(cost.data_ptr()), _dev(x, "x"), _dev(y, "y"), n,
                                      m, d, _dev(marginal, "marginal", n), _dev(phi, "phi", n),
                                      _dev(psi, "psi", m), float(reg), float(winf), float(p),
                                      _stream()), "culamp_residual_sk")
    return res, cost


def warp_logsumexp_spp_ct_fused(x, y, theta, reg, st, winf, p, out=None):
    """MirrorProxKernel.jl:833-938: LSE_j(-(C_ij st/(2W) + theta_j)/reg); `out`
    as for warp_logsumexp_ct_fused."""
    n, d = x.shape
    m = y.shape[0]
    out = _empty(n, x) if out is None else out
    h = _h(x)
    h.check(h._lib.culamp_lse_rows_spp(h.ptr, C.c_void_p(out.data_ptr()), _dev(x, "x"),
                                       _dev(y, "y"), n, m, d, _dev(theta, "theta", m), float(reg),
                                       float(st), float(winf), float(p), _stream()),
            "culamp_lse_rows_spp")
    return out


def residual_spp_c(x, y, marginal1, theta, logz, reg, st, winf, p):
    """MirrorProxKernel.jl:7-94: per column j, (sum_i P_ij, sum_i P_ij C_ij)."""
    n, d = x.shape
    m = y.shape[0]
    res, cost = _empty(m, x), _empty(m, x)
    h = _h(x)
    h.check(h._lib.culamp_col_residual_spp(h.ptr, C.c_void_p(res.data_ptr()),
                                           C.c_void_p(cost.data_ptr()), _dev(x, "x"), _dev(y, "y"),
                                           n, m, d, _dev(marginal1, "marginal1", n),
                                           _dev(theta, "theta", m), _dev(logz, "logz", n),
                                           float(reg), float(st), float(winf), float(p), _stream()),
            "culamp_col_residual_spp")
    return res, cost


def warp_min_reduce(x, y, theta, winf, p):
    """MirrorProxKernel.jl:941-1016: min_j (C_ij + 2 W theta_j)."""
    n, d = x.shape
    m = y.shape[0]
    out = _empty(n, x)
    h = _h(x)
    h.check(h._lib.culamp_min_reduce(h.ptr, C.c_void_p(out.data_ptr()), _dev(x, "x"), _dev(y, "y"),
                                     n, m, d, _dev(theta, "theta", m), float(winf), float(p),
                                     _stream()), "culamp_min_reduce")
    return out


def update_theta_residual(theta0, residual, c, eta_mu_i, eta_mu, adjust, minv, maxv, winf=1.0,
                          out=None):
    """MirrorProx.jl:159-180 (elementwise); `out` may alias theta0."""
    m = theta0.shape[0]
    out = _empty(m, theta0) if out is None else out
    h = _h(theta0)
    h.check(h._lib.culamp_theta_update(h.ptr, C.c_void_p(out.data_ptr()), _dev(theta0, "theta0"),
                                       _dev(residual, "residual"), _dev(c, "c"),
                                       _dev(eta_mu_i, "eta_mu_i"), float(eta_mu), int(bool(adjust)),
                                       float(minv), float(maxv), float(winf), m, _stream()),
            "culamp_theta_update")
    return out
