"""Dense-cost GPU solvers: the run_dot path without --kernel.

run_dot (CmdLineUtils.jl:189-204) builds or reads (--weights CSV) a cost matrix
W, divides it by max |W| and calls the dense solvers on the GPU:
sinkhorn_log (Sinkhorn.jl:8-84) and the GPU LAMP (MirrorProx.jl:397-503). Here
both run in libculamp_b200 (culamp_sinkhorn_dense / culamp_lamp_dense): W
stays in HBM and every pass streams it (or its transpose) once.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .args import EOTArgs
from .solvers import SolveResult, _log_rows, _stream, get_handle

_LOG_CAP = 100_000


def _as_dev(a, device=None):
    import torch
    if isinstance(a, torch.Tensor):
        return a.contiguous().to(torch.float64)
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64),
                           device=device or torch.device("cuda", 0))


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def solve_sinkhorn_dense(W, r, c, args: EOTArgs, frequency: int = 50, phi0=None, psi0=None,
                         want_plan: bool = False, log_cap: int = _LOG_CAP) -> SolveResult:
    """sinkhorn_log on the GPU; W (n x m) is used as given (K = -W / eta_p)."""
    import torch
    W = _as_dev(W)
    dev = W.device
    r, c = _as_dev(r, dev), _as_dev(c, dev)
    n, m = W.shape
    phi = torch.empty(n, dtype=torch.float64, device=dev)
    psi = torch.empty(m, dtype=torch.float64, device=dev)
    plan = torch.empty((n, m), dtype=torch.float64, device=dev) if want_plan else None
    p0 = _as_dev(phi0, dev) if phi0 is not None else None
    q0 = _as_dev(psi0, dev) if psi0 is not None else None
    a = args.to_c()
    stats = _lib.CStats()
    buf = (_lib.CLogRow * max(1, log_cap))()
    h = get_handle(dev.index)
    st = h._lib.culamp_sinkhorn_dense(h.ptr, _ptr(W), n, m, _ptr(r), _ptr(c), C.byref(a), int(frequency),
                                      _ptr(p0), _ptr(q0), _ptr(phi), _ptr(psi), _ptr(plan),
                                      C.byref(stats), buf, log_cap, _stream())
    h.check(st, "culamp_sinkhorn_dense")
    res = SolveResult(phi, psi, stats.residual, stats.objective, int(stats.iterations),
                      int(stats.num_iter), stats.winf, stats.elapsed_ms, int(stats.stopped),
                      log=_log_rows(buf, stats))
    res.plan = plan
    return res


def solve_lamp_dense(W, r, c, args: EOTArgs, frequency: int = 50, theta0=None,
                     want_plan: bool = True, log_cap: int = _LOG_CAP) -> SolveResult:
    """The GPU LAMP (MirrorProx.jl:397-503) on a dense cost W (n x m)."""
    import torch
    W = _as_dev(W)
    dev = W.device
    r, c = _as_dev(r, dev), _as_dev(c, dev)
    n, m = W.shape
    theta = torch.empty(m, dtype=torch.float64, device=dev)
    nu = torch.empty(m, dtype=torch.float64, device=dev)
    plan = torch.empty((n, m), dtype=torch.float64, device=dev) if want_plan else None
    t0 = _as_dev(theta0, dev) if theta0 is not None else None
    a = args.to_c()
    stats = _lib.CStats()
    buf = (_lib.CLogRow * max(1, log_cap))()
    h = get_handle(dev.index)
    st = h._lib.culamp_lamp_dense(h.ptr, _ptr(W), n, m, _ptr(r), _ptr(c), C.byref(a), int(frequency),
                                  _ptr(t0), _ptr(theta), _ptr(nu), _ptr(plan), C.byref(stats), buf,
                                  log_cap, _stream())
    h.check(st, "culamp_lamp_dense")
    res = SolveResult(None, None, stats.residual, stats.objective, int(stats.iterations),
                      int(stats.num_iter), stats.winf, stats.elapsed_ms, int(stats.stopped),
                      eta_t=stats.eta_t, s_t=stats.s_t, nu=nu, theta=theta, log=_log_rows(buf, stats))
    res.plan = plan
    return res


def sinkhorn_log(r, c, W, args: EOTArgs, frequency: int = 50, *, return_state: bool = False,
                 phi0=None, psi0=None):
    """Sinkhorn.jl:8-84 (reference name and argument order). Returns (p, phi, psi),
    or (p, phi, psi, obj, feas, num_iter) with return_state."""
    res = solve_sinkhorn_dense(W, r, c, args, frequency, phi0, psi0, want_plan=True)
    if return_state:
        return res.plan, res.phi, res.psi, res.objective, res.residual, res.num_iter
    return res.plan, res.phi, res.psi


def LAMP(r, c, W, args: EOTArgs, frequency: int = 50, *, theta0=None):  # noqa: N802 (reference name)
    """MirrorProx.jl:397-503 (reference name and argument order). Returns (r .* p, theta)."""
    res = solve_lamp_dense(W, r, c, args, frequency, theta0, want_plan=True)
    return res.plan, res.theta
