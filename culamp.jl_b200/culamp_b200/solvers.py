"""Reference-named solver API over the C ABI.

Function names, argument order and return shapes follow CuLAMP.jl's kernelized
solvers so call sites read the same:

* sinkhorn_color_transfer   (SinkhornKernel.jl:477-559)
* sinkhorn_euclidean        (SinkhornKernel.jl:579-608)
* extragradient_color_transfer (MirrorProxKernel.jl:1019-1132)
* extragradient_euclidean   (MirrorProxKernel.jl:1143-1185)
* annealed_sinkhorn_euclidean (AnnealedSinkhorn.jl:65-177)

Point clouds are (N, d) float64 arrays, point-major -- the memory layout of the
reference's 3 x N column-major CuArray. CUDA tensors (torch) run the
device-pointer entry points on the current torch stream; numpy arrays run the
host-buffer entry points (copy in, solve, copy out). Errors raise CulampError.
"""
from __future__ import annotations

import ctypes as C
import math
import threading
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .args import EOTArgs
from . import io as _io

_LOG_CAP = 100_000


class Handle:
    """Owns a culamp_handle (workspace + cached CUDA graphs) on one device."""

    def __init__(self, device: int = 0):
        self._lib = _lib.load()
        h = C.c_void_p()
        st = self._lib.culamp_create(C.byref(h), int(device))
        if st:
            raise _lib.CulampError(st, f"culamp_create(device={device}): {_lib.status_string(st)}")
        self.ptr = h
        self.device = device

    def check(self, st: int, what: str):
        if st:
            msg = self._lib.culamp_last_error(self.ptr)
            raise _lib.CulampError(st, f"{what}: {msg.decode() if msg else _lib.status_string(st)}")

    def close(self):
        if self.ptr:
            self._lib.culamp_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_handles: dict = {}
_hlock = threading.Lock()


def get_handle(device: int | None = None) -> Handle:
    """Per-(thread, device) cached handle."""
    if device is None:
        import torch
        device = torch.cuda.current_device()
    key = (threading.get_ident(), int(device))
    with _hlock:
        h = _handles.get(key)
        if h is None:
            h = Handle(int(device))
            _handles[key] = h
        return h


@dataclass
class SolveResult:
    phi: object
    psi: object
    residual: float
    objective: float
    iterations: int
    num_iter: int
    winf: float
    elapsed_ms: float
    stopped: int
    eta_t: float = math.nan
    s_t: float = math.nan
    nu: object = None
    theta: object = None
    log: list = field(default_factory=list)
    plan: object = None     # dense solvers: the transport plan (n x m), when requested


# ------------------------------------------------------------------ helpers

def _is_torch(a) -> bool:
    try:
        import torch
        return isinstance(a, torch.Tensor)
    except ImportError:
        return False


def _dev(t, name, shape0=None, ndim=None):
    import torch
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError(f"{name} must be a CUDA tensor")
    if t.dtype != torch.float64:
        raise TypeError(f"{name} must be float64 (got {t.dtype})")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    if ndim is not None and t.dim() != ndim:
        raise ValueError(f"{name} must have {ndim} dims")
    if shape0 is not None and t.shape[0] != shape0:
        raise ValueError(f"{name} has {t.shape[0]} entries, expected {shape0}")
    return C.c_void_p(t.data_ptr())


def _host(a, name, shape0=None, ndim=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if ndim is not None and a.ndim != ndim:
        raise ValueError(f"{name} must have {ndim} dims")
    if shape0 is not None and a.shape[0] != shape0:
        raise ValueError(f"{name} has {a.shape[0]} entries, expected {shape0}")
    return a


def _stream():
    import torch
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _log_rows(buf, stats):
    out = []
    for k in range(min(int(stats.log_rows), len(buf))):
        r = buf[k]
        out.append((r.time_s, int(r.iter), r.infeas, r.ot_objective, r.primal, r.dual))
    return out


def _points(img):
    if img.ndim != 2:
        raise ValueError("point clouds must be (N, d)")
    return img.shape[0], img.shape[1]


# ------------------------------------------------------------------ Sinkhorn

def solve_sinkhorn(x, y, r, c, args: EOTArgs, frequency: int = 100, p: float = 2.0,
                   phi0=None, psi0=None, flags: int = 0, handle: Handle | None = None,
                   log_cap: int = _LOG_CAP) -> SolveResult:
    """Kernelized log-domain Sinkhorn; returns every output and statistic."""
    n, d = _points(x)
    m, d2 = _points(y)
    if d != d2:
        raise ValueError("x and y must have the same dimension")
    a = args.to_c()
    stats = _lib.CStats()
    buf = (_lib.CLogRow * max(1, log_cap))()
    if _is_torch(x):
        import torch
        h = handle or get_handle(x.device.index)
        phi = torch.empty(n, dtype=torch.float64, device=x.device)
        psi = torch.empty(m, dtype=torch.float64, device=x.device)
        st = h._lib.culamp_sinkhorn(
            h.ptr, _dev(x, "x", n, 2), _dev(y, "y", m, 2), n, m, d, _dev(r, "r", n, 1),
            _dev(c, "c", m, 1), C.byref(a), int(frequency), float(p),
            _dev(phi0, "phi0", n, 1) if phi0 is not None else None,
            _dev(psi0, "psi0", m, 1) if psi0 is not None else None, int(flags),
            C.c_void_p(phi.data_ptr()), C.c_void_p(psi.data_ptr()), C.byref(stats), buf, log_cap,
            _stream())
    else:
        h = handle or get_handle(0)
        xh, yh = _host(x, "x", n, 2), _host(y, "y", m, 2)
        rh, ch = _host(r, "r", n, 1), _host(c, "c", m, 1)
        p0 = _host(phi0, "phi0", n, 1) if phi0 is not None else None
        q0 = _host(psi0, "psi0", m, 1) if psi0 is not None else None
        phi, psi = np.empty(n), np.empty(m)
        st = h._lib.culamp_sinkhorn_host(
            h.ptr, xh.ctypes.data, yh.ctypes.data, n, m, d, rh.ctypes.data, ch.ctypes.data,
            C.byref(a), int(frequency), float(p), p0.ctypes.data if p0 is not None else None,
            q0.ctypes.data if q0 is not None else None, int(flags), phi.ctypes.data,
            psi.ctypes.data, C.byref(stats), buf, log_cap)
    h.check(st, "culamp_sinkhorn")
    return SolveResult(phi, psi, stats.residual, stats.objective, int(stats.iterations),
                       int(stats.num_iter), stats.winf, stats.elapsed_ms, int(stats.stopped),
                       log=_log_rows(buf, stats))


def solve_symmetric_sinkhorn(x, r, args: EOTArgs, frequency: int = 100, p: float = 2.0, f0=None,
                             flags: int = 0, handle: Handle | None = None,
                             log_cap: int = _LOG_CAP) -> SolveResult:
    """Self-transport OT(r, r; x, x) by the averaged symmetric iteration
    f <- (f + T(f))/2 (culamp_symmetric_sinkhorn); phi and psi of the result
    are the same tensor f. Device tensors only."""
    import torch
    n, d = _points(x)
    if not _is_torch(x):
        raise TypeError("solve_symmetric_sinkhorn takes device tensors")
    a = args.to_c()
    stats = _lib.CStats()
    buf = (_lib.CLogRow * max(1, log_cap))()
    h = handle or get_handle(x.device.index)
    f = torch.empty(n, dtype=torch.float64, device=x.device)
    st = h._lib.culamp_symmetric_sinkhorn(
        h.ptr, _dev(x, "x", n, 2), n, d, _dev(r, "r", n, 1), C.byref(a), int(frequency), float(p),
        _dev(f0, "f0", n, 1) if f0 is not None else None, int(flags), C.c_void_p(f.data_ptr()),
        C.byref(stats), buf, log_cap, _stream())
    h.check(st, "culamp_symmetric_sinkhorn")
    return SolveResult(f, f, stats.residual, stats.objective, int(stats.iterations),
                       int(stats.num_iter), stats.winf, stats.elapsed_ms, int(stats.stopped),
                       log=_log_rows(buf, stats))


def sinkhorn_color_transfer(img1, img2, marginal1, marginal2, args: EOTArgs, frequency: int = 100,
                            p: float = 2, *, return_cuda: bool = False,
                            return_assignments: bool = True, phi0=None, psi0=None,
                            flags: int = 0):
    """SinkhornKernel.jl:477-559. Returns (phi, psi, objective, residual[, num_iter])
    when return_assignments is False, else (phi, psi, img1', img2') with the
    barycentric images."""
    res = solve_sinkhorn(img1, img2, marginal1, marginal2, args, frequency, p, phi0, psi0, flags)
    if args.verbose:
        _io.print_log(res.log, "sinkhorn_kernel", header="time(s),iter,infeas,ot_objective,dual")
    if not return_assignments:
        if return_cuda:
            return res.phi, res.psi, res.objective, res.residual, res.num_iter
        return _np(res.phi), _np(res.psi), res.objective, res.residual
    b1 = barycentric_map(img1, img2, res.phi, res.psi, args.eta_p, res.winf, p, flags)
    b2 = barycentric_map(img2, img1, res.psi, res.phi, args.eta_p, res.winf, p, flags)
    return _np(res.phi), _np(res.psi), _np(b1), _np(b2)


def sinkhorn_euclidean(marginal1, marginal2, location1, location2, out1: str, out2: str,
                       potentials: str, args: EOTArgs, frequency: int, p: float):
    """SinkhornKernel.jl:579-608: solve, then write `<potentials>.row/.col`."""
    phi, psi, a1, a2 = sinkhorn_color_transfer(location1, location2, marginal1, marginal2, args,
                                               frequency, p)
    if potentials:
        _io.write_potentials(potentials, row=phi, col=psi)
    if out1:
        _io.write_assignments(out1, a1)
    if out2:
        _io.write_assignments(out2, a2)
    return phi, psi


# ---------------------------------------------------------------------- LAMP

def solve_lamp(x, y, r, c, args: EOTArgs, frequency: int = 100, p: float = 2.0, flags: int = 0,
               handle: Handle | None = None, log_cap: int = _LOG_CAP) -> SolveResult:
    n, d = _points(x)
    m, _ = _points(y)
    a = args.to_c()
    stats = _lib.CStats()
    buf = (_lib.CLogRow * max(1, log_cap))()
    if _is_torch(x):
        import torch
        h = handle or get_handle(x.device.index)
        mk = lambda k: torch.empty(k, dtype=torch.float64, device=x.device)  # noqa: E731
        nu, phi, psi, th = mk(m), mk(n), mk(m), mk(m)
        st = h._lib.culamp_lamp(
            h.ptr, _dev(x, "x", n, 2), _dev(y, "y", m, 2), n, m, d, _dev(r, "r", n, 1),
            _dev(c, "c", m, 1), C.byref(a), int(frequency), float(p), int(flags),
            C.c_void_p(nu.data_ptr()), C.c_void_p(phi.data_ptr()), C.c_void_p(psi.data_ptr()),
            C.c_void_p(th.data_ptr()), C.byref(stats), buf, log_cap, _stream())
    else:
        h = handle or get_handle(0)
        xh, yh = _host(x, "x", n, 2), _host(y, "y", m, 2)
        rh, ch = _host(r, "r", n, 1), _host(c, "c", m, 1)
        nu, phi, psi, th = np.empty(m), np.empty(n), np.empty(m), np.empty(m)
        st = h._lib.culamp_lamp_host(
            h.ptr, xh.ctypes.data, yh.ctypes.data, n, m, d, rh.ctypes.data, ch.ctypes.data,
            C.byref(a), int(frequency), float(p), int(flags), nu.ctypes.data, phi.ctypes.data,
            psi.ctypes.data, th.ctypes.data, C.byref(stats), buf, log_cap)
    h.check(st, "culamp_lamp")
    return SolveResult(phi, psi, stats.residual, stats.objective, int(stats.iterations),
                       int(stats.num_iter), stats.winf, stats.elapsed_ms, int(stats.stopped),
                       eta_t=stats.eta_t, s_t=stats.s_t, nu=nu, theta=th,
                       log=_log_rows(buf, stats))


def extragradient_color_transfer(img1, img2, marginal1, marginal2, args: EOTArgs,
                                 frequency: int = 100, p: float = 2.0, flags: int = 0):
    """MirrorProxKernel.jl:1019-1132. Returns (nu, phi, psi, img1', img2')."""
    res = solve_lamp(img1, img2, marginal1, marginal2, args, frequency, p, flags)
    if args.verbose:
        _io.print_log(res.log, "lamp_kernel",
                      header="time(s),iter,infeas,ot_objective,primal,dual,solver")
    b1, b2 = lamp_barycentric_maps(img1, img2, marginal1, res, p)
    return _np(res.nu), _np(res.phi), _np(res.psi), _np(b1), _np(b2)


def extragradient_euclidean(marginal1, marginal2, location1, location2, out1: str, out2: str,
                            outmu: str, args: EOTArgs, frequency: int, p: float):
    """MirrorProxKernel.jl:1143-1185: solve, then write `<outmu>.spp_col/.row/.col`."""
    mu, phi, psi, a1, a2 = extragradient_color_transfer(location1, location2, marginal1,
                                                        marginal2, args, frequency, p)
    if outmu:
        _io.write_potentials(outmu, spp_col=mu, row=phi, col=psi)
    if out1:
        _io.write_assignments(out1, a1)
    if out2:
        _io.write_assignments(out2, a2)
    return mu, phi, psi


# ------------------------------------------------------------ annealed Sinkhorn

def solve_annealed_sinkhorn(x, y, r, c, args: EOTArgs, frequency: int = 10, p: float = 2.0,
                            flags: int = 0, handle: Handle | None = None,
                            log_cap: int = 10_000) -> SolveResult:
    import torch
    n, d = _points(x)
    m, _ = _points(y)
    on_host = not _is_torch(x)
    if on_host:
        dev = torch.device("cuda", 0)
        x, y, r, c = (torch.as_tensor(np.ascontiguousarray(v, dtype=np.float64), device=dev)
                      for v in (x, y, r, c))
    h = handle or get_handle(x.device.index)
    a = args.to_c()
    stats = _lib.CStats()
    buf = (_lib.CLogRow * max(1, log_cap))()
    phi = torch.empty(n, dtype=torch.float64, device=x.device)
    psi = torch.empty(m, dtype=torch.float64, device=x.device)
    st = h._lib.culamp_annealed_sinkhorn(
        h.ptr, _dev(x, "x", n, 2), _dev(y, "y", m, 2), n, m, d, _dev(r, "r", n, 1),
        _dev(c, "c", m, 1), C.byref(a), int(frequency), float(p), int(flags),
        C.c_void_p(phi.data_ptr()), C.c_void_p(psi.data_ptr()), C.byref(stats), buf, log_cap,
        _stream())
    h.check(st, "culamp_annealed_sinkhorn")
    if on_host:
        phi, psi = phi.cpu().numpy(), psi.cpu().numpy()
    return SolveResult(phi, psi, stats.residual, stats.objective, int(stats.iterations),
                       int(stats.num_iter), stats.winf, stats.elapsed_ms, int(stats.stopped),
                       eta_t=stats.eta_t, log=_log_rows(buf, stats))


def annealed_sinkhorn_euclidean(marginal1, marginal2, location1, location2, out1: str, out2: str,
                                potentials: str, args: EOTArgs, frequency: int, p: float,
                                flags: int = 0):
    """AnnealedSinkhorn.jl:65-177. Returns (phi, psi, objective)."""
    res = solve_annealed_sinkhorn(location1, location2, marginal1, marginal2, args, frequency, p,
                                  flags)
    if args.verbose:
        _io.print_log(res.log, "annealed_sinkhorn_kernel",
                      header="time(s),iter,infeas,ot_objective,eta,solver", eta_col=True)
    phi, psi = _np(res.phi), _np(res.psi)
    if potentials:
        _io.write_potentials(potentials, row=phi, col=psi)
    if out1 or out2:
        eta_final = args.epsilon
        b1 = barycentric_map(location1, location2, res.phi, res.psi, eta_final, res.winf, p, flags)
        b2 = barycentric_map(location2, location1, res.psi, res.phi, eta_final, res.winf, p, flags)
        if out1:
            _io.write_assignments(out1, _np(b1))
        if out2:
            _io.write_assignments(out2, _np(b2))
    return phi, psi, res.objective


# ------------------------------------------------------------ barycentric maps

def _to_dev(a, like=None):
    import torch
    if _is_torch(a):
        return a
    dev = like.device if like is not None and _is_torch(like) else torch.device("cuda", 0)
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=dev)


def barycentric_map(x, y, phi, psi, reg, winf, p, flags=0):
    """naive_findmaxindex_ct! (SinkhornKernel.jl:124-162) on the GPU. The
    reference evaluates this map with p==1 ? L1 : squared (quirk) unless
    FLAG_TRUE_PINF is set."""
    import torch
    x, y, phi, psi = (_to_dev(v, x) for v in (x, y, phi, psi))
    n, d = x.shape
    m = y.shape[0]
    cp = p if (flags & _lib.FLAG_TRUE_PINF) else (1.0 if p == 1 else 2.0)
    out = torch.empty_like(x)
    h = get_handle(x.device.index)
    st = h._lib.culamp_barycentric_sk(h.ptr, C.c_void_p(out.data_ptr()), _dev(x, "x"), _dev(y, "y"),
                                      n, m, d, _dev(phi, "phi"), _dev(psi, "psi"), float(reg),
                                      float(winf), float(cp), _stream())
    h.check(st, "culamp_barycentric_sk")
    return out


def lamp_barycentric_maps(x, y, r, res: SolveResult, p):
    """naive_findmaxindex_spp_ct! and _t! (MirrorProxKernel.jl:97-189): row-wise and
    column-wise barycentres of P_ij = r_i exp(-(C_ij s/(2W) + nu_j)/eta_t - logZ_i).
    Written as a Sinkhorn-form plan: phi_i = log r_i - logZ_i (res.phi),
    psi_j = -nu_j / eta_t and cost scale s/(2 W eta_t)."""
    import torch
    x, y = _to_dev(x), _to_dev(y)
    phi = _to_dev(res.phi, x)
    nu = _to_dev(res.nu, x)
    et, s = res.eta_t, res.s_t
    if math.isinf(et):
        psi = torch.zeros_like(nu)
        reg, winf = math.inf, 1.0
    else:
        psi = -nu / et
        reg, winf = 1.0, 2.0 * res.winf * et / s   # -C/(reg*winf) = -C s/(2 W eta_t)
    b1 = barycentric_map(x, y, phi, psi, reg, winf, p, _lib.FLAG_TRUE_PINF)
    b2 = barycentric_map(y, x, psi, phi, reg, winf, p, _lib.FLAG_TRUE_PINF)
    return b1, b2


def marginal_error_fp64(x, y, r, c, phi, psi, reg, winf, p):
    """FP64 (exp included) L1 row / column marginal errors of a Sinkhorn-form plan."""
    x, y, r, c, phi, psi = (_to_dev(v) for v in (x, y, r, c, phi, psi))
    n, d = x.shape
    m = y.shape[0]
    h = get_handle(x.device.index)
    rl, cl = C.c_double(), C.c_double()
    st = h._lib.culamp_marginal_error_fp64(h.ptr, _dev(x, "x"), _dev(y, "y"), n, m, d,
                                           _dev(r, "r"), _dev(c, "c"), _dev(phi, "phi"),
                                           _dev(psi, "psi"), float(reg), float(winf), float(p),
                                           C.byref(rl), C.byref(cl), _stream())
    h.check(st, "culamp_marginal_error_fp64")
    return rl.value, cl.value


def _np(a):
    if _is_torch(a):
        return a.detach().cpu().numpy()
    return a


# ------------------------------------------------------------------ batched solves

@dataclass
class BatchResult:
    results: list            # one SolveResult per instance (phi, psi on the device)
    elapsed_ms: float        # device time of the solve loop
    tune_ms: float           # device time spent timing shape candidates (0 when cached)
    target_ctas_per_sm: int
    feat_tiles_per_unit: int
    unroll: int
    launches_per_iteration: int
    phases: int


def solve_batched_sinkhorn(instances, args: EOTArgs, frequency: int = 100, p: float = 2.0,
                           flags: int = 0, handle: Handle | None = None) -> BatchResult:
    """Many independent kernel Sinkhorn problems of uneven n, m, d in one solve
    (culamp_batched_sinkhorn). `instances`: sequence of (x, y, r, c) float64
    CUDA tensors on one device. Each result equals what solve_sinkhorn gives for
    that instance alone (same iterations and stopping rule)."""
    import torch
    inst = list(instances)
    if not inst:
        raise ValueError("empty batch")
    dev = inst[0][0].device
    h = handle or get_handle(dev.index)
    arr = (_lib.CInstance * len(inst))()
    outs = []
    for k, (x, y, r, c) in enumerate(inst):
        n, d = _points(x)
        m, d2 = _points(y)
        if d != d2:
            raise ValueError(f"instance {k}: x and y dimensions differ")
        phi = torch.empty(n, dtype=torch.float64, device=dev)
        psi = torch.empty(m, dtype=torch.float64, device=dev)
        e = arr[k]
        e.x, e.y = _dev(x, "x", n, 2), _dev(y, "y", m, 2)
        e.r, e.c = _dev(r, "r", n, 1), _dev(c, "c", m, 1)
        e.phi, e.psi = phi.data_ptr(), psi.data_ptr()
        e.n, e.m, e.d = n, m, d
        outs.append((phi, psi))
    stats = (_lib.CBatchStats * len(inst))()
    info = _lib.CBatchInfo()
    a = args.to_c()
    st = h._lib.culamp_batched_sinkhorn(h.ptr, arr, len(inst), C.byref(a), int(frequency), float(p),
                                        int(flags), stats, C.byref(info), _stream())
    h.check(st, "culamp_batched_sinkhorn")
    res = [SolveResult(phi, psi, s.residual, s.objective, int(s.iterations), int(s.num_iter), s.winf,
                       math.nan, int(s.stopped)) for (phi, psi), s in zip(outs, stats)]
    return BatchResult(res, info.elapsed_ms, info.tune_ms, info.target_ctas_per_sm,
                       info.feat_tiles_per_unit, info.unroll, info.launches_per_iteration,
                       info.phases)
