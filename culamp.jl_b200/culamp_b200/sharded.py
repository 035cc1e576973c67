"""Row-sharded kernel Sinkhorn over torch.distributed ranks.

The reference runs sinkhorn_color_transfer (SinkhornKernel.jl:477-559) on one
GPU. Here the rows of x (and the matching row marginal r and potential phi)
are split into shards; every shard also holds the full y, c and psi (small).
One iteration, identical in arithmetic to the single-GPU solver:

  * row half-step phi = log r - LSE_j(-C/(eta W) + psi): local to each shard
    (culamp_lse_rows_sk over the shard's rows);
  * column half-step psi = log c - LSE_i(-C/(eta W) + phi): each shard reduces
    over its own rows (culamp_lse_rows_sk with the roles swapped, giving
    out_g = log c - LSE over shard g), the shards' outputs are gathered
    (one all_gather of m doubles per rank) and combined by culamp_lse_combine,
    psi = -log sum_g exp(-out_g) -- the log-sum-exp over all rows;
  * W_inf = max over shards (all_reduce MAX) once; on check iterations
    ((it - 1) % frequency == 0, SinkhornKernel.jl:527-537) the residual L1 and
    transport cost are summed over shards (all_reduce SUM) and every rank takes
    the same stopping decision.

Row-sharded LAMP (sharded_lamp, MirrorProxKernel.jl:1019-1132) splits the
rows the same way; its column quantities are sums over all rows, so each
shard computes partial column masses (and costs on check iterations) over its
rows (culamp_col_residual_spp) and one all_reduce(SUM) of the m-vector per
infeas(.) call gives the full residual; theta, nu, theta_bar, nu_bar and the
eta_t / s recursions are replicated and bit-identical on every rank (they
only see all-reduced values). The row-weighted scalars of the primal / dual
values (r.logZ, r.LSE(theta) or r.min) are shard sums, all-reduced on check
iterations.

A process may own several shards (its row blocks are reduced locally first),
so the same driver runs one rank per GPU over NCCL, several row blocks on one
GPU, or -- with compute ops that run on the host -- gloo ranks on CPU. Every
rank issues the same collectives in the same order. With the CUDA ops the
Sinkhorn driver captures the `frequency` iterations between two checks (the
passes, the combines and the all_gather on the NCCL stream) in one CUDA graph
and replays it, so the host takes part once per check. tmax is tested on check
iterations (the reference tests it every iteration; a per-iteration test would
need a collective per iteration to keep the ranks in step).
"""
from __future__ import annotations

import ctypes as C
import math
import time
from dataclasses import dataclass

import torch
import torch.distributed as dist

from . import kernels as K
from .args import EOTArgs
from .solvers import _dev, _stream, get_handle


@dataclass
class ShardedResult:
    phi: list            # this rank's row potentials, one tensor per shard
    psi: torch.Tensor    # column potentials (replicated)
    residual: float
    objective: float
    iterations: int
    num_iter: int
    winf: float
    stopped: int         # 1 tolerance, 2 itermax, 3 tmax
    elapsed_s: float


class CudaOps:
    """Compute of one shard on its GPU through the C ABI."""

    def max_cost(self, x, y, p):
        _, winf = K.max_logsumexp_spp_ct(x, y, p)
        return winf

    def lse_rows(self, out, x, y, marg, pot, reg, winf, p):
        K.warp_logsumexp_ct_fused(x, y, marg, pot, reg, winf, p, out=out)

    def residual(self, x, y, marg, phi, psi, reg, winf, p):
        res, cost = K.residual_opt(x, y, marg, phi, psi, reg, winf, p)
        return res.abs().sum(), cost.sum()

    def spp_lse(self, out, x, y, theta, reg, st, winf, p):
        K.warp_logsumexp_spp_ct_fused(x, y, theta, reg, st, winf, p, out=out)

    def col_residual(self, x, y, r, theta, logz, reg, st, winf, p):
        return K.residual_spp_c(x, y, r, theta, logz, reg, st, winf, p)

    def min_reduce(self, x, y, theta, winf, p):
        return K.warp_min_reduce(x, y, theta, winf, p)

    def theta_update(self, theta0, res, c, emu, eta_mu, adjust, minv, maxv):
        return K.update_theta_residual(theta0, res, c, emu, eta_mu, adjust, minv, maxv, 1.0)

    def combine(self, parts):
        g, m = parts.shape
        psi = torch.empty(m, dtype=torch.float64, device=parts.device)
        h = get_handle(parts.device.index)
        h.check(h._lib.culamp_lse_combine(h.ptr, C.c_void_p(psi.data_ptr()), _dev(parts, "parts"), g, m,
                                          _stream()), "culamp_lse_combine")
        return psi


def shard_rows(n: int, shards: int, index: int) -> tuple[int, int]:
    """Even split of n rows into `shards` blocks: rows [start, end) of block `index`."""
    base, extra = divmod(n, shards)
    start = index * base + min(index, extra)
    return start, start + base + (1 if index < extra else 0)


def _reduce(t, op, group):
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(t, op=op, group=group)
    return t


def sharded_sinkhorn(x_shards, r_shards, y, c, args: EOTArgs, frequency: int = 100, p: float = 2.0,
                     group=None, ops=None, phi0=None, psi0=None, graph: bool | None = None) -> ShardedResult:
    """Kernel Sinkhorn with the rows split over shards and ranks (see module doc).
    x_shards / r_shards: this rank's row blocks (same device); y, c: full.
    Without an initialised process group the shards are those of one process.

    graph (default: on for the CUDA ops): the `frequency` iterations between
    two checks -- passes, the combine and the all_gather -- are captured once
    in a CUDA graph and replayed, so the host meets the device once per check
    instead of once per pass; the first iteration runs eagerly (it warms the
    kernels, the scratch and the communicator before the capture)."""
    ops = ops or CudaOps()
    if frequency < 1:
        raise ValueError("frequency must be >= 1")
    if not args.eta_p > 0:
        raise ValueError("Sinkhorn needs eta_p > 0")
    if len(x_shards) != len(r_shards) or not x_shards:
        raise ValueError("one row marginal per x shard")
    dev = y.device
    ip = 2.0 if math.isinf(p) else p                 # SinkhornKernel.jl:518-520
    rp = 1.0 if p == 1 else 2.0                      # SinkhornKernel.jl:38-42
    world = dist.get_world_size(group) if (dist.is_available() and dist.is_initialized()) else 1
    m = y.shape[0]
    eta = args.eta_p
    winf_t = torch.tensor([max(ops.max_cost(x, y, p) for x in x_shards)], dtype=torch.float64, device=dev)
    winf = float(_reduce(winf_t, dist.ReduceOp.MAX, group).item())
    phis = [torch.zeros(x.shape[0], dtype=torch.float64, device=dev) if phi0 is None else phi0[k].clone()
            for k, x in enumerate(x_shards)]
    psi = torch.zeros(m, dtype=torch.float64, device=dev) if psi0 is None else psi0.clone()
    outs = [torch.zeros(m, dtype=torch.float64, device=dev) for _ in x_shards]
    gathered = [torch.empty(m, dtype=torch.float64, device=dev) for _ in range(world)]
    t0 = time.perf_counter()
    num_iter, it, stopped = 0, 0, 2

    def resid():
        s = torch.zeros(2, dtype=torch.float64, device=dev)
        for x, r, ph in zip(x_shards, r_shards, phis):
            l1, cost = ops.residual(x, y, r, ph, psi, eta, winf, rp)
            s[0] += l1
            s[1] += cost
        return _reduce(s, dist.ReduceOp.SUM, group)

    def iterate():
        # one iteration; phi and psi are updated in place (a captured graph
        # replays on the same buffers)
        for x, r, ph in zip(x_shards, r_shards, phis):
            ops.lse_rows(ph, x, y, r, psi, eta, winf, ip)
        for x, ph, out in zip(x_shards, phis, outs):
            ops.lse_rows(out, y, x, c, ph, eta, winf, ip)
        local = ops.combine(torch.stack(outs)) if len(outs) > 1 else outs[0]
        if world > 1:
            dist.all_gather(gathered, local.contiguous(), group=group)
            psi.copy_(ops.combine(torch.stack(gathered)))
        else:
            psi.copy_(local)

    use_graph = (isinstance(ops, CudaOps) if graph is None else graph) and y.is_cuda and frequency > 1
    cg = None
    it = 0
    while it < args.itermax:
        if cg is not None and it + frequency <= args.itermax:
            # iterations it + 1 .. it + frequency: the last is the next check
            # iteration ((it - 1) % frequency == 0 below); the others count here
            cg.replay()
            it += frequency
            num_iter += frequency - 1
        else:
            iterate()
            it += 1
        if (it - 1) % frequency == 0:
            s = resid()
            if float(s[0]) <= args.epsilon / 6.0:
                stopped = 1
                break
            el = torch.tensor([time.perf_counter() - t0], dtype=torch.float64, device=dev)
            if float(_reduce(el, dist.ReduceOp.MAX, group).item()) > args.tmax:
                num_iter += 1
                stopped = 3
                break
        num_iter += 1
        if use_graph and cg is None and it == 1:
            # record (not run) one block of `frequency` iterations
            torch.cuda.synchronize()
            cg = torch.cuda.CUDAGraph()
            with torch.cuda.graph(cg):
                for _ in range(frequency):
                    iterate()
    s = resid()
    return ShardedResult(phis, psi, float(s[0]), float(s[1]), it, num_iter, winf, stopped,
                         time.perf_counter() - t0)


@dataclass
class ShardedLampResult:
    nu: torch.Tensor     # averaged dual (replicated)
    theta: torch.Tensor  # (replicated)
    phi: list            # this rank's log r - logZ, one tensor per shard
    psi: torch.Tensor    # -2 W_inf nu / eta_p (replicated)
    residual: float
    objective: float
    iterations: int
    winf: float
    eta_t: float
    s_t: float
    stopped: int         # 1 tolerance, 2 itermax, 3 tmax
    log: list            # (iter, infeas, ot_objective, primal, dual) per check
    elapsed_s: float


def sharded_lamp(x_shards, r_shards, y, c, args: EOTArgs, frequency: int = 100, p: float = 2.0,
                 check: bool | None = None, marginal_only: bool = False, group=None,
                 ops=None) -> ShardedLampResult:
    """Kernel LAMP (MirrorProxKernel.jl:1019-1132) with the rows split over
    shards and ranks (see module doc). `check` defaults to args.verbose (the
    reference checks only when verbose, :1081); marginal_only drops the gap
    test of :1098. Every rank takes the same collective steps."""
    ops = ops or CudaOps()
    if frequency < 1:
        raise ValueError("frequency must be >= 1")
    if len(x_shards) != len(r_shards) or not x_shards:
        raise ValueError("one row marginal per x shard")
    dev = y.device
    m = y.shape[0]
    check = bool(args.verbose) if check is None else bool(check)
    winf_t = torch.tensor([max(ops.max_cost(x, y, p) for x in x_shards)], dtype=torch.float64, device=dev)
    winf = float(_reduce(winf_t, dist.ReduceOp.MAX, group).item())
    n_t = torch.tensor([float(sum(x.shape[0] for x in x_shards))], dtype=torch.float64, device=dev)
    n_total = float(_reduce(n_t, dist.ReduceOp.SUM, group).item())
    hr_t = torch.zeros(1, dtype=torch.float64, device=dev)
    for r in r_shards:
        hr_t += (r * torch.log(r)).sum()
    eta = args.eta_p / (2.0 * winf)
    hr = eta * float(_reduce(hr_t, dist.ReduceOp.SUM, group).item())
    emu = (c + args.alpha / n_total) / args.tau_mu
    theta = torch.zeros(m, dtype=torch.float64, device=dev)
    nu = torch.zeros(m, dtype=torch.float64, device=dev)
    s_t, eta_t, tau_p = 1.0, math.inf, 1.0       # tau_p hard-coded in the reference (:1073)
    minv, maxv = math.tanh(-args.B / 2.0), math.tanh(args.B / 2.0)
    logz = [torch.zeros(x.shape[0], dtype=torch.float64, device=dev) for x in x_shards]

    def infeas(th, et, st, want_cost=False):
        """Column mass (and cost) over all rows; row logZ of the shards."""
        acc = torch.zeros(2 * m, dtype=torch.float64, device=dev)
        for x, r, lz in zip(x_shards, r_shards, logz):
            ops.spp_lse(lz, x, y, th, et, st, winf, p)
            res, cost = ops.col_residual(x, y, r, th, lz, et, st, winf, p)
            acc[:m] += res
            if want_cost:
                acc[m:] += cost
        _reduce(acc, dist.ReduceOp.SUM, group)
        return acc[:m], acc[m:]

    def shard_dot(vals):
        t = torch.zeros(1, dtype=torch.float64, device=dev)
        for r, v in zip(r_shards, vals):
            t += torch.dot(r, v)
        return float(_reduce(t, dist.ReduceOp.SUM, group).item())

    t0 = time.perf_counter()
    log, stopped, it = [], 2, 0
    for it in range(1, args.itermax + 1):
        el = torch.tensor([time.perf_counter() - t0], dtype=torch.float64, device=dev)
        if float(_reduce(el, dist.ReduceOp.MAX, group).item()) > args.tmax:
            stopped = 3
            it -= 1
            break
        if check and (it - 1) % frequency == 0:
            res, cost = infeas(nu, eta_t, s_t, want_cost=True)
            residual_value = float((res - c).abs().sum())
            objective = float(cost.sum())
            q = eta / eta_t
            primal = (objective * (1.0 - q) - q * float(torch.dot(res, nu)) + q * shard_dot(logz)
                      + 2.0 * winf * residual_value)
            if eta > 0:
                tmp = []
                for x in x_shards:
                    t = torch.empty(x.shape[0], dtype=torch.float64, device=dev)
                    ops.spp_lse(t, x, y, theta, eta, 1.0, winf, p)
                    tmp.append(t)
                dual = -2.0 * eta * shard_dot(tmp) - 2.0 * winf * float(torch.dot(c, theta)) + 2.0 * hr
            else:
                tmp = [ops.min_reduce(x, y, theta, winf, p) for x in x_shards]
                dual = shard_dot(tmp) - 2.0 * winf * float(torch.dot(c, theta))
            log.append((it, residual_value, objective, primal, dual))
            gap_ok = True if marginal_only else (primal - dual < args.epsilon / 6.0)
            if gap_ok and residual_value < args.epsilon / 6.0:
                stopped = 1
                break
        res, _ = infeas(nu, eta_t, s_t)
        thb = ops.theta_update(theta, res, c, emu, args.eta_mu, False, minv, maxv)
        eta_t = 1.0 / (tau_p + (1.0 / eta_t) * (1.0 - eta))
        nub = (1.0 - eta_t) * nu + eta_t * theta
        s_t = (1.0 - eta_t) * s_t + eta_t
        res, _ = infeas(nub, eta_t, s_t)
        theta = ops.theta_update(theta, res, c, emu, args.eta_mu, True, minv, maxv)
        nu = (1.0 - eta_t) * nu + eta_t * thb
    res, cost = infeas(nu, eta_t, s_t, want_cost=True)
    phis = [torch.log(r) - lz for r, lz in zip(r_shards, logz)]
    psi = -2.0 * winf * nu / args.eta_p if args.eta_p != 0 else torch.full_like(nu, math.nan)
    return ShardedLampResult(nu, theta, phis, psi, float((res - c).abs().sum()), float(cost.sum()), it, winf,
                             eta_t, s_t, stopped, log, time.perf_counter() - t0)
