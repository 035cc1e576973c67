"""Differentiable entropic OT and the Sinkhorn divergence.

OT_eps(a, b; x, y) is the value of the entropic problem
    min_P <P, C> + eps sum_ij P_ij log P_ij   s.t. P 1 = a, P^T 1 = b,
solved by the kernel Sinkhorn with P_ij = exp(phi_i + psi_j - C_ij / eps). At
the optimum it equals the dual value eps (a.phi + b.psi). `eps` here is
absolute (cost units): each solve runs with eta_p = eps / W_inf of its own
point pair, so the three terms of the divergence share one eps.

Gradients (envelope theorem, eps fixed -- W_inf does not enter):
  * d OT / d x_i = sum_j P_ij grad_x C(x_i, y_j): culamp_adjoint_sk, one pass
    over all pairs that recomputes P_ij and never stores the n x m plan;
  * d OT / d y_j: the same pass with the roles of the clouds swapped;
  * d OT / d a_i = eps phi_i, d OT / d b_j = eps psi_j (the potentials; defined
    up to a constant because sum a = sum b = 1).

S_eps(a, b) = OT(a, b) - OT(a, a)/2 - OT(b, b)/2. The self terms have a
symmetric optimal plan and one potential f = phi = psi; they are solved by the
averaged symmetric iteration f <- (f + T(f))/2 (culamp_symmetric_sinkhorn), one
row pass per iteration, which reaches the tolerance in tens of passes where
the alternating iteration takes hundreds. In OT(a, a; x, x) the cloud x enters
both sides, so its gradient is the row pass plus the column pass.

SinkhornDivergence is a torch.autograd.Function -- the Python counterpart of a
ChainRulesCore rrule.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import torch

from . import kernels as K
from .args import EOTArgs
from .solvers import _dev, _stream, get_handle, solve_sinkhorn, solve_symmetric_sinkhorn


@dataclass
class OTResult:
    value: float          # eps (a.phi + b.psi)
    phi: torch.Tensor
    psi: torch.Tensor
    eps: float
    eta_p: float
    winf: float
    iterations: int
    residual: float


def entropic_ot(x, y, a, b, eps: float, p: float = 2.0, tol: float = 1e-7, frequency: int = 10,
                itermax: int = 200_000, phi0=None, psi0=None) -> OTResult:
    """Kernel Sinkhorn at absolute regularisation eps, to L1 marginal error tol."""
    _, winf = K.max_logsumexp_spp_ct(x, y, p, rows=False)
    eta_p = eps / winf
    args = EOTArgs(eta_p=eta_p, epsilon=6.0 * tol, itermax=itermax, verbose=False)
    res = solve_sinkhorn(x, y, a, b, args, frequency, p, phi0=phi0, psi0=psi0)
    value = eps * (float(torch.dot(a, res.phi)) + float(torch.dot(b, res.psi)))
    return OTResult(value, res.phi, res.psi, eps, eta_p, winf, res.iterations, res.residual)


def entropic_ot_self(x, a, eps: float, p: float = 2.0, tol: float = 1e-7, frequency: int = 10,
                     itermax: int = 200_000, f0=None) -> OTResult:
    """OT_eps(a, a; x, x) by the symmetric iteration, to L1 marginal error tol."""
    _, winf = K.max_logsumexp_spp_ct(x, x, p, rows=False)
    eta_p = eps / winf
    args = EOTArgs(eta_p=eta_p, epsilon=6.0 * tol, itermax=itermax, verbose=False)
    res = solve_symmetric_sinkhorn(x, a, args, frequency, p, f0=f0)
    value = 2.0 * eps * float(torch.dot(a, res.phi))
    return OTResult(value, res.phi, res.psi, eps, eta_p, winf, res.iterations, res.residual)


def adjoint(x, y, phi, psi, eps: float, p: float = 2.0, want_mass: bool = False):
    """sum_j P_ij grad_x C(x_i, y_j) for P_ij = exp(phi_i + psi_j - C_ij/eps)."""
    n, d = x.shape
    m = y.shape[0]
    grad = torch.empty_like(x)
    mass = torch.empty(n, dtype=torch.float64, device=x.device) if want_mass else None
    h = get_handle(x.device.index)
    h.check(h._lib.culamp_adjoint_sk(h.ptr, C.c_void_p(grad.data_ptr()),
                                     C.c_void_p(mass.data_ptr()) if want_mass else None,
                                     _dev(x, "x"), _dev(y, "y"), n, m, d, _dev(phi, "phi", n),
                                     _dev(psi, "psi", m), float(eps), 1.0, float(p), _stream()),
            "culamp_adjoint_sk")
    return (grad, mass) if want_mass else grad


@dataclass
class DivergenceParts:
    value: float
    xy: OTResult
    xx: OTResult
    yy: OTResult


def sinkhorn_divergence(x, y, a, b, eps: float, p: float = 2.0, tol: float = 1e-7,
                        frequency: int = 10, warm=None) -> DivergenceParts:
    """S_eps = OT(a,b) - OT(a,a)/2 - OT(b,b)/2 (three solves sharing eps)."""
    w = warm or (None, None, None)
    xy = entropic_ot(x, y, a, b, eps, p, tol, frequency,
                     phi0=w[0].phi if w[0] else None, psi0=w[0].psi if w[0] else None)
    xx = entropic_ot_self(x, a, eps, p, tol, frequency, f0=w[1].phi if w[1] else None)
    yy = entropic_ot_self(y, b, eps, p, tol, frequency, f0=w[2].phi if w[2] else None)
    return DivergenceParts(xy.value - 0.5 * xx.value - 0.5 * yy.value, xy, xx, yy)


def divergence_grads(x, y, parts: DivergenceParts, p: float = 2.0):
    """(dS/dx, dS/dy, dS/da, dS/db) at the solved potentials."""
    eps = parts.xy.eps
    xy, xx, yy = parts.xy, parts.xx, parts.yy
    gx = adjoint(x, y, xy.phi, xy.psi, eps, p) - 0.5 * (adjoint(x, x, xx.phi, xx.psi, eps, p) +
                                                          adjoint(x, x, xx.psi, xx.phi, eps, p))
    gy = adjoint(y, x, xy.psi, xy.phi, eps, p) - 0.5 * (adjoint(y, y, yy.phi, yy.psi, eps, p) +
                                                          adjoint(y, y, yy.psi, yy.phi, eps, p))
    ga = eps * xy.phi - 0.5 * eps * (xx.phi + xx.psi)
    gb = eps * xy.psi - 0.5 * eps * (yy.phi + yy.psi)
    return gx, gy, ga, gb


class SinkhornDivergence(torch.autograd.Function):
    """S_eps(a, b; x, y) with gradients for x, y, a and b."""

    @staticmethod
    def forward(ctx, x, y, a, b, eps, p=2.0, tol=1e-7):
        x, y, a, b = (t.detach().contiguous() for t in (x, y, a, b))
        parts = sinkhorn_divergence(x, y, a, b, float(eps), float(p), float(tol))
        ctx.save_for_backward(x, y)
        ctx.parts = parts
        ctx.p = float(p)
        return torch.tensor(parts.value, dtype=torch.float64, device=x.device)

    @staticmethod
    def backward(ctx, g):
        x, y = ctx.saved_tensors
        gx, gy, ga, gb = divergence_grads(x, y, ctx.parts, ctx.p)
        return g * gx, g * gy, g * ga, g * gb, None, None, None


def sinkhorn_divergence_fn(x, y, a, b, eps, p=2.0, tol=1e-7):
    return SinkhornDivergence.apply(x, y, a, b, eps, p, tol)
