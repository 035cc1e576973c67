"""Adjoint pass and Sinkhorn divergence.

* The adjoint (culamp_adjoint_sk) against the FP64 envelope gradient
  sum_j P_ij grad_x C (oracle) at the same potentials: 1e-6 relative.
* The divergence gradient against central finite differences of FP64 oracle
  solves: h = 1e-3 on 64 coordinates at eta_p = 1e-2 (n = 256), and h = 2e-4
  on 12 coordinates at the divergence workload's eta_p = 1e-3 (n = 1024):
  1e-4 relative (the gradient parity bar). eps is held fixed across the perturbed
  solves.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def T(a):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device="cuda")


@pytest.mark.parametrize("p", [1.0, 2.0, math.inf, 3.0])
@pytest.mark.parametrize("shape", [(300, 200, 3), (64, 500, 2), (1031, 777, 1), (40, 60, 4)])
def test_adjoint_matches_envelope_gradient(oracle, p, shape):
    from culamp_b200.divergence import adjoint
    n, m, d = shape
    g = np.random.Generator(np.random.PCG64(7 + n + m + d))
    x, y = g.uniform(size=(n, d)), g.uniform(size=(m, d))
    phi, psi = g.normal(-math.log(n), 1.0, n), g.normal(-math.log(m), 1.0, m)
    eps = 0.05
    grad, mass = adjoint(T(x), T(y), T(phi), T(psi), eps, p, want_mass=True)
    want, wmass = oracle.envelope_grad(x, y, phi, psi, eps, 1.0, p)
    got = grad.cpu().numpy()
    assert np.abs(got - want).max() <= 1e-6 * np.abs(want).max()
    np.testing.assert_allclose(mass.cpu().numpy(), wmass, rtol=1e-6)


def _oracle_ot(O, x, y, a, b, eps, p, phi0, psi0):
    winf = O.max_cost(x, y, p)
    args = O.Args(eta_p=eps / winf, epsilon=6e-14, itermax=200000, verbose=False)
    phi, psi, st, _ = O.sinkhorn_kernel(x, y, a, b, args, frequency=5, p=p, phi0=phi0, psi0=psi0)
    return eps * (a @ phi + b @ psi)


def test_divergence_gradient_matches_finite_differences(oracle):
    from culamp_b200 import datasets as D
    from culamp_b200.divergence import divergence_grads, sinkhorn_divergence
    n = 256
    x, y, a, b = D.rgb_instance(n, n)
    eps = 1e-2 * oracle.max_cost(x, y, 2.0)
    parts = sinkhorn_divergence(T(x), T(y), T(a), T(b), eps, 2.0, tol=1e-10)
    gx, gy, ga, gb = divergence_grads(T(x), T(y), parts, 2.0)
    gx = gx.cpu().numpy()
    oracle.set_threads(0)
    rng = np.random.Generator(np.random.PCG64(11))
    idx = rng.choice(n * 3, size=64, replace=False)
    h = 1e-3
    phi_xy, psi_xy = parts.xy.phi.cpu().numpy(), parts.xy.psi.cpu().numpy()
    phi_xx, psi_xx = parts.xx.phi.cpu().numpy(), parts.xx.psi.cpu().numpy()
    fd = np.empty(64)
    for q, flat in enumerate(idx):
        i, k = divmod(int(flat), 3)
        vals = []
        for s in (+1.0, -1.0):
            xp = x.copy()
            xp[i, k] += s * h
            oxy = _oracle_ot(oracle, xp, y, a, b, eps, 2.0, phi_xy, psi_xy)
            oxx = _oracle_ot(oracle, xp, xp, a, a, eps, 2.0, phi_xx, psi_xx)
            vals.append(oxy - 0.5 * oxx)       # OT(b, b) does not depend on x
        fd[q] = (vals[0] - vals[1]) / (2 * h)
    adj = np.array([gx[divmod(int(f), 3)] for f in idx])
    assert np.linalg.norm(adj - fd) <= 1e-4 * np.linalg.norm(fd)


def test_divergence_gradient_fd_at_the_config_eta(oracle):
    """The same check at the divergence workload's eta_p = 1e-3 (eps = 1e-3
    W_inf) on n = m = 1024 RGB points: 12 coordinates, h = 2e-4, the cross
    term by warm-started FP64 oracle solves to L1 <= 1e-9 (the dual value's
    error is second order in the residual), the self term by the oracle's
    symmetric iteration from the solved potential."""
    import time
    from culamp_b200 import datasets as D
    from culamp_b200.divergence import divergence_grads, sinkhorn_divergence
    n = 1024
    x, y, a, b = D.rgb_instance(n, n)
    eps = 1e-3 * oracle.max_cost(x, y, 2.0)
    parts = sinkhorn_divergence(T(x), T(y), T(a), T(b), eps, 2.0, tol=1e-8)
    gx = divergence_grads(T(x), T(y), parts, 2.0)[0].cpu().numpy()
    oracle.set_threads(0)
    rng = np.random.Generator(np.random.PCG64(13))
    idx = rng.choice(n * 3, size=12, replace=False)
    h = 2e-4
    phi_xy, psi_xy = parts.xy.phi.cpu().numpy(), parts.xy.psi.cpu().numpy()
    f_xx = parts.xx.phi.cpu().numpy()
    fd = np.empty(len(idx))
    t0 = time.time()
    for q, flat in enumerate(idx):
        i, k = divmod(int(flat), 3)
        vals = []
        for s in (+1.0, -1.0):
            xp = x.copy()
            xp[i, k] += s * h
            winf = oracle.max_cost(xp, y, 2.0)
            args = oracle.Args(eta_p=eps / winf, epsilon=6e-9, itermax=200000, verbose=False)
            phi, psi, _, _ = oracle.sinkhorn_kernel(xp, y, a, b, args, frequency=10, p=2.0,
                                                     phi0=phi_xy, psi0=psi_xy)
            oxy = eps * (a @ phi + b @ psi)
            wxx = oracle.np_cost(xp, xp, 2.0).max()
            f, *_ = oracle.np_symmetric_sinkhorn(xp, a, eps / wxx, 5000, epsilon=6e-12, p=2.0,
                                                 f0=f_xx, winf=wxx)
            oxx = eps * 2.0 * (a @ f)
            vals.append(oxy - 0.5 * oxx)       # OT(b, b) does not depend on x
        fd[q] = (vals[0] - vals[1]) / (2 * h)
    print(f"12 FD coordinates in {time.time() - t0:.1f} s")
    adj = np.array([gx[divmod(int(f), 3)] for f in idx])
    assert np.linalg.norm(adj - fd) <= 1e-4 * np.linalg.norm(fd)


def test_autograd_function_and_identity(oracle):
    import torch
    from culamp_b200 import datasets as D
    from culamp_b200.divergence import (divergence_grads, sinkhorn_divergence,
                                        sinkhorn_divergence_fn)
    x, y, a, b = (T(v) for v in D.rgb_instance(512, 400))
    eps = 0.02
    xr = x.clone().requires_grad_(True)
    ar = a.clone().requires_grad_(True)
    s = sinkhorn_divergence_fn(xr, y, ar, b, eps, 2.0, 1e-8)
    s.backward()
    parts = sinkhorn_divergence(x, y, a, b, eps, 2.0, tol=1e-8)
    gx, _, ga, _ = divergence_grads(x, y, parts, 2.0)
    assert abs(float(s.detach()) - parts.value) <= 1e-9 * max(1.0, abs(parts.value))
    assert torch.allclose(xr.grad, gx, rtol=1e-6, atol=1e-12)
    assert torch.allclose(ar.grad, ga, rtol=1e-6, atol=1e-12)
    same = sinkhorn_divergence(x, x, a, a, eps, 2.0, tol=1e-8)
    assert abs(same.value) <= 1e-6 * abs(same.xy.value)
