"""Barycentric colour-transfer maps against FP64 restatements of the reference.

Sinkhorn maps (naive_findmaxindex_ct!, SinkhornKernel.jl:124-162):
out_i = sum_j y_j P_ij / sum_j P_ij, P_ij = exp(-C_ij/(eta_p W_inf) + phi_i + psi_j),
with the reference's cost choice (p == 1 ? L1 : squared). Checked against the
C oracle's or_barycentric_sk on the GPU solve's own potentials, so the test
isolates the map kernel from solver rounding.

LAMP maps (naive_findmaxindex_spp_ct! / _t!, MirrorProxKernel.jl:97-189):
w_ij = r_i exp(-(C_ij/(2 W_inf) + nu_j)/eta_t - logZ_i), the row map
sum_j y_j w_ij / sum_j w_ij and the column map sum_i x_i w_ij / sum_i w_ij,
logZ the final log-sum-exp of MirrorProxKernel.jl:1124. The library evaluates
them through the Sinkhorn-form rewrite (culamp_b200.solvers.lamp_barycentric_maps);
here they are restated directly from the reference formulas in numpy.

Both are FP64 end to end on the GPU (exp in FP64), so the bar is 1e-10
relative to the coordinate range.
"""
import math
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAP_ATOL = 1e-10


def _fixtures(golden_dir):
    g8 = np.load(os.path.join(golden_dir, "solvers_grid8.npz"))
    rg = np.load(os.path.join(golden_dir, "solvers_ragged.npz"))
    return {"grid8": g8, "ragged": rg}


def np_cost(x, y, p):
    d = x[:, None, :] - y[None, :, :]
    if p == 1:
        return np.abs(d).sum(-1)
    if p == 2:
        return (d * d).sum(-1)
    if math.isinf(p):
        return np.abs(d).max(-1)
    return (np.abs(d) ** p).sum(-1)


def np_logz(x, y, nu, eta_t, s_t, winf, p):
    """logZ of MirrorProxKernel.jl:1124 (two-pass LSE, :702-829), FP64."""
    a = -(np_cost(x, y, p) * s_t / (2.0 * winf) + nu[None, :]) / eta_t
    mx = a.max(axis=1, keepdims=True)
    return (np.log(np.exp(a - mx).sum(axis=1, keepdims=True)) + mx)[:, 0]


def np_lamp_maps(x, y, r, nu, eta_t, s_t, winf, p, logz=None):
    """MirrorProxKernel.jl:97-189 given logZ (default: np_logz)."""
    C = np_cost(x, y, p)
    if logz is None:
        logz = np_logz(x, y, nu, eta_t, s_t, winf, p)
    # the map kernels themselves use C / (2 W_inf) without s (s_t == 1 here)
    w = r[:, None] * np.exp(-(C / (2.0 * winf) + nu[None, :]) / eta_t - logz[:, None])
    b1 = (w @ y) / w.sum(axis=1, keepdims=True)
    b2 = (w.T @ x) / w.sum(axis=0)[:, None]
    return b1, b2


@pytest.mark.parametrize("name", ["grid8", "ragged"])
@pytest.mark.parametrize("p", [1.0, 2.0, math.inf])
def test_sinkhorn_maps_match_oracle(golden_dir, oracle, name, p):
    import culamp_b200 as cb
    g = _fixtures(golden_dir)[name]
    eta_p = 1e-2 if name == "grid8" else 5e-2
    a = cb.EOTArgs(eta_p=eta_p, epsilon=0.0, itermax=120, verbose=False)
    res = cb.solve_sinkhorn(g["x"], g["y"], g["r"], g["c"], a, frequency=10, p=p)
    b1 = cb.barycentric_map(g["x"], g["y"], res.phi, res.psi, eta_p, res.winf, p).cpu().numpy()
    b2 = cb.barycentric_map(g["y"], g["x"], res.psi, res.phi, eta_p, res.winf, p).cpu().numpy()
    cost_p = 1.0 if p == 1 else 2.0          # the reference map's cost (SinkhornKernel.jl:143-147)
    w1 = oracle.barycentric_sk(g["x"], g["y"], res.phi, res.psi, eta_p, res.winf, cost_p)
    w2 = oracle.barycentric_sk(g["y"], g["x"], res.psi, res.phi, eta_p, res.winf, cost_p)
    np.testing.assert_allclose(b1, w1, rtol=0, atol=MAP_ATOL)
    np.testing.assert_allclose(b2, w2, rtol=0, atol=MAP_ATOL)
    # a wrong weight would move the images; they also stay inside the hull
    assert b1.min() >= g["y"].min() - 1e-12 and b1.max() <= g["y"].max() + 1e-12


@pytest.mark.parametrize("name", ["grid8", "ragged"])
@pytest.mark.parametrize("p", [1.0, 2.0, math.inf])
def test_lamp_maps_match_reference_formula(golden_dir, name, p):
    import culamp_b200 as cb
    g = _fixtures(golden_dir)[name]
    eta_p = 1e-2 if name == "grid8" else 5e-2
    a = cb.EOTArgs(eta_p=eta_p, epsilon=0.0, itermax=60, verbose=False, B=1.1)
    res = cb.solve_lamp(g["x"], g["y"], g["r"], g["c"], a, frequency=10, p=p)
    b1, b2 = cb.lamp_barycentric_maps(g["x"], g["y"], g["r"], res, p)
    assert abs(res.s_t - 1.0) < 1e-12
    nu = np.asarray(res.nu)
    # logZ enters the column map's weights; the solver's final logZ (FP32 exp
    # sums) matches the FP64 one to the log-sum-exp tolerance, and the maps
    # are checked in FP64 on that logZ
    logz = np.log(g["r"]) - np.asarray(res.phi)
    want_logz = np_logz(g["x"], g["y"], nu, res.eta_t, res.s_t, res.winf, p)
    np.testing.assert_allclose(logz, want_logz, rtol=0, atol=2e-6)
    w1, w2 = np_lamp_maps(g["x"], g["y"], g["r"], nu, res.eta_t, res.s_t, res.winf, p, logz)
    np.testing.assert_allclose(b1.cpu().numpy(), w1, rtol=0, atol=MAP_ATOL)
    np.testing.assert_allclose(b2.cpu().numpy(), w2, rtol=0, atol=MAP_ATOL)


def test_color_transfer_entry_points_return_the_maps(golden_dir):
    """sinkhorn_color_transfer / extragradient_color_transfer return exactly the
    maps of the standalone calls on their own potentials."""
    import culamp_b200 as cb
    g = _fixtures(golden_dir)["grid8"]
    a = cb.EOTArgs(eta_p=1e-2, epsilon=0.0, itermax=80, verbose=False)
    phi, psi, img1, img2 = cb.sinkhorn_color_transfer(g["x"], g["y"], g["r"], g["c"], a, 10, 2)
    res = cb.solve_sinkhorn(g["x"], g["y"], g["r"], g["c"], a, 10, 2.0)
    b1 = cb.barycentric_map(g["x"], g["y"], phi, psi, 1e-2, res.winf, 2.0).cpu().numpy()
    assert np.array_equal(img1, b1)
    b = cb.EOTArgs(eta_p=1e-2, epsilon=0.0, itermax=40, verbose=False, B=1.1)
    nu, phil, _, l1, l2 = cb.extragradient_color_transfer(g["x"], g["y"], g["r"], g["c"], b, 10, 2.0)
    lr = cb.solve_lamp(g["x"], g["y"], g["r"], g["c"], b, 10, 2.0)
    w1, w2 = np_lamp_maps(g["x"], g["y"], g["r"], nu, lr.eta_t, lr.s_t, lr.winf, 2.0,
                          np.log(g["r"]) - phil)
    np.testing.assert_allclose(l1, w1, rtol=0, atol=MAP_ATOL)
    np.testing.assert_allclose(l2, w2, rtol=0, atol=MAP_ATOL)
