"""Solver-level parity through the C ABI against the FP64 oracle and the
committed golden fixtures: same iteration counts / stopping iteration, same
convergence-log rows, potentials and objectives within tolerance.

Potentials are compared two ways. (1) Raw, at the 1e-5 parity bar: max error
<= 1e-5 of max |potential|. (2) Gauge-fixed (the r-weighted mean removed), at
5e-6 absolute for Sinkhorn: Sinkhorn's plan exp(phi_i + psi_j - C/eps) is
invariant to phi + k, psi - k, and LAMP's to a uniform shift of nu, and those
directions are not contracted by the iteration, so FP32-exp rounding drifts
along them (a few 1e-6 over 200 iterations) while the plan itself stays within
rounding. LAMP: nu / theta 2e-6 / 5e-6 absolute after gauge fixing; residuals
and objectives 1e-5 relative; eta_t bit-exact.
"""
import math
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

POT_ATOL = 5e-6
REL = 1e-5


@pytest.fixture(scope="module")
def grid8(golden_dir):
    return np.load(os.path.join(golden_dir, "solvers_grid8.npz"))


def pk(p):
    return "inf" if math.isinf(p) else f"{p:g}"


def gauge(v, w):
    v = np.asarray(v, dtype=np.float64)
    return v - np.dot(w, v) / np.sum(w)


def assert_potentials(got, want, w, atol):
    got, want = np.asarray(got), np.asarray(want)
    assert np.abs(got - want).max() <= 1e-5 * max(1.0, np.abs(want).max())   # raw, relative bar
    np.testing.assert_allclose(gauge(got, w), gauge(want, w), atol=atol, rtol=0)


@pytest.mark.parametrize("p,tag,flags", [(1.0, "ref", 0), (2.0, "ref", 0), (math.inf, "ref", 0),
                                         (math.inf, "true", 1)])
def test_sinkhorn_matches_golden(grid8, p, tag, flags):
    import culamp_b200 as cb
    g = grid8
    a = cb.EOTArgs(eta_p=1e-2, epsilon=0.0, itermax=200, verbose=True)
    res = cb.solve_sinkhorn(g["x"], g["y"], g["r"], g["c"], a, frequency=7, p=p, flags=flags)
    pre = f"sk_{pk(p)}_{tag}"
    st = g[pre + "_stats"]
    assert res.iterations == st[0] and res.num_iter == st[1]
    assert_potentials(res.phi, g[pre + "_phi"], g["r"], POT_ATOL)
    assert_potentials(res.psi, g[pre + "_psi"], g["c"], POT_ATOL)
    assert res.residual == pytest.approx(st[2], rel=1e-3, abs=1e-9)
    assert res.objective == pytest.approx(st[3], rel=REL)
    assert res.winf == st[4]
    log = np.array([row[1:4] for row in res.log])
    want = g[pre + "_log"][:, 1:4]
    assert log.shape == want.shape
    assert np.array_equal(log[:, 0], want[:, 0])            # same check iterations
    np.testing.assert_allclose(log[:, 2], want[:, 2], rtol=REL)


def test_sinkhorn_stops_at_same_iteration(grid8):
    import culamp_b200 as cb
    g = grid8
    a = cb.EOTArgs(eta_p=1e-2, epsilon=6e-4, itermax=500, verbose=True)
    res = cb.solve_sinkhorn(g["x"], g["y"], g["r"], g["c"], a, frequency=5, p=2.0)
    st = g["skstop_stats"]
    assert res.stopped == 1
    assert res.iterations == st[0] and res.num_iter == st[1]
    assert_potentials(res.phi, g["skstop_phi"], g["r"], POT_ATOL)


@pytest.mark.parametrize("eta_tag,eta_p", [("eta", 1e-2), ("zero", 0.0)])
@pytest.mark.parametrize("p", [1.0, 2.0, math.inf])
def test_lamp_matches_golden(grid8, eta_tag, eta_p, p):
    import culamp_b200 as cb
    g = grid8
    a = cb.EOTArgs(eta_p=eta_p, epsilon=1e-12, itermax=120, verbose=True, B=1.1)
    res = cb.solve_lamp(g["x"], g["y"], g["r"], g["c"], a, frequency=10, p=p)
    pre = f"lamp_{eta_tag}_{pk(p)}"
    st = g[pre + "_stats"]
    assert res.iterations == st[0]
    assert res.eta_t == st[4]                                 # bit-exact recursion
    assert_potentials(res.nu, g[pre + "_nu"], g["c"], 2e-6)
    np.testing.assert_allclose(res.theta, g[pre + "_theta"], atol=5e-6)
    # phi = log r - logZ amplifies nu's error by 1/eta_t: relative bar only
    assert np.abs(res.phi - g[pre + "_phi"]).max() <= 1e-5 * np.abs(g[pre + "_phi"]).max()
    assert res.residual == pytest.approx(st[1], rel=1e-3, abs=1e-8)
    assert res.objective == pytest.approx(st[2], rel=REL)
    log = np.array([row[1:6] for row in res.log])
    want = g[pre + "_log"][:, 1:6]
    assert log.shape == want.shape
    assert np.array_equal(log[:, 0], want[:, 0])
    np.testing.assert_allclose(log[:, 2], want[:, 2], rtol=REL)          # ot_objective
    np.testing.assert_allclose(log[:, 3:5], want[:, 3:5], rtol=1e-4, atol=1e-6)  # primal, dual


def test_annealed_matches_golden(grid8):
    import culamp_b200 as cb
    g = grid8
    a = cb.EOTArgs(eta_p=0.1, epsilon=2e-3, anneal_mult=0.5, itermax=300, verbose=False)
    res = cb.solve_annealed_sinkhorn(g["x"], g["y"], g["r"], g["c"], a, frequency=10, p=2.0)
    st = g["ann_stats"]
    assert res.iterations == st[0] and res.num_iter == st[1]
    assert_potentials(res.phi, g["ann_phi"], g["r"], 1e-5)
    assert_potentials(res.psi, g["ann_psi"], g["c"], 1e-5)
    assert res.objective == pytest.approx(st[3], rel=REL)


def test_ragged_solvers(golden_dir):
    import culamp_b200 as cb
    g = np.load(os.path.join(golden_dir, "solvers_ragged.npz"))
    a = cb.EOTArgs(eta_p=5e-2, epsilon=0.0, itermax=150, verbose=False)
    res = cb.solve_sinkhorn(g["x"], g["y"], g["r"], g["c"], a, frequency=50, p=2.0)
    assert_potentials(res.phi, g["sk_phi"], g["r"], POT_ATOL)
    assert_potentials(res.psi, g["sk_psi"], g["c"], POT_ATOL)
    assert res.objective == pytest.approx(g["sk_stats"][1], rel=REL)
    b = cb.EOTArgs(eta_p=5e-2, epsilon=0.0, itermax=80, verbose=False, B=1.1)
    lr = cb.solve_lamp(g["x"], g["y"], g["r"], g["c"], b, frequency=50, p=2.0)
    assert_potentials(lr.nu, g["lamp_nu"], g["c"], 2e-6)
    np.testing.assert_allclose(lr.theta, g["lamp_theta"], atol=5e-6)
    assert lr.eta_t == g["lamp_stats"][3]


def test_device_host_and_nograph_paths_agree(grid8):
    import torch
    import culamp_b200 as cb
    g = grid8
    a = cb.EOTArgs(eta_p=1e-2, epsilon=0.0, itermax=60, verbose=False)
    host = cb.solve_sinkhorn(g["x"], g["y"], g["r"], g["c"], a, frequency=3, p=2.0)
    dev = [torch.as_tensor(g[k], device="cuda") for k in ("x", "y", "r", "c")]
    d0 = cb.solve_sinkhorn(*dev, a, frequency=3, p=2.0)
    # the pass-per-launch loop, as a graph and launched from the host
    d1 = cb.solve_sinkhorn(*dev, a, frequency=3, p=2.0, flags=cb.FLAG_NO_PERSIST)
    d2 = cb.solve_sinkhorn(*dev, a, frequency=3, p=2.0, flags=cb.FLAG_NO_GRAPH)
    assert np.array_equal(host.phi, d0.phi.cpu().numpy())
    assert np.array_equal(d1.phi.cpu().numpy(), d2.phi.cpu().numpy())
    # the persistent loop sums the same FP32 terms in another order (~1e-7
    # relative per log-sum-exp)
    want = d1.phi.cpu().numpy()
    np.testing.assert_allclose(d0.phi.cpu().numpy(), want, rtol=0, atol=2e-6 * max(1.0, np.abs(want).max()))
    assert host.iterations == d0.iterations == d1.iterations == d2.iterations


def test_warm_start_continues_the_iteration(grid8):
    import culamp_b200 as cb
    g = grid8
    a40 = cb.EOTArgs(eta_p=1e-2, epsilon=0.0, itermax=40, verbose=False)
    a20 = cb.EOTArgs(eta_p=1e-2, epsilon=0.0, itermax=20, verbose=False)
    full = cb.solve_sinkhorn(g["x"], g["y"], g["r"], g["c"], a40, frequency=100, p=2.0)
    half = cb.solve_sinkhorn(g["x"], g["y"], g["r"], g["c"], a20, frequency=100, p=2.0)
    cont = cb.solve_sinkhorn(g["x"], g["y"], g["r"], g["c"], a20, frequency=100, p=2.0,
                             phi0=half.phi, psi0=half.psi)
    np.testing.assert_allclose(cont.phi, full.phi, atol=1e-9)


def test_plain_form_runs_and_is_close(grid8, oracle):
    import culamp_b200 as cb
    g = grid8
    a = cb.EOTArgs(eta_p=1e-2, epsilon=0.0, itermax=200, verbose=False)
    res = cb.solve_sinkhorn(g["x"], g["y"], g["r"], g["c"], a, frequency=7, p=2.0,
                            flags=cb.FLAG_FORM_PLAIN)
    np.testing.assert_allclose(res.phi, g["sk_2_ref_phi"], atol=5e-3)
    b = cb.EOTArgs(eta_p=1e-2, epsilon=1e-12, itermax=120, verbose=True, B=1.1)
    lr = cb.solve_lamp(g["x"], g["y"], g["r"], g["c"], b, frequency=10, p=2.0,
                       flags=cb.FLAG_FORM_PLAIN)
    np.testing.assert_allclose(lr.nu, g["lamp_eta_2_nu"], atol=1e-4)
    assert lr.iterations == 120


def test_reference_named_api(tmp_path, grid8):
    import culamp_b200 as cb
    from culamp_b200 import io as cio
    g = grid8
    a = cb.EOTArgs(eta_p=1e-2, epsilon=0.0, itermax=50, verbose=False)
    phi, psi, obj, resid = cb.sinkhorn_color_transfer(g["x"], g["y"], g["r"], g["c"], a, 10, 2,
                                                      return_assignments=False)
    assert phi.shape == (64,) and np.isfinite(obj) and resid >= 0
    phi2, psi2, img1, img2 = cb.sinkhorn_color_transfer(g["x"], g["y"], g["r"], g["c"], a, 10, 2)
    assert img1.shape == g["x"].shape and np.isfinite(img1).all()
    prefix = str(tmp_path / "pot")
    cb.sinkhorn_euclidean(g["r"], g["c"], g["x"], g["y"], "", "", prefix, a, 10, 2.0)
    assert np.array_equal(cio.read_potentials(prefix, ".row"), phi2)
    b = cb.EOTArgs(eta_p=1e-2, epsilon=0.0, itermax=30, verbose=False, B=1.1)
    mu, phil, psil, b1, b2 = cb.extragradient_color_transfer(g["x"], g["y"], g["r"], g["c"], b, 10, 2.0)
    np.testing.assert_allclose(psil, -2 * 2.0 * mu / 1e-2, rtol=1e-14)   # psi = -2 W nu / eta_p
    assert np.isfinite(b1).all() and np.isfinite(b2).all()


def test_invalid_arguments_raise():
    import culamp_b200 as cb
    from culamp_b200 import _lib
    x = np.zeros((4, 3)); r = np.full(4, 0.25)
    with pytest.raises(cb.CulampError) as e:
        cb.solve_sinkhorn(x, x, r, r, cb.EOTArgs(eta_p=0.0), 1, 2.0)
    assert e.value.status == _lib.ERR_INVALID_ARG
    with pytest.raises(cb.CulampError):
        cb.solve_sinkhorn(x, x, -r, r, cb.EOTArgs(eta_p=0.1), 1, 2.0)
    with pytest.raises(cb.CulampError):
        cb.solve_sinkhorn(x, x, r, r, cb.EOTArgs(eta_p=0.1), 1, 0.0)
    with pytest.raises(cb.CulampError):
        cb.solve_sinkhorn(x, x, r, r, cb.EOTArgs(eta_p=0.1), 0, 2.0)


def test_itermax_zero_and_tmax_zero(grid8):
    import culamp_b200 as cb
    g = grid8
    r0 = cb.solve_sinkhorn(g["x"], g["y"], g["r"], g["c"], cb.EOTArgs(eta_p=1e-2, itermax=0), 1, 2.0)
    assert r0.iterations == 0 and np.all(r0.phi == 0)
    rt = cb.solve_sinkhorn(g["x"], g["y"], g["r"], g["c"], cb.EOTArgs(eta_p=1e-2, itermax=1000, tmax=0.0,
                                                                      epsilon=0.0), 1000, 2.0)
    assert rt.stopped == 3 and rt.iterations <= 2
