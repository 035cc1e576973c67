"""The oracle is pinned before anything is checked against it (CPU only).

Pins: the reference's archived W_inf values, a second independent numpy
restatement, closed forms, self-consistency and an exact LP optimum.
"""
import json
import math
import os

import numpy as np
import pytest

from culamp_b200 import datasets as D


def test_winf_matches_reference_logs(oracle, golden_dir):
    ref = json.load(open(os.path.join(golden_dir, "winf_reference.json")))
    X = D.grid_coords(64, 64, scaled=False)   # CmdLineUtils.jl:208-212
    for key, want in ref["winf"].items():
        p = math.inf if key == "inf" else float(key)
        assert oracle.max_cost(X, X, p) == want


@pytest.mark.parametrize("p", [1.0, 2.0, math.inf, 3.0])
def test_c_oracle_matches_numpy_sinkhorn(oracle, p):
    x, y, r, c = D.grid_instance(6, 7, "mixture")
    a = oracle.Args(eta_p=2e-2, epsilon=0.0, itermax=40, verbose=False)
    phi, psi, st, _ = oracle.sinkhorn_kernel(x, y, r, c, a, frequency=1, p=p)
    nphi, npsi, res, cost, it, winf = oracle.np_sinkhorn_kernel(x, y, r, c, 2e-2, 40, 1, 0.0, p)
    assert np.allclose(phi, nphi, atol=1e-11, rtol=0)
    assert np.allclose(psi, npsi, atol=1e-11, rtol=0)
    assert st.residual == pytest.approx(res, rel=1e-9, abs=1e-14)
    assert st.objective == pytest.approx(cost, rel=1e-9)
    assert st.winf == winf and st.iterations == it == 40


@pytest.mark.parametrize("p", [1.0, 2.0, math.inf])
@pytest.mark.parametrize("eta_p", [1e-2, 0.0])
def test_c_oracle_matches_numpy_lamp(oracle, p, eta_p):
    x, y, r, c = D.grid_instance(6, 6, "uniform")
    a = oracle.Args(eta_p=eta_p, epsilon=0.0, itermax=25, verbose=False, B=1.1)
    nu, phi, psi, th, st, _ = oracle.lamp_kernel(x, y, r, c, a, frequency=5, p=p)
    nnu, nphi, npsi, nth, res, cost, et = oracle.np_lamp_kernel(x, y, r, c, eta_p, 25, p=p, B=1.1)
    assert np.allclose(nu, nnu, atol=1e-12)
    assert np.allclose(th, nth, atol=1e-12)
    assert np.allclose(phi, nphi, atol=1e-10)
    assert st.eta_t == pytest.approx(et, rel=1e-15)
    assert st.residual == pytest.approx(res, rel=1e-9, abs=1e-14)


def test_sinkhorn_quirk_pinf_uses_squared_cost(oracle):
    """SinkhornKernel.jl:518-520: p=Inf iterates with the squared-Euclidean
    `_opt` kernel while W_inf is the Chebyshev max."""
    x, y, r, c = D.grid_instance(5, 5, "uniform")
    a = oracle.Args(eta_p=5e-2, epsilon=0.0, itermax=10, verbose=False)
    phi_q, _, st_q, _ = oracle.sinkhorn_kernel(x, y, r, c, a, frequency=1, p=math.inf)
    phi_t, _, st_t, _ = oracle.sinkhorn_kernel(x, y, r, c, a, frequency=1, p=math.inf,
                                               flags=oracle.TRUE_PINF)
    winf = oracle.max_cost(x, y, math.inf)
    nphi, *_ = oracle.np_sinkhorn_kernel(x, y, r, c, 5e-2, 10, 1, 0.0, math.inf)
    assert st_q.winf == st_t.winf == winf
    assert np.allclose(phi_q, nphi, atol=1e-11)
    assert not np.allclose(phi_q, phi_t, atol=1e-6)


def test_closed_form_eta_inf_gives_uniform_rows(oracle):
    """eta_t = Inf (LAMP's first iteration, MirrorProxKernel.jl:1071): logZ = log m."""
    x, y = D.grid_coords(4, 4), D.grid_coords(3, 5)
    theta = np.linspace(-0.5, 0.5, 15)
    out = oracle.spp_lse(x, y, theta, math.inf, 1.0, 1.0, 2.0)
    assert np.allclose(out, math.log(15), atol=1e-15)


def test_column_marginals_exact_after_column_update(oracle):
    x, y, r, c = D.grid_instance(6, 6, "mixture")
    a = oracle.Args(eta_p=1e-2, epsilon=0.0, itermax=7, verbose=False)
    phi, psi, st, _ = oracle.sinkhorn_kernel(x, y, r, c, a, frequency=100, p=2.0)
    res_c, _ = oracle.sk_residual(y, x, c, psi, phi, 1e-2, st.winf, 2.0)
    assert np.abs(res_c).sum() < 1e-13


def test_small_eta_approaches_exact_lp(oracle):
    """As eta -> 0 the entropic transport cost tends to the exact OT optimum
    (scipy HiGHS LP)."""
    from scipy.optimize import linprog
    g = np.random.Generator(np.random.PCG64(3))
    n = 9
    x, y = g.uniform(size=(n, 2)), g.uniform(size=(n, 2))
    r = g.uniform(0.5, 1.0, n); r /= r.sum()
    c = g.uniform(0.5, 1.0, n); c /= c.sum()
    Cm = oracle.np_cost(x, y, 2.0)
    A = np.zeros((2 * n, n * n))
    for i in range(n):
        A[i, i * n:(i + 1) * n] = 1
        A[n + i, i::n] = 1
    lp = linprog(Cm.ravel(), A_eq=A, b_eq=np.concatenate([r, c]), bounds=(0, None), method="highs")
    a = oracle.Args(eta_p=5e-4, epsilon=6e-10, itermax=200000, verbose=False)
    _, _, st, _ = oracle.sinkhorn_kernel(x, y, r, c, a, frequency=10, p=2.0)
    assert st.objective == pytest.approx(lp.fun, rel=2e-2)


def test_oracle_against_golden(oracle, golden_dir):
    g = np.load(os.path.join(golden_dir, "passes_small.npz"))
    x, y, r, pot = g["x"], g["y"], g["r"], g["pot"]
    for p, k in ((1.0, "1"), (2.0, "2"), (math.inf, "inf"), (3.0, "3")):
        winf = oracle.max_cost(x, y, p)
        assert winf == g[f"winf_{k}"]
        assert np.array_equal(oracle.sk_lse(x, y, r, pot, 0.05, winf, p), g[f"sk_lse_{k}"])
    s = np.load(os.path.join(golden_dir, "solvers_grid8.npz"))
    a = oracle.Args(eta_p=1e-2, epsilon=0.0, itermax=200, verbose=True)
    phi, psi, st, _ = oracle.sinkhorn_kernel(s["x"], s["y"], s["r"], s["c"], a, frequency=7, p=2.0)
    assert np.array_equal(phi, s["sk_2_ref_phi"])


def test_dense_solvers_converge(oracle, golden_dir):
    g = np.load(os.path.join(golden_dir, "dense_grid8.npz"))
    a = oracle.Args(eta_p=1e-2, epsilon=1e-6, itermax=400, verbose=True)
    phi, psi, st, log = oracle.sinkhorn_dense(g["W"], g["r"], g["c"], a, frequency=20)
    assert np.array_equal(phi, g["sk_phi"])
    feas = [row[2] for row in log]
    assert feas[-1] < feas[0]
    b = oracle.Args(eta_p=1e-2, epsilon=1e-6, itermax=300, verbose=True, B=1.1)
    th, nu, _, st2, log2 = oracle.lamp_dense(g["W"], g["r"], g["c"], b, frequency=20)
    assert np.array_equal(nu, g["lamp_nu"])
    assert log2[-1][2] < log2[0][2]


def test_bf16_split_emulation(oracle):
    """The split-precision cost model of the tensor-core feature path: bf16
    rounding matches torch's on float-representable inputs (ties to even), the
    pieces reconstruct the value, and BF16x3 / BF16x6 inner products sit at
    their expected error levels."""
    import torch
    g = np.random.default_rng(3)
    a = g.uniform(-4, 4, 200000).astype(np.float32).astype(np.float64)
    want = torch.from_numpy(a.astype(np.float32)).to(torch.bfloat16).to(torch.float64).numpy()
    assert np.array_equal(oracle.bf16_rn(a), want)
    v = g.uniform(0, 1, 5000)
    p = oracle.bf16_pieces(v, 3)
    assert np.abs(p[0] + p[1] + p[2] - v).max() <= 2.0 ** -24 * np.abs(v).max()
    x, y = g.uniform(0, 1, (40, 256)), g.uniform(0, 1, (30, 256))
    exact = x @ y.T
    e3 = np.abs(oracle.split_dot(x, y, 2) - exact).max() / np.abs(exact).max()
    e6 = np.abs(oracle.split_dot(x, y, 3) - exact).max() / np.abs(exact).max()
    assert 1e-7 < e3 < 2e-5 and e6 < 1e-8
    c = oracle.feature_cost(x, y)
    assert np.allclose(c, ((x[:, None, :] - y[None, :, :]) ** 2).sum(-1), rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("p", [1.0, 2.0])
def test_symmetric_iteration_reaches_the_sinkhorn_fixed_point(oracle, p):
    """The averaged symmetric iteration (self-transport terms of the Sinkhorn
    divergence) converges to the alternating Sinkhorn solution: its f equals
    (phi + psi)/2 of the alternating fixed point, and the two OT values agree."""
    x, _, _, _ = D.rgb_instance(200, 200)
    r = D.uniform_marginal(200, seed=3)
    eta = 5e-2
    f, res, cost, done, winf = oracle.np_symmetric_sinkhorn(x, r, eta, 500, epsilon=6e-12, p=p)
    assert res <= 1e-12 and 0 < done < 100
    phi, psi, res2, cost2, it, _ = oracle.np_sinkhorn_kernel(x, x, r, r, eta, 50000, 1, 6e-12, p)
    assert res2 <= 1e-12 and it > 3 * done
    np.testing.assert_allclose(f, 0.5 * (phi + psi), rtol=0, atol=1e-9)
    ot_sym = eta * winf * 2 * np.dot(r, f)
    ot_alt = eta * winf * (np.dot(r, phi) + np.dot(r, psi))
    assert ot_sym == pytest.approx(ot_alt, rel=1e-9)
    assert cost == pytest.approx(cost2, rel=1e-8)
