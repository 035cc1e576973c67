"""Dense-cost GPU solvers (run_dot without --kernel) against the FP64 oracles.

* sinkhorn_log (Sinkhorn.jl:8-84): culamp_sinkhorn_dense against the C oracle
  (or_sinkhorn_dense, square W) and the numpy restatement (any n x m):
  iteration counters, log rows (feas, <p, W>, primal, dual), potentials.
* GPU LAMP (MirrorProx.jl:397-503): culamp_lamp_dense against the numpy
  restatement np_lamp_dense_gpu: eta_t bit-exact, theta / nu, the plan
  r .* softmax(...), log rows including the rounded objective
  (Utilities.jl:158-165) and primalv / dualv (MirrorProx.jl:7-32).

Iteration passes use FP32 ex2 sums (log-sum-exp within ~1e-7 relative);
check passes are exact FP64. Potentials: within 1e-5 of max |potential| raw,
5e-6 absolute after removing the r-weighted mean (the gauge direction of
Sinkhorn, not contracted by the iteration).
"""
import math
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def gauge(v, w):
    v = np.asarray(v, dtype=np.float64)
    return v - np.dot(w, v) / np.sum(w)


def pots_close(got, want, w, atol=5e-6):
    got, want = np.asarray(got), np.asarray(want)
    assert np.abs(got - want).max() <= 1e-5 * max(1.0, np.abs(want).max())
    np.testing.assert_allclose(gauge(got, w), gauge(want, w), atol=atol, rtol=0)


def _np(t):
    return t.cpu().numpy() if hasattr(t, "cpu") else np.asarray(t)


@pytest.fixture(scope="module")
def grid8(golden_dir):
    return np.load(os.path.join(golden_dir, "dense_grid8.npz"))


def ragged(n, m, seed):
    g = np.random.Generator(np.random.PCG64(seed))
    W = g.uniform(0.0, 1.0, size=(n, m)) ** 2
    W /= np.abs(W).max()
    r = g.uniform(0.2, 1.0, n)
    c = g.uniform(0.2, 1.0, m)
    return W, r / r.sum(), c / c.sum()


@pytest.mark.parametrize("eta_p", [1e-2, 3e-3])
def test_sinkhorn_dense_matches_c_oracle(oracle, grid8, eta_p):
    import culamp_b200 as cb
    from culamp_b200.dense import solve_sinkhorn_dense
    W, r, c = grid8["W"], grid8["r"], grid8["c"]
    a = cb.EOTArgs(eta_p=eta_p, epsilon=0.0, itermax=200, verbose=False)
    phi, psi, st, log = oracle.sinkhorn_dense(W, r, c, oracle.Args(eta_p=eta_p, epsilon=0.0, itermax=200,
                                                                   verbose=False), frequency=20)
    res = solve_sinkhorn_dense(W, r, c, a, frequency=20, want_plan=True)
    assert res.iterations == st.iterations and res.num_iter == st.num_iter
    pots_close(_np(res.phi), phi, r)
    pots_close(_np(res.psi), psi, c)
    got = np.array([row[1:6] for row in res.log])
    want = np.array([row[1:6] for row in log])
    assert got.shape == want.shape and np.array_equal(got[:, 0], want[:, 0])
    # feas: within 1e-3 relative, or 2e-8 absolute where it approaches the floor
    # of the FP32-exp iteration passes (~1e-7 relative log-sum-exp)
    np.testing.assert_allclose(got[:, 1], want[:, 1], rtol=1e-3, atol=2e-8)
    np.testing.assert_allclose(got[:, 2:5], want[:, 2:5], rtol=1e-5, atol=1e-9)  # obj, primal, dual
    plan = _np(res.plan)
    want_plan = np.exp(-W / eta_p + phi[:, None] + psi[None, :])
    np.testing.assert_allclose(plan, want_plan, rtol=2e-5, atol=1e-12)


def test_sinkhorn_dense_ragged_and_stop(oracle):
    from culamp_b200 import EOTArgs
    from culamp_b200.dense import solve_sinkhorn_dense
    W, r, c = ragged(150, 97, 3)
    eta = 1e-3
    p, phi, psi, log, it, num_iter, stopped = oracle.np_sinkhorn_dense(W, r, c, eta, 300, 10, 0.0)
    res = solve_sinkhorn_dense(W, r, c, EOTArgs(eta_p=eta, epsilon=0.0, itermax=300, verbose=False), 10)
    assert res.iterations == it and res.num_iter == num_iter
    pots_close(_np(res.phi), phi, r)
    pots_close(_np(res.psi), psi, c)
    # stop at a tolerance placed between two logged checks (decisive)
    q = [max(row[1], row[3] - row[4]) for row in log]
    k = next(k for k in range(2, len(q)) if min(q[:k]) > 1.1 * q[k])
    eps = 6.0 * math.sqrt(q[k] * min(q[:k]))
    *_, it2, ni2, st2 = oracle.np_sinkhorn_dense(W, r, c, eta, 300, 10, eps)
    r2 = solve_sinkhorn_dense(W, r, c, EOTArgs(eta_p=eta, epsilon=eps, itermax=300, verbose=False), 10)
    assert st2 == 1 and r2.stopped == 1
    assert r2.iterations == it2 == log[k][0] and r2.num_iter == ni2


@pytest.mark.parametrize("eta_p", [1e-2, 0.0])
def test_lamp_dense_matches_restatement(oracle, grid8, eta_p):
    from culamp_b200 import EOTArgs
    from culamp_b200.dense import solve_lamp_dense
    W, r, c = grid8["W"], grid8["r"], grid8["c"]
    plan, th, nu, log, it, eta_t, stopped = oracle.np_lamp_dense_gpu(W, r, c, eta_p, 120, 10, 0.0, B=1.1)
    res = solve_lamp_dense(W, r, c, EOTArgs(eta_p=eta_p, epsilon=0.0, itermax=120, verbose=False, B=1.1),
                           frequency=10)
    assert res.iterations == it and res.eta_t == eta_t
    np.testing.assert_allclose(_np(res.theta), th, atol=5e-6, rtol=0)
    np.testing.assert_allclose(_np(res.nu), nu, atol=2e-6, rtol=0)
    np.testing.assert_allclose(_np(res.plan), plan, atol=1e-7, rtol=1e-4)
    got = np.array([row[1:6] for row in res.log])
    want = np.array(log)
    assert got.shape == want.shape and np.array_equal(got[:, 0], want[:, 0])
    np.testing.assert_allclose(got[:, 1], want[:, 1], rtol=1e-3, atol=1e-9)      # feas
    np.testing.assert_allclose(got[:, 2:5], want[:, 2:5], rtol=1e-4, atol=1e-7)   # obj, primal, dual


def test_lamp_dense_ragged_stop_and_reference_names(oracle):
    import culamp_b200 as cb
    from culamp_b200.dense import LAMP, sinkhorn_log, solve_lamp_dense
    W, r, c = ragged(120, 77, 5)
    *_, log, it, eta_t, stopped = oracle.np_lamp_dense_gpu(W, r, c, 1e-2, 200, 10, 0.0)
    q = [max(row[1], row[3] - row[4]) for row in log]
    k = next(k for k in range(2, len(q)) if min(q[:k]) > 1.1 * q[k])
    eps = 2.0 * math.sqrt(q[k] * min(q[:k]))
    plan, th, nu, log2, it2, eta2, st2 = oracle.np_lamp_dense_gpu(W, r, c, 1e-2, 200, 10, eps)
    res = solve_lamp_dense(W, r, c, cb.EOTArgs(eta_p=1e-2, epsilon=eps, itermax=200, verbose=False), 10)
    assert st2 == 1 and res.stopped == 1 and res.iterations == it2 == log[k][0]
    assert res.eta_t == eta2
    np.testing.assert_allclose(_np(res.theta), th, atol=5e-6, rtol=0)
    p, theta = LAMP(r, c, W, cb.EOTArgs(eta_p=1e-2, epsilon=eps, itermax=200, verbose=False), 10)
    assert p.shape == (120, 77) and theta.shape == (77,)
    np.testing.assert_allclose(_np(p).sum(1), r, rtol=1e-12)     # r .* softmax(rows)
    pk, phi, psi = sinkhorn_log(r, c, W, cb.EOTArgs(eta_p=2e-2, epsilon=0.0, itermax=50, verbose=False), 10)
    assert pk.shape == (120, 77) and phi.shape == (120,) and psi.shape == (77,)


def test_dense_large_pass_against_numpy(oracle):
    """A 1500 x 1100 problem (a few lanes' worth of columns per warp, ragged tail)
    at eta_p = 1e-3: 30 Sinkhorn iterations against the numpy restatement."""
    from culamp_b200 import EOTArgs
    from culamp_b200.dense import solve_sinkhorn_dense
    W, r, c = ragged(1500, 1100, 9)
    _, phi, psi, log, it, ni, _ = oracle.np_sinkhorn_dense(W, r, c, 1e-3, 30, 10, 0.0)
    res = solve_sinkhorn_dense(W, r, c, EOTArgs(eta_p=1e-3, epsilon=0.0, itermax=30, verbose=False), 10)
    pots_close(_np(res.phi), phi, r)
    pots_close(_np(res.psi), psi, c)
    got = np.array([row[2:6] for row in res.log])
    np.testing.assert_allclose(got[:, 1:], np.array(log)[:, 2:], rtol=1e-5, atol=1e-9)


def test_dense_invalid_arguments():
    import culamp_b200 as cb
    from culamp_b200.dense import solve_sinkhorn_dense
    W = np.ones((4, 4)); r = np.full(4, 0.25)
    with pytest.raises(cb.CulampError):
        solve_sinkhorn_dense(W, r, r, cb.EOTArgs(eta_p=0.0), 1)
    with pytest.raises(cb.CulampError):
        solve_sinkhorn_dense(W, r, r, cb.EOTArgs(eta_p=0.1), 0)
