"""Parity on the 64x64-grid workload (n = m = 4096): the chosen form against
the FP64 C oracle on the same seeded instance.

Instance: datasets.grid_instance(64, 64, "mixture") -- the grid coordinates
in [0,1]^2 (stored d = 3, z = 0) with marginals from seeded mixtures of 5
isotropic Gaussians + 1e-4 floor. Cost |x - y|_p for p in {1, 2, Inf},
eta_p in {1e-3, 1e-4}.

* Sinkhorn (SinkhornKernel.jl:477-559), LAMP (MirrorProxKernel.jl:1019-1132)
  and annealed Sinkhorn (AnnealedSinkhorn.jl:65-177) at a fixed iteration
  count: same iteration / num_iter counters, same convergence-log check
  iterations, potentials within 1e-5 of max |potential| (the parity bar),
  objective within 1e-5 relative, LAMP's eta_t recursion bit-exact.
* Stopping rules: the Sinkhorn solve to 1e-6 L1 (eta_p = 1e-3, p = 2, check
  every 10) stops at the oracle's own iteration; LAMP with its full rule
  (primal-dual gap and marginal test, MirrorProxKernel.jl:1098) and with the
  marginal test alone stops at the oracle's iteration for a tolerance placed
  between two of the oracle's logged check values (a decisive threshold).

The oracle runs here, on the host cores (OpenMP): about 30 ms per Sinkhorn
iteration at this size on 16 threads.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL = 1e-5
ETAS = [1e-3, 1e-4]
PS = [1.0, 2.0, math.inf]


@pytest.fixture(scope="module")
def inst():
    from culamp_b200 import datasets as D
    return D.grid_instance(64, 64, "mixture")


@pytest.fixture(scope="module")
def dev_inst(inst):
    import torch
    return tuple(torch.as_tensor(v, device="cuda") for v in inst)


def pot_close(got, want, what):
    got, want = np.asarray(got), np.asarray(want)
    err = np.abs(got - want).max()
    bar = REL * max(1.0, np.abs(want).max())
    assert err <= bar, f"{what}: max error {err:.3e} > {bar:.3e}"


def _np(t):
    return t.cpu().numpy() if hasattr(t, "cpu") else np.asarray(t)


@pytest.mark.parametrize("eta_p", ETAS)
@pytest.mark.parametrize("p", PS)
def test_sinkhorn_fixed_iterations(oracle, inst, dev_inst, p, eta_p):
    import culamp_b200 as cb
    x, y, r, c = inst
    K, F = 100, 10
    phi, psi, st, log = oracle.sinkhorn_kernel(
        x, y, r, c, oracle.Args(eta_p=eta_p, epsilon=0.0, itermax=K, verbose=True), frequency=F, p=p)
    res = cb.solve_sinkhorn(*dev_inst, cb.EOTArgs(eta_p=eta_p, epsilon=0.0, itermax=K, verbose=True),
                            frequency=F, p=p)
    assert res.iterations == st.iterations and res.num_iter == st.num_iter
    assert res.winf == st.winf
    pot_close(_np(res.phi), phi, "phi")
    pot_close(_np(res.psi), psi, "psi")
    assert res.objective == pytest.approx(st.objective, rel=REL)
    assert res.residual == pytest.approx(st.residual, rel=1e-3, abs=1e-9)
    got = np.array([row[1:4] for row in res.log])
    want = np.array([row[1:4] for row in log])
    assert got.shape == want.shape
    assert np.array_equal(got[:, 0], want[:, 0])                    # same check iterations
    np.testing.assert_allclose(got[:, 1], want[:, 1], rtol=1e-3, atol=1e-9)   # L1 residual
    np.testing.assert_allclose(got[:, 2], want[:, 2], rtol=REL)      # transport cost


@pytest.mark.parametrize("eta_p", ETAS)
@pytest.mark.parametrize("p", PS)
def test_lamp_fixed_iterations(oracle, inst, dev_inst, p, eta_p):
    import culamp_b200 as cb
    x, y, r, c = inst
    K, F = 60, 10
    nu, phi, psi, theta, st, log = oracle.lamp_kernel(
        x, y, r, c, oracle.Args(eta_p=eta_p, epsilon=0.0, itermax=K, verbose=True, B=1.1),
        frequency=F, p=p)
    res = cb.solve_lamp(*dev_inst, cb.EOTArgs(eta_p=eta_p, epsilon=0.0, itermax=K, verbose=True,
                                              B=1.1), frequency=F, p=p)
    assert res.iterations == st.iterations
    assert res.eta_t == st.eta_t                                      # bit-exact recursion
    pot_close(_np(res.nu), nu, "nu")
    pot_close(_np(res.theta), theta, "theta")
    pot_close(_np(res.psi), psi, "psi")
    pot_close(_np(res.phi), phi, "phi")
    assert res.objective == pytest.approx(st.objective, rel=REL)
    got = np.array([row[1:6] for row in res.log])
    want = np.array([row[1:6] for row in log])
    assert got.shape == want.shape
    assert np.array_equal(got[:, 0], want[:, 0])
    np.testing.assert_allclose(got[:, 1], want[:, 1], rtol=1e-3, atol=1e-9)   # L1 residual
    np.testing.assert_allclose(got[:, 2], want[:, 2], rtol=REL)                # ot objective
    # primal and dual values (MirrorProxKernel.jl:1084-1092), sign of the gap included
    np.testing.assert_allclose(got[:, 3:5], want[:, 3:5], rtol=1e-4, atol=1e-6)
    assert np.array_equal(np.sign(got[:, 3] - got[:, 4]), np.sign(want[:, 3] - want[:, 4]))


@pytest.mark.parametrize("eta_p,p", [(1e-3, 1.0), (1e-3, 2.0), (1e-3, math.inf), (1e-4, 2.0)])
def test_annealed_sinkhorn(oracle, inst, dev_inst, eta_p, p):
    import culamp_b200 as cb
    x, y, r, c = inst
    # stages eta = 4 eta_p, 2 eta_p, eta_p; inner tolerance = final eta (Q4); <= 60 iterations each
    kw = dict(eta_p=4 * eta_p, epsilon=eta_p, anneal_mult=0.5, itermax=60, verbose=False)
    phi, psi, st, _ = oracle.annealed_sinkhorn_kernel(x, y, r, c, oracle.Args(**kw), frequency=10, p=p)
    res = cb.solve_annealed_sinkhorn(*dev_inst, cb.EOTArgs(**kw), frequency=10, p=p)
    assert res.iterations == st.iterations and res.num_iter == st.num_iter
    pot_close(_np(res.phi), phi, "phi")
    pot_close(_np(res.psi), psi, "psi")
    assert res.objective == pytest.approx(st.objective, rel=REL)


def test_sinkhorn_stops_at_the_oracles_iteration(oracle, inst, dev_inst):
    """The bench workload's solve (eta_p = 1e-3, p = 2, L1 <= 1e-6, check every
    10): the oracle's stopping iteration, measured here, equals the GPU's."""
    import culamp_b200 as cb
    x, y, r, c = inst
    kw = dict(eta_p=1e-3, epsilon=6e-6, itermax=20000, verbose=True)
    phi, psi, st, log = oracle.sinkhorn_kernel(x, y, r, c, oracle.Args(**kw), frequency=10, p=2.0)
    assert st.stopped == 1 and st.residual <= 1e-6
    res = cb.solve_sinkhorn(*dev_inst, cb.EOTArgs(**kw), frequency=10, p=2.0)
    assert res.stopped == 1
    assert res.iterations == st.iterations and res.num_iter == st.num_iter
    pot_close(_np(res.phi), phi, "phi")
    pot_close(_np(res.psi), psi, "psi")
    rl, cl = cb.marginal_error_fp64(*dev_inst, res.phi, res.psi, 1e-3, res.winf, 2.0)
    assert rl <= 1e-6 and cl <= 1e-6


def _decisive_tolerance(log, use_gap):
    """epsilon/6 strictly between the first logged check value that the rule
    would accept and every earlier one, with >= 2 % margin either side."""
    q = [max(row[2], row[4] - row[5]) if use_gap else row[2] for row in log]
    for k in range(2, len(q)):
        lo, hi = q[k], min(q[:k])
        if hi > 1.04 * lo:
            return 6.0 * math.sqrt(lo * hi), int(log[k][1])
    return None, None


@pytest.mark.parametrize("use_gap", [True, False])
def test_lamp_stopping_rule(oracle, inst, dev_inst, use_gap):
    import culamp_b200 as cb
    x, y, r, c = inst
    F, K = 10, 120
    base = dict(eta_p=1e-3, itermax=K, verbose=True, B=1.1)
    flags = 0 if use_gap else oracle.CHECK_ALWAYS | oracle.MARGINAL_ONLY
    *_, log = oracle.lamp_kernel(x, y, r, c, oracle.Args(epsilon=0.0, **base), frequency=F, p=2.0,
                                 flags=flags)
    eps, it_stop = _decisive_tolerance(log, use_gap)
    assert eps is not None, "no decisive threshold in the oracle's log"
    nu, *_, st, olog = oracle.lamp_kernel(x, y, r, c, oracle.Args(epsilon=eps, **base), frequency=F,
                                          p=2.0, flags=flags)
    assert st.stopped == 1 and int(olog[-1][1]) == it_stop
    gflags = 0 if use_gap else cb.FLAG_CHECK_ALWAYS | cb.FLAG_MARGINAL_ONLY
    res = cb.solve_lamp(*dev_inst, cb.EOTArgs(epsilon=eps, **base), frequency=F, p=2.0, flags=gflags)
    assert res.stopped == 1
    # the stop happens at the check of iteration it_stop, before its update: the
    # log's last row names it; the returned state is the same averaged potential
    assert int(res.log[-1][1]) == it_stop
    assert len(res.log) == len(olog)
    pot_close(_np(res.nu), nu, "nu")
