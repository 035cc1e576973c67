"""Batched uneven Sinkhorn solves (culamp_batched_sinkhorn).

Every instance of a batch must come out as if solved alone. On the FP64-
exponent pair path (d <= 3, and other d on the FP64 loops): the same stopping
iteration as culamp_sinkhorn's pass-per-launch loop (CULAMP_FLAG_NO_PERSIST,
the passes a batch runs) at a tolerance the residual crosses decisively,
and the same potentials up to summation order (the batch sizes its column
splits for the batch, not for the instance alone), gauge-fixed within 5e-6.
At epsilon = 1e-6 the residual decays slowly through the threshold, and the
rounding that differs with the split geometry (FP32 exp; on the tensor-core
feature path also the FP32 partial sums) may move the stop by a few checks:
iterations within ITERS_REL there, potentials within 5e-6 / FEAT_ATOL. A few
members are also checked against the FP64 oracle directly.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FEAT_ATOL = 1e-4
ITERS_REL = 0.1


def gauge(v, w):
    v = np.asarray(v, dtype=np.float64)
    return v - np.dot(w, v) / np.sum(w)


def T(a):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device="cuda")


@pytest.fixture(scope="module")
def batch():
    from culamp_b200 import datasets as D
    inst = D.batched_instances(14, lo=100, hi=1200, dims=(2, 3, 5, 40), seed=4)
    return [tuple(T(v) for v in t) for t in inst], inst


@pytest.mark.parametrize("frequency", [1, 10])
def test_batch_matches_single_solves(batch, frequency):
    import culamp_b200 as cb
    dev, host = batch
    a = cb.EOTArgs(eta_p=1e-2, epsilon=1e-6, itermax=3000, verbose=False)
    out = cb.solve_batched_sinkhorn(dev, a, frequency=frequency, p=2.0)
    assert out.target_ctas_per_sm in (2, 4, 8, 16, 32, 64)
    assert len(out.results) == len(dev)
    for k, ((x, y, r, c), res) in enumerate(zip(dev, out.results)):
        one = cb.solve_sinkhorn(x, y, r, c, a, frequency, 2.0, flags=cb.FLAG_NO_PERSIST)
        feat = x.shape[1] >= 32
        assert res.stopped == one.stopped == 1, k
        # at 1e-6 the residual crosses the threshold slowly, so rounding that
        # differs with the split geometry may move the stop by a few checks
        assert abs(res.iterations - one.iterations) <= ITERS_REL * one.iterations + 2 * frequency, k
        assert res.winf == one.winf
        tol = FEAT_ATOL if feat else 5e-6
        rr, cc = host[k][2], host[k][3]
        np.testing.assert_allclose(gauge(res.phi.cpu().numpy(), rr), gauge(one.phi.cpu().numpy(), rr), atol=tol, rtol=0)
        np.testing.assert_allclose(gauge(res.psi.cpu().numpy(), cc), gauge(one.psi.cpu().numpy(), cc), atol=tol, rtol=0)
        if not feat:
            # residuals near 1.6e-7 sit within ~1e-8 of the FP32-exp rounding floor, and the
            # batched and single passes split the columns differently
            assert res.residual == pytest.approx(one.residual, rel=1e-3, abs=1e-8)
        assert res.residual <= 1e-6 / 6 * 1.5
        assert res.objective == pytest.approx(one.objective, rel=1e-5)


def test_batch_stops_at_single_solver_iteration(batch):
    """At a tolerance the residual crosses decisively (6e-4), every member on
    the FP64-exponent pair path stops at exactly the single-solve iteration."""
    import culamp_b200 as cb
    dev, _ = batch
    a = cb.EOTArgs(eta_p=1e-2, epsilon=6e-4, itermax=3000, verbose=False)
    out = cb.solve_batched_sinkhorn(dev, a, frequency=5, p=2.0)
    for k, ((x, y, r, c), res) in enumerate(zip(dev, out.results)):
        if x.shape[1] >= 32:
            continue
        one = cb.solve_sinkhorn(x, y, r, c, a, 5, 2.0, flags=cb.FLAG_NO_PERSIST)
        assert (res.iterations, res.num_iter, res.stopped) == (one.iterations, one.num_iter, 1), k


def test_batch_members_match_oracle(oracle, batch):
    import culamp_b200 as cb
    dev, host = batch
    a = cb.EOTArgs(eta_p=1e-2, epsilon=0.0, itermax=120, verbose=False)
    out = cb.solve_batched_sinkhorn(dev, a, frequency=10, p=2.0, flags=cb.FLAG_FEAT_X6)
    for k in range(len(host)):
        x, y, r, c = host[k]
        res = out.results[k]
        assert res.iterations == 120 and res.stopped == 2
        cost = oracle.feature_cost(x, y, 3) if x.shape[1] >= 32 else None
        phi, psi, *_ = oracle.np_sinkhorn_kernel(x, y, r, c, 1e-2, 120, frequency=10, p=2.0,
                                                 cost=cost, winf=res.winf)
        tol = FEAT_ATOL if x.shape[1] >= 32 else 5e-6
        np.testing.assert_allclose(gauge(res.phi.cpu().numpy(), r), gauge(phi, r), atol=tol, rtol=0)
        np.testing.assert_allclose(gauge(res.psi.cpu().numpy(), c), gauge(psi, c), atol=tol, rtol=0)


def test_batch_repeat_uses_cached_shape_and_is_deterministic(batch):
    import culamp_b200 as cb
    dev, _ = batch
    a = cb.EOTArgs(eta_p=1e-2, epsilon=1e-5, itermax=2000, verbose=False)
    o1 = cb.solve_batched_sinkhorn(dev, a, frequency=5, p=2.0)
    o2 = cb.solve_batched_sinkhorn(dev, a, frequency=5, p=2.0)
    assert o2.tune_ms == 0.0 and o2.target_ctas_per_sm == o1.target_ctas_per_sm
    for r1, r2 in zip(o1.results, o2.results):
        assert r1.iterations == r2.iterations
        assert np.array_equal(r1.phi.cpu().numpy(), r2.phi.cpu().numpy())


def test_batch_l1_cost_and_graphless_loop(batch):
    import culamp_b200 as cb
    dev, host = batch
    small = [t for t in dev if t[0].shape[1] <= 5][:5]
    a = cb.EOTArgs(eta_p=1e-2, epsilon=1e-6, itermax=2000, verbose=False)
    g = cb.solve_batched_sinkhorn(small, a, frequency=3, p=1.0)
    h = cb.solve_batched_sinkhorn(small, a, frequency=3, p=1.0, flags=cb.FLAG_NO_GRAPH)
    for (x, y, r, c), rg, rh in zip(small, g.results, h.results):
        one = cb.solve_sinkhorn(x, y, r, c, a, 3, 1.0, flags=cb.FLAG_NO_PERSIST)
        assert rg.iterations == one.iterations == rh.iterations
        assert np.array_equal(rg.phi.cpu().numpy(), rh.phi.cpu().numpy())


def test_batch_rejects_bad_input(batch):
    import torch
    import culamp_b200 as cb
    dev, _ = batch
    a = cb.EOTArgs(eta_p=1e-2, epsilon=1e-6, itermax=10, verbose=False)
    with pytest.raises(cb.CulampError):
        cb.solve_batched_sinkhorn(dev[:2], a, frequency=1, p=3.0)
    with pytest.raises(cb.CulampError):
        cb.solve_batched_sinkhorn(dev[:2], a.copy(eta_p=0.0), frequency=1, p=2.0)
    bad = list(dev[:2]) + [(torch.zeros((3, 300), dtype=torch.float64, device="cuda"),) + dev[0][1:]]
    with pytest.raises((cb.CulampError, ValueError)):
        cb.solve_batched_sinkhorn(bad, a, frequency=1, p=2.0)
