"""Symmetric Sinkhorn (culamp_symmetric_sinkhorn): the self-transport terms
OT(a, a; x, x) of the Sinkhorn divergence, one averaged row pass per iteration.

* A fixed number of iterations against the FP64 oracle restatement
  (oracle.np_symmetric_sinkhorn): f within 1e-5 of max(1, max |f|) on the
  FP64-exponent pair paths (packed d <= 3 with the fixed-reference loop, the
  generic d loop, p = 1); on the tensor-core feature path against the oracle
  run on the same split-precision cost, within FEAT_ATOL.
* The stopping rule: at a tolerance the residual crosses decisively the GPU
  stops at the oracle's iteration, with the residual at the returned f.
* The fixed point: converged f equals (phi + psi)/2 of the alternating
  Sinkhorn solve of the same problem, and the OT values agree.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FEAT_ATOL = 1e-4
# The in-loop residual (tolerance test) and the final residual pass sum FP32
# exponents along different loops; their L1 residuals differ by up to ~6e-8
# (measured), so a stop at residual <= tol reads back below tol + RESID_FLOOR.
RESID_FLOOR = 1e-7


def T(a):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device="cuda")


def cloud(n, d, seed):
    from culamp_b200 import datasets as D
    g = np.random.Generator(np.random.PCG64(seed))
    x = g.uniform(0.0, 1.0, size=(n, d))
    return x, D.uniform_marginal(n, seed=seed + 1)


@pytest.mark.parametrize("n,d,p", [(700, 3, 2.0), (513, 2, 2.0), (300, 1, 2.0), (450, 5, 2.0),
                                   (600, 3, 1.0), (257, 4, 1.0)])
def test_fixed_iterations_match_oracle(oracle, n, d, p):
    import culamp_b200 as cb
    x, r = cloud(n, d, 5 + d)
    its = 9
    a = cb.EOTArgs(eta_p=1e-2, epsilon=0.0, itermax=its, verbose=False)
    res = cb.solve_symmetric_sinkhorn(T(x), T(r), a, frequency=1, p=p)
    assert res.iterations == its and res.stopped == 2
    f, resid, cost, done, winf = oracle.np_symmetric_sinkhorn(x, r, 1e-2, its, p=p)
    assert res.winf == pytest.approx(winf, rel=1e-14)
    got = res.phi.cpu().numpy()
    assert np.abs(got - f).max() <= 1e-5 * max(1.0, np.abs(f).max())
    # residual and cost come from FP32 exponents (~1e-6 relative per P_ij) over
    # a plan of total mass 1: absolute 1e-6 on the L1 residual
    assert res.residual == pytest.approx(resid, rel=0, abs=1e-6)
    assert res.objective == pytest.approx(cost, rel=1e-5)


@pytest.mark.parametrize("pieces,flag", [(2, 0), (3, 32)], ids=["bf16x3", "bf16x6"])
def test_feature_path_matches_split_cost_oracle(oracle, pieces, flag):
    import culamp_b200 as cb
    from culamp_b200 import datasets as D
    x, _, r, _ = D.feature_instance(500, 500, 72)
    its = 8
    a = cb.EOTArgs(eta_p=1e-2, epsilon=0.0, itermax=its, verbose=False)
    res = cb.solve_symmetric_sinkhorn(T(x), T(r), a, frequency=1, p=2.0, flags=flag)
    assert res.iterations == its
    cost = oracle.feature_cost(x, x, pieces)
    f, *_ = oracle.np_symmetric_sinkhorn(x, r, 1e-2, its, cost=cost, winf=res.winf)
    assert np.abs(res.phi.cpu().numpy() - f).max() <= FEAT_ATOL


def test_stops_at_oracle_iteration(oracle):
    import culamp_b200 as cb
    x, r = cloud(800, 3, 21)
    a = cb.EOTArgs(eta_p=2e-3, epsilon=6e-5, itermax=1000, verbose=False)
    res = cb.solve_symmetric_sinkhorn(T(x), T(r), a, frequency=1, p=2.0)
    f, resid, _, done, _ = oracle.np_symmetric_sinkhorn(x, r, 2e-3, 1000, epsilon=6e-5)
    assert res.stopped == 1 and res.iterations == done
    assert res.residual <= 1e-5 + RESID_FLOOR and res.residual == pytest.approx(resid, rel=0, abs=1e-6)
    assert np.abs(res.phi.cpu().numpy() - f).max() <= 1e-5 * max(1.0, np.abs(f).max())


@pytest.mark.parametrize("eta_p", [1e-2, 1e-3])
def test_fixed_point_is_the_sinkhorn_solution(eta_p):
    """Both solves to L1 residual 1e-7. Their potentials then differ by the
    alternating solve's slow-mode error (measured 1.3e-7 / 1.1e-6 of max |f| at
    eta_p = 1e-2 / 1e-3); the OT values are stationary and agree to ~1e-11."""
    import torch
    import culamp_b200 as cb
    x, r = cloud(2000, 3, 33)
    xs, rs = T(x), T(r)
    a = cb.EOTArgs(eta_p=eta_p, epsilon=6e-7, itermax=200_000, verbose=False)
    sym = cb.solve_symmetric_sinkhorn(xs, rs, a, frequency=10, p=2.0)
    alt = cb.solve_sinkhorn(xs, xs, rs, rs, a, frequency=10, p=2.0)
    assert sym.stopped == 1 and alt.stopped == 1
    assert sym.iterations * 3 < alt.iterations
    assert sym.residual <= 1e-7 + RESID_FLOOR
    half = 0.5 * (alt.phi + alt.psi)
    scale = max(1.0, float(half.abs().max()))
    assert float((sym.phi - half).abs().max()) <= 1e-5 * scale
    v_sym = 2.0 * float(torch.dot(rs, sym.phi))
    v_alt = float(torch.dot(rs, alt.phi) + torch.dot(rs, alt.psi))
    assert v_sym == pytest.approx(v_alt, rel=1e-9)


def test_graphless_loop_warm_start_and_log():
    import culamp_b200 as cb
    x, r = cloud(3000, 2, 41)
    xs, rs = T(x), T(r)
    a = cb.EOTArgs(eta_p=1e-2, epsilon=1e-6, itermax=500, verbose=True)
    g = cb.solve_symmetric_sinkhorn(xs, rs, a, frequency=2, p=2.0)
    h = cb.solve_symmetric_sinkhorn(xs, rs, a, frequency=2, p=2.0, flags=cb.FLAG_NO_GRAPH)
    assert g.stopped == h.stopped == 1 and g.iterations == h.iterations
    assert np.array_equal(g.phi.cpu().numpy(), h.phi.cpu().numpy())
    assert [row[1] for row in g.log] == list(range(0, g.iterations + 1, 2))
    assert g.residual <= 1e-6 / 6 + RESID_FLOOR < g.log[0][2]
    # warm start from the solution: stops at once (or within a pass or two if
    # the first, reference-free pass rounds the residual above the tolerance)
    w = cb.solve_symmetric_sinkhorn(xs, rs, a, frequency=2, p=2.0, f0=g.phi)
    assert w.stopped == 1 and w.iterations <= 2
    if w.iterations == 0:
        assert np.array_equal(w.phi.cpu().numpy(), g.phi.cpu().numpy())


def test_rejects_bad_input():
    import culamp_b200 as cb
    x, r = cloud(100, 3, 1)
    a = cb.EOTArgs(eta_p=0.0, epsilon=1e-6, itermax=10, verbose=False)
    with pytest.raises(cb.CulampError):
        cb.solve_symmetric_sinkhorn(T(x), T(r), a, frequency=1, p=2.0)
    with pytest.raises(cb.CulampError):
        cb.solve_symmetric_sinkhorn(T(x), T(-r), a.copy(eta_p=1e-2), frequency=1, p=2.0)
    with pytest.raises(cb.CulampError):
        cb.solve_symmetric_sinkhorn(T(x), T(r), a.copy(eta_p=1e-2), frequency=1, p=2.0,
                                    flags=cb.FLAG_FORM_PLAIN)
