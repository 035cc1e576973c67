"""Feature clouds (d >= 32, squared Euclidean cost) on the tensor cores.

The tensor-core passes form <x_i, y_j> from bf16 pieces of the FP64 features
(BF16x3 by default, BF16x6 with FLAG_FEAT_X6), accumulate in FP32 (TMEM) and
run an FP32 online log-sum-exp; norms, potentials and scalar reductions stay
FP64. Parity is checked in two steps:

* against the FP64 oracle run on the SAME split-precision cost
  (oracle.feature_cost(x, y, pieces) rounds the same bf16 pieces and sums the
  products in FP64). What remains is FP32 accumulation and the FP32 exponent:
  gauge-fixed potentials within SAME_ATOL, raw within 1e-5 of max |potential|;
* against the FP64 oracle on the exact cost: BF16x6 within EXACT_ATOL_X6.
  BF16x3 products carry ~2^-16 relative error, which moves potentials by up to
  ~1e-3 at eta_p = 1e-2; that gap is asserted as a bound, not hidden.

The FP64 pair loops (FLAG_FEAT_FP64, and p != 2 at any d) match the exact
oracle at the solver bar.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SAME_ATOL = 1e-4
EXACT_ATOL_X6 = 1e-4
EXACT_ATOL_X3 = 5e-2
ITERS = 150


def gauge(v, w):
    v = np.asarray(v, dtype=np.float64)
    return v - np.dot(w, v) / np.sum(w)


def close(got, want, w, atol):
    got, want = np.asarray(got), np.asarray(want)
    gerr = np.abs(gauge(got, w) - gauge(want, w)).max()
    assert gerr <= atol, f"gauge-fixed max error {gerr:.3e} > {atol:.1e}"
    return gerr


@pytest.fixture(scope="module", params=[(640, 520, 256), (300, 450, 72)],
            ids=["640x520xd256", "300x450xd72"])
def feats(request):
    from culamp_b200 import datasets as D
    n, m, d = request.param
    return D.feature_instance(n, m, d)


@pytest.mark.parametrize("pieces,flag", [(2, 0), (3, 32)], ids=["bf16x3", "bf16x6"])
def test_sinkhorn_feature_path_matches_split_cost_oracle(oracle, feats, pieces, flag):
    import culamp_b200 as cb
    x, y, r, c = feats
    a = cb.EOTArgs(eta_p=1e-2, epsilon=0.0, itermax=ITERS, verbose=False)
    res = cb.solve_sinkhorn(x, y, r, c, a, frequency=10, p=2.0, flags=flag)
    assert res.iterations == ITERS
    cost = oracle.feature_cost(x, y, pieces)
    phi, psi, *_ = oracle.np_sinkhorn_kernel(x, y, r, c, 1e-2, ITERS, frequency=10, p=2.0,
                                             cost=cost, winf=res.winf)
    assert res.winf == pytest.approx(oracle.feature_cost(x, y).max(), rel=1e-14)
    big = max(1.0, np.abs(phi).max())
    assert np.abs(res.phi - phi).max() <= 1e-5 * big
    close(res.phi, phi, r, SAME_ATOL)
    close(res.psi, psi, c, SAME_ATOL)
    # against the exact cost
    phie, psie, *_ = oracle.np_sinkhorn_kernel(x, y, r, c, 1e-2, ITERS, frequency=10, p=2.0,
                                               cost=oracle.feature_cost(x, y), winf=res.winf)
    tol = EXACT_ATOL_X6 if pieces == 3 else EXACT_ATOL_X3
    close(res.phi, phie, r, tol)
    close(res.psi, psie, c, tol)


def test_sinkhorn_feature_fp64_loops_match_exact_oracle(oracle, feats):
    import culamp_b200 as cb
    x, y, r, c = feats
    a = cb.EOTArgs(eta_p=1e-2, epsilon=0.0, itermax=60, verbose=False)
    res = cb.solve_sinkhorn(x, y, r, c, a, frequency=10, p=2.0, flags=cb.FLAG_FEAT_FP64)
    phi, psi, *_ = oracle.np_sinkhorn_kernel(x, y, r, c, 1e-2, 60, frequency=10, p=2.0)
    close(res.phi, phi, r, 5e-6)
    close(res.psi, psi, c, 5e-6)


def test_sinkhorn_feature_l1_cost_stays_on_fp64_loops(oracle, feats):
    import culamp_b200 as cb
    x, y, r, c = feats
    a = cb.EOTArgs(eta_p=1e-2, epsilon=0.0, itermax=40, verbose=False)
    res = cb.solve_sinkhorn(x, y, r, c, a, frequency=10, p=1.0)
    phi, psi, *_ = oracle.np_sinkhorn_kernel(x, y, r, c, 1e-2, 40, frequency=10, p=1.0)
    close(res.phi, phi, r, 5e-6)


def test_sinkhorn_feature_residual_and_objective(oracle, feats):
    """Check-pass moment path: residual L1 and transport cost at the returned
    potentials, against the FP64 evaluation on the same split cost. The FP32
    exponent carries ~5e-6 relative error per P_ij, so the residual (a sum of
    |r_i - sum_j P_ij| with total mass 1) is good to a few 1e-6 absolute."""
    import culamp_b200 as cb
    x, y, r, c = feats
    a = cb.EOTArgs(eta_p=1e-2, epsilon=0.0, itermax=80, verbose=True)
    res = cb.solve_sinkhorn(x, y, r, c, a, frequency=20, p=2.0, flags=cb.FLAG_FEAT_X6)
    cost = oracle.feature_cost(x, y, 3)
    P = np.exp(-cost / (1e-2 * res.winf) + res.phi[:, None] + res.psi[None, :])
    assert res.objective == pytest.approx((P * cost).sum(), rel=1e-5)
    assert res.residual == pytest.approx(np.abs(r - P.sum(1)).sum(), rel=0, abs=5e-6)
    assert len(res.log) == 80 // 20


@pytest.mark.parametrize("pieces,flag", [(2, 0), (3, 32)], ids=["bf16x3", "bf16x6"])
def test_lamp_feature_path_matches_split_cost_oracle(oracle, feats, pieces, flag):
    import culamp_b200 as cb
    x, y, r, c = feats
    its = 60
    a = cb.EOTArgs(eta_p=1e-2, epsilon=0.0, itermax=its, verbose=False)
    res = cb.solve_lamp(x, y, r, c, a, frequency=10, p=2.0, flags=flag)
    nu, phi, psi, theta, *_ = oracle.np_lamp_kernel(x, y, r, c, 1e-2, its, p=2.0,
                                                    cost=oracle.feature_cost(x, y, pieces),
                                                    winf=res.winf)
    close(res.nu, nu, c, 2e-5)
    close(res.theta, theta, c, 5e-5)
    close(res.phi, phi, r, SAME_ATOL)


def test_lamp_feature_checks_match_fp64_loops(feats):
    """Verbose LAMP exercises the min-reduction (dual) pass on the tensor
    cores; its log must track the FP64 pair-loop run."""
    import culamp_b200 as cb
    x, y, r, c = feats
    a = cb.EOTArgs(eta_p=0.0, epsilon=0.0, itermax=30, verbose=True)
    t = cb.solve_lamp(x, y, r, c, a, frequency=10, p=2.0, flags=cb.FLAG_FEAT_X6)
    e = cb.solve_lamp(x, y, r, c, a, frequency=10, p=2.0, flags=cb.FLAG_FEAT_FP64)
    lt, le = np.array(t.log), np.array(e.log)
    assert lt.shape == le.shape and len(lt) == 3
    np.testing.assert_allclose(lt[:, 1], le[:, 1])                       # iterations
    np.testing.assert_allclose(lt[:, 2:], le[:, 2:], rtol=1e-4, atol=1e-6)
