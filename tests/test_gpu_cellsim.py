"""Cell-similarity metrics on the GPU passes (culamp_b200.cellsim): cosine and
correlation run on the tensor-core squared-Euclidean path (d = 64 cells), l1 on
the FP64 pair loops. Compared with the oracle's Sinkhorn / LAMP on the
metric's cost matrix: for the tensor-core metrics on the same split-precision
(BF16x3) inner products, as the feature-path tests do (gauge-fixed potentials
within 1e-4), and on the exact cost at the BF16x3 bound."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def gauge(v, w):
    v = np.asarray(v, dtype=np.float64)
    return v - np.dot(w, v) / np.sum(w)


def counts(n, d, seed):
    g = np.random.Generator(np.random.PCG64(seed))
    a = np.log1p(g.negative_binomial(0.5, 0.2, size=(n, d)).astype(float))
    a *= g.uniform(size=(n, d)) >= 0.7
    a[a.sum(1) == 0, 0] = 1.0
    a[:, 1] += 0.01
    return a


@pytest.mark.parametrize("metric", ["cosine", "correlation", "l1"])
def test_sinkhorn_cellsim_matches_oracle(oracle, metric):
    from culamp_b200 import EOTArgs
    from culamp_b200.cellsim import cell_points, sinkhorn_cellsim
    a = counts(400, 64, 7)
    g = np.random.Generator(np.random.PCG64(8))
    r = g.uniform(0.2, 1, 400); r /= r.sum()
    c = g.uniform(0.2, 1, 400); c /= c.sum()
    res = sinkhorn_cellsim(a, metric, r, c, EOTArgs(eta_p=1e-2, epsilon=0.0, itermax=100, verbose=False), 10)
    pts, p, factor = cell_points(a, metric)
    exact = oracle.np_cell_cost(a, metric)
    assert res.winf == pytest.approx(exact.max(), rel=1e-12)
    if p == 2.0:
        # the BF16x3 inner products; what remains is the FP32 (TMEM) accumulation
        # of 64-term dot products of unit vectors, ~1e-6 relative, which the
        # exponent scales by 1/(eta_p W_inf): 5e-5 of max |potential|
        cost = factor * oracle.feature_cost(pts, pts, 2)
        tol_same, tol_exact = None, 5e-2
    else:
        cost, tol_same, tol_exact = exact, 5e-6, 5e-6
    phi, psi, *_ = oracle.np_sinkhorn_kernel(pts, pts, r, c, 1e-2, 100, frequency=10, p=p, cost=cost,
                                             winf=res.winf)
    got_phi, got_psi = res.phi.cpu().numpy(), res.psi.cpu().numpy()
    if tol_same is None:
        tol_same = 5e-5 * np.abs(phi).max()
    assert np.abs(gauge(got_phi, r) - gauge(phi, r)).max() <= tol_same
    assert np.abs(gauge(got_psi, c) - gauge(psi, c)).max() <= tol_same
    phie, *_ = oracle.np_sinkhorn_kernel(pts, pts, r, c, 1e-2, 100, frequency=10, p=p, cost=exact,
                                         winf=res.winf)
    assert np.abs(gauge(got_phi, r) - gauge(phie, r)).max() <= tol_exact


def test_lamp_cellsim_runs_on_the_metric(oracle):
    from culamp_b200 import EOTArgs
    from culamp_b200.cellsim import cell_points, lamp_cellsim
    a = counts(300, 48, 11)
    r = np.full(300, 1 / 300)
    res = lamp_cellsim(a, "l1", r, r, EOTArgs(eta_p=1e-2, epsilon=0.0, itermax=40, verbose=False, B=1.1), 10)
    pts, p, factor = cell_points(a, "l1")
    nu, *_ = oracle.np_lamp_kernel(pts, pts, r, r, 1e-2, 40, p=p, B=1.1)
    np.testing.assert_allclose(gauge(res.nu.cpu().numpy(), r), gauge(nu, r), atol=2e-6, rtol=0)
