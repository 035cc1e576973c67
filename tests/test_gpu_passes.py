"""Pass-level parity: every hot kernel vs the FP64 oracle on the same seeded inputs.

Tolerances (chosen form: FP64 exponent, FP32 MUFU exp, compensated FP32 sums):
  * max-cost / min-reduce: exact FP64 (rtol 1e-14 for general p, which uses pow)
  * log-sum-exp outputs: absolute 2e-6 in natural-log units
  * residual / cost / column masses: relative 2e-6 of the row's mass
"""
import math
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PS = [1.0, 2.0, math.inf, 3.0]
SHAPES = [(1, 1, 1), (31, 257, 2), (257, 31, 3), (1031, 777, 3), (300, 200, 5), (64, 700, 16)]
LSE_ATOL = 2e-6
MASS_RTOL = 2e-6


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    assert torch.cuda.is_available()
    return torch


def T(torch, a):
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device="cuda")


def case(n, m, d, seed=0):
    g = np.random.Generator(np.random.PCG64(1000 + seed + n + 7 * m + 13 * d))
    x, y = g.uniform(size=(n, d)), g.uniform(size=(m, d))
    r = g.uniform(0.1, 1.0, n); r /= r.sum()
    c = g.uniform(0.1, 1.0, m); c /= c.sum()
    return dict(x=x, y=y, r=r, c=c, pot=g.normal(0, 3, m), phi=g.normal(0, 3, n),
                theta=g.uniform(-0.9, 0.9, m), logz=g.normal(0, 1, n))


@pytest.mark.parametrize("p", PS)
@pytest.mark.parametrize("shape", SHAPES)
def test_max_cost_and_min_reduce(torch_cuda, oracle, p, shape):
    from culamp_b200 import kernels as K
    n, m, d = shape
    cs = case(n, m, d)
    x, y = T(torch_cuda, cs["x"]), T(torch_cuda, cs["y"])
    rowmax, winf = K.max_logsumexp_spp_ct(x, y, p)
    want = oracle.max_cost_rows(cs["x"], cs["y"], p)
    tol = 0 if p in (1.0, 2.0) or math.isinf(p) else 1e-14
    np.testing.assert_allclose(rowmax.cpu().numpy(), want, rtol=tol, atol=0)
    assert winf == pytest.approx(want.max(), rel=tol, abs=0)
    mn = K.warp_min_reduce(x, y, T(torch_cuda, cs["theta"]), winf, p)
    np.testing.assert_allclose(mn.cpu().numpy(), oracle.min_reduce(cs["x"], cs["y"], cs["theta"], winf, p),
                               rtol=1e-13, atol=1e-13)


@pytest.mark.parametrize("p", PS)
@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("reg", [0.05, 1e-3])
def test_sinkhorn_lse_and_residual(torch_cuda, oracle, p, shape, reg):
    from culamp_b200 import kernels as K
    n, m, d = shape
    cs = case(n, m, d, 1)
    x, y = T(torch_cuda, cs["x"]), T(torch_cuda, cs["y"])
    winf = oracle.max_cost(cs["x"], cs["y"], p)
    out = K.warp_logsumexp_ct_fused(x, y, T(torch_cuda, cs["r"]), T(torch_cuda, cs["pot"]), reg, winf, p)
    want = oracle.sk_lse(cs["x"], cs["y"], cs["r"], cs["pot"], reg, winf, p)
    np.testing.assert_allclose(out.cpu().numpy(), want, rtol=0, atol=LSE_ATOL)
    # residual at a near-feasible point: phi from the row update above
    phi = want
    res, cost = K.residual_opt(x, y, T(torch_cuda, cs["r"]), T(torch_cuda, phi), T(torch_cuda, cs["pot"]),
                               reg, winf, p)
    wres, wcost = oracle.sk_residual(cs["x"], cs["y"], cs["r"], phi, cs["pot"], reg, winf, p)
    np.testing.assert_allclose(res.cpu().numpy(), wres, rtol=0, atol=MASS_RTOL * cs["r"].max())
    np.testing.assert_allclose(cost.cpu().numpy(), wcost, rtol=MASS_RTOL, atol=1e-300)


@pytest.mark.parametrize("p", PS)
@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("reg", [0.02, 1e-3, math.inf])
def test_spp_lse_and_column_residual(torch_cuda, oracle, p, shape, reg):
    from culamp_b200 import kernels as K
    n, m, d = shape
    cs = case(n, m, d, 2)
    x, y = T(torch_cuda, cs["x"]), T(torch_cuda, cs["y"])
    winf = oracle.max_cost(cs["x"], cs["y"], p)
    out = K.warp_logsumexp_spp_ct_fused(x, y, T(torch_cuda, cs["theta"]), reg, 1.0, winf, p)
    want = oracle.spp_lse(cs["x"], cs["y"], cs["theta"], reg, 1.0, winf, p)
    np.testing.assert_allclose(out.cpu().numpy(), want, rtol=0, atol=LSE_ATOL)
    res, cost = K.residual_spp_c(x, y, T(torch_cuda, cs["r"]), T(torch_cuda, cs["theta"]),
                                 T(torch_cuda, want), reg, 1.0, winf, p)
    wres, wcost = oracle.spp_col_residual(cs["x"], cs["y"], cs["r"], cs["theta"], want, reg, 1.0, winf, p)
    np.testing.assert_allclose(res.cpu().numpy(), wres, rtol=MASS_RTOL, atol=1e-300)
    np.testing.assert_allclose(cost.cpu().numpy(), wcost, rtol=MASS_RTOL, atol=1e-300)


def test_theta_update_matches_oracle(torch_cuda, oracle, golden_dir):
    from culamp_b200 import kernels as K
    g = np.load(os.path.join(golden_dir, "passes_small.npz"))
    n = g["x"].shape[0]
    emu = (g["c"] + 0.01 / n) / 1.0
    for adjust, key in ((False, "theta_upd_a0"), (True, "theta_upd_a1")):
        out = K.update_theta_residual(T(torch_cuda, g["theta"]), T(torch_cuda, g["spp_res_2"]),
                                      T(torch_cuda, g["c"]), T(torch_cuda, emu), 0.0, adjust, -0.5, 0.5)
        np.testing.assert_allclose(out.cpu().numpy(), g[key], rtol=1e-14, atol=1e-15)


def test_golden_passes(torch_cuda, golden_dir):
    """The committed oracle fixture (n=37, m=23, d=3), no live oracle."""
    from culamp_b200 import kernels as K
    g = np.load(os.path.join(golden_dir, "passes_small.npz"))
    x, y = T(torch_cuda, g["x"]), T(torch_cuda, g["y"])
    for p, k in ((1.0, "1"), (2.0, "2"), (math.inf, "inf"), (3.0, "3")):
        rowmax, winf = K.max_logsumexp_spp_ct(x, y, p)
        np.testing.assert_allclose(rowmax.cpu().numpy(), g[f"rowmax_{k}"], rtol=1e-14)
        out = K.warp_logsumexp_ct_fused(x, y, T(torch_cuda, g["r"]), T(torch_cuda, g["pot"]), 0.05, winf, p)
        np.testing.assert_allclose(out.cpu().numpy(), g[f"sk_lse_{k}"], atol=LSE_ATOL, rtol=0)
        out = K.warp_logsumexp_spp_ct_fused(x, y, T(torch_cuda, g["theta"]), 0.02, 1.0, winf, p)
        np.testing.assert_allclose(out.cpu().numpy(), g[f"spp_lse_{k}"], atol=LSE_ATOL, rtol=0)


def test_reference_grid_winf(torch_cuda, golden_dir):
    """W_inf of the reference's integer 64x64 grid equals its archived logs."""
    import json
    from culamp_b200 import datasets as D, kernels as K
    ref = json.load(open(os.path.join(golden_dir, "winf_reference.json")))
    X = T(torch_cuda, D.grid_coords(64, 64, scaled=False))
    for key, want in ref["winf"].items():
        p = math.inf if key == "inf" else float(key)
        _, w = K.max_logsumexp_spp_ct(X, X, p)
        assert w == want


def test_large_pass_properties(torch_cuda):
    """Full-size (n = m = 65536, d = 3) size-independent checks: after a column
    update the column masses equal c exactly (up to FP32-exp rounding), and the
    LSE is invariant to a constant shift of the potentials."""
    from culamp_b200 import datasets as D, kernels as K
    x, y, r, c = D.rgb_instance(65536, 65536)
    X, Y, R, Cc = (T(torch_cuda, v) for v in (x, y, r, c))
    _, winf = K.max_logsumexp_spp_ct(X, Y, 2.0)
    phi = torch_cuda.zeros(65536, dtype=torch_cuda.float64, device="cuda")
    psi = K.warp_logsumexp_ct_fused(Y, X, Cc, phi, 1e-3, winf, 2.0)   # column update
    res_c, _ = K.residual_opt(Y, X, Cc, psi, phi, 1e-3, winf, 2.0)
    assert float(res_c.abs().sum()) < 1e-5
    psi2 = K.warp_logsumexp_ct_fused(Y, X, Cc, phi + 123.25, 1e-3, winf, 2.0)
    assert float((psi2 + 123.25 - psi).abs().max()) < 1e-6
