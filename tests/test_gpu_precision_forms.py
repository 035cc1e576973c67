"""The FP32-exponent form and the FP32 -> FP64 precision ladder of Sinkhorn
(SinkhornKernel.jl:477-559, p = 2, d <= 3) on the 64x64-grid workload.

* CULAMP_FLAG_FORM_FP32 runs the chosen form's engine (tiling, fixed row
  reference, graph loop) with every exponent formed in FP32. Its check passes
  stay FP64, so its logged L1 residuals are exact for the potentials it
  reached. At a fixed iteration count its potentials follow the FP64-exponent
  form within the FP32 rounding of the exponent (~|g| 2^-24 per term, |g|
  up to ~1e3 in log2 units at eta_p = 1e-3): checked at 1e-4 of max |phi|
  after removing the Sinkhorn gauge.
* CULAMP_FLAG_LADDER switches from FP32 to FP64 passes on the device; the
  solve stops on the FP64 check only, so the bench workload's 1e-6 L1 holds
  under an independent FP64 re-evaluation of both marginals (exp included).
* Both flags leave costs other than the squared one bit-identical to the
  default form (p = Inf iterates on the squared cost, SinkhornKernel.jl:518-520,
  so it takes them too).
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev_inst():
    import torch
    from culamp_b200 import datasets as D
    return tuple(torch.as_tensor(v, device="cuda") for v in D.grid_instance(64, 64, "mixture"))


def _np(t):
    return t.cpu().numpy() if hasattr(t, "cpu") else np.asarray(t)


def gauge_free(phi, psi, r):
    """Sinkhorn's potentials are defined up to (phi + k, psi - k)."""
    phi, psi = _np(phi), _np(psi)
    k = np.dot(_np(r), phi) / np.sum(_np(r))
    return phi - k, psi + k


@pytest.mark.parametrize("eta_p", [1e-3, 1e-4])
def test_fp32_form_follows_fp64_form(dev_inst, eta_p):
    import culamp_b200 as cb
    x, y, r, c = dev_inst
    a = cb.EOTArgs(eta_p=eta_p, epsilon=0.0, itermax=100, verbose=True)
    ref = cb.solve_sinkhorn(x, y, r, c, a, frequency=10, p=2.0)
    f32 = cb.solve_sinkhorn(x, y, r, c, a, frequency=10, p=2.0, flags=cb.FLAG_FORM_FP32)
    assert f32.iterations == ref.iterations and f32.num_iter == ref.num_iter
    p0, q0 = gauge_free(ref.phi, ref.psi, r)
    p1, q1 = gauge_free(f32.phi, f32.psi, r)
    scale = max(1.0, np.abs(p0).max(), np.abs(q0).max())
    err = max(np.abs(p1 - p0).max(), np.abs(q1 - q0).max()) / scale
    print(f"eta_p={eta_p}: FP32-form potential error {err:.3e} of max |potential| {scale:.3e}")
    assert err <= 1e-4
    assert not np.array_equal(_np(f32.phi), _np(ref.phi))        # the FP32 kernels ran
    # the FP64 check passes log the same check iterations, residuals close
    g = np.array([row[1:3] for row in f32.log])
    w = np.array([row[1:3] for row in ref.log])
    assert np.array_equal(g[:, 0], w[:, 0])
    np.testing.assert_allclose(g[:, 1], w[:, 1], rtol=0.2, atol=1e-8)


def test_ladder_reaches_tolerance_certified_in_fp64(oracle, dev_inst):
    import culamp_b200 as cb
    x, y, r, c = dev_inst
    kw = dict(eta_p=1e-3, epsilon=6e-6, itermax=20000, verbose=True)
    ref = cb.solve_sinkhorn(x, y, r, c, cb.EOTArgs(**kw), frequency=10, p=2.0, flags=cb.FLAG_FORM_FP64)
    lad = cb.solve_sinkhorn(x, y, r, c, cb.EOTArgs(**kw), frequency=10, p=2.0, flags=cb.FLAG_LADDER)
    assert ref.stopped == 1 and lad.stopped == 1
    assert lad.residual <= 1e-6
    rl, cl = cb.marginal_error_fp64(x, y, r, c, lad.phi, lad.psi, 1e-3, lad.winf, 2.0)
    print(f"ladder: {lad.iterations} iterations ({ref.iterations} FP64), {lad.elapsed_ms:.2f} ms "
          f"({ref.elapsed_ms:.2f} ms FP64), FP64 marginal L1 {rl:.3e} / {cl:.3e}")
    assert rl <= 1e-6 and cl <= 1e-6
    # the iteration count stays within a few checks of the FP64 form's
    assert abs(lad.iterations - ref.iterations) <= 0.1 * ref.iterations + 20
    # both stop at the same fixed point to the solve's own accuracy
    p0, q0 = gauge_free(ref.phi, ref.psi, r)
    p1, q1 = gauge_free(lad.phi, lad.psi, r)
    scale = max(1.0, np.abs(p0).max())
    assert np.abs(p1 - p0).max() <= 1e-5 * scale
    assert np.abs(q1 - q0).max() <= 1e-5 * scale
    # the last logged check and the post-loop residual pass (residual_opt!,
    # SinkhornKernel.jl:541-544) evaluate the same potentials; their FP32 term
    # sums may run in different orders (persistent loop vs pass engine)
    res = [row[2] for row in lad.log]
    assert res[-1] <= 1e-6
    assert res[-1] == pytest.approx(lad.residual, rel=5e-2)


@pytest.mark.parametrize("p", [1.0, 3.0])
@pytest.mark.parametrize("flag", ["FLAG_FORM_FP32", "FLAG_LADDER"])
def test_flags_leave_other_costs_unchanged(dev_inst, p, flag):
    import culamp_b200 as cb
    x, y, r, c = dev_inst
    a = cb.EOTArgs(eta_p=1e-3, epsilon=0.0, itermax=30, verbose=True)
    ref = cb.solve_sinkhorn(x, y, r, c, a, frequency=10, p=p)
    got = cb.solve_sinkhorn(x, y, r, c, a, frequency=10, p=p, flags=getattr(cb, flag))
    assert np.array_equal(_np(got.phi), _np(ref.phi))
    assert np.array_equal(_np(got.psi), _np(ref.psi))
    assert got.iterations == ref.iterations and got.residual == ref.residual


def test_ladder_without_a_tolerance_switches_on_stall(dev_inst):
    """epsilon = 0 never reaches the switch threshold: the stall rule moves the
    ladder to FP64 once the FP32 iteration stops gaining, and the residuals of
    the late checks match the FP64 form's (a ladder stuck in FP32 would show
    its floor instead)."""
    import culamp_b200 as cb
    x, y, r, c = dev_inst
    a = cb.EOTArgs(eta_p=1e-3, epsilon=0.0, itermax=2500, verbose=True)
    ref = cb.solve_sinkhorn(x, y, r, c, a, frequency=10, p=2.0)
    lad = cb.solve_sinkhorn(x, y, r, c, a, frequency=10, p=2.0, flags=cb.FLAG_LADDER)
    f32 = cb.solve_sinkhorn(x, y, r, c, a, frequency=10, p=2.0, flags=cb.FLAG_FORM_FP32)
    print(f"2500 iterations: residual FP64 {ref.residual:.3e}, ladder {lad.residual:.3e}, "
          f"FP32 {f32.residual:.3e}")
    assert lad.residual <= 2.0 * ref.residual + 1e-12


def test_fp32_pass_against_fp64_pass():
    """culamp_lse_rows_sk_form (FP32 exponents) against culamp_lse_rows_sk on a
    20000 x 18000 RGB instance after a few Sinkhorn iterations: the FP32 pass's
    error is the exponent rounding, a few 2^-24 of the largest exponent term
    (|alpha C| + |psi| ~ 3e3 here), so <= 1e-3 absolute in log units."""
    import torch
    import culamp_b200 as cb
    from culamp_b200 import datasets as D, kernels as K
    x, y, r, c = (torch.as_tensor(v, device="cuda") for v in D.rgb_instance(20000, 18000))
    s = cb.solve_sinkhorn(x, y, r, c, cb.EOTArgs(eta_p=1e-3, epsilon=0.0, itermax=20, verbose=False),
                          frequency=10, p=2.0)
    want = s.phi.clone()
    K.warp_logsumexp_ct_fused(x, y, r, s.psi, 1e-3, s.winf, 2.0, out=want)
    got = s.phi.clone()
    K.warp_logsumexp_ct_fused(x, y, r, s.psi, 1e-3, s.winf, 2.0, out=got, flags=cb.FLAG_FORM_FP32)
    err = (got - want).abs().max().item()
    print(f"FP32 pass: max |error| {err:.3e} (|phi| <= {want.abs().max().item():.3e})")
    assert err <= 1e-3
    assert err > 0.0                                        # the FP32 kernel ran
    # a stale hint (zeros) takes the FP64 fallbacks and gives the same result
    cold = torch.zeros_like(want)
    K.warp_logsumexp_ct_fused(x, y, r, s.psi, 1e-3, s.winf, 2.0, out=cold, flags=cb.FLAG_FORM_FP32)
    assert (cold - want).abs().max().item() <= 1e-3


def test_fp32_pass_rejects_other_costs():
    import torch
    import culamp_b200 as cb
    from culamp_b200 import kernels as K
    x = torch.rand(64, 3, dtype=torch.float64, device="cuda")
    r = torch.full((64,), 1 / 64, dtype=torch.float64, device="cuda")
    out = torch.zeros(64, dtype=torch.float64, device="cuda")
    with pytest.raises(cb.CulampError):
        K.warp_logsumexp_ct_fused(x, x, r, torch.zeros_like(r), 1e-2, 1.0, 1.0, out=out,
                                  flags=cb.FLAG_FORM_FP32)
    x5 = torch.rand(64, 5, dtype=torch.float64, device="cuda")
    with pytest.raises(cb.CulampError):
        K.warp_logsumexp_ct_fused(x5, x5, r, torch.zeros_like(r), 1e-2, 1.0, 2.0, out=out,
                                  flags=cb.FLAG_FORM_FP32)


def test_default_form_takes_the_ladder_above_16384_squared():
    """At n m >= 16384^2 the default is the ladder: same result as
    FLAG_LADDER bit for bit, and FLAG_FORM_FP64 gives the FP64 form; both
    certified to 1e-6 by the FP64 re-check."""
    import torch
    import culamp_b200 as cb
    from culamp_b200 import datasets as D
    x, y, r, c = (torch.as_tensor(v, device="cuda") for v in D.rgb_instance(16384, 16384))
    a = cb.EOTArgs(eta_p=1e-3, epsilon=6e-6, itermax=5000, verbose=False)
    dflt = cb.solve_sinkhorn(x, y, r, c, a, frequency=25, p=2.0)
    lad = cb.solve_sinkhorn(x, y, r, c, a, frequency=25, p=2.0, flags=cb.FLAG_LADDER)
    f64 = cb.solve_sinkhorn(x, y, r, c, a, frequency=25, p=2.0, flags=cb.FLAG_FORM_FP64)
    print(f"16384: default {dflt.iterations} it {dflt.elapsed_ms:.1f} ms, FP64 form "
          f"{f64.iterations} it {f64.elapsed_ms:.1f} ms")
    assert torch.equal(dflt.phi, lad.phi) and dflt.iterations == lad.iterations
    for res in (dflt, f64):
        assert res.stopped == 1
        rl, cl = cb.marginal_error_fp64(x, y, r, c, res.phi, res.psi, 1e-3, res.winf, 2.0)
        assert rl <= 1e-6 and cl <= 1e-6


def test_lamp_ladder_reaches_tolerance_certified_in_fp64(dev_inst):
    """LAMP (MirrorProxKernel.jl:1019-1132) with the precision ladder: the
    logZ and column passes in FP32 exponents until a check's FP64 marginal
    residual is within 32x of the tolerance; the checks themselves (cost
    moment, dual value) stay FP64, so the stop is FP64-decided. The plan's
    column marginal, recomputed in FP64 from the returned Sinkhorn-form
    potentials (phi = log r - logZ, psi = -nu / eta_t), meets the tolerance."""
    import culamp_b200 as cb
    x, y, r, c = dev_inst
    a = cb.EOTArgs(eta_p=1e-3, epsilon=6e-6, itermax=100_000, verbose=False, B=1.1)
    fl = cb.FLAG_CHECK_ALWAYS | cb.FLAG_MARGINAL_ONLY
    ref = cb.solve_lamp(x, y, r, c, a, 10, 2.0, flags=fl)
    lad = cb.solve_lamp(x, y, r, c, a, 10, 2.0, flags=fl | cb.FLAG_LADDER)
    print(f"LAMP ladder: {lad.iterations} iterations ({ref.iterations} FP64), {lad.elapsed_ms:.2f} ms "
          f"({ref.elapsed_ms:.2f} ms FP64)")
    assert ref.stopped == 1 and lad.stopped == 1
    assert lad.residual <= 1e-6
    assert abs(lad.iterations - ref.iterations) <= 0.1 * ref.iterations + 20
    # Sinkhorn form of the LAMP plan: psi = -nu / eta_t, cost scale s / (2 W eta_t)
    rl, cl = cb.marginal_error_fp64(x, y, r, c, lad.phi, -lad.nu / lad.eta_t, 1.0,
                                    2.0 * lad.winf * lad.eta_t / lad.s_t, 2.0)
    assert cl <= 1.5e-6 and rl <= 1e-6
    # the FP32 phase moves the iteration LAMP stops at, and with it eta_t (a
    # function of the iteration count) and the returned plan's entropy: the
    # transport cost agrees to ~1e-3, not to the FP64 form's 1e-5 -- which is
    # why the LAMP ladder is opt-in
    assert lad.objective == pytest.approx(ref.objective, rel=3e-3)


def test_lamp_ladder_needs_checks(dev_inst):
    """Without checks (verbose off, no CHECK_ALWAYS) LAMP cannot leave the FP32
    phase, so the ladder flag leaves it in the FP64 form (the same passes; the
    fixed-reference hints left in the workspace by the previous solve may route
    a few rows through the online loop, so agreement is to FP32-sum rounding,
    far below the FP32-exponent form's ~1e-4)."""
    import culamp_b200 as cb
    x, y, r, c = dev_inst
    a = cb.EOTArgs(eta_p=1e-3, epsilon=6e-6, itermax=40, verbose=False, B=1.1)
    ref = cb.solve_lamp(x, y, r, c, a, 10, 2.0)
    lad = cb.solve_lamp(x, y, r, c, a, 10, 2.0, flags=cb.FLAG_LADDER)
    assert ref.iterations == lad.iterations
    want = _np(ref.nu)
    np.testing.assert_allclose(_np(lad.nu), want, rtol=0, atol=1e-7 * max(1.0, np.abs(want).max()))
