"""The persistent Sinkhorn loop (csrc/persist.cu: every iteration of a small
solve in one cooperative launch) against the pass-per-launch graph loop
(CULAMP_FLAG_NO_PERSIST), SinkhornKernel.jl:477-559.

The two run the same arithmetic per term (fixed-reference exponent, FP32 ex2
sums) in different summation orders, so potentials agree to the log-sum-exp
rounding (~1e-7 relative per pass); counters, check iterations, stop reasons
and log rows agree exactly. Parity against the FP64 oracle on the 64x64-grid
workload is tests/test_gpu_config2.py, which runs this loop by default.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _np(t):
    return t.cpu().numpy() if hasattr(t, "cpu") else np.asarray(t)


def close(got, want, rel=2e-6):
    got, want = _np(got), _np(want)
    assert np.abs(got - want).max() <= rel * max(1.0, np.abs(want).max())


def both(x, y, r, c, a, freq, p, **kw):
    import culamp_b200 as cb
    fl = kw.pop("flags", 0)
    per = cb.solve_sinkhorn(x, y, r, c, a, freq, p, flags=fl, **kw)
    ref = cb.solve_sinkhorn(x, y, r, c, a, freq, p, flags=fl | cb.FLAG_NO_PERSIST, **kw)
    return per, ref


def same_control(per, ref):
    assert per.iterations == ref.iterations and per.num_iter == ref.num_iter
    assert per.stopped == ref.stopped
    assert len(per.log) == len(ref.log)
    g = np.array([row[1:6] for row in per.log]) if per.log else np.zeros((0, 5))
    w = np.array([row[1:6] for row in ref.log]) if ref.log else np.zeros((0, 5))
    assert np.array_equal(g[:, 0], w[:, 0])
    # FP32 term sums in another order: residuals to the FP32 floor, the cost
    # moment (FP32 products) and the dual value to ~1e-7 relative
    np.testing.assert_allclose(g[:, 1], w[:, 1], rtol=1e-3, atol=5e-8)      # L1 residual
    np.testing.assert_allclose(g[:, 2], w[:, 2], rtol=1e-6)                 # transport cost
    np.testing.assert_allclose(g[:, 4], w[:, 4], rtol=1e-6)                 # dual value


@pytest.fixture(scope="module")
def grid():
    import torch
    from culamp_b200 import datasets as D
    return tuple(torch.as_tensor(v, device="cuda") for v in D.grid_instance(64, 64, "mixture"))


@pytest.mark.parametrize("eta_p", [1e-3, 1e-4])
@pytest.mark.parametrize("p", [1.0, 2.0, math.inf])
def test_fixed_iterations_match_graph_loop(grid, p, eta_p):
    import culamp_b200 as cb
    a = cb.EOTArgs(eta_p=eta_p, epsilon=0.0, itermax=100, verbose=True)
    per, ref = both(*grid, a, 10, p)
    same_control(per, ref)
    close(per.phi, ref.phi)
    close(per.psi, ref.psi)
    assert per.objective == pytest.approx(ref.objective, rel=1e-6)


def test_stops_where_the_graph_loop_stops(grid):
    import culamp_b200 as cb
    a = cb.EOTArgs(eta_p=1e-3, epsilon=6e-6, itermax=20000, verbose=True)
    per, ref = both(*grid, a, 10, 2.0)
    assert per.stopped == 1 and ref.stopped == 1
    same_control(per, ref)
    print(f"4096 solve: persistent {per.elapsed_ms:.2f} ms, graph loop {ref.elapsed_ms:.2f} ms, "
          f"{per.iterations} iterations")
    assert per.residual <= 1e-6


@pytest.mark.parametrize("itermax,freq", [(37, 10), (1, 10), (25, 1), (40, 7)])
def test_itermax_and_cadence(grid, itermax, freq):
    import culamp_b200 as cb
    a = cb.EOTArgs(eta_p=1e-2, epsilon=0.0, itermax=itermax, verbose=True)
    per, ref = both(*grid, a, freq, 2.0)
    same_control(per, ref)
    close(per.phi, ref.phi)


def test_tmax_stops_after_the_first_iteration(grid):
    import culamp_b200 as cb
    a = cb.EOTArgs(eta_p=1e-3, epsilon=0.0, itermax=1000, verbose=True, tmax=0.0)
    per, ref = both(*grid, a, 10, 2.0)
    assert per.iterations == ref.iterations == 1
    same_control(per, ref)


@pytest.mark.parametrize("n,m,d", [(5, 7, 3), (1000, 3000, 3), (2500, 1200, 2), (777, 1500, 1),
                                   (8192, 8192, 3), (8192, 16384, 3)])
def test_ragged_shapes(n, m, d):
    import torch
    import culamp_b200 as cb
    g = np.random.Generator(np.random.PCG64(n * 31 + m))
    x = torch.as_tensor(g.uniform(0, 1, (n, d)), device="cuda")
    y = torch.as_tensor(g.uniform(0, 1, (m, d)), device="cuda")
    r = torch.as_tensor(g.uniform(0.5, 1.0, n), device="cuda")
    c = torch.as_tensor(g.uniform(0.5, 1.0, m), device="cuda")
    r, c = r / r.sum(), c / c.sum()
    a = cb.EOTArgs(eta_p=5e-3, epsilon=0.0, itermax=30, verbose=True)
    per, ref = both(x, y, r, c, a, 10, 2.0)
    same_control(per, ref)
    close(per.phi, ref.phi)
    close(per.psi, ref.psi)


def test_far_starting_point_takes_the_exact_rows(grid):
    """A starting potential far from the solution puts every row outside the
    fixed-reference window at the first iteration: those rows are recomputed
    with the FP64 online log-sum-exp, and the solve continues identically."""
    import torch
    import culamp_b200 as cb
    x, y, r, c = grid
    phi0 = torch.full_like(r, 400.0)
    psi0 = torch.full_like(c, -900.0)
    a = cb.EOTArgs(eta_p=1e-3, epsilon=0.0, itermax=20, verbose=True)
    per, ref = both(x, y, r, c, a, 10, 2.0, phi0=phi0, psi0=psi0)
    same_control(per, ref)
    close(per.phi, ref.phi)
    close(per.psi, ref.psi)


def test_annealed_solve_uses_the_same_loop(grid):
    import culamp_b200 as cb
    kw = dict(eta_p=4e-3, epsilon=1e-3, anneal_mult=0.5, itermax=60, verbose=False)
    per = cb.solve_annealed_sinkhorn(*grid, cb.EOTArgs(**kw), frequency=10, p=2.0)
    ref = cb.solve_annealed_sinkhorn(*grid, cb.EOTArgs(**kw), frequency=10, p=2.0, flags=cb.FLAG_NO_PERSIST)
    assert per.iterations == ref.iterations and per.num_iter == ref.num_iter
    close(per.phi, ref.phi)


def test_ladder_in_the_persistent_loop(grid):
    """CULAMP_FLAG_LADDER in the persistent loop: FP32-exponent row and column
    passes until a check's FP64 residual is within 32x the tolerance, then the
    FP64 passes; the stop is decided by FP64 checks only, and the result is the
    FP64 form's fixed point to the solve's accuracy."""
    import culamp_b200 as cb
    x, y, r, c = grid
    a = cb.EOTArgs(eta_p=1e-3, epsilon=6e-6, itermax=20000, verbose=True)
    f64 = cb.solve_sinkhorn(x, y, r, c, a, 10, 2.0)
    lad = cb.solve_sinkhorn(x, y, r, c, a, 10, 2.0, flags=cb.FLAG_LADDER)
    glad = cb.solve_sinkhorn(x, y, r, c, a, 10, 2.0, flags=cb.FLAG_LADDER | cb.FLAG_NO_PERSIST)
    print(f"4096 ladder: persistent {lad.elapsed_ms:.2f} ms / {lad.iterations} it, graph loop "
          f"{glad.elapsed_ms:.2f} ms / {glad.iterations} it, FP64 persistent {f64.elapsed_ms:.2f} ms / "
          f"{f64.iterations} it")
    for res in (lad, glad):
        assert res.stopped == 1 and res.residual <= 1e-6
        rl, cl = cb.marginal_error_fp64(x, y, r, c, res.phi, res.psi, 1e-3, res.winf, 2.0)
        assert rl <= 1e-6 and cl <= 1e-6
        assert abs(res.iterations - f64.iterations) <= 0.05 * f64.iterations + 20
    rr = _np(r)
    k0 = np.dot(rr, _np(f64.phi)) / rr.sum()
    k1 = np.dot(rr, _np(lad.phi)) / rr.sum()
    scale = max(1.0, np.abs(_np(f64.phi)).max())
    assert np.abs((_np(lad.phi) - k1) - (_np(f64.phi) - k0)).max() <= 1e-5 * scale
    assert np.abs((_np(lad.psi) + k1) - (_np(f64.psi) + k0)).max() <= 1e-5 * scale


# ----------------------------------------------------------------- LAMP

def lamp_both(x, y, r, c, a, freq, p, flags=0):
    import culamp_b200 as cb
    per = cb.solve_lamp(x, y, r, c, a, freq, p, flags=flags)
    ref = cb.solve_lamp(x, y, r, c, a, freq, p, flags=flags | cb.FLAG_NO_PERSIST)
    return per, ref


def lamp_same(per, ref):
    """Counters, eta_t (a function of the iteration count: bit-exact), the
    check rows; theta / nu to the FP32 term-sum rounding amplified by the
    mirror step's 1 / eta_mu_j (~m), as for the sharded LAMP."""
    assert per.iterations == ref.iterations and per.stopped == ref.stopped
    assert per.eta_t == ref.eta_t and per.s_t == ref.s_t
    assert len(per.log) == len(ref.log)
    if per.log:
        g = np.array([row[1:6] for row in per.log])
        w = np.array([row[1:6] for row in ref.log])
        assert np.array_equal(g[:, 0], w[:, 0])
        np.testing.assert_allclose(g[:, 1], w[:, 1], rtol=1e-3, atol=2e-7)     # marginal residual
        np.testing.assert_allclose(g[:, 2], w[:, 2], rtol=1e-5, atol=1e-7)      # cost
        np.testing.assert_allclose(g[:, 3:5], w[:, 3:5], rtol=1e-4, atol=1e-6)  # primal, dual
    np.testing.assert_allclose(_np(per.theta), _np(ref.theta), rtol=0, atol=5e-5)
    np.testing.assert_allclose(_np(per.nu), _np(ref.nu), rtol=0, atol=5e-5)
    assert per.objective == pytest.approx(ref.objective, rel=1e-5)


@pytest.mark.parametrize("eta_p", [1e-3, 1e-4])
@pytest.mark.parametrize("p", [1.0, 2.0, math.inf])
def test_lamp_fixed_iterations_match_graph_loop(grid, p, eta_p):
    import culamp_b200 as cb
    a = cb.EOTArgs(eta_p=eta_p, epsilon=0.0, itermax=60, verbose=True, B=1.1)
    per, ref = lamp_both(*grid, a, 10, p)
    lamp_same(per, ref)


@pytest.mark.parametrize("flags", ["full", "marginal"])
def test_lamp_stops_where_the_graph_loop_stops(grid, flags):
    import culamp_b200 as cb
    fl = cb.FLAG_CHECK_ALWAYS | (cb.FLAG_MARGINAL_ONLY if flags == "marginal" else 0)
    # the full rule's gap does not close to 1e-6 on this instance: both loops
    # run to itermax there, with the same check rows
    a = cb.EOTArgs(eta_p=1e-3, epsilon=6e-6, itermax=2000, verbose=False, B=1.1)
    per, ref = lamp_both(*grid, a, 10, 2.0, fl)
    print(f"4096 LAMP ({flags}): persistent {per.elapsed_ms:.2f} ms, graph loop {ref.elapsed_ms:.2f} ms, "
          f"{per.iterations} iterations")
    lamp_same(per, ref)


@pytest.mark.parametrize("n,m,d", [(5, 7, 3), (1000, 3000, 3), (2500, 1200, 2), (8192, 8192, 3)])
def test_lamp_ragged_shapes(n, m, d):
    import torch
    import culamp_b200 as cb
    g = np.random.Generator(np.random.PCG64(n * 37 + m))
    x = torch.as_tensor(g.uniform(0, 1, (n, d)), device="cuda")
    y = torch.as_tensor(g.uniform(0, 1, (m, d)), device="cuda")
    r = torch.as_tensor(g.uniform(0.5, 1.0, n), device="cuda")
    c = torch.as_tensor(g.uniform(0.5, 1.0, m), device="cuda")
    r, c = r / r.sum(), c / c.sum()
    a = cb.EOTArgs(eta_p=5e-3, epsilon=0.0, itermax=25, verbose=True, B=1.1)
    per, ref = lamp_both(x, y, r, c, a, 5, 2.0)
    lamp_same(per, ref)


def test_lamp_itermax_and_tmax(grid):
    import culamp_b200 as cb
    for kw in (dict(itermax=7), dict(itermax=1000, tmax=0.0)):
        a = cb.EOTArgs(eta_p=1e-2, epsilon=0.0, verbose=True, B=1.1, **kw)
        per, ref = lamp_both(*grid, a, 3, 2.0)
        lamp_same(per, ref)
