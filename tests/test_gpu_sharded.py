"""Row-sharded Sinkhorn on the GPU: several row blocks driven by one process
through the real pass kernels and culamp_lse_combine must match the
single-GPU solver and the FP64 oracle: potentials gauge-fixed within 5e-6 after
a fixed number of iterations (the FP32-exp rounding differs with the row
split), and the same stopping iteration at a tolerance the residual crosses
decisively. (At epsilon = 1e-6 with a check every iteration the residual
decays slowly through the threshold, and ~1e-9 of rounding moves the crossing
by a few iterations between any two split geometries.) A one-rank NCCL process
group exercises the collective path."""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ATOL = 5e-6


def gauge(v, w):
    v = np.asarray(v, dtype=np.float64)
    return v - np.dot(w, v) / np.sum(w)


def test_lse_combine_matches_numpy():
    import torch
    import culamp_b200  # noqa: F401  (loads the library)
    from culamp_b200.sharded import CudaOps
    g = np.random.default_rng(0)
    parts = g.normal(0, 30, (3, 1000))
    got = CudaOps().combine(torch.as_tensor(parts, device="cuda")).cpu().numpy()
    a = -parts
    want = -(a.max(0) + np.log(np.exp(a - a.max(0)).sum(0)))
    np.testing.assert_allclose(got, want, rtol=1e-14, atol=1e-12)


def _blocks_run(shards, p, frequency, args):
    import torch
    import culamp_b200 as cb
    from culamp_b200 import datasets as D
    from culamp_b200.sharded import shard_rows, sharded_sinkhorn
    x, y, r, c = D.grid_instance(24, 24, "mixture")
    X, Y, R, Cc = (torch.as_tensor(v, device="cuda") for v in (x, y, r, c))
    blocks = [shard_rows(x.shape[0], shards, k) for k in range(shards)]
    res = sharded_sinkhorn([X[s:e].contiguous() for s, e in blocks], [R[s:e].contiguous() for s, e in blocks],
                           Y, Cc, args, frequency=frequency, p=p)
    one = cb.solve_sinkhorn(X, Y, R, Cc, args, frequency, p)
    return (x, y, r, c), res, one


@pytest.mark.parametrize("p", [2.0, 1.0])
@pytest.mark.parametrize("shards", [1, 2, 3])
def test_row_blocks_match_single_solver_and_oracle(oracle, p, shards):
    """Fixed iteration count: potentials against the single-GPU solver and the oracle."""
    import culamp_b200 as cb
    a = cb.EOTArgs(eta_p=1e-2, epsilon=0.0, itermax=150, verbose=False)
    (x, y, r, c), res, one = _blocks_run(shards, p, 10, a)
    phi = np.concatenate([v.cpu().numpy() for v in res.phi])
    assert res.iterations == one.iterations == 150 and res.stopped == 2
    assert res.winf == one.winf
    np.testing.assert_allclose(gauge(phi, r), gauge(one.phi.cpu().numpy(), r), atol=ATOL, rtol=0)
    np.testing.assert_allclose(gauge(res.psi.cpu().numpy(), c), gauge(one.psi.cpu().numpy(), c), atol=ATOL, rtol=0)
    wphi, wpsi, wst, _ = oracle.sinkhorn_kernel(x, y, r, c, oracle.Args(eta_p=1e-2, epsilon=0.0, itermax=150,
                                                                        verbose=False), frequency=10, p=p)
    np.testing.assert_allclose(gauge(phi, r), gauge(wphi, r), atol=ATOL, rtol=0)
    np.testing.assert_allclose(gauge(res.psi.cpu().numpy(), c), gauge(wpsi, c), atol=ATOL, rtol=0)
    assert res.objective == pytest.approx(wst.objective, rel=1e-5)
    assert res.residual == pytest.approx(wst.residual, rel=1e-3)


@pytest.mark.parametrize("p,frequency", [(2.0, 5), (1.0, 1)])
@pytest.mark.parametrize("shards", [2, 3])
def test_row_blocks_stop_at_the_oracle_iteration(oracle, p, frequency, shards):
    """Stopping rule at a tolerance the residual crosses decisively (epsilon
    6e-4): the same check iteration as the oracle and the single-GPU solver."""
    import culamp_b200 as cb
    a = cb.EOTArgs(eta_p=1e-2, epsilon=6e-4, itermax=3000, verbose=False)
    (x, y, r, c), res, one = _blocks_run(shards, p, frequency, a)
    _, _, wst, _ = oracle.sinkhorn_kernel(x, y, r, c, oracle.Args(eta_p=1e-2, epsilon=6e-4, itermax=3000,
                                                                 verbose=False), frequency=frequency, p=p)
    assert res.stopped == one.stopped == 1 and wst.stopped == 1
    assert res.iterations == one.iterations == wst.iterations
    assert res.num_iter == one.num_iter == wst.num_iter


@pytest.mark.parametrize("p,eta_p", [(2.0, 1e-2), (1.0, 1e-2), (2.0, 0.0)])
@pytest.mark.parametrize("shards", [2, 3])
def test_row_blocks_lamp_match_single_solver_and_oracle(oracle, p, eta_p, shards):
    """Row-sharded LAMP through the real passes (partial column masses summed
    over the blocks): nu / theta against the single-GPU LAMP and the oracle,
    the log rows (marginal, objective, primal, dual) and eta_t exactly."""
    import torch
    import culamp_b200 as cb
    from culamp_b200 import datasets as D
    from culamp_b200.sharded import shard_rows, sharded_lamp
    x, y, r, c = D.grid_instance(20, 20, "mixture")
    X, Y, R, Cc = (torch.as_tensor(v, device="cuda") for v in (x, y, r, c))
    blocks = [shard_rows(x.shape[0], shards, k) for k in range(shards)]
    a = cb.EOTArgs(eta_p=eta_p, epsilon=1e-12, itermax=80, verbose=True, B=1.1)
    res = sharded_lamp([X[s:e].contiguous() for s, e in blocks], [R[s:e].contiguous() for s, e in blocks],
                       Y, Cc, a, frequency=10, p=p)
    one = cb.solve_lamp(X, Y, R, Cc, a, 10, p)
    nu, _, _, theta, wst, log = oracle.lamp_kernel(x, y, r, c, oracle.Args(eta_p=eta_p, epsilon=1e-12, itermax=80,
                                                                           verbose=True, B=1.1), frequency=10, p=p)
    assert res.iterations == one.iterations == wst.iterations
    assert res.eta_t == one.eta_t == wst.eta_t
    got_nu = res.nu.cpu().numpy()
    # nu averages the theta iterates; the FP32-exp column sums of a different
    # row split round differently (a few 1e-6 after 80 iterations)
    np.testing.assert_allclose(gauge(got_nu, c), gauge(one.nu.cpu().numpy(), c), atol=5e-6, rtol=0)
    np.testing.assert_allclose(gauge(got_nu, c), gauge(nu, c), atol=5e-6, rtol=0)
    # theta's mirror step divides the column residual by eta_mu_j = (c_j + alpha/n) / tau_mu,
    # about 1/m, so the ~1e-7 rounding of FP32-exp column sums reaches theta amplified
    # by ~m (here 400): 5e-5
    np.testing.assert_allclose(res.theta.cpu().numpy(), theta, atol=5e-5, rtol=0)
    np.testing.assert_allclose(res.theta.cpu().numpy(), one.theta.cpu().numpy(), atol=5e-5, rtol=0)
    got = np.array(res.log)
    want = np.array([row[1:6] for row in log])
    assert got.shape == want.shape and np.array_equal(got[:, 0], want[:, 0])
    np.testing.assert_allclose(got[:, 1], want[:, 1], rtol=1e-3, atol=1e-9)
    # objective, primal, dual: the dual is evaluated at theta, which carries the
    # 5e-5 above
    np.testing.assert_allclose(got[:, 2:], want[:, 2:], rtol=1e-4, atol=5e-5)


def test_single_rank_nccl_group(tmp_path):
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    script = f"""
import os, sys, json, datetime
sys.path.insert(0, {os.path.join(root, 'culamp.jl_b200')!r})
import torch, torch.distributed as dist
import culamp_b200 as cb
from culamp_b200 import datasets as D
from culamp_b200.sharded import sharded_sinkhorn
os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT="29561")
dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60))
torch.cuda.set_device(0)
x, y, r, c = (torch.as_tensor(v, device="cuda") for v in D.grid_instance(16, 16, "mixture"))
a = cb.EOTArgs(eta_p=1e-2, epsilon=6e-4, itermax=2000, verbose=False)
res = sharded_sinkhorn([x[:100].contiguous(), x[100:].contiguous()], [r[:100].contiguous(), r[100:].contiguous()], y, c, a, 5, 2.0)
one = cb.solve_sinkhorn(x, y, r, c, a, 5, 2.0)
print(json.dumps([res.iterations, one.iterations, res.stopped]))
dist.destroy_process_group()
"""
    out = subprocess.run([sys.executable, "-c", script], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    it, one_it, stopped = eval(out.stdout.strip().splitlines()[-1])
    assert it == one_it and stopped == 1


@pytest.mark.parametrize("itermax,eps", [(57, 0.0), (5000, 6e-6)])
def test_graph_replayed_blocks_equal_the_eager_loop(itermax, eps):
    """The default loop captures the `frequency` iterations between checks in
    one CUDA graph; it must give exactly what the eager loop gives (same
    kernels on the same buffers): potentials bit for bit, counters, stop."""
    import torch
    import culamp_b200 as cb
    from culamp_b200 import datasets as D
    from culamp_b200.sharded import shard_rows, sharded_sinkhorn
    x, y, r, c = D.grid_instance(24, 24, "mixture")
    X, Y, R, Cc = (torch.as_tensor(v, device="cuda") for v in (x, y, r, c))
    blocks = [shard_rows(x.shape[0], 3, k) for k in range(3)]
    xs = [X[s:e].contiguous() for s, e in blocks]
    rs = [R[s:e].contiguous() for s, e in blocks]
    a = cb.EOTArgs(eta_p=1e-2, epsilon=eps, itermax=itermax, verbose=False)
    g = sharded_sinkhorn(xs, rs, Y, Cc, a, frequency=10, p=2.0)
    e = sharded_sinkhorn(xs, rs, Y, Cc, a, frequency=10, p=2.0, graph=False)
    assert (g.iterations, g.num_iter, g.stopped) == (e.iterations, e.num_iter, e.stopped)
    for pg, pe in zip(g.phi, e.phi):
        assert torch.equal(pg, pe)
    assert torch.equal(g.psi, e.psi)
    if eps > 0:
        assert g.stopped == 1
