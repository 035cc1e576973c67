"""Row-sharded Sinkhorn driver (culamp_b200.sharded) on CPU: world-size-2
gloo ranks run the driver with the FP64 oracle as their compute ops and must
reproduce the oracle's single-process solve (SinkhornKernel.jl:477-559): same
iteration counts and stopping reason, potentials equal to FP64 rounding (the
column LSE is summed shard by shard, a different order than one pass)."""
import math
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

ATOL = 1e-11


class OracleOps:
    """Host compute of one shard through the C oracle (test infrastructure)."""

    def __init__(self, O):
        self.O = O

    def max_cost(self, x, y, p):
        return self.O.max_cost(x.numpy(), y.numpy(), p)

    def lse_rows(self, out, x, y, marg, pot, reg, winf, p):
        out.copy_(torch.from_numpy(self.O.sk_lse(x.numpy(), y.numpy(), marg.numpy(), pot.numpy(), reg, winf, p)))

    def residual(self, x, y, marg, phi, psi, reg, winf, p):
        res, cost = self.O.sk_residual(x.numpy(), y.numpy(), marg.numpy(), phi.numpy(), psi.numpy(), reg, winf, p)
        return float(np.abs(res).sum()), float(np.sum(cost))

    def spp_lse(self, out, x, y, theta, reg, st, winf, p):
        out.copy_(torch.from_numpy(self.O.spp_lse(x.numpy(), y.numpy(), theta.numpy(), reg, st, winf, p)))

    def col_residual(self, x, y, r, theta, logz, reg, st, winf, p):
        res, cost = self.O.spp_col_residual(x.numpy(), y.numpy(), r.numpy(), theta.numpy(), logz.numpy(),
                                            reg, st, winf, p)
        return torch.from_numpy(res), torch.from_numpy(cost)

    def min_reduce(self, x, y, theta, winf, p):
        return torch.from_numpy(self.O.min_reduce(x.numpy(), y.numpy(), theta.numpy(), winf, p))

    def theta_update(self, theta0, res, c, emu, eta_mu, adjust, minv, maxv):
        return torch.from_numpy(self.O.theta_update(theta0.numpy(), res.numpy(), c.numpy(), emu.numpy(),
                                                    eta_mu, adjust, minv, maxv, 1.0))

    def combine(self, parts):
        a = -parts.numpy()
        mx = a.max(0)
        return torch.from_numpy(-(mx + np.log(np.exp(a - mx).sum(0))))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, case, out_dir, oracle_dir):
    import sys
    import torch.distributed as dist
    sys.path.insert(0, oracle_dir)
    sys.path.insert(0, os.path.join(os.path.dirname(oracle_dir), "culamp.jl_b200"))
    import oracle as O
    from culamp_b200.args import EOTArgs
    from culamp_b200.sharded import shard_rows, sharded_sinkhorn
    O.set_threads(1)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    x, y, r, c = (torch.from_numpy(v) for v in case["data"])
    per_rank = case["shards_per_rank"]
    blocks = [shard_rows(x.shape[0], world * per_rank, rank * per_rank + k) for k in range(per_rank)]
    xs = [x[a:b].contiguous() for a, b in blocks]
    rs = [r[a:b].contiguous() for a, b in blocks]
    if case.get("lamp"):
        from culamp_b200.sharded import sharded_lamp
        a = EOTArgs(eta_p=case["eta_p"], epsilon=case["epsilon"], itermax=case["itermax"], verbose=True,
                    B=case["B"])
        res = sharded_lamp(xs, rs, y, c, a, frequency=case["frequency"], p=case["p"], ops=OracleOps(O),
                           marginal_only=case["marginal_only"])
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), phi=np.concatenate([v.numpy() for v in res.phi]),
                 psi=res.psi.numpy(), nu=res.nu.numpy(), theta=res.theta.numpy(), log=np.array(res.log),
                 stats=np.array([res.iterations, res.stopped, res.residual, res.objective, res.winf,
                                 res.eta_t, res.s_t]))
        dist.destroy_process_group()
        return
    a = EOTArgs(eta_p=case["eta_p"], epsilon=case["epsilon"], itermax=case["itermax"], verbose=False)
    res = sharded_sinkhorn(xs, rs, y, c, a, frequency=case["frequency"], p=case["p"], ops=OracleOps(O))
    np.savez(os.path.join(out_dir, f"rank{rank}.npz"), phi=np.concatenate([v.numpy() for v in res.phi]),
             psi=res.psi.numpy(), stats=np.array([res.iterations, res.num_iter, res.stopped, res.residual,
                                                  res.objective, res.winf]))
    dist.destroy_process_group()


def _run(case, tmp_path, world=2):
    oracle_dir = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle")
    mp.spawn(_worker, args=(world, _free_port(), case, str(tmp_path), oracle_dir), nprocs=world, join=True)
    outs = [np.load(os.path.join(tmp_path, f"rank{k}.npz")) for k in range(world)]
    phi = np.concatenate([o["phi"] for o in outs])
    return phi, outs[0]["psi"], outs[0]["stats"], outs


def _grid(n_side, seed):
    g = np.random.Generator(np.random.PCG64(seed))
    t = np.linspace(0, 1, n_side)
    pts = np.stack(np.meshgrid(t, t, indexing="ij"), -1).reshape(-1, 2)
    w = g.uniform(0.1, 1.0, pts.shape[0])
    return pts, w / w.sum()


@pytest.mark.parametrize("p,frequency,shards_per_rank,n_side", [(2.0, 1, 1, 7), (1.0, 5, 2, 6), (math.inf, 3, 1, 5)])
def test_two_gloo_ranks_match_single_oracle(oracle, tmp_path, p, frequency, shards_per_rank, n_side):
    x, r = _grid(n_side, 0)
    y, c = _grid(n_side + 1, 1)
    x = x[:-3]                                    # ragged: rows do not split evenly
    r = r[:-3] / r[:-3].sum()
    case = {"data": (x, y, r, c), "eta_p": 5e-2, "epsilon": 1e-9, "itermax": 400, "frequency": frequency,
            "p": p, "shards_per_rank": shards_per_rank}
    phi, psi, st, outs = _run(case, tmp_path)
    for o in outs[1:]:
        assert np.array_equal(o["psi"], outs[0]["psi"]) and np.array_equal(o["stats"], outs[0]["stats"])
    args = oracle.Args(eta_p=5e-2, epsilon=1e-9, itermax=400, verbose=False)
    wphi, wpsi, wst, _ = oracle.sinkhorn_kernel(x, y, r, c, args, frequency=frequency, p=p)
    assert int(st[0]) == wst.iterations and int(st[1]) == wst.num_iter
    assert int(st[2]) == (1 if wst.stopped == 1 else 2)
    np.testing.assert_allclose(phi, wphi, rtol=0, atol=ATOL)
    np.testing.assert_allclose(psi, wpsi, rtol=0, atol=ATOL)
    assert st[3] == pytest.approx(wst.residual, rel=1e-6, abs=1e-15)
    assert st[4] == pytest.approx(wst.objective, rel=1e-12)
    assert st[5] == wst.winf


def test_shard_rows_cover_every_row_once():
    from culamp_b200.sharded import shard_rows
    for n in (1, 7, 64, 1001):
        for g in (1, 2, 3, 8):
            blocks = [shard_rows(n, g, k) for k in range(g)]
            assert blocks[0][0] == 0 and blocks[-1][1] == n
            assert all(b[0] == a[1] for a, b in zip(blocks, blocks[1:]))
            assert max(b - a for a, b in blocks) - min(b - a for a, b in blocks) <= 1


@pytest.mark.parametrize("p,eta_p,shards_per_rank,marginal_only", [(2.0, 5e-2, 1, False), (1.0, 5e-2, 2, True),
                                                                   (math.inf, 0.0, 1, False)])
def test_two_gloo_ranks_lamp_match_single_oracle(oracle, tmp_path, p, eta_p, shards_per_rank, marginal_only):
    """Row-sharded LAMP: partial column masses all-reduced per infeas(.) call;
    the replicated duals, eta_t / s recursion, log rows and the gathered row
    potentials equal the single-process oracle to FP64 rounding."""
    x, r = _grid(6, 2)
    y, c = _grid(7, 3)
    x = x[:-5]
    r = r[:-5] / r[:-5].sum()
    case = {"data": (x, y, r, c), "eta_p": eta_p, "epsilon": 1e-12, "itermax": 60, "frequency": 7, "p": p,
            "shards_per_rank": shards_per_rank, "lamp": True, "B": 1.1, "marginal_only": marginal_only}
    phi, _, st, outs = _run(case, tmp_path)
    for o in outs[1:]:
        assert np.array_equal(o["nu"], outs[0]["nu"]) and np.array_equal(o["stats"], outs[0]["stats"])
    flags = oracle.CHECK_ALWAYS | (oracle.MARGINAL_ONLY if marginal_only else 0)
    args = oracle.Args(eta_p=eta_p, epsilon=1e-12, itermax=60, verbose=True, B=1.1)
    nu, wphi, psi, theta, wst, log = oracle.lamp_kernel(x, y, r, c, args, frequency=7, p=p, flags=flags)
    o = outs[0]
    assert int(o["stats"][0]) == wst.iterations
    assert o["stats"][5] == wst.eta_t and o["stats"][6] == wst.s_t
    np.testing.assert_allclose(o["nu"], nu, rtol=0, atol=ATOL)
    np.testing.assert_allclose(o["theta"], theta, rtol=0, atol=ATOL)
    np.testing.assert_allclose(phi, wphi, rtol=0, atol=1e-9)
    want = np.array([row[1:6] for row in log])
    assert o["log"].shape == want.shape and np.array_equal(o["log"][:, 0], want[:, 0])
    np.testing.assert_allclose(o["log"][:, 1:], want[:, 1:], rtol=1e-10, atol=1e-12)
    assert o["stats"][2] == pytest.approx(wst.residual, rel=1e-8, abs=1e-14)
    assert o["stats"][3] == pytest.approx(wst.objective, rel=1e-12)
