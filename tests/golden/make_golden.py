"""Generate the golden fixtures in tests/golden/ from the FP64 oracle.

    python tests/golden/make_golden.py

Inputs are seeded (numpy PCG64) synthetic instances; outputs come from
oracle/culamp_oracle.c. `winf_reference.json` is different: its values were
read from the reference's own archived run logs
(data_archive/data/updated_pnorm.csv, column `maxval`, one value per p for the
integer 64x64 grid), so it pins the max-cost pass to reference output.
"""
from __future__ import annotations

import json
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "culamp.jl_b200"))

import oracle as O  # noqa: E402
from culamp_b200 import datasets as D  # noqa: E402

PS = (1.0, 2.0, math.inf, 3.0)


def pkey(p):
    return "inf" if math.isinf(p) else f"{p:g}"


def ragged_points(seed, n, d):
    g = np.random.Generator(np.random.PCG64(seed))
    return g.uniform(0.0, 1.0, size=(n, d))


def passes_case():
    n, m, d = 37, 23, 3
    x, y = ragged_points(11, n, d), ragged_points(12, m, d)
    g = np.random.Generator(np.random.PCG64(13))
    r = g.uniform(0.1, 1.0, n); r /= r.sum()
    c = g.uniform(0.1, 1.0, m); c /= c.sum()
    pot = g.normal(0.0, 3.0, m)
    phi = g.normal(0.0, 3.0, n)
    theta = g.uniform(-0.9, 0.9, m)
    logz = g.normal(0.0, 1.0, n)
    out = dict(x=x, y=y, r=r, c=c, pot=pot, phi=phi, theta=theta, logz=logz)
    for p in PS:
        k = pkey(p)
        winf = O.max_cost(x, y, p)
        out[f"rowmax_{k}"] = O.max_cost_rows(x, y, p)
        out[f"winf_{k}"] = np.array(winf)
        out[f"sk_lse_{k}"] = O.sk_lse(x, y, r, pot, 0.05, winf, p)
        res, cost = O.sk_residual(x, y, r, phi, pot, 0.05, winf, p)
        out[f"sk_res_{k}"], out[f"sk_cost_{k}"] = res, cost
        out[f"spp_lse_{k}"] = O.spp_lse(x, y, theta, 0.02, 1.0, winf, p)
        res, cost = O.spp_col_residual(x, y, r, theta, logz, 0.02, 1.0, winf, p)
        out[f"spp_res_{k}"], out[f"spp_cost_{k}"] = res, cost
        out[f"minred_{k}"] = O.min_reduce(x, y, theta, winf, p)
    emu = (c + 0.01 / n) / 1.0
    out["theta_upd_a0"] = O.theta_update(theta, out["spp_res_2"], c, emu, 0.0, False, -0.5, 0.5)
    out["theta_upd_a1"] = O.theta_update(theta, out["spp_res_2"], c, emu, 0.0, True, -0.5, 0.5)
    np.savez_compressed(os.path.join(HERE, "passes_small.npz"), **out)


def solver_cases():
    x, y, r, c = D.grid_instance(8, 8, "mixture")
    out = dict(x=x, y=y, r=r, c=c)
    a = O.Args(eta_p=1e-2, epsilon=0.0, itermax=200, verbose=True)
    for p in (1.0, 2.0, math.inf):
        k = pkey(p)
        for flags, tag in ((0, "ref"), (O.TRUE_PINF, "true")):
            if flags and not math.isinf(p):
                continue
            phi, psi, st, log = O.sinkhorn_kernel(x, y, r, c, a, frequency=7, p=p, flags=flags)
            pre = f"sk_{k}_{tag}"
            out[pre + "_phi"], out[pre + "_psi"] = phi, psi
            out[pre + "_stats"] = np.array([st.iterations, st.num_iter, st.residual,
                                            st.objective, st.winf])
            out[pre + "_log"] = np.array(log, dtype=np.float64)
    # early stop: tolerance met part-way (num_iter semantics)
    a2 = O.Args(eta_p=1e-2, epsilon=6e-4, itermax=500, verbose=True)
    phi, psi, st, log = O.sinkhorn_kernel(x, y, r, c, a2, frequency=5, p=2.0)
    out["skstop_phi"], out["skstop_psi"] = phi, psi
    out["skstop_stats"] = np.array([st.iterations, st.num_iter, st.residual, st.objective, st.winf])
    out["skstop_log"] = np.array(log, dtype=np.float64)
    # LAMP: eta_p > 0 with verbose checks, and eta_p = 0 (min-reduce dual)
    for eta_p, tag in ((1e-2, "eta"), (0.0, "zero")):
        b = O.Args(eta_p=eta_p, epsilon=1e-12, itermax=120, verbose=True, B=1.1)
        for p in (1.0, 2.0, math.inf):
            nu, phi, psi, th, st, log = O.lamp_kernel(x, y, r, c, b, frequency=10, p=p)
            pre = f"lamp_{tag}_{pkey(p)}"
            out[pre + "_nu"], out[pre + "_phi"], out[pre + "_theta"] = nu, phi, th
            out[pre + "_stats"] = np.array([st.iterations, st.residual, st.objective, st.winf,
                                            st.eta_t, st.s_t])
            out[pre + "_log"] = np.array(log, dtype=np.float64)
    # annealed Sinkhorn
    c3 = O.Args(eta_p=0.1, epsilon=2e-3, anneal_mult=0.5, itermax=300, verbose=False)
    phi, psi, st, log = O.annealed_sinkhorn_kernel(x, y, r, c, c3, frequency=10, p=2.0)
    out["ann_phi"], out["ann_psi"] = phi, psi
    out["ann_stats"] = np.array([st.iterations, st.num_iter, st.residual, st.objective])
    out["ann_log"] = np.array(log, dtype=np.float64)
    np.savez_compressed(os.path.join(HERE, "solvers_grid8.npz"), **out)


def ragged_solver_case():
    n, m, d = 37, 23, 3
    x, y = ragged_points(21, n, d), ragged_points(22, m, d)
    g = np.random.Generator(np.random.PCG64(23))
    r = g.uniform(0.1, 1.0, n); r /= r.sum()
    c = g.uniform(0.1, 1.0, m); c /= c.sum()
    out = dict(x=x, y=y, r=r, c=c)
    a = O.Args(eta_p=5e-2, epsilon=0.0, itermax=150, verbose=False)
    phi, psi, st, _ = O.sinkhorn_kernel(x, y, r, c, a, frequency=50, p=2.0)
    out["sk_phi"], out["sk_psi"] = phi, psi
    out["sk_stats"] = np.array([st.residual, st.objective, st.winf])
    b = O.Args(eta_p=5e-2, epsilon=0.0, itermax=80, verbose=False, B=1.1)
    nu, phi, psi, th, st, _ = O.lamp_kernel(x, y, r, c, b, frequency=50, p=2.0)
    out["lamp_nu"], out["lamp_phi"], out["lamp_theta"] = nu, phi, th
    out["lamp_stats"] = np.array([st.residual, st.objective, st.winf, st.eta_t])
    np.savez_compressed(os.path.join(HERE, "solvers_ragged.npz"), **out)


def dense_case():
    W = D.dense_grid_cost(8, 8)
    r = D.uniform_marginal(64, 0)
    c = D.uniform_marginal(64, 1)
    a = O.Args(eta_p=1e-2, epsilon=1e-6, itermax=400, verbose=True)
    phi, psi, st, log = O.sinkhorn_dense(W, r, c, a, frequency=20)
    b = O.Args(eta_p=1e-2, epsilon=1e-6, itermax=300, verbose=True, B=1.1)
    th, nu, _, st2, log2 = O.lamp_dense(W, r, c, b, frequency=20)
    np.savez_compressed(os.path.join(HERE, "dense_grid8.npz"), W=W, r=r, c=c, sk_phi=phi,
                        sk_psi=psi, sk_stats=np.array([st.iterations, st.residual, st.objective]),
                        lamp_theta=th, lamp_nu=nu,
                        lamp_stats=np.array([st2.iterations, st2.residual, st2.eta_t]),
                        sk_log=np.array(log), lamp_log=np.array(log2))


def winf_reference():
    data = {
        "source": "data_archive/data/updated_pnorm.csv column maxval (reference run logs), "
                  "integer 64x64 grid of CmdLineUtils.jl:208-212",
        "grid": [64, 64],
        "winf": {"1": 126.0, "2": 7938.0, "inf": 63.0},
    }
    with open(os.path.join(HERE, "winf_reference.json"), "w") as f:
        json.dump(data, f, indent=1)


if __name__ == "__main__":
    O.build()
    winf_reference()
    passes_case()
    solver_cases()
    ragged_solver_case()
    dense_case()
    for fn in sorted(os.listdir(HERE)):
        print(fn, os.path.getsize(os.path.join(HERE, fn)))
