"""Seeded synthetic OT instances with the shapes of CuLAMP.jl's benchmarks.

DOTmark and OT-scOmics (the reference's public inputs) are not available, so
these generators stand in for them with the same sizes and value ranges:

* ``grid_instance``      -- h x w grid (DOTmark-shaped), coordinates either the
  reference's integer (row, col, 0) layout (CmdLineUtils.jl:208-212) or scaled
  to [0,1]^2; marginals Uniform(0,1)+1e-3 or a 5-component Gaussian mixture.
* ``feature_instance``   -- n points in R^d, log1p(negative-binomial counts)
  with 90% zeros, rows L2-normalised (single-cell-like features).
* ``batched_instances``  -- many uneven instances (n, m log-uniform, d mixed).
* ``rgb_instance``       -- colour-transfer-sized RGB clouds from two seeded
  8-component Gaussian mixtures in [0,1]^3.

All draws use numpy's PCG64 with the documented seeds (0 for the first
cloud / row marginal, 1 for the second / column marginal).
"""
from __future__ import annotations

import numpy as np


def _rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(seed))


def grid_coords(h: int, w: int, scaled: bool = True) -> np.ndarray:
    """Point-major (h*w, 3) coordinates of an h x w grid, z = 0.

    Point i (0-based) is (i // w, i % w, 0) -- the reference's column-major
    3 x N `locations` array (CmdLineUtils.jl:208-212) has the same memory
    layout. With ``scaled`` the coordinates are divided by (h-1, w-1).
    """
    idx = np.arange(h * w)
    pts = np.zeros((h * w, 3), dtype=np.float64)
    pts[:, 0] = idx // w
    pts[:, 1] = idx % w
    if scaled:
        pts[:, 0] /= max(h - 1, 1)
        pts[:, 1] /= max(w - 1, 1)
    return pts


def uniform_marginal(n: int, seed: int, floor: float = 1e-3) -> np.ndarray:
    v = _rng(seed).uniform(0.0, 1.0, size=n) + floor
    return v / v.sum()


def gaussian_mixture_marginal(h: int, w: int, seed: int, k: int = 5,
                              floor: float = 1e-4) -> np.ndarray:
    """Mixture of k isotropic 2-D Gaussians evaluated on the [0,1]^2 grid."""
    g = _rng(seed)
    centres = g.uniform(0.0, 1.0, size=(k, 2))
    sigma = g.uniform(0.05, 0.2, size=k)
    weights = g.dirichlet(np.ones(k))
    pts = grid_coords(h, w, scaled=True)[:, :2]
    dens = np.zeros(h * w)
    for c, s, wt in zip(centres, sigma, weights):
        d2 = ((pts - c) ** 2).sum(axis=1)
        dens += wt * np.exp(-0.5 * d2 / s**2) / (2 * np.pi * s**2)
    dens = dens + floor
    return dens / dens.sum()


def dotmark_smoothing(v: np.ndarray) -> np.ndarray:
    """`normalize(marginal .+ 1e-6, 1)` of run_dot (CmdLineUtils.jl:187-188)."""
    v = np.asarray(v, dtype=np.float64) + 1e-6
    return v / np.abs(v).sum()


def grid_instance(h: int = 64, w: int = 64, marginals: str = "mixture",
                  scaled: bool = True):
    """(x, y, r, c) for a grid problem with x == y (the reference's
    `img1 === img2` locations)."""
    x = grid_coords(h, w, scaled=scaled)
    if marginals == "mixture":
        r = gaussian_mixture_marginal(h, w, seed=0)
        c = gaussian_mixture_marginal(h, w, seed=1)
    elif marginals == "uniform":
        r = uniform_marginal(h * w, seed=0)
        c = uniform_marginal(h * w, seed=1)
    else:
        raise ValueError(f"unknown marginals {marginals!r}")
    return x, x.copy(), r, c


def dense_grid_cost(h: int, w: int) -> np.ndarray:
    """Squared-Euclidean grid cost normalised by its max (run_dot's
    `W ./= W_inf`, CmdLineUtils.jl:193-198)."""
    x = grid_coords(h, w, scaled=False)[:, :2]
    W = ((x[:, None, :] - x[None, :, :]) ** 2).sum(-1)
    return W / W.max()


def feature_instance(n: int = 16384, m: int = 16384, d: int = 256,
                     mean: float = 2.0, dispersion: float = 0.5,
                     sparsity: float = 0.9):
    """Nonnegative features log1p(NB(mean, dispersion)) with `sparsity`
    Bernoulli zeros; rows L2-normalised, all-zero rows resampled."""
    def cloud(seed, count):
        g = _rng(seed)
        # NB(r, p) with mean mu and dispersion k: r = k, p = k / (k + mu)
        p = dispersion / (dispersion + mean)
        out = np.empty((count, d), dtype=np.float64)
        filled = np.zeros(count, dtype=bool)
        while not filled.all():
            todo = np.flatnonzero(~filled)
            cnt = g.negative_binomial(dispersion, p, size=(todo.size, d)).astype(np.float64)
            mask = g.uniform(size=(todo.size, d)) >= sparsity
            vals = np.log1p(cnt) * mask
            norms = np.linalg.norm(vals, axis=1)
            ok = norms > 0
            out[todo[ok]] = vals[ok] / norms[ok, None]
            filled[todo[ok]] = True
        return out
    x = cloud(0, n)
    y = cloud(1, m)
    r = np.full(n, 1.0 / n)
    c = np.full(m, 1.0 / m)
    return x, y, r, c


def _gmm_points(g: np.random.Generator, count: int, d: int, k: int) -> np.ndarray:
    centres = g.uniform(0.1, 0.9, size=(k, d))
    sigma = g.uniform(0.03, 0.15, size=k)
    weights = g.dirichlet(np.ones(k))
    comp = g.choice(k, size=count, p=weights)
    pts = centres[comp] + sigma[comp, None] * g.standard_normal((count, d))
    return np.clip(pts, 0.0, 1.0)


def rgb_instance(n: int = 65536, m: int = 65536, k: int = 8):
    """Two RGB clouds in [0,1]^3 from seeded k-component Gaussian mixtures,
    uniform marginals (colour-transfer sized)."""
    x = _gmm_points(_rng(0), n, 3, k)
    y = _gmm_points(_rng(1), m, 3, k)
    return x, y, np.full(n, 1.0 / n), np.full(m, 1.0 / m)


def batched_instances(count: int = 512, lo: int = 256, hi: int = 8192,
                      dims=(2, 3, 64), seed: int = 0):
    """`count` independent instances, n and m log-uniform in [lo, hi],
    d drawn uniformly from `dims`, Gaussian-mixture points clipped to
    [0,1]^d, Dirichlet(1) marginals."""
    g = _rng(seed)
    out = []
    for _ in range(count):
        n = int(round(np.exp(g.uniform(np.log(lo), np.log(hi)))))
        m = int(round(np.exp(g.uniform(np.log(lo), np.log(hi)))))
        d = int(g.choice(np.asarray(dims)))
        x = _gmm_points(g, n, d, 4)
        y = _gmm_points(g, m, d, 4)
        r = g.dirichlet(np.ones(n))
        c = g.dirichlet(np.ones(m))
        r = np.maximum(r, 1e-300)
        c = np.maximum(c, 1e-300)
        out.append((x, y, r / r.sum(), c / c.sum()))
    return out
