"""Cell-similarity feature costs (CellUtilities.jl:127-172) on the solver passes.

CuLAMP.jl's cellsim solvers transport mass between the rows of one data matrix
(features x cells; a point is a row, its coordinates are the cells) under a
feature cost with the row-sum normalisation of CellCostKernel
(CellUtilities.jl:14-112): row i is read as data[i, :] / s_i with s_i its sum
(1 when the sum is 0, or when normalize_features is off). Three of the
metrics are exactly a constant multiple of a cost the passes already compute,
on preprocessed points, so they run on the existing kernels -- cosine and
correlation on the tensor-core squared-Euclidean path for d >= 32:

* l1:          C = sum_k |a_k/s_i - b_k/s_j| / 2            -> p = 1 on u_i = a/s_i, x 1/2
* cosine:      C = (1 - <u_i, u_j> / (|u_i| |u_j|)) / 2      -> p = 2 on u_i / |u_i|,   x 1/4
               (|u - v|^2 = 2 - 2 cos for unit vectors)
* correlation: C = (1 - <u_i - mu_i, u_j - mu_j> / (|.| |.|)) / 2
                                                             -> p = 2 on the centred,
                                                                normalised rows, x 1/4
  (d mu_i mu_j subtracted from the dot product is the centring; the row-sum
  scale s_i cancels in both normalised metrics).

The solvers normalise every cost by its own maximum W_inf (MirrorProxCellSim.jl:115-117,
SinkhornCellSim.jl:269-270), so a constant multiple leaves every iterate
unchanged; only the reported transport cost carries the factor, applied here.
The clamp of the similarity to [-1, 1] is implied (|u - v|^2 >= 0).
Rows of zero norm (cosine) or zero variance (correlation) have a special case
in the reference (cost 0, or 0 / 1/scale) that no such multiple reproduces;
they are rejected. The l2 metric (a square root of the squared distance) is
not a multiple of a pass cost and is not offered here.
"""
from __future__ import annotations

import numpy as np

from .args import EOTArgs

METRICS = ("l1", "cosine", "correlation")


def cell_points(data, metric: str = "correlation", normalize_features: bool = True):
    """(points, p, factor): C_metric(i, j) = factor * C_p(points_i, points_j)."""
    metric = "correlation" if metric.lower() == "pearson" else metric.lower()
    if metric not in METRICS:
        raise ValueError(f"cell metric {metric!r}: supported are {METRICS} (and 'pearson')")
    a = np.asarray(data, dtype=np.float64)
    s = a.sum(axis=1) if normalize_features else np.ones(a.shape[0])
    if normalize_features:
        s = np.where(s > 0, s, 1.0)                     # row_scales (CellUtilities.jl:69-80)
    u = a / s[:, None]
    if metric == "l1":
        return u, 1.0, 0.5
    if metric == "correlation":
        u = u - u.mean(axis=1, keepdims=True)
    norms = np.linalg.norm(u, axis=1)
    if not np.all(norms > 0):
        bad = int(np.flatnonzero(~(norms > 0))[0])
        raise ValueError(f"row {bad} has zero {'variance' if metric == 'correlation' else 'norm'}: "
                         "the reference's special-case cost is not supported")
    return u / norms[:, None], 2.0, 0.25


def _solve(kind, data, metric, marginal1, marginal2, args, frequency, normalize_features, flags):
    import torch
    from . import solvers as S
    pts, p, factor = cell_points(data, metric, normalize_features)
    X = torch.as_tensor(pts, device="cuda")
    r = torch.as_tensor(np.asarray(marginal1, dtype=np.float64), device="cuda")
    c = torch.as_tensor(np.asarray(marginal2, dtype=np.float64), device="cuda")
    fn = S.solve_sinkhorn if kind == "sinkhorn" else S.solve_lamp
    res = fn(X, X, r, c, args, frequency, p, flags=flags)
    res.objective *= factor
    res.winf *= factor
    res.log = [(t, it, inf, obj * factor, pr, du) for (t, it, inf, obj, pr, du) in res.log]
    return res


def sinkhorn_cellsim(data, metric: str, marginal1, marginal2, args: EOTArgs, frequency: int = 100,
                     normalize_features: bool = True, flags: int = 0):
    """Kernel Sinkhorn between two distributions over the rows of `data`
    (SinkhornCellSim.jl:240-310) under a cell metric; returns the solver result
    with the transport cost and W_inf in the metric's units."""
    return _solve("sinkhorn", data, metric, marginal1, marginal2, args, frequency, normalize_features, flags)


def lamp_cellsim(data, metric: str, marginal1, marginal2, args: EOTArgs, frequency: int = 100,
                 normalize_features: bool = True, flags: int = 0):
    """Kernel LAMP over the rows of `data` under a cell metric
    (MirrorProxCellSim.jl:100-200)."""
    return _solve("lamp", data, metric, marginal1, marginal2, args, frequency, normalize_features, flags)
