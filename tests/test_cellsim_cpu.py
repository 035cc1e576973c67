"""Cell metrics (CellUtilities.jl:127-172) as constant multiples of pass costs
on preprocessed points: the identities culamp_b200.cellsim relies on, checked
against the oracle's direct restatement of the reference formulas."""
import numpy as np
import pytest

from culamp_b200.cellsim import cell_points


def counts(n, d, seed):
    g = np.random.Generator(np.random.PCG64(seed))
    a = np.log1p(g.negative_binomial(0.5, 0.2, size=(n, d)).astype(float))
    a *= g.uniform(size=(n, d)) >= 0.7
    a[a.sum(1) == 0, 0] = 1.0
    a[:, 1] += 0.01                      # every row has some spread
    return a


@pytest.mark.parametrize("metric", ["l1", "cosine", "correlation", "pearson"])
@pytest.mark.parametrize("normalize", [True, False])
def test_cell_metric_is_a_multiple_of_a_pass_cost(oracle, metric, normalize):
    a = counts(60, 24, 1)
    pts, p, factor = cell_points(a, metric, normalize)
    want = oracle.np_cell_cost(a, metric, normalize)
    got = factor * oracle.np_cost(pts, pts, p)
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-13)


def test_degenerate_rows_are_rejected():
    a = counts(10, 6, 2)
    a[3] = 0.0
    with pytest.raises(ValueError):
        cell_points(a, "cosine")
    b = counts(10, 6, 3)
    b[4] = 2.0
    with pytest.raises(ValueError):
        cell_points(b, "correlation")
    with pytest.raises(ValueError):
        cell_points(b, "l2")
