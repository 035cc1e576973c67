"""W_inf = max_ij C(x_i, y_j) (maxcost.cu), the normaliser every solver
computes before iterating: bit-identical to the FP64 oracle for p = 1, 2, Inf
(each pair's cost is formed with the same correctly rounded operations in the
same order), within 1e-14 for other p (CUDA's pow and the host's differ by an
ulp), on ragged sizes (tiles of 64 pairs x 64 pairs cut by n and m), d from 1
to 256, and through the batched solve's one launch over many instances."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def T(a):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device="cuda")


@pytest.mark.parametrize("n,m,d", [(1, 1, 1), (1, 700, 3), (65, 63, 2), (129, 200, 5), (640, 1, 17),
                                   (300, 450, 72), (77, 2000, 256), (4100, 70, 33)])
@pytest.mark.parametrize("p", [1.0, 2.0, math.inf, 3.0])
def test_winf_is_bit_identical_to_oracle(oracle, n, m, d, p):
    import culamp_b200 as cb
    g = np.random.Generator(np.random.PCG64(n * 7 + m * 3 + d))
    x = g.normal(size=(n, d))
    y = g.normal(size=(m, d)) + 0.5
    r = np.full(n, 1.0 / n)
    c = np.full(m, 1.0 / m)
    a = cb.EOTArgs(eta_p=1e-2, epsilon=0.0, itermax=0, verbose=False)
    flags = cb.FLAG_TRUE_PINF if math.isinf(p) else 0
    res = cb.solve_sinkhorn(T(x), T(y), T(r), T(c), a, 10, p, flags=flags)
    if p in (1.0, 2.0, math.inf):
        assert res.winf == oracle.max_cost(x, y, p)
    else:
        assert res.winf == pytest.approx(oracle.max_cost(x, y, p), rel=1e-14)


def test_batched_winf_one_launch_matches_oracle(oracle):
    import culamp_b200 as cb
    from culamp_b200 import datasets as D
    inst = D.batched_instances(40, lo=64, hi=3000, dims=(2, 3, 40), seed=9)
    dev = [tuple(T(v) for v in t) for t in inst]
    a = cb.EOTArgs(eta_p=1e-2, epsilon=0.0, itermax=1, verbose=False)
    for p in (1.0, 2.0):
        out = cb.solve_batched_sinkhorn(dev, a, frequency=1, p=p)
        for (x, y, _, _), res in zip(inst, out.results):
            assert res.winf == oracle.max_cost(x, y, p)


@pytest.mark.parametrize("d,p", [(3, 2.0), (64, 2.0), (7, 1.0), (5, math.inf)])
def test_pass_level_winf_only_matches_row_maxima(d, p):
    """culamp_max_cost with rowmax NULL (tiled maximum) against the row-max
    pass of the same call with rowmax given."""
    from culamp_b200 import kernels as K
    g = np.random.Generator(np.random.PCG64(d))
    x, y = T(g.uniform(size=(1500, d))), T(g.uniform(size=(999, d)))
    rowmax, w_rows = K.max_logsumexp_spp_ct(x, y, p)
    none, w_tiled = K.max_logsumexp_spp_ct(x, y, p, rows=False)
    assert none is None
    assert w_tiled == w_rows == float(rowmax.max())
