"""The scratch-free Sinkhorn row pass, culamp_lse_rows_sk_noalloc.

It exists for callers that cannot let the library allocate device memory at
the call site -- code recording a CUDA stream capture (cudaMalloc cannot be
captured) and hosts that own all device memory through their own pool or
budget. It uses fixed file-scope device scratch instead of the handle's
cudaMalloc-grown scratch, so it must give the same result as the handle path
(culamp_lse_rows_sk), call after call. Collected last on purpose: it must pass
both alone in a fresh process and after every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LSE_ATOL = 2e-6   # the tolerance of the pass-level log-sum-exp tests


def _case(n, m, d, seed):
    g = np.random.Generator(np.random.PCG64(seed))
    x, y = g.uniform(size=(n, d)), g.uniform(size=(m, d))
    r = g.uniform(0.1, 1.0, n)
    return x, y, r / r.sum(), g.normal(0.0, 3.0, m)


# (1031, 777, 3): several splits, partials fit; (40000, 5000, 2): splits reduced
# to fit the fixed partials; (140000, 600, 3): n alone exceeds the partials, a
# single split; (40000, 2000, 5): the generic d > 3 tile with reduced splits.
@pytest.mark.parametrize("n,m,d,reg", [(1031, 777, 3, 0.05), (40000, 5000, 2, 1e-3),
                                       (5, 9, 1, 0.5), (140000, 600, 3, 1e-2),
                                       (40000, 2000, 5, 5e-2)])
def test_noalloc_matches_handle_path_two_calls(n, m, d, reg):
    import torch
    from culamp_b200 import _lib, kernels as K
    lib = _lib.load()
    fn = lib.culamp_lse_rows_sk_noalloc
    x, y, r, pot = _case(n, m, d, n + m)
    X, Y, R, POT = (torch.as_tensor(v, device="cuda") for v in (x, y, r, pot))
    _, winf = K.max_logsumexp_spp_ct(X, Y, 2.0)
    want = K.warp_logsumexp_ct_fused(X, Y, R, POT, reg, winf, 2.0).cpu().numpy()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for k in range(2):   # the fixed scratch keeps the previous call's contents
        # first call: no usable reference in out; second: the previous result
        # minus a shift as the (ignored-for-correctness) hint
        out = (torch.full((n,), float("nan"), dtype=torch.float64, device="cuda") if k == 0
               else torch.as_tensor(want - 0.25, device="cuda"))
        st = fn(C.c_void_p(out.data_ptr()), C.c_void_p(X.data_ptr()), C.c_void_p(Y.data_ptr()),
                n, m, d, C.c_void_p(R.data_ptr()), C.c_void_p(POT.data_ptr()), reg, winf, 2.0,
                stream)
        assert st == 0
        torch.cuda.synchronize()
        np.testing.assert_allclose(out.cpu().numpy(), want, rtol=0, atol=LSE_ATOL)


def test_noalloc_rejects_bad_arguments():
    from culamp_b200 import _lib
    fn = _lib.load().culamp_lse_rows_sk_noalloc
    assert fn(None, None, None, 4, 4, 3, None, None, 0.1, 1.0, 2.0, None) == _lib.ERR_INVALID_ARG


def test_noalloc_rejects_rows_beyond_the_fixed_tickets():
    """n above 8,388,608 rows is refused on the host before any launch."""
    import torch
    from culamp_b200 import _lib
    fn = _lib.load().culamp_lse_rows_sk_noalloc
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    ptr = C.c_void_p(buf.data_ptr())
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for d in (3, 5):
        assert fn(ptr, ptr, ptr, 8388609, 4, d, ptr, ptr, 0.1, 1.0, 2.0, stream) == _lib.ERR_UNSUPPORTED
    torch.cuda.synchronize()
