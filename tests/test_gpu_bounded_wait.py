"""Failure detection without a GPU fault: the tensor-core path's bounded
mbarrier wait (ft_wait, used by every role of the feature pass) runs on a
barrier phase that nothing completes, and the persistent loops' grid barrier
on a barrier one CTA never reaches; each must give up after its limit, set
its abort flag and let the host see CULAMP_ERR_DEVICE_TIMEOUT, and the device
context must stay usable for the next solve."""
import ctypes as C
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_bounded_wait_gives_up_and_the_context_stays_usable():
    import torch
    import culamp_b200 as cb
    from culamp_b200 import _lib
    h = cb.get_handle(0)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    t0 = time.perf_counter()
    st = h._lib.culamp_probe_wait(h.ptr, 50_000_000, stream)      # 50 ms limit
    dt = time.perf_counter() - t0
    assert st == _lib.ERR_DEVICE_TIMEOUT
    assert b"gave up" in h._lib.culamp_last_error(h.ptr)
    assert 0.04 < dt < 5.0
    # the context is intact: a solve on the same handle and stream
    g = np.random.Generator(np.random.PCG64(3))
    x, y = g.uniform(size=(300, 3)), g.uniform(size=(200, 3))
    r, c = np.full(300, 1 / 300), np.full(200, 1 / 200)
    res = cb.solve_sinkhorn(x, y, r, c, cb.EOTArgs(eta_p=5e-2, epsilon=0.0, itermax=30, verbose=False), 10, 2.0)
    assert res.iterations == 30 and np.isfinite(res.phi).all()
    torch.cuda.synchronize()


def test_bounded_wait_limit_is_checked():
    import culamp_b200 as cb
    from culamp_b200 import _lib
    h = cb.get_handle(0)
    assert h._lib.culamp_probe_wait(h.ptr, 0, None) == _lib.ERR_INVALID_ARG
    assert h._lib.culamp_probe_wait(h.ptr, 20_000_000_000, None) == _lib.ERR_INVALID_ARG


def test_grid_barrier_wait_gives_up_and_the_context_stays_usable():
    """The persistent loops' grid barrier (two co-resident CTAs, one never
    arrives): the waiting CTA gives up after its limit, publishes the abort on
    the barrier counter, and the host sees CULAMP_ERR_DEVICE_TIMEOUT; then a
    persistent solve on the same handle runs normally."""
    import torch
    import culamp_b200 as cb
    from culamp_b200 import _lib, datasets as D
    h = cb.get_handle(0)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    t0 = time.perf_counter()
    st = h._lib.culamp_probe_grid_wait(h.ptr, 50_000_000, stream)
    dt = time.perf_counter() - t0
    assert st == _lib.ERR_DEVICE_TIMEOUT
    assert b"gave up" in h._lib.culamp_last_error(h.ptr)
    assert 0.04 < dt < 5.0
    assert h._lib.culamp_probe_grid_wait(h.ptr, 0, None) == _lib.ERR_INVALID_ARG
    x, y, r, c = (torch.as_tensor(v, device="cuda") for v in D.grid_instance(32, 32, "mixture"))
    res = cb.solve_sinkhorn(x, y, r, c, cb.EOTArgs(eta_p=1e-2, epsilon=0.0, itermax=30, verbose=False), 10, 2.0)
    assert res.iterations == 30 and bool(torch.isfinite(res.phi).all())
