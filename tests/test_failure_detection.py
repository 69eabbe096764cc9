"""Failure detection without a GPU fault: the bounded waits that guard every
bulk copy and tensor-core commit in the stage kernels give up by themselves.
A kernel waits on a barrier that nothing completes; it must report that it
gave up after about the limit and leave the context usable (a solve run
right after it still matches a fresh run)."""
import numpy as np
import pytest

import mojoxm_b200 as M
from tests import dgcases as C


@pytest.mark.gpu
def test_bounded_wait_gives_up_and_context_survives():
    phys = C.euler(M.FLUX_RUSANOV)
    s = M.Solver(M.Mesh(3, 3, 3), phys, P=2, precision="f64")
    q = C.random_state(s.shape, phys, seed=5)
    s.upload_state(q)
    s.step_n(1e-3, 2)
    before = s.download_state()
    gave_up, waited = M.selftest_wait_timeout(50.0)
    assert gave_up == 1
    assert 45.0 <= waited < 2000.0, waited
    s.synchronize()  # no device error recorded by the stage kernels
    s.upload_state(q)
    s.step_n(1e-3, 2)
    assert np.array_equal(s.download_state(), before)
    s.close()


def test_selftest_rejects_bad_limits():
    # argument checks happen before any device work
    import ctypes
    g, w = ctypes.c_int32(), ctypes.c_double()
    assert M.lib().mxm_dg_selftest_wait_timeout(0.0, ctypes.byref(g), ctypes.byref(w)) == M.EINVAL
    assert M.lib().mxm_dg_selftest_wait_timeout(1e6, ctypes.byref(g), ctypes.byref(w)) == M.EINVAL
