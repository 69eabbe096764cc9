"""C-ABI library checks that need no GPU: it loads, exports every function
include/mxm_dg.h declares, reports errors without crashing, and its host FP64
operators agree with the oracle's restatement of the reference construction."""
import ctypes
import os
import re

import numpy as np
import pytest

import mojoxm_b200 as M

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "mxm_dg.h")).read()
    return sorted(set(re.findall(r"^int (mxm_dg_\w+)\(", src, re.M)))


def test_header_and_wrapper_agree():
    assert header_functions() == sorted(M.EXPORTED)


def test_library_exports_every_declared_symbol():
    L = M.lib()
    for name in header_functions():
        assert hasattr(L, name), name
    assert L.mxm_dg_version() == 20100


def test_bad_arguments_return_einval():
    L = M.lib()
    md, pd = M._MeshDesc(), M._PhysDesc()
    md.dim, md.nx, md.ny, md.nz = 3, 2, 2, 2
    h = ctypes.c_void_p()
    assert L.mxm_dg_create(ctypes.byref(md), ctypes.byref(pd), 9, 0, ctypes.byref(h)) == M.EINVAL
    assert "order" in M._err(None)
    md.dim = 4
    assert L.mxm_dg_create(ctypes.byref(md), ctypes.byref(pd), 2, 0, ctypes.byref(h)) == M.EINVAL
    md.dim = 3
    pd.kind, pd.flux_type = M.PHYS_EULER, M.FLUX_HLLC  # HLLC exists only in 2D
    assert L.mxm_dg_create(ctypes.byref(md), ctypes.byref(pd), 2, 0, ctypes.byref(h)) == M.EINVAL
    assert L.mxm_dg_step_ssprk3(None, 0.1) == M.EINVAL


@pytest.mark.parametrize("P", [1, 2, 3, 4, 5])
def test_operators_vs_oracle(oracle_mod, P):
    r = oracle_mod.refelem3d(P)
    D, Lf, w = M.reference_operators(3, P)
    assert np.abs(D - r["D"]).max() <= 1e-13 * np.abs(r["D"]).max()
    assert np.abs(Lf - r["Lift"]).max() <= 1e-13 * np.abs(r["Lift"]).max()
    assert np.abs(w - r["w"]).max() <= 1e-15
    r2 = oracle_mod.refelem2d(P)
    D2, L2, w2 = M.reference_operators(2, P)
    # the reference's 2D edge-mass construction loses digits at high P
    # (equispaced 1D Vandermonde, reference_2d.mojo:278-306)
    tol = {1: 1e-14, 2: 1e-13, 3: 1e-11, 4: 1e-10, 5: 1e-8}[P]
    assert np.abs(D2[0] - r2["Dr"]).max() <= tol * 10 and np.abs(D2[1] - r2["Ds"]).max() <= tol * 10
    assert np.abs(L2 - r2["Lift"]).max() <= tol
    assert np.abs(w2 - r2["w"]).max() <= 1e-14


def test_create_without_gpu_fails_cleanly():
    """On a machine without a GPU the product must refuse, not fall back."""
    try:
        import torch  # noqa: F401  (only to know whether a GPU is present)

        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("GPU present")
    with pytest.raises(M.DGError) as ei:
        M.Solver(M.Mesh(2, 2, 2), M.Advection(1.0, 0.0, 0.0), P=1)
    assert ei.value.rc in (M.ECUDA, M.ENOMEM)
