"""The allocation-free reduction entry point against the allocating one.

mxm_dg_reduce_conserved_noalloc keeps its scratch in a static device array
of the library instead of a per-handle buffer; with nblocks = 0 it runs the
same two-pass reduction with the same block count, so its results must agree
with mxm_dg_reduce_conserved to round-off (bit-identical in practice) on two
calls in a row.  This file is named to be collected last, and it also passes
alone in a fresh process (the first call does the scratch set-up)."""
import ctypes

import numpy as np
import pytest

import mojoxm_b200 as M
from tests.dgcases import random_state

TOL = 1e-12  # relative; both paths sum the same partials in the same order


def _noalloc(s, c, which=0, kind=0, nblocks=0):
    v = ctypes.c_double()
    rc = M.lib().mxm_dg_reduce_conserved_noalloc(s.h, which, c, kind, nblocks, ctypes.byref(v))
    return rc, v.value


def _alloc(s, c, which=0, kind=0):
    v = ctypes.c_double()
    rc = M.lib().mxm_dg_reduce_conserved(s.h, which, c, kind, ctypes.byref(v))
    return rc, v.value


@pytest.mark.gpu
@pytest.mark.parametrize("dim,prec", [(3, "f64"), (3, "f32"), (2, "f64")])
def test_noalloc_reduction_matches_allocating_entry(dim, prec):
    if dim == 3:
        mesh = M.Mesh(6, 5, 4)
    else:
        mesh = M.Mesh(9, 7, dim=2)
    phys = M.Euler(flux_type=M.FLUX_RUSANOV)
    s = M.Solver(mesh, phys, P=3, precision=prec)
    q = random_state(s.shape, phys, seed=11 + dim)
    s.upload_state(q)
    for _ in range(2):  # two calls in a row: the static scratch is reused as is
        for kind in (0, 1, 2):
            for c in range(s.NC):
                rc_a, a = _alloc(s, c, kind=kind)
                rc_b, b = _noalloc(s, c, kind=kind)
                assert rc_a == M.OK and rc_b == M.OK, M._err(s.h)
                assert abs(a - b) <= TOL * max(1.0, abs(a)), (kind, c, a, b)
    s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("nblocks", [7, 1500, 4096])
def test_noalloc_other_block_counts(nblocks):
    """Block counts other than the default one.  36^3 x 6 = 279,936 elements
    need 1094 blocks of 256, so the default (capped at 1024 partials) uses
    1024; nblocks 7 runs the grid-stride loop with 7 blocks, 1500 and 4096
    are capped at 1094 blocks, a count the allocating entry never uses."""
    phys = M.Euler(flux_type=M.FLUX_RUSANOV)
    s = M.Solver(M.Mesh(36, 36, 36), phys, P=1, precision="f64")
    assert s.num_elements == 279936
    q = random_state(s.shape, phys, seed=5)
    s.upload_state(q)
    for _ in range(2):
        for kind in (0, 1, 2, 3):
            _, a = _alloc(s, 4, kind=kind)
            rc, b = _noalloc(s, 4, kind=kind, nblocks=nblocks)
            assert rc == M.OK, M._err(s.h)
            if kind == 2:
                assert a == b
            else:
                assert abs(a - b) <= 1e-12 * abs(a), (kind, nblocks, a, b)
    s.close()


@pytest.mark.gpu
def test_noalloc_rejects_oversized_scratch():
    s = M.Solver(M.Mesh(2, 2, 2), M.Euler(flux_type=M.FLUX_RUSANOV), P=2, precision="f64")
    rc, _ = _noalloc(s, 0, nblocks=4097)
    assert rc == M.EINVAL
    assert "static reduction scratch" in M._err(s.h)
    rc, _ = _noalloc(s, 0, nblocks=-1)
    assert rc == M.EINVAL
    s.close()
