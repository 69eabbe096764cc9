"""Batched 2D engine (mxm_dg_batch_*): every member of a batch of uneven
solves (mesh size, order P, physics, limiter on/off) must end where the same
solve advanced alone ends.  The batched kernel runs the same per-tile code
as the single-solve kernel, so the states agree bit for bit."""
import numpy as np
import pytest

import mojoxm_b200 as M
from tests import dgcases as C

CASES = [  # (n, P, physics name, limiter, bcs)
    (6, 1, "euler_hlle", True, "walls"),
    (9, 2, "euler_hlle", True, "periodic"),
    (5, 3, "euler_hlle", False, "inflow_outflow"),
    (7, 4, "euler_hlle", True, "mixed_hi_only"),
    (4, 5, "euler_hlle", True, "periodic"),
    (8, 3, "euler_rusanov", False, "periodic"),
    (6, 2, "shallow_water", True, "walls"),
    (3, 5, "maxwell", False, "walls"),
]


def _make(prec, n, P, name, lim, bcn):
    phys = C.PHYSICS_2D[name]()
    bcs = M.BoundaryConditions(*C.BCS_2D[bcn], 0, 0)
    mesh = M.Mesh(n, n + 1, 1, 1.0, 0.9, 1.0, bcs=bcs, dim=2)
    s = M.Solver(mesh, phys, P=P, precision=prec)
    if lim:
        s.enable_cell_limiter(True, 0.05)
    return s, phys


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_batch_members_match_alone(prec):
    batch = M.Batch()
    pairs = []
    for k, (n, P, name, lim, bcn) in enumerate(CASES):
        a, phys = _make(prec, n, P, name, lim, bcn)
        b, _ = _make(prec, n, P, name, lim, bcn)
        q = C.random_state(a.shape, phys, seed=100 + k)
        a.upload_state(q)
        b.upload_state(q)
        dt = 1e-3 * (1 + k % 3)
        batch.add(a, dt)
        pairs.append((a, b, dt))
    nsteps = 3
    batch.step(nsteps)
    batch.synchronize()
    for a, b, dt in pairs:
        b.step_n(dt, nsteps)
        qa, qb = a.download_state(), b.download_state()
        assert np.isfinite(qa).all()
        assert np.array_equal(qa, qb), (a.P, a.physics, np.abs(qa - qb).max())
    for i in range(len(CASES)):
        assert batch.tile_cells(i) in (1, 2, 4, 8, 16, 32, 64)
    # 3 physics groups; the Euler-HLLE and SW groups have limited members
    assert batch.launches_per_step() == 3 * 3 + 3 * 1 + 3 * 3 + 3 * 1
    batch.close()


@pytest.mark.gpu
def test_batch_rejects_3d_and_mixed_precision():
    batch = M.Batch()
    s3 = M.Solver(M.Mesh(2, 2, 2), C.PHYSICS_3D["euler_rusanov"](), P=2, precision="f32")
    with pytest.raises(M.DGError):
        batch.add(s3, 1e-3)
    a = M.Solver(M.Mesh(4, 4, dim=2), C.PHYSICS_2D["euler_hlle"](), P=2, precision="f32")
    b = M.Solver(M.Mesh(4, 4, dim=2), C.PHYSICS_2D["euler_hlle"](), P=2, precision="f64")
    batch.add(a, 1e-3)
    with pytest.raises(M.DGError):
        batch.add(b, 1e-3)
    with pytest.raises(M.DGError):
        batch.add(a, 1e-3)  # already a member
    batch.close()
