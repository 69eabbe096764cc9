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


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_batch_mhd2d_members_match_alone(prec):
    """2D MHD in a batch (plain and GLM, limited and not, uneven dt): each
    member equals the same solve stepped alone, psi damping included."""
    cases = [(6, 3, "mhd_glm", True, "walls", 1e-3), (5, 2, "mhd_plain", False, "periodic", 2e-3),
             (4, 4, "mhd_glm", False, "inflow_outflow", 5e-4), (7, 1, "euler_hlle", True, "periodic", 1e-3)]
    solo, mem, b = [], [], M.Batch()
    for k, (n, P, name, lim, bcn, dt) in enumerate(cases):
        for lst in (solo, mem):
            s, phys = _make(prec, n, P, name, lim, bcn)
            q = C.random_state(s.shape, phys, seed=200 + k)
            s.upload_state(q)
            lst.append((s, dt))
        b.add(mem[-1][0], dt)
    b.step(4)
    b.synchronize()
    for (s1, dt), (s2, _) in zip(solo, mem):
        s1.step_n(dt, 4)
        a, c = s1.download_state(), s2.download_state()
        assert np.array_equal(a, c)
        s1.close()
    b.close()
    for s2, _ in mem:
        s2.close()
