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
def test_batch_rejects_mixed_state_widths_and_repeats():
    batch = M.Batch()
    a = M.Solver(M.Mesh(4, 4, dim=2), C.PHYSICS_2D["euler_hlle"](), P=2, precision="f32")
    b = M.Solver(M.Mesh(4, 4, dim=2), C.PHYSICS_2D["euler_hlle"](), P=2, precision="f64")
    s3 = M.Solver(M.Mesh(2, 2, 2), C.PHYSICS_3D["euler_rusanov"](), P=2, precision="f64")
    batch.add(a, 1e-3)
    with pytest.raises(M.DGError):
        batch.add(b, 1e-3)  # FP64 state beside FP32 state
    with pytest.raises(M.DGError):
        batch.add(s3, 1e-3)
    with pytest.raises(M.DGError):
        batch.add(a, 1e-3)  # already a member
    batch.close()


# 3D members: (n cubes, P, physics, precision, limiter, bcs).  Tensor-core
# members of one (physics, order, operand kind) share one batched launch;
# the uneven meshes make tiles of several solves meet inside one block's
# tile range, and the last tile of every solve partial.
CASES_3D = [
    ((3, 4, 2), 3, "euler_rusanov", "mixed", False, "periodic"),
    ((5, 3, 3), 3, "euler_rusanov", "mixed", False, "walls"),
    ((2, 2, 3), 3, "euler_rusanov", "mixed", False, "periodic"),
    ((4, 3, 2), 3, "euler_hllec", "mixed", True, "outflow_x_wall_yz"),
    ((3, 3, 3), 2, "euler_hllec", "mixed", True, "walls"),
    ((3, 2, 2), 4, "maxwell", "tf32", False, "walls"),
    ((2, 3, 2), 4, "maxwell", "tf32", False, "periodic"),
    ((3, 2, 2), 5, "euler_hlle", "mixed", False, "inflow_outflow"),
    ((3, 3, 2), 2, "mhd", "mixed", True, "periodic"),
    ((2, 2, 2), 1, "euler_rusanov", "mixed", False, "periodic"),  # P1: the FP32 SIMT stage
    ((3, 2, 2), 3, "shallow_water", "f32", False, "walls"),       # FP32 SIMT stage
]


@pytest.mark.gpu
def test_batch_3d_members_match_alone():
    """3D members (split-BF16 and split-TF32 tensor-core stages, limited and
    not, and FP32 SIMT members) beside 2D members in one batch: every member
    ends where the same solve stepped alone ends, bit for bit."""
    batch = M.Batch()
    pairs = []
    for k, (n, P, name, prec, lim, bcn) in enumerate(CASES_3D):
        phys = C.PHYSICS_3D[name]()
        bcs = M.BoundaryConditions(*C.BCS_3D[bcn])
        L = (1.0, 0.9, 1.1)
        a = M.Solver(M.Mesh(*n, *L, bcs=bcs), phys, P=P, precision=prec)
        b = M.Solver(M.Mesh(*n, *L, bcs=bcs), phys, P=P, precision=prec)
        q = C.random_state(a.shape, phys, seed=300 + k)
        for s in (a, b):
            s.upload_state(q)
            if lim:
                s.enable_cell_limiter(True, 0.05)
        dt = 2e-4 * (1 + k % 3) / (2 * P + 1)
        batch.add(a, dt)
        pairs.append((a, b, dt))
    s2, phys2 = _make("f32", 6, 3, "euler_hlle", True, "walls")  # a 2D member too
    t2, _ = _make("f32", 6, 3, "euler_hlle", True, "walls")
    q2 = C.random_state(s2.shape, phys2, seed=399)
    s2.upload_state(q2)
    t2.upload_state(q2)
    batch.add(s2, 1e-3)
    pairs.append((s2, t2, 1e-3))
    nsteps = 3
    batch.step(nsteps)
    batch.synchronize()
    for a, b, dt in pairs:
        b.step_n(dt, nsteps)
        qa, qb = a.download_state(), b.download_state()
        assert np.isfinite(qa).all()
        assert np.array_equal(qa, qb), (a.P, a.precision, np.abs(qa - qb).max())
    for k, (n, P, name, prec, lim, bcn) in enumerate(CASES_3D):
        tc = P >= 2 and prec in ("mixed", "tf32")
        assert (batch.tile_cells(k) > 0) == tc
    batch.close()
    for a, b, _ in pairs:
        a.close()
        b.close()


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
