"""CUDA path vs the CPU oracle on identical seeded inputs (through the C ABI).

Element-wise RHS parity for every (physics, flux, entropy-fix, P, BC arm),
full SSPRK3 steps with and without the cell limiter, 2D kernels, node
coordinates, FP64 reductions and the max wave speed.  Meshes are small and
anisotropic (dx != dy != dz) so permutation and scaling mistakes show.
"""
import numpy as np
import pytest

import mojoxm_b200 as M
from tests import dgcases as C

pytestmark = pytest.mark.gpu


def make_pair(oracle, phys, P, n, L, bcs, prec="f64", dim=3):
    bc = M.BoundaryConditions(*bcs) if dim == 3 else M.BoundaryConditions(*bcs, 0, 0)
    mesh = M.Mesh(*n, *L, bcs=bc, dim=dim) if dim == 3 else M.Mesh(n[0], n[1], 1, L[0], L[1], 1.0, bcs=bc, dim=2)
    s = M.Solver(mesh, phys, P=P, precision=prec)
    real = "f64" if prec == "f64" else "f32"
    if dim == 3:
        o = oracle.Oracle3D(P, n, L, M.physics_dict(phys), bcs=bcs, real=real)
    else:
        o = oracle.Oracle2D(P, n, L, M.physics_dict(phys), bcs=bcs, real=real)
    return s, o


N3, L3 = (3, 4, 2), (1.0, 1.3, 0.7)
N2, L2 = (4, 3), (1.0, 0.8)


@pytest.mark.parametrize("P", [1, 2, 3, 4, 5])
@pytest.mark.parametrize("name", list(C.PHYSICS_3D))
def test_rhs3d_f64_periodic(oracle_mod, name, P):
    phys = C.PHYSICS_3D[name]()
    s, o = make_pair(oracle_mod, phys, P, N3, L3, C.BCS_3D["periodic"])
    q = C.random_state(s.shape, phys, seed=100 + P)
    r_gpu, r_cpu = s.rhs(q), o.rhs(q)
    assert C.rel_err(r_gpu, r_cpu) <= C.TOL_F64_3D[P]


@pytest.mark.parametrize("bcname", [b for b in C.BCS_3D if b != "periodic"])
@pytest.mark.parametrize("name", ["advection", "euler_hllec_fix", "euler_rusanov", "maxwell", "shallow_water", "mhd"])
@pytest.mark.parametrize("P", [2, 3])
def test_rhs3d_f64_boundaries(oracle_mod, name, bcname, P):
    phys = C.PHYSICS_3D[name]()
    s, o = make_pair(oracle_mod, phys, P, N3, L3, C.BCS_3D[bcname])
    q = C.random_state(s.shape, phys, seed=7)
    assert C.rel_err(s.rhs(q), o.rhs(q)) <= C.TOL_F64_3D[P]


@pytest.mark.parametrize("name", ["euler_hllec", "euler_roe_fix", "maxwell", "advection", "shallow_water", "mhd"])
@pytest.mark.parametrize("P", [1, 3, 5])
def test_rhs3d_f32(oracle_mod, name, P):
    phys = C.PHYSICS_3D[name]()
    s, o = make_pair(oracle_mod, phys, P, N3, L3, C.BCS_3D["walls"], prec="f32")
    q = C.random_state(s.shape, phys, seed=11)
    qf = q.astype(np.float32).astype(np.float64)
    assert C.rel_err(s.rhs(qf), o.rhs(qf)) <= C.TOL_F32


@pytest.mark.parametrize("limiter", [False, True])
@pytest.mark.parametrize("P", [2, 4])
def test_ssprk3_steps_f64(oracle_mod, P, limiter):
    phys = C.PHYSICS_3D["euler_hllec_fix"]()
    s, o = make_pair(oracle_mod, phys, P, N3, L3, C.BCS_3D["outflow_x_wall_yz"])
    q = C.random_state(s.shape, phys, seed=3)
    s.upload_state(q)
    o.set(q)
    if limiter:
        s.enable_cell_limiter(True, 0.05)
        o.enable_limiter(True, 0.05)
    dt = 2e-3
    s.step_n(dt, 3)
    o.step(dt, 3)
    assert C.rel_err(s.download_state(0), o.get(0)) <= 50 * C.TOL_F64_3D[P]


@pytest.mark.parametrize("P", [1, 2, 3, 4, 5])
@pytest.mark.parametrize("name", list(C.PHYSICS_2D))
def test_rhs2d_f64(oracle_mod, name, P):
    phys = C.PHYSICS_2D[name]()
    for bcname in ("periodic", "inflow_outflow"):
        s, o = make_pair(oracle_mod, phys, P, N2, L2, C.BCS_2D[bcname], dim=2)
        q = C.random_state(s.shape, phys, seed=21 + P)
        assert C.rel_err(s.rhs(q), o.rhs(q)) <= C.TOL_F64_2D[P], bcname


@pytest.mark.parametrize("P", [2, 3])
@pytest.mark.parametrize("bcname", list(C.BCS_2D))
def test_ssprk3_2d_limited(oracle_mod, bcname, P):
    phys = C.PHYSICS_2D["euler_hllc"]()
    s, o = make_pair(oracle_mod, phys, P, N2, L2, C.BCS_2D[bcname], dim=2)
    q = C.random_state(s.shape, phys, seed=5)
    s.upload_state(q)
    o.set(q)
    s.enable_cell_limiter(True, 0.02)
    o.enable_limiter(True, 0.02)
    s.step_n(1e-3, 2)
    o.step(1e-3, 2)
    assert C.rel_err(s.download_state(0), o.get(0)) <= 50 * C.TOL_F64_2D[P]


def test_limiter_alone_3d(oracle_mod):
    phys = C.PHYSICS_3D["euler_hllec"]()
    s, o = make_pair(oracle_mod, phys, 3, N3, L3, C.BCS_3D["walls"])
    q = C.random_state(s.shape, phys, seed=9)
    s.upload_state(q)
    o.set(q)
    s.enable_cell_limiter(True, 0.01)
    o.enable_limiter(True, 0.01)
    s.limit(0)
    o.limit(0)
    out = s.download_state(0)
    assert C.rel_err(out, o.get(0)) <= 1e-13
    assert np.abs(out - q).max() > 1e-3  # the limiter fired


def test_node_xyz(oracle_mod):
    for dim, n, L in ((3, N3, L3), (2, N2, L2)):
        phys = M.Advection(1.0, 0.5, 0.0)
        s, o = make_pair(oracle_mod, phys, 3, n, L, (0,) * (2 * dim), dim=dim)
        x_gpu = s.node_xyz()
        x_cpu = o.node_xyz() if dim == 3 else o.node_xy()
        assert np.abs(x_gpu - x_cpu).max() < 1e-14


def test_reductions_and_wavespeed(oracle_mod):
    phys = C.PHYSICS_3D["euler_hllec"]()
    s, o = make_pair(oracle_mod, phys, 3, N3, L3, C.BCS_3D["inflow_outflow"])
    q = C.random_state(s.shape, phys, seed=13)
    s.upload_state(q)
    o.set(q)
    w = oracle_mod.refelem3d(3)["w"]
    vol = (L3[0] / N3[0]) * (L3[1] / N3[1]) * (L3[2] / N3[2]) / 6.0
    for c in range(5):
        want = vol * float((q[..., c] * w[None, :]).sum())
        assert abs(s.integral(c) - want) <= 1e-13 * abs(want)
        assert abs(s.integral(c, kind=2) - np.abs(q[..., c]).max()) == 0.0
    assert abs(s.max_wavespeed() - o.max_face_speed()) <= 1e-13 * o.max_face_speed()


# Mixed precision (FP32 state, split-BF16 tcgen05 contraction) vs the FP64
# oracle: element-wise RHS error relative to max |RHS|.  Split-BF16 keeps
# 8 + 8 significant bits of each operand and drops the lo x lo product, so
# each product is off by up to ~2^-16 relative; the derivative and lift sums
# over K = 3 NP + 4 NFP columns add and partly cancel those errors.  Measured
# on a B200 for every physics here at P2..P5: 3.2e-6 .. 1.7e-5 (largest:
# shallow water P4); the bound is about 3x the largest.
TOL_MIXED = 5e-5
TOL_MIXED_P = {2: TOL_MIXED, 3: TOL_MIXED, 4: TOL_MIXED, 5: TOL_MIXED}


# Split-TF32 (tcgen05 kind::tf32, 11 + 11 significant bits per operand): the
# contraction is accurate to ~2^-21, so the RHS error is that of FP32
# arithmetic in the fluxes (the FP32 SIMT kernel's own level on these
# random states) rather than of the operand split.  P = 5 runs the FP32
# kernel (its TF32 operands exceed a block's shared memory).  Measured:
# 1.3e-7 .. 2.1e-6.
TOL_TF32 = {2: 5e-6, 3: 5e-6, 4: 5e-6, 5: 5e-6}


@pytest.mark.parametrize("prec", ["mixed", "tf32"])
@pytest.mark.parametrize("P", [2, 3, 4, 5])
@pytest.mark.parametrize("name", ["euler_rusanov", "euler_hllec_fix", "maxwell", "advection", "shallow_water", "mhd"])
def test_rhs3d_mixed_vs_f64(oracle_mod, name, P, prec):
    phys = C.PHYSICS_3D[name]()
    s, o = make_pair(oracle_mod, phys, P, N3, L3, C.BCS_3D["outflow_x_wall_yz"], prec=prec)
    q = C.random_state(s.shape, phys, seed=31)
    qf = q.astype(np.float32).astype(np.float64)
    o64 = oracle_mod.Oracle3D(P, N3, L3, M.physics_dict(phys), bcs=C.BCS_3D["outflow_x_wall_yz"], real="f64")
    err = C.rel_err(s.rhs(qf), o64.rhs(qf))
    print(f"{prec} {name} P={P}: rel err vs FP64 oracle {err:.2e}")
    assert err <= (TOL_MIXED_P[P] if prec == "mixed" else TOL_TF32[P])


@pytest.mark.parametrize("prec", ["mixed", "tf32"])
def test_mixed_large_mesh_vs_f32(oracle_mod, prec):
    """Many tiles, partial last tile, tensor-core kernel vs the FP32 SIMT kernel."""
    phys = C.PHYSICS_3D["euler_hllec"]()
    n, L = (7, 5, 3), (1.0, 1.0, 1.0)
    sm = M.Solver(M.Mesh(*n, *L), phys, P=3, precision=prec)
    sf = M.Solver(M.Mesh(*n, *L), phys, P=3, precision="f32")
    q = C.random_state(sm.shape, phys, seed=41)
    err = C.rel_err(sm.rhs(q), sf.rhs(q))
    print(f"{prec} vs f32 on {n}: {err:.2e}")
    assert err <= (TOL_MIXED if prec == "mixed" else TOL_TF32[3])


@pytest.mark.parametrize("limiter", [False, True])
@pytest.mark.parametrize("P", [2, 3])
def test_mhd_ssprk3_steps_f64(oracle_mod, P, limiter):
    """Ideal MHD with GLM cleaning: three SSPRK3 steps (conducting walls in x,
    outflow in y, periodic z), with and without the cell limiter."""
    phys = C.PHYSICS_3D["mhd"]()
    bcs = (1, 1, 2, 2, 0, 0)
    s, o = make_pair(oracle_mod, phys, P, N3, L3, bcs)
    q = C.random_state(s.shape, phys, seed=41)
    s.upload_state(q)
    o.set(q)
    if limiter:
        s.enable_cell_limiter(True, 0.1)
        o.enable_limiter(True, 0.1)
    dt = 0.02 / (2 * P + 1)
    s.step_n(dt, 3)
    o.step(dt, 3)
    assert C.rel_err(s.download_state(0), o.get(0)) <= 50 * C.TOL_F64_3D[P]


@pytest.mark.parametrize("prec", ["f64", "f32", "mixed"])
def test_mhd_constant_state_preserved(prec):
    """A uniform magnetised state on a periodic mesh is a steady solution."""
    s = M.Solver(M.Mesh(3, 2, 2), C.PHYSICS_3D["mhd"](), P=3, precision=prec)
    q = np.zeros(s.shape)
    q[..., 0], q[..., 1:4], q[..., 5:8] = 1.2, [0.3, -0.2, 0.1], [0.4, 0.1, -0.3]
    q[..., 4] = 1.0 / (5.0 / 3.0 - 1) + 0.5 * (0.3 ** 2 + 0.2 ** 2 + 0.1 ** 2) / 1.2 + 0.5 * 0.26
    r = s.rhs(q)
    s.close()
    assert np.abs(r).max() <= (1e-11 if prec == "f64" else 2e-4)


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("bcname", list(C.BCS_2D))
@pytest.mark.parametrize("name", ["mhd_glm", "mhd_plain"])
def test_mhd2d_steps(oracle_mod, name, bcname, prec):
    """2D MHD (plain and GLM): every BC arm, three SSPRK3 steps with the
    limiter; with GLM the psi damping exp(-alpha_d dt) after every step."""
    P = 3
    phys = C.PHYSICS_2D[name]()
    s, o = make_pair(oracle_mod, phys, P, N2, L2, C.BCS_2D[bcname], prec=prec, dim=2)
    q = C.random_state(s.shape, phys, seed=61)
    if prec == "f32":
        q = q.astype(np.float32).astype(np.float64)
    s.upload_state(q)
    o.set(q)
    s.enable_cell_limiter(True, 0.05)
    o.enable_limiter(True, 0.05)
    s.step_n(2e-3, 3)
    o.step(2e-3, 3)
    assert C.rel_err(s.download_state(0), o.get(0)) <= (50 * C.TOL_F64_2D[P] if prec == "f64" else 1e-4)


def test_mhd_wavespeed_and_integrals(oracle_mod):
    """3D MHD: the CFL reduction (max Rusanov alpha over face nodes) and the
    FP64 integrals of all nine components."""
    phys = C.PHYSICS_3D["mhd"]()
    s, o = make_pair(oracle_mod, phys, 3, N3, L3, C.BCS_3D["inflow_outflow"])
    q = C.random_state(s.shape, phys, seed=17)
    s.upload_state(q)
    o.set(q)
    w = oracle_mod.refelem3d(3)["w"]
    vol = (L3[0] / N3[0]) * (L3[1] / N3[1]) * (L3[2] / N3[2]) / 6.0
    for c in range(9):
        want = vol * float((q[..., c] * w[None, :]).sum())
        assert abs(s.integral(c) - want) <= 1e-13 * max(abs(want), 1e-3)
    assert abs(s.max_wavespeed() - o.max_face_speed()) <= 1e-13 * o.max_face_speed()


@pytest.mark.parametrize("bcname", list(C.BCS_3D))
@pytest.mark.parametrize("P", [1, 2, 3, 4])
def test_two_fluid_rhs_f64(oracle_mod, bcname, P):
    phys = C.two_fluid()
    s, o = make_pair(oracle_mod, phys, P, N3, L3, C.BCS_3D[bcname])
    q = C.random_state(s.shape, phys, seed=71 + P)
    assert C.rel_err(s.rhs(q), o.rhs(q)) <= C.TOL_F64_3D[P]


@pytest.mark.parametrize("prec", ["f32", "mixed"])
@pytest.mark.parametrize("P", [2, 3, 5])
def test_two_fluid_rhs_reduced(oracle_mod, prec, P):
    """17 components: MIXED runs the FP32 kernel (no tensor-core tile)."""
    phys = C.two_fluid()
    s, o = make_pair(oracle_mod, phys, P, N3, L3, C.BCS_3D["walls"], prec=prec)
    q = C.random_state(s.shape, phys, seed=81)
    qf = q.astype(np.float32).astype(np.float64)
    assert C.rel_err(s.rhs(qf), o.rhs(qf)) <= C.TOL_F32


@pytest.mark.parametrize("limiter", [False, True])
def test_two_fluid_steps_f64(oracle_mod, limiter):
    phys = C.two_fluid()
    s, o = make_pair(oracle_mod, phys, 2, N3, L3, C.BCS_3D["inflow_outflow"])
    q = C.random_state(s.shape, phys, seed=91)
    s.upload_state(q)
    o.set(q)
    if limiter:
        s.enable_cell_limiter(True, 0.1)
        o.enable_limiter(True, 0.1)
    s.step_n(1e-3, 3)
    o.step(1e-3, 3)
    assert C.rel_err(s.download_state(0), o.get(0)) <= 50 * C.TOL_F64_3D[2]
    assert abs(s.max_wavespeed() - o.max_face_speed()) <= 1e-13 * o.max_face_speed()


def test_two_fluid_f64_p5_refused():
    with pytest.raises(M.DGError):
        M.Solver(M.Mesh(2, 2, 2), C.two_fluid(), P=5, precision="f64")


def test_reference_diagnostics_rows(tmp_path):
    """DiagnosticsWriter rows (src/diagnostics.mojo:162-229) from device
    reductions: sum q and sum q^2 over all nodes times domain volume /
    (elements x nodes), and max |q|, against the same sums in numpy."""
    phys = C.PHYSICS_3D["euler_rusanov"]()
    s = M.Solver(M.Mesh(*N3, *L3), phys, P=3, precision="f32")
    q = C.random_state(s.shape, phys, seed=23).astype(np.float32).astype(np.float64)
    s.upload_state(q)
    dw = M.DiagnosticsWriter(s, M.DiagComponents().linear("mass", 0).squared("rho2", 0).maxabs("maxE", 4),
                             csv_path=str(tmp_path / "diag.csv"))
    row = dw.record(0.5)
    scale = L3[0] * L3[1] * L3[2] / (q.shape[0] * q.shape[1])
    assert abs(row[0] - q[..., 0].sum() * scale) <= 1e-13 * abs(row[0])
    assert abs(row[1] - (q[..., 0] ** 2).sum() * scale) <= 1e-13 * abs(row[1])
    assert row[2] == np.abs(q[..., 4]).max()
    lines = open(tmp_path / "diag.csv").read().splitlines()
    assert lines[0] == "t,mass,rho2,maxE" and lines[1].startswith("0.5,")
    s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["f64", "mixed"])
def test_advance_host_async_pipeline_matches_sync(prec):
    """Pipelined host entry: three calls in flight with distinct inputs and
    outputs give the synchronous entry's results bit for bit."""
    phys = C.euler(M.FLUX_RUSANOV)
    mesh = M.Mesh(4, 4, 4)
    s = M.Solver(mesh, phys, P=3, precision=prec)
    ref = M.Solver(mesh, phys, P=3, precision=prec)
    ins = [M.PinnedArray(s.shape, s.dtype) for _ in range(3)]
    outs = [M.PinnedArray(s.shape, s.dtype) for _ in range(3)]
    for k, p in enumerate(ins):
        p.array[...] = C.random_state(s.shape, phys, seed=20 + k)
    for p_in, p_out in zip(ins, outs):
        s.advance_host_async(p_in.array, 2, 1e-3, p_out.array)
    s.synchronize()
    for p_in, p_out in zip(ins, outs):
        want = ref.advance_host(p_in.array, 2, 1e-3)
        assert np.array_equal(p_out.array, want)
    for p in ins + outs:
        p.free()
