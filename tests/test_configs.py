"""End-to-end runs of the benchmark configurations' physics at test sizes.

* Isentropic vortex (3D Euler, [0,10]^3 periodic, 8^3 x 6 tets, P = 2,
  HLLEC with and without the entropy fix, SSPRK3 at CFL 0.3 to T = 1): the
  oracle and the product agree, and both stay within the reference's own
  analytic gate (L2 <= 0.10 relative to the translated vortex,
  benchmarks/bench_euler_vortex_3d.mojo:75).
* Maxwell PEC cavity mode (E_z = sin(pi x) sin(pi y) at t = 0, PEC on x and
  y, periodic z): after one period the field returns to its initial state;
  FP64 and split-BF16 runs are checked against that and against each other."""
import json
import os

import numpy as np
import pytest

import mojoxm_b200 as M
from tests import dgcases as C

GAMMA = 1.4
HERE = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(HERE, "golden", "known_answers.json")) as _f:
    G = json.load(_f)["values"]

BETA, X0, Y0, UBG, VBG = 5.0, 5.0, 5.0, 1.0, 1.0


def vortex_state(xyz, t=0.0, L=10.0):
    """Shu isentropic vortex advected by (UBG, VBG, 0), nearest periodic image."""
    dx = xyz[..., 0] - (X0 + UBG * t)
    dy = xyz[..., 1] - (Y0 + VBG * t)
    dx -= L * np.floor(dx / L + 0.5)
    dy -= L * np.floor(dy / L + 0.5)
    r2 = dx * dx + dy * dy
    f = BETA / (2 * np.pi)
    ex = np.exp(0.5 * (1 - r2))
    u, v = UBG - f * dy * ex, VBG + f * dx * ex
    T = 1 - (GAMMA - 1) * f * f / (2 * GAMMA) * np.exp(1 - r2)
    rho = T ** (1 / (GAMMA - 1))
    p = rho ** GAMMA
    q = np.zeros(xyz.shape[:-1] + (5,))
    q[..., 0] = rho
    q[..., 1] = rho * u
    q[..., 2] = rho * v
    q[..., 4] = p / (GAMMA - 1) + 0.5 * rho * (u * u + v * v)
    return q


def vortex_steps(P=2, n=8, L=10.0, T=1.0, cfl=0.3):
    # examples/euler_vortex.mojo:137-144: dt = CFL h / (lambda (2P+1))
    lam = np.hypot(UBG, VBG) + BETA / (2 * np.pi) + np.sqrt(GAMMA)
    dt = cfl * (L / n) / (lam * (2 * P + 1))
    nsteps = int(np.ceil(T / dt))
    return T / nsteps, nsteps


def rel_l2(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


@pytest.mark.parametrize("efix", [False, True])
def test_vortex_oracle_within_reference_gate(oracle_mod, efix):
    ph = C.euler(M.FLUX_HLLEC, efix=efix)
    o = oracle_mod.Oracle3D(2, 8, 10.0, M.physics_dict(ph))
    xyz = o.node_xyz()
    o.set(vortex_state(xyz))
    dt, n = vortex_steps()
    o.step(dt, n)
    err = rel_l2(o.get(), vortex_state(xyz, t=1.0))
    assert err <= G["vortex_3d.l2_max_rel"], err


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("efix", [False, True])
def test_vortex_product_vs_oracle(oracle_mod, prec, efix):
    ph = C.euler(M.FLUX_HLLEC, efix=efix)
    o = oracle_mod.Oracle3D(2, 8, 10.0, M.physics_dict(ph), real=prec)
    s = M.Solver(M.Mesh(8, 8, 8, 10.0, 10.0, 10.0), ph, P=2, precision=prec)
    xyz = o.node_xyz()
    q0 = vortex_state(xyz)
    o.set(q0)
    s.upload_state(q0)
    dt, n = vortex_steps()
    o.step(dt, n)
    s.step_n(dt, n)
    qs = s.download_state().astype(np.float64)
    assert rel_l2(qs, o.get()) <= (1e-11 if prec == "f64" else 2e-5)
    assert rel_l2(qs, vortex_state(xyz, t=1.0)) <= G["vortex_3d.l2_max_rel"]
    # the device IC fill gives the same field
    s.fill_ic(M.IC_VORTEX, [BETA, X0, Y0, UBG, VBG, 0.0, 1.0])
    assert rel_l2(s.download_state().astype(np.float64), q0) < (1e-7 if prec == "f64" else 1e-6)
    s.close()


def cavity_steps(P, n, cfl=0.2):
    # bench_maxwell_cavity_3d.mojo:56,128-130: dt = CFL h / (c (2P+1)), T one period
    T = np.sqrt(2.0)  # omega = sqrt(2) pi for the (1, 1) mode on the unit square
    dt = cfl * (1.0 / n) / (2 * P + 1)
    nsteps = int(np.ceil(T / dt))
    return T / nsteps, nsteps


@pytest.mark.gpu
def test_maxwell_cavity_one_period():
    n, P = 6, 3
    bcs = M.BoundaryConditions(1, 1, 1, 1, 0, 0)  # PEC on x and y, periodic z
    phys = M.Maxwell(1.0, *([0.0] * 12))
    dt, nsteps = cavity_steps(P, n)
    out = {}
    for prec in ("f64", "f32", "mixed", "tf32"):
        s = M.Solver(M.Mesh(n, n, n, bcs=bcs), phys, P=P, precision=prec)
        s.fill_ic(M.IC_CAVITY, [1.0, 1.0, 1.0])
        q0 = s.download_state().astype(np.float64)
        s.step_n(dt, nsteps)
        out[prec] = s.download_state().astype(np.float64)
        s.close()
    # after one period E_z is back and B vanishes: error of the DG scheme
    err64 = rel_l2(out["f64"], q0)
    assert err64 < 5e-3, err64
    e32, emx, etf = (rel_l2(out[p], out["f64"]) for p in ("f32", "mixed", "tf32"))
    print(f"cavity one period vs FP64: f32 {e32:.2e}, split-BF16 {emx:.2e}, split-TF32 {etf:.2e}")
    assert emx < 1e-4
    # the split-TF32 operator is ~2^6 times closer to the FP64 one than the
    # split-BF16 operator: the period ends at FP32-state accuracy (measured
    # 2.7e-6 here, 4.5e-6 on the 24^3 P4 benchmark cavity against 9.5e-6
    # for the FP32 kernel there)
    assert etf < 5e-6 and etf < emx / 4, (etf, emx)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["f32", "mixed", "tf32"])
@pytest.mark.parametrize("P", [2, 3, 4, 5])
def test_reduced_precision_steps_track_f64(P, prec):
    """Several SSPRK3 steps of the smooth density wave in FP32 / split-BF16
    stay within FP32-state accuracy of the FP64 kernels.  5^3 cubes do not
    fill whole tiles, so the last tile of every launch takes the partial-tile
    path (plain loads where the bulk copy does not fit)."""
    n = 5
    phys = C.euler(M.FLUX_RUSANOV)
    mesh = M.Mesh(n, n, n)
    s64 = M.Solver(mesh, phys, P=P, precision="f64")
    s64.fill_ic(M.IC_SINE_WAVE, [1.0, 0.2, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0])
    q0 = s64.download_state()
    h = 1.0 / n
    dt = 0.1 * h / ((np.sqrt(3.0) + np.sqrt(GAMMA)) * (2 * P + 1))
    s64.step_n(dt, 12)
    q64 = s64.download_state()
    s64.close()
    s = M.Solver(mesh, phys, P=P, precision=prec)
    s.upload_state(q0)
    s.step_n(dt, 12)
    q = s.download_state().astype(np.float64)
    s.close()
    assert rel_l2(q, q64) < 5e-6, rel_l2(q, q64)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["f32", "mixed"])
@pytest.mark.parametrize("P", [3, 4, 5])
def test_reduced_precision_l2_after_100_steps(P, prec):
    """Regression bound on a coarse 8^3 mesh: relative L2 against the FP64
    kernels after 100 SSPRK3 steps of the Euler smooth wave <= 2e-6
    (measured 0.7e-6 at P3; 1.2e-6 FP32 and 1.6e-6 split-BF16 at P4/P5).
    The error is FP32 state rounding, a random walk of ~0.7e-6 after 300
    stages, plus the FP32 flux and, for split-BF16, the 16-bit hi+lo
    operator.  Without exact stage weights (the reference's a q_a + b q_b
    with a = 1/3 and b = 2/3 rounded separately to FP32 sums to 1 + 3e-8)
    every variant drifts to ~3e-6.  The 1e-6 target is checked at the
    configuration sizes below."""
    err = _l2_after_100_steps(8, P, prec)
    print(f"8^3 P{P} {prec}: rel L2 vs FP64 after 100 steps {err:.2e}")
    assert err <= 2e-6, err


def _l2_after_100_steps(n, P, prec):
    phys = C.euler(M.FLUX_RUSANOV)
    mesh = M.Mesh(n, n, n)
    s64 = M.Solver(mesh, phys, P=P, precision="f64")
    s64.fill_ic(M.IC_SINE_WAVE, [1.0, 0.2, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0])
    q0 = s64.download_state()
    dt = 0.1 * (1.0 / n) / ((np.sqrt(3.0) + np.sqrt(GAMMA)) * (2 * P + 1))
    s64.step_n(dt, 100)
    q64 = s64.download_state()
    s64.close()
    s = M.Solver(mesh, phys, P=P, precision=prec)
    s.upload_state(q0)
    s.step_n(dt, 100)
    err = rel_l2(s.download_state().astype(np.float64), q64)
    s.close()
    return err


# The 1e-6 target after 100 steps, at the sizes the Euler configurations
# run: P3 on the 32^3 headline mesh (measured 7.0e-7 split-BF16, 7.4e-7
# FP32), P4 on 24^3 (9.3e-7, 8.1e-7), P5 on 16^3.  P5 misses it (1.20e-6
# split-BF16, 1.32e-6 FP32): the FP32 state alone, with FP64 fluxes and
# operator, is 0.7e-6 from FP64 after 300 roundings and the FP32 fluxes add
# the rest.  That case is an expected failure, strict, so that the miss
# stays visible here and a fix would show up as an unexpected pass.
P5_MISS = pytest.mark.xfail(strict=True, reason="FP32-state floor: P5 on 16^3 is 1.2e-6 to 1.3e-6 after 100 "
                                                "steps against the 1e-6 target")


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["mixed", "f32"])
@pytest.mark.parametrize("P,n", [(3, 32), (4, 24), pytest.param(5, 16, marks=P5_MISS)])
def test_l2_target_at_config_sizes(P, n, prec):
    err = _l2_after_100_steps(n, P, prec)
    print(f"{n}^3 P{P} {prec}: rel L2 vs FP64 after 100 steps {err:.2e}")
    assert err <= 1e-6, err


def alfven_case():
    """benchmarks/bench_mhd_alfven_3d_p3.mojo: 16 x 4 x 4 periodic slab, P=3,
    one Alfven period with dt = CFL h / (max(c_f, c_h) (2P+1))."""
    nx, ny, nz, lx, ly, lz = G["mhd_alfven_3d_p3.mesh"]
    gamma, rho0, b0, p0, amp = G["mhd_alfven_3d_p3.gamma_rho0_b0_p0_amp"]
    c_h, alpha_d = G["mhd_alfven_3d_p3.c_h_alpha_d"]
    ph = M.IdealMHD(gamma, 1e-6, 1e-6, c_h, alpha_d)
    cf = np.sqrt(gamma * p0 / rho0 + (b0 * b0 + amp * amp) / rho0)
    P = 3
    dt_est = G["mhd_alfven_3d_p3.cfl"] * (lx / nx) / (max(cf, c_h) * (2 * P + 1))
    nsteps = int(1.0 / dt_est) + 1
    mesh = (int(nx), int(ny), int(nz)), (lx, ly, lz)
    return ph, P, mesh, 1.0 / nsteps, nsteps, (rho0, b0, p0, amp, 1.0)


def alfven_state(xyz, gamma, rho0, b0, p0, amp, k, lx=1.0):
    s = np.sin(2 * np.pi * k * xyz[..., 0] / lx)
    q = np.zeros(xyz.shape[:-1] + (9,))
    v, by = amp * s, -amp * np.sqrt(rho0) * s
    q[..., 0], q[..., 2] = rho0, rho0 * v
    q[..., 4] = p0 / (gamma - 1) + 0.5 * rho0 * v * v + 0.5 * (b0 * b0 + by * by)
    q[..., 5], q[..., 6] = b0, by
    return q


_ALFVEN_ORACLE = {}


def alfven_oracle(oracle_mod):
    """(initial state, state after one period) of the FP64 oracle, computed once."""
    if "q" not in _ALFVEN_ORACLE:
        ph, P, (n, L), dt, nsteps, prm = alfven_case()
        o = oracle_mod.Oracle3D(P, n, L, M.physics_dict(ph))
        q0 = alfven_state(o.node_xyz(), ph.gamma, *prm)
        o.set(q0)
        o.step(dt, nsteps)
        _ALFVEN_ORACLE["q0"], _ALFVEN_ORACLE["q"] = q0, o.get()
    return _ALFVEN_ORACLE["q0"], _ALFVEN_ORACLE["q"]


def test_mhd_alfven_gate_oracle(oracle_mod):
    """The oracle's ideal MHD passes the reference bench's one-period gate."""
    q0, q = alfven_oracle(oracle_mod)
    assert np.isfinite(q).all()
    assert rel_l2(q, q0) < G["mhd_alfven_3d_p3.l2_max_rel"], rel_l2(q, q0)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["f64", "f32", "mixed"])
def test_mhd_alfven_gate_product(oracle_mod, prec):
    ph, P, (n, L), dt, nsteps, prm = alfven_case()
    s = M.Solver(M.Mesh(*n, *L), ph, P=P, precision=prec)
    s.fill_ic(M.IC_ALFVEN, list(prm))
    q0 = s.download_state().astype(np.float64)
    assert rel_l2(q0, alfven_state(s.node_xyz(), ph.gamma, *prm)) < (1e-14 if prec == "f64" else 1e-7)
    s.step_n(dt, nsteps)
    q = s.download_state().astype(np.float64)
    s.close()
    assert np.isfinite(q).all()
    err = rel_l2(q, q0)
    assert err < G["mhd_alfven_3d_p3.l2_max_rel"], err
    q0o, qo = alfven_oracle(oracle_mod)
    assert rel_l2(q0, q0o) < (1e-14 if prec == "f64" else 1e-7)
    d = rel_l2(q, qo)
    print(f"alfven {prec}: rel L2 vs IC {err:.3e}, vs oracle FP64 {d:.2e}")
    assert d < (1e-10 if prec == "f64" else 2e-4)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_two_fluid_langmuir_gate(prec):
    """benchmarks/bench_two_fluid_langmuir_3d_p3.mojo: a uniform electron
    velocity perturbation oscillates at the plasma frequency; after one
    period the mean electron momentum is back within 2 % and the mean E_x
    within 2 % of A m_e n0 omega_p."""
    nx, ny, nz, lx, ly, lz = G["langmuir_3d_p3.mesh"]
    ge, gi, qe, me, qi, mi, eps0, c = G["langmuir_3d_p3.species"]
    n0, pe, pi, a = G["langmuir_3d_p3.n0_pe_pi_upert"]
    c_h, alpha_d, rho_min, p_min = G["langmuir_3d_p3.c_h_alpha_d_rhomin_pmin"]
    ph = M.FiveMomentTwoFluid(ge, gi, qe, me, qi, mi, eps0, c, c_h, alpha_d, rho_min, p_min)
    P = 3
    s = M.Solver(M.Mesh(int(nx), int(ny), int(nz), lx, ly, lz), ph, P=P, precision=prec)
    rho_e, rho_i = me * n0, mi * n0
    state = [rho_e, rho_e * a, 0.0, 0.0, pe / (ge - 1) + 0.5 * rho_e * a * a,
             rho_i, 0.0, 0.0, 0.0, pi / (gi - 1)] + [0.0] * 7
    s.fill_ic(M.IC_CONSTANT, state)
    T = G["langmuir_3d_p3.t_final"]
    dt_est = G["langmuir_3d_p3.cfl"] * (lx / nx) / (max(c, c_h) * (2 * P + 1))
    nsteps = int(T / dt_est) + 1
    s.step_n(T / nsteps, nsteps)
    q = s.download_state().astype(np.float64)
    s.close()
    assert np.isfinite(q).all()
    wp = np.sqrt(n0 * (qe * qe / me + qi * qi / mi) / eps0)
    mom_err = abs(q[..., 1].mean() - a * me * n0) / (a * me * n0)
    ex_rel = abs(q[..., 10].mean()) / (a * me * n0 * wp)
    print(f"langmuir {prec}: {nsteps} steps, momentum drift {mom_err:.2e}, E_x {ex_rel:.2e}")
    assert mom_err < G["langmuir_3d_p3.drift_tol_rel"], mom_err
    assert ex_rel < G["langmuir_3d_p3.drift_tol_rel"], ex_rel
