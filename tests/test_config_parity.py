"""CUDA path vs the CPU oracle at the benchmark configurations' full sizes.

The small-mesh parity tables (test_gpu_parity.py) cover every physics, flux,
order and boundary arm on meshes of a few tiles.  Tile-boundary and
occupancy effects show only at the sizes the benchmarks run, where a
launch has thousands of tiles, every block loops over many of them and the
state spills out of L2.  So here the product is compared with the FP64
oracle at those sizes:

* 3D Euler smooth density wave, periodic [0,1]^3, 32^3 x 6 = 196,608 tets,
  P = 3, Rusanov: the RHS and one SSPRK3 stage, in FP64 and in the
  tensor-core precision (FP32 state, split-BF16 tcgen05 contraction);
* 3D Maxwell PEC cavity, 24^3 x 6 = 82,944 tets, P = 4, Rusanov: the RHS in
  FP64 and in the tensor-core precisions;
* batched 2D Euler (HLLE, limiter on): the first 16 members of the batched
  workload's seeded draw (n in {16..256}, P in 1..5, vortex / Sod ICs), one
  batched SSPRK3 step against the oracle stepping each member alone.

Errors are per component: relative L2 (||a - b|| / ||b||) and relative L-inf
(max |a - b| / max |b|); the bounds are written beside each case.
"""
import numpy as np
import pytest

import bench
import mojoxm_b200 as M
from tests import dgcases as C

pytestmark = pytest.mark.gpu


def per_component(a, b):
    """[(rel L2, rel Linf)] per component of (..., NC) arrays."""
    a = np.asarray(a, np.float64).reshape(-1, a.shape[-1])
    b = np.asarray(b, np.float64).reshape(-1, b.shape[-1])
    out = []
    for c in range(a.shape[1]):
        d = a[:, c] - b[:, c]
        out.append((float(np.linalg.norm(d) / max(np.linalg.norm(b[:, c]), 1e-300)),
                    float(np.abs(d).max() / max(np.abs(b[:, c]).max(), 1e-300))))
    return out


def smooth_wave_perturbed(xyz, seed):
    """The headline initial state (rho = 1 + 0.2 sin(2 pi (x+y+z)), u = (1,1,1),
    p = 1) with a seeded 1 % nodal perturbation of every component, so that
    no component's RHS is degenerate."""
    q = bench.smooth_wave_state(xyz)
    rng = np.random.default_rng(seed)
    return q * (1.0 + 0.01 * rng.uniform(-1, 1, q.shape))


# Bounds at 32^3 P3 (relative per component).  FP64: operator rounding only
# (the product builds its operators in binary128, the oracle as the
# reference does in FP64).  Tensor-core precision: FP32 fluxes and
# Riemann solves plus the 16-bit split operands; the stage adds dt * RHS to
# an FP32 state, so its error is the state's rounding (6e-8) plus dt times
# the RHS error.
C2_RHS = {"f64": (2e-13, 5e-13), "mixed": (3e-5, 5e-5)}
C2_STAGE = {"f64": (5e-16, 5e-15), "mixed": (1e-7, 5e-7)}


@pytest.mark.parametrize("prec", ["f64", "mixed"])
def test_c2_rhs_and_stage_vs_oracle(oracle_mod, prec):
    n, P = 32, 3
    phys = M.Euler(1.4, 1e-6, 1e-6, M.FLUX_RUSANOV, False)
    s = M.Solver(M.Mesh(n, n, n), phys, P=P, precision=prec)
    o = oracle_mod.Oracle3D(P, n, 1.0, M.physics_dict(phys))
    q = smooth_wave_perturbed(o.node_xyz(), seed=3)
    if prec != "f64":
        q = q.astype(np.float32).astype(np.float64)
    errs = per_component(s.rhs(q), o.rhs(q))
    print(f"C2 {prec} RHS per component (rel L2, rel Linf): " + ", ".join(f"({a:.2e}, {b:.2e})" for a, b in errs))
    l2_bound, inf_bound = C2_RHS[prec]
    for l2, linf in errs:
        assert l2 <= l2_bound and linf <= inf_bound
    dt = bench.dt_for(n, P)
    s.upload_state(q)
    o.set(q)
    s.rk_stage(0, dt)
    o.stage(0, dt)
    errs = per_component(s.download_state(1), o.get(1))
    print(f"C2 {prec} stage 0 per component: " + ", ".join(f"({a:.2e}, {b:.2e})" for a, b in errs))
    l2_bound, inf_bound = C2_STAGE[prec]
    for l2, linf in errs:
        assert l2 <= l2_bound and linf <= inf_bound
    s.close()


C3_RHS = {"f64": (1e-13, 2e-13), "mixed": (2e-5, 5e-5), "tf32": (2e-6, 5e-6)}


@pytest.mark.parametrize("prec", ["f64", "mixed", "tf32"])
def test_c3_maxwell_rhs_vs_oracle(oracle_mod, prec):
    n, P = 24, 4
    bcs = (1, 1, 1, 1, 0, 0)
    phys = M.Maxwell(1.0, *([0.0] * 12))
    s = M.Solver(M.Mesh(n, n, n, bcs=M.BoundaryConditions(*bcs)), phys, P=P, precision=prec)
    o = oracle_mod.Oracle3D(P, n, 1.0, M.physics_dict(phys), bcs=bcs)
    s.fill_ic(M.IC_CAVITY, [1.0, 1.0, 1.0])
    q = s.download_state().astype(np.float64)
    rng = np.random.default_rng(5)
    q = q + 0.05 * rng.uniform(-1, 1, q.shape)  # every field component non-zero
    if prec != "f64":
        q = q.astype(np.float32).astype(np.float64)
    errs = per_component(s.rhs(q), o.rhs(q))
    print(f"C3 {prec} RHS per component (rel L2, rel Linf): " + ", ".join(f"({a:.2e}, {b:.2e})" for a, b in errs))
    l2_bound, inf_bound = C3_RHS[prec]
    for l2, linf in errs:
        assert l2 <= l2_bound and linf <= inf_bound
    s.close()


# One batched SSPRK3 step (limiter on) against the oracle stepping each
# member alone from the same initial state with the same dt.  FP64: the
# operator discrepancy of the 2D construction (C.TOL_F64_2D) with slack for
# the three stages; FP32: against the oracle in FP32 (the reference's own
# arithmetic), within the FP32 parity bound.
C4_MEMBERS = 16
# one limited FP32 SSPRK3 step against the FP32 oracle's: the RHS
# differences of FP32 summation order pass through three stages and the
# limiter's theta.  Measured on a B200 over the 16 members: 1.7e-7 ..
# 5.9e-7; the bound is about 3x the largest.
C4_TOL_F32 = 2e-6


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_c4_batched_members_vs_oracle(oracle_mod, prec):
    rng = np.random.default_rng(2024)  # the batched workload's seed
    batch = M.Batch()
    members = []
    for _ in range(C4_MEMBERS):
        s, kind, h = bench.batch_member(M, rng, prec)
        dt = 0.3 * h / ((2 * s.P + 1) * s.max_wavespeed())
        q0 = s.download_state().astype(np.float64)
        batch.add(s, dt)
        members.append((s, kind, dt, q0))
    batch.step(1)
    batch.synchronize()
    worst = 0.0
    for s, kind, dt, q0 in members:
        m = s.mesh
        o = oracle_mod.Oracle2D(s.P, (m.nx, m.ny), (m.lx, m.ly), M.physics_dict(s.physics),
                                bcs=tuple(m.bcs.as_list()[:4]), real=prec)
        o.enable_limiter(True, 0.1)
        o.set(q0)
        o.step(dt, 1)
        got, want = s.download_state().astype(np.float64), o.get(0)
        err = C.rel_err(got, want)
        bound = 50 * C.TOL_F64_2D[s.P] if prec == "f64" else C4_TOL_F32
        print(f"C4 {prec} member n={m.nx} P={s.P} {kind}: rel err {err:.2e} (bound {bound:.0e})")
        assert err <= bound, (m.nx, s.P, kind, err)
        worst = max(worst, err)
    print(f"C4 {prec}: worst member rel err {worst:.2e}")
    batch.close()
    for s, *_ in members:
        s.close()
