"""Shared case builders for the parity tests: physics descriptors, seeded
states and tolerance rules.  Used by tests only."""
from __future__ import annotations

import numpy as np

import mojoxm_b200 as M

GAMMA = 1.4


def euler(flux, efix=False, g=(0.0, 0.0, 0.0), inflow=None):
    inflow = inflow or (0.0,) * 5
    return M.Euler(GAMMA, 1e-6, 1e-6, flux, efix, *g, *inflow)


PHYSICS_3D = {
    "advection": lambda: M.Advection(0.7, -0.4, 0.3, inflow_q=0.25),
    "euler_rusanov": lambda: euler(M.FLUX_RUSANOV, g=(0.1, -0.2, 0.3), inflow=(1.1, 0.2, -0.1, 0.05, 2.7)),
    "euler_roe": lambda: euler(M.FLUX_ROE, inflow=(1.1, 0.2, -0.1, 0.05, 2.7)),
    "euler_roe_fix": lambda: euler(M.FLUX_ROE, efix=True),
    "euler_hlle": lambda: euler(M.FLUX_HLLE, inflow=(1.1, 0.2, -0.1, 0.05, 2.7)),
    "euler_hlle_fix": lambda: euler(M.FLUX_HLLE, efix=True),
    "euler_hllec": lambda: euler(M.FLUX_HLLEC, inflow=(1.1, 0.2, -0.1, 0.05, 2.7)),
    "euler_hllec_fix": lambda: euler(M.FLUX_HLLEC, efix=True),
    "maxwell": lambda: M.Maxwell(1.0, 0.1, -0.2, 0.05, 0.02, 0.0, -0.03, 0.1, 0.2, -0.1, 0.05, 0.0, 0.1),
    "shallow_water": lambda: M.ShallowWater(9.81, 1e-6, 1.5, 0.2, -0.1),
    "mhd": lambda: M.IdealMHD(5.0 / 3.0, 1e-6, 1e-6, 1.3, 0.4, 1.1, 0.2, -0.1, 0.05, 3.0, 0.3, -0.2, 0.1, 0.02),
}

# 17 components, FP64 at P <= 4 only (P5 exceeds the stage tile), so kept
# out of the tables the generic parity tests iterate over
def two_fluid():
    return M.FiveMomentTwoFluid(5.0 / 3.0, 5.0 / 3.0, -1.0, 1.0, 1.0, 25.0, 1.0, 10.0, 12.0, 0.5, 1e-6, 1e-8,
                                inflow=(1.1, 0.1, 0.0, 0.0, 0.8, 26.0, 0.5, 0.0, 0.0, 1.2,
                                        0.0, 0.1, 0.0, 0.3, 0.0, 0.0, 0.0))


PHYSICS_2D = {
    "advection": lambda: M.Advection(0.7, -0.4, 0.0, inflow_q=0.25),
    "euler_rusanov": lambda: euler(M.FLUX_RUSANOV, g=(0.1, -0.2, 0.0), inflow=(1.1, 0.2, -0.1, 0.0, 2.7)),
    "euler_hllc": lambda: euler(M.FLUX_HLLC, inflow=(1.1, 0.2, -0.1, 0.0, 2.7)),
    "euler_hlle": lambda: euler(M.FLUX_HLLE, inflow=(1.1, 0.2, -0.1, 0.0, 2.7)),
    "maxwell": lambda: M.Maxwell(1.0, 0.1, -0.2, 0.05, 0.02, 0.0, -0.03, 0.1, 0.2, -0.1, 0.05, 0.0, 0.1),
    "shallow_water": lambda: M.ShallowWater(9.81, 1e-6, 1.5, 0.2, -0.1),
    "shallow_water_hll": lambda: M.ShallowWater(9.81, 1e-6, 1.5, 0.2, -0.1, flux_type=M.FLUX_HLL),
    "mhd_glm": lambda: M.IdealMHD(5.0 / 3.0, 1e-6, 1e-6, 1.3, 0.4, 1.1, 0.2, -0.1, 0.0, 3.0, 0.3, -0.2, 0.0, 0.02),
    "mhd_plain": lambda: M.IdealMHDPlain(5.0 / 3.0, 1e-6, 1e-6, 0.0, 0.0, 1.1, 0.2, -0.1, 0.0, 3.0, 0.3, -0.2),
}

BCS_3D = {
    "periodic": (0, 0, 0, 0, 0, 0),
    "walls": (1, 1, 1, 1, 1, 1),
    "outflow_x_wall_yz": (2, 2, 1, 1, 1, 1),
    "inflow_outflow": (3, 2, 1, 1, 0, 0),
    "mixed_lo_only": (1, 0, 0, 2, 0, 0),
}
BCS_2D = {
    "periodic": (0, 0, 0, 0),
    "walls": (1, 1, 1, 1),
    "inflow_outflow": (3, 2, 1, 1),
    "mixed_hi_only": (0, 2, 1, 0),
}


def random_state(shape, physics, seed, xyz=None):
    """Seeded non-constant admissible state (positive density/pressure/depth)."""
    rng = np.random.default_rng(seed)
    ne, npn, nc = shape
    q = np.zeros(shape)
    k = physics.kind
    if k == M.PHYS_EULER:
        rho = 1.0 + 0.2 * rng.uniform(-1, 1, (ne, npn))
        vel = 0.5 * rng.uniform(-1, 1, (ne, npn, 3))
        p = 1.0 + 0.2 * rng.uniform(-1, 1, (ne, npn))
        if nc == 5:
            q[..., 0] = rho
            q[..., 1:4] = rho[..., None] * vel
            q[..., 4] = p / (GAMMA - 1) + 0.5 * rho * (vel ** 2).sum(-1)
        else:
            q[..., 0] = rho
            q[..., 1:3] = rho[..., None] * vel[..., :2]
            q[..., 3] = p / (GAMMA - 1) + 0.5 * rho * (vel[..., :2] ** 2).sum(-1)
    elif k in (M.PHYS_MHD, M.PHYS_MHD_PLAIN) and nc in (6, 7):  # 2D (rho, mx, my, Bx, By, E[, psi])
        rho = 1.0 + 0.2 * rng.uniform(-1, 1, (ne, npn))
        vel = 0.5 * rng.uniform(-1, 1, (ne, npn, 2))
        B = 0.5 * rng.uniform(-1, 1, (ne, npn, 2))
        p = 1.0 + 0.2 * rng.uniform(-1, 1, (ne, npn))
        q[..., 0] = rho
        q[..., 1:3] = rho[..., None] * vel
        q[..., 3:5] = B
        q[..., 5] = p / (5.0 / 3.0 - 1) + 0.5 * rho * (vel ** 2).sum(-1) + 0.5 * (B ** 2).sum(-1)
        if nc == 7:
            q[..., 6] = 0.1 * rng.uniform(-1, 1, (ne, npn))
    elif k == M.PHYS_MHD:
        rho = 1.0 + 0.2 * rng.uniform(-1, 1, (ne, npn))
        vel = 0.5 * rng.uniform(-1, 1, (ne, npn, 3))
        B = 0.5 * rng.uniform(-1, 1, (ne, npn, 3))
        p = 1.0 + 0.2 * rng.uniform(-1, 1, (ne, npn))
        q[..., 0] = rho
        q[..., 1:4] = rho[..., None] * vel
        q[..., 4] = p / (5.0 / 3.0 - 1) + 0.5 * rho * (vel ** 2).sum(-1) + 0.5 * (B ** 2).sum(-1)
        q[..., 5:8] = B
        q[..., 8] = 0.1 * rng.uniform(-1, 1, (ne, npn))
    elif k == M.PHYS_TWO_FLUID:
        for off, rho0 in ((0, 1.0), (5, 25.0)):  # electrons, ions
            rho = rho0 * (1.0 + 0.2 * rng.uniform(-1, 1, (ne, npn)))
            vel = 0.3 * rng.uniform(-1, 1, (ne, npn, 3))
            p = 0.5 + 0.1 * rng.uniform(-1, 1, (ne, npn))
            q[..., off] = rho
            q[..., off + 1:off + 4] = rho[..., None] * vel
            q[..., off + 4] = p / (5.0 / 3.0 - 1) + 0.5 * rho * (vel ** 2).sum(-1)
        q[..., 10:13] = 0.2 * rng.uniform(-1, 1, (ne, npn, 3))
        q[..., 13:16] = 0.3 * rng.uniform(-1, 1, (ne, npn, 3))
        q[..., 16] = 0.05 * rng.uniform(-1, 1, (ne, npn))
    elif k == M.PHYS_SHALLOW_WATER:
        h = 1.0 + 0.3 * rng.uniform(-1, 1, (ne, npn))
        q[..., 0] = h
        q[..., 1:3] = h[..., None] * 0.5 * rng.uniform(-1, 1, (ne, npn, 2))
    else:
        q[:] = rng.uniform(-1, 1, shape)
    return q


def rel_err(a, b):
    """max |a - b| / max |b| (per whole array)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


# FP64 RHS parity bound product-vs-oracle.  The product builds its operators
# in binary128 (correctly rounded FP64); the oracle follows the reference's
# FP64 construction, whose own rounding grows with P (3D D/Lift: 1e-15 at
# P2 .. 6e-14 at P5; 2D edge lift: up to 1.4e-9 at P5, reference_2d.mojo:
# 278-306).  The bound is that operator discrepancy plus accumulation slack.
TOL_F64_3D = {1: 1e-12, 2: 1e-12, 3: 1e-12, 4: 2e-12, 5: 5e-12}
TOL_F64_2D = {1: 1e-12, 2: 1e-12, 3: 1e-11, 4: 2e-10, 5: 1e-8}
# FP32 product vs FP32 oracle RHS (both mimic the reference's Float32
# arithmetic; summation order and fused multiply-adds differ).  Measured on a
# B200 for every 3D physics at P1..P5 and the two-fluid state: 1.7e-7 ..
# 1.2e-6 (largest: shallow water P5); the bound is about 3x the largest.
TOL_F32 = 4e-6
