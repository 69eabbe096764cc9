"""The Euler positivity floor (`limit_state`, src/euler.mojo:758-792) recovers
the pressure in FP64 in every precision.

Near vacuum the total energy E and the kinetic energy |m|^2 / 2 rho agree to
a few FP32 ulps, so an FP32 difference decides the floor on rounding noise.
One SSPRK3 stage with dt = 0 leaves q unchanged and then applies the floor,
so the stage output is the floor of the input; it must equal the FP64 floor
evaluated on the same FP32 inputs bit for bit.
"""
import numpy as np
import pytest

import mojoxm_b200 as M
from tests import dgcases as C

GAMMA, RHO_MIN, P_MIN = 1.4, 1e-6, 1e-6


def near_vacuum_state(shape, seed):
    """rho ~ U[0.5, 3], |u| ~ U[10, 1000] in a random direction, E within
    +-4 FP32 ulps of the kinetic energy (FP32 values)."""
    rng = np.random.default_rng(seed)
    n = shape[0] * shape[1]
    rho = rng.uniform(0.5, 3.0, n).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    u = d * rng.uniform(10.0, 1000.0, (n, 1))
    m = (rho[:, None].astype(np.float64) * u).astype(np.float32)
    m64 = m.astype(np.float64)
    ke = 0.5 * (m64[:, 0] * m64[:, 0] + m64[:, 1] * m64[:, 1] + m64[:, 2] * m64[:, 2]) * (1.0 / rho.astype(np.float64))
    E = (ke + ke * rng.uniform(-4.0, 4.0, n) * 2.0 ** -24).astype(np.float32)
    q = np.zeros((n, 5), np.float32)
    q[:, 0], q[:, 1:4], q[:, 4] = rho, m, E
    return q.reshape(shape)


def floor_f64(q):
    """The floor in FP64 on FP32 inputs, in the kernel's operation order."""
    q = q.reshape(-1, 5)
    out = q.copy()
    g1 = float(np.float32(GAMMA)) - 1.0
    pm = float(np.float32(P_MIN))
    rho = q[:, 0].astype(np.float64)
    m = q[:, 1:4].astype(np.float64)
    m2 = m[:, 0] * m[:, 0] + m[:, 1] * m[:, 1] + m[:, 2] * m[:, 2]
    ke = 0.5 * m2 * (1.0 / rho)
    p = g1 * (q[:, 4].astype(np.float64) - ke)
    low = ~(p > pm)
    out[low, 4] = (ke[low] + pm / g1).astype(np.float32)
    return out, low


def floor_f32(q):
    """The same floor evaluated in FP32 arithmetic (the reference's Float32)."""
    q = q.reshape(-1, 5)
    f = np.float32
    g1 = f(GAMMA) - f(1)
    m2 = q[:, 1] * q[:, 1] + q[:, 2] * q[:, 2] + q[:, 3] * q[:, 3]
    ke = f(0.5) * m2 / q[:, 0]
    p = g1 * (q[:, 4] - ke)
    return ~(p > f(P_MIN))


def test_near_vacuum_states_straddle_the_floor():
    """The test states are ones where FP32 and FP64 disagree about the floor
    for some nodes (otherwise the GPU test below could not tell them apart)."""
    q = near_vacuum_state((48 * 10, 1, 5), seed=5)
    _, low64 = floor_f64(q)
    low32 = floor_f32(q)
    assert 0 < low64.sum() < low64.size
    assert (low32 != low64).sum() > 0


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["f32", "mixed"])
@pytest.mark.parametrize("P", [2, 3])
def test_floor_is_fp64_on_fp32_inputs(prec, P):
    s = M.Solver(M.Mesh(2, 2, 2), C.euler(M.FLUX_RUSANOV), P=P, precision=prec)
    q = near_vacuum_state(s.shape, seed=11 + P)
    s.upload_state(q.astype(np.float64))
    s.rk_stage(0, 0.0)  # q1 = q + 0 * dt * rhs, then the floor
    out = s.download_state(1).reshape(-1, 5).astype(np.float32)
    s.close()
    want, low = floor_f64(q)
    assert 0 < low.sum() < low.size
    np.testing.assert_array_equal(out, want)
