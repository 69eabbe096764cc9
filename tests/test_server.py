"""Serving loop (mxm_dg_server_*) and the device IC fill it uses.

* Each request's result is the same alone and in a mix of concurrent
  requests (bit for bit: every solve runs single-solve arithmetic on its own
  buffers), and equals the same solve run directly through a solver handle.
* Admission respects the HBM budget: with room for one solve at a time the
  peak concurrency is 1 and everything still completes.
* The device IC fill matches the IC formula evaluated at the node
  coordinates."""
import numpy as np
import pytest

import mojoxm_b200 as M
from tests import dgcases as C

GAMMA = 1.4


def _euler3d():
    return C.euler(M.FLUX_RUSANOV)


def _requests():
    # (mesh, physics, P, precision, ic kind, ic params, dt, nsteps, limiter eps)
    wave = [1.0, 0.2, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0]
    return [
        (M.Mesh(6, 6, 6), _euler3d(), 2, "f32", M.IC_SINE_WAVE, wave, 1e-3, 23, None),
        (M.Mesh(16, 12, lx=10.0, ly=10.0, dim=2), C.euler(M.FLUX_HLLE), 3, "f32", M.IC_VORTEX,
         [5.0, 5.0, 5.0, 1.0, 1.0, 0.0, 1.0], 2e-3, 31, 0.1),
        (M.Mesh(20, 4, lx=1.0, ly=0.2, dim=2, bcs=M.BoundaryConditions(1, 1, 1, 1)), M.ShallowWater(9.81, 1e-6, 1.0, 0, 0),
         2, "f32", M.IC_DAM_BREAK, [2.0, 1.0, 0.5, 0.02], 1e-4, 17, None),
        (M.Mesh(4, 4, 3, bcs=M.BoundaryConditions(1, 1, 1, 1, 0, 0)), M.Maxwell(1.0, *([0.0] * 12)), 4, "f32",
         M.IC_CAVITY, [1.0, 1.0, 1.0], 5e-4, 12, None),
        (M.Mesh(5, 5, 5), _euler3d(), 3, "mixed", M.IC_SINE_WAVE, wave, 5e-4, 9, None),
        (M.Mesh(12, 3, dim=2, bcs=M.BoundaryConditions(2, 2, 1, 1)), C.euler(M.FLUX_HLLE), 2, "f64", M.IC_SOD,
         [1.0, 1.0, 0.125, 0.1, 0.5, 0.02], 1e-3, 14, 0.1),
    ]


def _direct(req):
    mesh, phys, P, prec, kind, prm, dt, n, eps = req
    s = M.Solver(mesh, phys, P=P, precision=prec)
    if eps is not None:
        s.enable_cell_limiter(True, eps)
    s.fill_ic(kind, prm)
    s.step_n(dt, n)
    out = s.download_state()
    s.close()
    return out


@pytest.mark.gpu
def test_result_alone_equals_in_mix_and_direct():
    reqs = _requests()
    probe = 1  # the 2D vortex
    alone = M.Server(hbm_budget_bytes=8e9, max_active=8, steps_per_chunk=4)
    rid = alone.submit(*reqs[probe])
    q_alone = alone.result(rid).copy()
    alone.close()

    mix = M.Server(hbm_budget_bytes=8e9, max_active=8, steps_per_chunk=4)
    ids = [mix.submit(*r) for r in reqs]
    outs = [mix.result(i).copy() for i in ids]
    st = mix.stats()
    mix.close()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert st["p99_ms"] >= st["p50_ms"] > 0
    assert st["peak_concurrent"] >= 2  # they did overlap
    assert np.array_equal(outs[probe], q_alone)
    for r, o in zip(reqs, outs):
        assert np.isfinite(o).all()
        assert np.array_equal(o, _direct(r)), r[1]


@pytest.mark.gpu
def test_admission_by_hbm_budget():
    # three equal requests, budget for one and a half of them
    req = _requests()[0]
    mesh, phys, P, prec, *_ = req
    ne, NP, NC = M.state_shape(mesh, phys, P)
    one = (3 * ne * NP * NC + ne * NC) * (8 if prec == "f64" else 4)
    srv = M.Server(hbm_budget_bytes=1.5 * one, max_active=8, steps_per_chunk=8)
    ids = [srv.submit(*req) for _ in range(3)]
    for i in ids:
        srv.wait(i)
    st = srv.stats()
    outs = [srv.result(i) for i in ids]
    srv.close()
    assert st["completed"] == 3 and st["peak_concurrent"] == 1
    assert one <= st["peak_bytes"] <= 1.5 * one
    assert all(np.array_equal(o, outs[0]) for o in outs)


@pytest.mark.gpu
def test_server_rejects_bad_requests():
    srv = M.Server(hbm_budget_bytes=1e6, max_active=2)
    with pytest.raises(M.DGError):  # larger than the budget
        srv.submit(M.Mesh(16, 16, 16), _euler3d(), 3, "f64", M.IC_CONSTANT, [1, 0, 0, 0, 2.5], 1e-3, 1)
    with pytest.raises(M.DGError):  # order out of range
        srv.submit(M.Mesh(2, 2, 2), _euler3d(), 7, "f64", M.IC_CONSTANT, [1, 0, 0, 0, 2.5], 1e-3, 1)
    srv.close()


@pytest.mark.gpu
def test_fill_ic_matches_formula():
    s = M.Solver(M.Mesh(4, 5, 3, 1.0, 1.2, 0.8), _euler3d(), P=3, precision="f64")
    s.fill_ic(M.IC_SINE_WAVE, [1.0, 0.2, 0.5, -0.3, 0.2, 0.9, 1.0, 2.0, 1.0])
    q = s.download_state()
    x = s.node_xyz()  # FP32 node coordinates of the reference's construction
    rho = 1.0 + 0.2 * np.sin(2 * np.pi * (x[..., 0] + 2 * x[..., 1] + x[..., 2]))
    assert np.abs(q[..., 0] - rho).max() < 1e-6
    assert np.allclose(q[..., 1] / q[..., 0], 0.5, atol=1e-12)
    E = 0.9 / (GAMMA - 1) + 0.5 * rho * (0.25 + 0.09 + 0.04)
    assert np.abs(q[..., 4] - E).max() < 1e-6
    s.close()
    # 2D vortex at its centre: density minimum T^(1/(g-1)) near (x0, y0)
    s2 = M.Solver(M.Mesh(20, 20, lx=10.0, ly=10.0, dim=2), C.euler(M.FLUX_HLLE), P=2, precision="f64")
    s2.fill_ic(M.IC_VORTEX, [5.0, 5.0, 5.0, 0.0, 0.0, 0.0, 0.0])
    q2 = s2.download_state()
    beta = 5.0
    T0 = 1 - (GAMMA - 1) * beta ** 2 / (8 * GAMMA * np.pi ** 2) * np.e
    assert q2[..., 0].min() >= T0 ** (1 / (GAMMA - 1)) - 1e-12
    assert q2[..., 0].max() <= 1.0
    s2.close()
