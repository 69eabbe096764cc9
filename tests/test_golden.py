"""Known answers from the reference's own tests (tests/golden/known_answers.json,
made by tests/golden/make_golden.py from the cited reference files).

CPU tests pin the oracle to those answers: the Gauss-Jordan inverse, the P=2
node weights, the exact Sod solver, the SSPRK3 stage plans, constant-state
preservation and limiter mean conservation.  The GPU tests hold the product
(through the C ABI) to the same answers."""
import json
import os

import numpy as np
import pytest

import mojoxm_b200 as M
from tests import dgcases as C

HERE = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(HERE, "golden", "known_answers.json")) as _f:
    G = json.load(_f)["values"]


# ------------------------------------------------------------- oracle (CPU)
@pytest.mark.parametrize("case", ["case_2x2", "case_pivot"])
def test_mat_inv_known_answers(oracle_mod, case):
    a = np.array(G[f"mat_inv.{case}.in"]).reshape(2, 2)
    want = np.array(G[f"mat_inv.{case}.out"]).reshape(2, 2)
    assert np.abs(oracle_mod.mat_inv(a) - want).max() <= G["mat_inv.tol"]
    assert np.abs(oracle_mod.mat_inv(np.eye(3)) - np.eye(3)).max() <= G["mat_inv.tol"]


def test_p2_node_weights(oracle_mod):
    w = np.sort(oracle_mod.refelem3d(2)["w"])
    want = np.sort([G["refelem.p2_vertex_weight"]] * 4 + [G["refelem.p2_edge_weight"]] * 6)
    assert np.abs(w - want).max() <= 1e-14


@pytest.mark.parametrize("P", [1, 2, 3, 4, 5])
def test_weights_sum_and_node_separation(oracle_mod, P):
    r = oracle_mod.refelem3d(P)
    assert abs(r["w"].sum() - 1.0) <= 1e-13
    x = r["node_pos"]
    d = np.sqrt(((x[:, None, :] - x[None, :, :]) ** 2).sum(-1)) + np.eye(len(x)) * 10
    assert d.min() >= G["refelem.min_node_separation_factor"] / P * 0.99
    assert abs(oracle_mod.refelem2d(P)["w"].sum() - 1.0) <= 1e-12
    # the library's own binary128 operators carry the same weights
    _, _, w = M.reference_operators(3, P)
    assert np.abs(np.sort(w) - np.sort(r["w"])).max() <= 1e-14


def _shock_speed(rhoR, pR, gamma, ps, uR=0.0):
    aR = np.sqrt(gamma * pR / rhoR)
    return uR + aR * np.sqrt((gamma + 1) / (2 * gamma) * ps / pR + (gamma - 1) / (2 * gamma))


def test_sod_canonical(oracle_mod):
    rL, pL, rR, pR, g = G["sod.canonical.state"]
    t, tight, loose = G["sod.canonical.samples_t"], G["sod.eps_tight"], G["sod.eps_loose"]
    x = np.array([0.0, 1.0, G["sod.canonical.x_star_L"], G["sod.canonical.x_star_R"]])
    rho, _, _ = oracle_mod.sod_exact(x, t, rL, 0.0, pL, rR, 0.0, pR, g)
    assert abs(rho[0] - rL) <= tight and abs(rho[1] - rR) <= tight
    assert abs(rho[2] - G["sod.canonical.rho_star_L"]) <= loose
    assert abs(rho[3] - G["sod.canonical.rho_star_R"]) <= loose
    ps = oracle_mod.sod_star(rL, 0.0, pL, rR, 0.0, pR, g)[0]
    assert abs(_shock_speed(rR, pR, g, ps) - G["sod.canonical.S_R"]) <= loose
    fan, _, _ = oracle_mod.sod_exact(np.array(G["sod.canonical.fan_x"]), t, rL, 0.0, pL, rR, 0.0, pR, g)
    assert np.all(np.diff(fan) <= 1e-12)
    uni, _, _ = oracle_mod.sod_exact(np.array([0.5]), t, rL, 0.0, pL, rL, 0.0, pL, g)
    assert abs(uni[0] - rL) <= tight


def test_sod_toro3(oracle_mod):
    rL, pL, rR, pR, g = G["sod.toro3.state"]
    t, loose = G["sod.toro3.t"], G["sod.eps_loose"]
    rho, _, _ = oracle_mod.sod_exact(np.array([G["sod.toro3.x_star_L"], G["sod.toro3.x_star_R"]]), t,
                                     rL, 0.0, pL, rR, 0.0, pR, g)
    assert abs(rho[0] - G["sod.toro3.rho_star_L"]) <= loose
    assert abs(rho[1] - G["sod.toro3.rho_star_R"]) <= loose
    ps = oracle_mod.sod_star(rL, 0.0, pL, rR, 0.0, pR, g)[0]
    assert abs(_shock_speed(rR, pR, g, ps) - G["sod.toro3.S_R"]) <= G["sod.toro3.S_R_tol"]


def _stage_plan_probe(run_stage, set_buf, get_buf, shape, seed=5):
    """Recover (q_in, q_a, q_b, q_out) routing and (a, b) of each stage with a
    zero right-hand side: three random buffers, one stage, least squares."""
    rng = np.random.default_rng(seed)
    names = ["q", "q1", "q2"]
    plans = []
    for s in range(3):
        bufs = [rng.uniform(0.5, 1.5, shape) for _ in range(3)]
        for k in range(3):
            set_buf(bufs[k], k)
        run_stage(s)
        outs = [get_buf(k) for k in range(3)]
        changed = [k for k in range(3) if np.abs(outs[k] - bufs[k]).max() > 1e-12]
        assert len(changed) == 1
        o = changed[0]
        A = np.stack([b.reshape(-1) for b in bufs], 1)
        coef, *_ = np.linalg.lstsq(A, outs[o].reshape(-1), rcond=None)
        plans.append((o, coef))
    for s, (o, coef) in enumerate(plans):
        a, b, _ = G["ssprk3.coeffs"][s]
        route = G["ssprk3.routing"][s]
        assert names[o] == route[3]
        want = np.zeros(3)
        want[names.index(route[1])] += a
        want[names.index(route[2])] += b
        assert np.abs(coef - want).max() <= 1e-12, (s, coef, want)


def test_ssprk3_stage_plans_oracle(oracle_mod):
    ph = M.Advection(0.0, 0.0, 0.0)
    o = oracle_mod.Oracle3D(2, 2, 1.0, M.physics_dict(ph))
    _stage_plan_probe(lambda s: o.stage(s, 0.1), o.set, o.get, o.shape)


def _const_state():
    r, u, v, w, p, g = G["euler3d_const.state"]
    return np.array([r, r * u, r * v, r * w, p / (g - 1) + 0.5 * r * (u * u + v * v + w * w)]), (r, u, v, w, p, g)


def _const_dt(P):
    nx, _, _, L = G["euler3d_const.mesh"]
    _, (r, u, v, w, p, g) = _const_state()
    speed = np.sqrt(u * u + v * v + w * w) + np.sqrt(g * p / r)
    return G["euler3d_const.cfl"] * (L / nx) / (speed * (2 * P + 1))


@pytest.mark.parametrize("real", ["f32", "f64"])
@pytest.mark.parametrize("P", [2, 3, 4, 5])
def test_constant_state_oracle(oracle_mod, P, real):
    nx, ny, nz, L = G["euler3d_const.mesh"]
    ph = C.euler(M.FLUX_HLLEC)
    o = oracle_mod.Oracle3D(P, (nx, ny, nz), L, M.physics_dict(ph), real=real)
    q0 = np.broadcast_to(_const_state()[0], o.shape).copy()
    o.set(q0)
    o.step(_const_dt(P), G["euler3d_const.steps"])
    assert np.abs(o.get() - q0).max() <= G["euler3d_const.tol"]


def _jitter_state(shape):
    q = np.broadcast_to(np.array(G["limiter3d.background"]), shape).copy()
    j = G["limiter3d.jitter"]
    q[:, 0::2, 0] += j
    q[:, 1::2, 0] -= j
    return q


def _cell_means(q, w):
    return np.einsum("enc,n->ec", q, w)


@pytest.mark.parametrize("real", ["f32", "f64"])
def test_limiter_conservation_oracle(oracle_mod, real):
    P = G["limiter3d.P"]
    o = oracle_mod.Oracle3D(P, 4, 1.0, M.physics_dict(C.euler(M.FLUX_HLLEC)), real=real)
    w = oracle_mod.refelem3d(P)["w"]
    o.enable_limiter(True, G["limiter3d.eps"])
    qc = np.broadcast_to(np.array(G["limiter3d.background"]), o.shape).copy()
    o.set(qc)
    o.limit()
    assert np.abs(o.get() - qc).max() <= G["limiter3d.const_tol"]
    q = _jitter_state(o.shape)
    o.set(q)
    o.limit()
    out = o.get()
    assert np.abs(_cell_means(out, w) - _cell_means(q, w)).max() <= G["limiter3d.mean_tol"]
    assert np.abs(out - q).max() > G["limiter3d.fired_min"]


# ------------------------------------------------------------ product (GPU)
@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_ssprk3_stage_plans_product(prec):
    s = M.Solver(M.Mesh(2, 2, 2), M.Advection(0.0, 0.0, 0.0), P=2, precision=prec)

    def get(k):
        return s.download_state(k).astype(np.float64)

    if prec == "f64":
        _stage_plan_probe(lambda st: s.rk_stage(st, 0.1), lambda q, k: s.upload_state(q, k), get, s.shape)
    else:
        # FP32 buffers: compare with the stated combine directly, to FP32 round-off
        rng = np.random.default_rng(5)
        names = ["q", "q1", "q2"]
        for st in range(3):
            bufs = [rng.uniform(0.5, 1.5, s.shape).astype(np.float32).astype(np.float64) for _ in range(3)]
            for k in range(3):
                s.upload_state(bufs[k], k)
            s.rk_stage(st, 0.1)
            a, b, _ = G["ssprk3.coeffs"][st]
            route = G["ssprk3.routing"][st]
            want = a * bufs[names.index(route[1])] + b * bufs[names.index(route[2])]
            assert np.abs(get(names.index(route[3])) - want).max() <= 4e-7
    s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["f64", "f32", "mixed"])
@pytest.mark.parametrize("P", [2, 3, 4, 5])
def test_constant_state_product(P, prec):
    nx, ny, nz, L = G["euler3d_const.mesh"]
    s = M.Solver(M.Mesh(nx, ny, nz, L, L, L), C.euler(M.FLUX_HLLEC), P=P, precision=prec)
    q0 = np.broadcast_to(_const_state()[0], s.shape).copy()
    s.upload_state(q0)
    s.step_n(_const_dt(P), G["euler3d_const.steps"])
    assert np.abs(s.download_state().astype(np.float64) - q0).max() <= G["euler3d_const.tol"]
    s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_limiter_conservation_product(prec):
    P = G["limiter3d.P"]
    s = M.Solver(M.Mesh(4, 4, 4), C.euler(M.FLUX_HLLEC), P=P, precision=prec)
    _, _, w = M.reference_operators(3, P)
    s.enable_cell_limiter(True, G["limiter3d.eps"])
    qc = np.broadcast_to(np.array(G["limiter3d.background"]), s.shape).copy()
    s.upload_state(qc)
    s.limit()
    assert np.abs(s.download_state().astype(np.float64) - qc).max() <= G["limiter3d.const_tol"]
    q = _jitter_state(s.shape)
    s.upload_state(q)
    s.limit()
    out = s.download_state().astype(np.float64)
    assert np.abs(_cell_means(out, w) - _cell_means(q, w)).max() <= G["limiter3d.mean_tol"]
    assert np.abs(out - q).max() > G["limiter3d.fired_min"]
    s.close()


def test_oracle_mhd_constant_state_and_conducting_wall(oracle_mod):
    """Ideal MHD (src/mhd.mojo): a uniform magnetised state is steady on a
    periodic mesh, and at a conducting wall a state at rest with B tangent to
    the wall gives no mass or normal-B flux (the ghost reflects u_n and B_n)."""
    ph = M.IdealMHD(5.0 / 3.0, 1e-6, 1e-6, 1.0, 0.2)
    o = oracle_mod.Oracle3D(2, 2, 1.0, M.physics_dict(ph))
    q = np.zeros((o.Ne, o.NP, o.NC))
    q[..., 0], q[..., 1:4], q[..., 5:8] = 1.2, [0.3, -0.2, 0.1], [0.4, 0.1, -0.3]
    q[..., 4] = 1.5 + 0.5 * 0.14 / 1.2 + 0.13
    assert np.abs(o.rhs(q)).max() < 1e-12
    ow = oracle_mod.Oracle3D(2, 2, 1.0, M.physics_dict(ph), bcs=(1, 1, 1, 1, 1, 1))
    qw = np.zeros((ow.Ne, ow.NP, ow.NC))
    qw[..., 0], qw[..., 4] = 1.0, 2.0
    qw[..., 7] = 0.5  # B along z: tangent to the x and y walls, normal to the z walls
    r = ow.rhs(qw)
    assert np.abs(r[..., 0]).max() < 1e-12  # no mass flux anywhere
