"""Outputs of the reference itself: the relative L2 error against the initial
condition after one period that the reference's README reports for three
periodic 2D drivers (advection of a Gaussian, the isentropic Euler vortex,
the ideal-MHD Alfven wave), re-run here with the drivers' own mesh, order,
IC, CFL rule and step count.  Both the oracle (FP32, the reference's
arithmetic) and the product's FP32 kernels must land on the reported value
within the digits the README gives (INTERVAL says how each is read).

Error definition (each driver's last lines): sqrt(sum (q - ic)^2) /
sqrt(sum ic^2) over all stored values.
"""
import json
import os

import numpy as np
import pytest

import mojoxm_b200 as M

HERE = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(HERE, "golden", "known_answers.json")) as _f:
    G = json.load(_f)["values"]
f32 = np.float32


def adv_case():
    """examples/advection_gaussian_2d_gpu.mojo:29-126 (dt arithmetic in Float32)."""
    P, nx, ny, lx, ly, vx, vy, T, frames, cfl, sig, cx, cy = G["adv2d_gauss.config"]
    h = f32(lx) / f32(nx)
    vmag = np.sqrt(f32(vx) * f32(vx) + f32(vy) * f32(vy))
    dt_est = f32(cfl) * h / (vmag * f32(2 * P + 1))
    spf = int(f32(T) / (f32(frames) * dt_est)) + 1
    total = int(frames) * spf
    dt = float(f32(T) / f32(total))

    def ic(xy):
        x, y = xy[..., 0].astype(f32), xy[..., 1].astype(f32)
        dx, dy = x - f32(cx), y - f32(cy)
        dx = np.where(dx > f32(lx * 0.5), dx - f32(lx), dx)
        dx = np.where(dx < -f32(lx * 0.5), dx + f32(lx), dx)
        dy = np.where(dy > f32(ly * 0.5), dy - f32(ly), dy)
        dy = np.where(dy < -f32(ly * 0.5), dy + f32(ly), dy)
        s2 = f32(sig) * f32(sig)
        return np.exp(-(dx * dx + dy * dy) / (f32(2.0) * s2))[..., None].astype(f32)

    return M.Advection(vx, vy, 0.0), int(P), (int(nx), int(ny)), (lx, ly), dt, total, ic


def vortex_case():
    """examples/euler_vortex_2d_gpu.mojo:36-154 (2D Rusanov face flux, dt in Float64)."""
    P, nx, ny, lx, ly, T, frames, cfl, gamma, tinf, u0, v0, beta, cx, cy = G["euler2d_vortex.config"]
    h = lx / nx
    two_pi = 2.0 * np.pi
    wave = np.sqrt(u0 * u0 + v0 * v0) + np.sqrt(gamma * tinf) + beta / two_pi
    dt_est = cfl * h / (wave * (2 * P + 1))
    spf = int(T / (frames * dt_est)) + 1
    total = int(frames) * spf
    dt = float(f32(T / total))

    def ic(xy):
        x, y = xy[..., 0].astype(np.float64), xy[..., 1].astype(np.float64)
        dx, dy = x - cx, y - cy
        dx = np.where(dx > lx * 0.5, dx - lx, dx)
        dx = np.where(dx < -lx * 0.5, dx + lx, dx)
        dy = np.where(dy > ly * 0.5, dy - ly, dy)
        dy = np.where(dy < -ly * 0.5, dy + ly, dy)
        r2 = dx * dx + dy * dy
        factor = (gamma - 1.0) * beta * beta / (8.0 * gamma * two_pi * two_pi)
        Tv = tinf - factor * np.exp(1.0 - r2)
        e_half = np.exp(0.5 * (1.0 - r2))
        u = u0 - (beta / two_pi) * dy * e_half
        v = v0 + (beta / two_pi) * dx * e_half
        rho = Tv ** (1.0 / (gamma - 1.0))
        p = rho * Tv
        E = p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v)
        return np.stack([rho, rho * u, rho * v, E], -1).astype(f32)

    ph = M.Euler(gamma, 1e-6, 1e-6, M.FLUX_RUSANOV, False)
    return ph, int(P), (int(nx), int(ny)), (lx, ly), dt, total, ic


def alfven_case():
    """examples/mhd_alfven_2d_gpu.mojo:39-149 (plain 2D MHD, dt in Float64)."""
    P, nx, ny, lx, ly, gamma, rho0, b0, p0, amp, T, frames, cfl = G["mhd2d_alfven.config"]
    cf = np.sqrt(gamma * p0 / rho0 + (b0 / np.sqrt(rho0)) ** 2)
    dt_est = cfl * (lx / nx) / (cf * (2 * P + 1))
    spf = int(T / (frames * dt_est)) + 1
    total = int(frames) * spf
    dt = float(f32(T / total))

    def ic(xy):
        sv = np.sin(2.0 * np.pi / lx * xy[..., 0].astype(np.float64))
        uy, by = amp * sv, -amp * sv
        q = np.zeros(xy.shape[:-1] + (6,))
        q[..., 0], q[..., 2], q[..., 3], q[..., 4] = rho0, rho0 * uy, b0, by
        q[..., 5] = p0 / (gamma - 1.0) + 0.5 * rho0 * uy * uy + 0.5 * (b0 * b0 + by * by)
        return q.astype(f32)

    ph = M.IdealMHDPlain(gamma, 1e-6, 1e-6)
    return ph, int(P), (int(nx), int(ny)), (lx, ly), dt, total, ic


CASES = {"adv2d_gauss": adv_case, "euler2d_vortex": vortex_case, "mhd2d_alfven": alfven_case}
# What the README's digits admit.  "0.07 %" and "6.8 %" as rounded values
# (this code gives 0.0725 % and 6.798 %).  For "0.36 %" this code gives
# 0.366 %, which rounds to 0.37 %: the interval is the truncated reading,
# [0.36, 0.37) %, and the rounded reading is missed by 0.0012 points.
INTERVAL = {"adv2d_gauss": (0.00065, 0.00075), "euler2d_vortex": (0.0675, 0.0685),
            "mhd2d_alfven": (0.0036, 0.0037)}


def rel_l2(q, ic):
    q, ic = q.astype(np.float64), ic.astype(np.float64)
    return float(np.sqrt(((q - ic) ** 2).sum() / (ic ** 2).sum()))


@pytest.mark.parametrize("name", list(CASES))
def test_oracle_reproduces_reported_output(oracle_mod, name):
    ph, P, n, L, dt, steps, ic = CASES[name]()
    o = oracle_mod.Oracle2D(P, n, L, M.physics_dict(ph), real="f32")
    q0 = ic(o.node_xy())
    o.set(q0.astype(np.float64))
    o.step(dt, steps)
    err = rel_l2(o.get(), q0)
    want = G[f"reported.{name}.rel_l2"]
    print(f"oracle {name}: {steps} steps, rel L2 {100 * err:.4f} % (reported {100 * want:g} %)")
    lo, hi = INTERVAL[name]
    assert lo <= err < hi, err


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_product_reproduces_reported_output(name):
    ph, P, n, L, dt, steps, ic = CASES[name]()
    s = M.Solver(M.Mesh(n[0], n[1], 1, L[0], L[1], 1.0, dim=2), ph, P=P, precision="f32")
    q0 = ic(s.node_xyz())
    s.upload_state(q0.astype(np.float64))
    s.step_n(dt, steps)
    err = rel_l2(s.download_state(), q0)
    s.close()
    want = G[f"reported.{name}.rel_l2"]
    print(f"product {name}: {steps} steps, rel L2 {100 * err:.4f} % (reported {100 * want:g} %)")
    lo, hi = INTERVAL[name]
    assert lo <= err < hi, err


def vortex3d_case(P):
    """benchmarks/bench_euler_vortex_3d.mojo(+_p3): the 2D vortex extruded in z
    on 32 x 32 x 4 cubes, HLLEC without the entropy fix, T = 10; IC and dt in
    Float32 (:78-117, :162-167)."""
    nx, ny, nz, lx, ly, T, cfl, gamma, tinf, u0, v0, beta, cx, cy = G["euler3d_vortex.config"]
    lz = nz / nx * lx
    two_pi = f32(2.0) * f32(np.pi)
    wave = np.sqrt(f32(u0) * f32(u0) + f32(v0) * f32(v0)) + np.sqrt(f32(gamma) * f32(tinf)) + f32(beta) / two_pi
    dt_est = f32(cfl) * (f32(lx) / f32(nx)) / (wave * f32(5.0))
    steps = int(f32(T) / dt_est) + 1
    dt = float(f32(T) / f32(steps))

    def ic(xyz):
        x, y = xyz[..., 0].astype(f32), xyz[..., 1].astype(f32)
        dx, dy = x - f32(cx), y - f32(cy)
        dx = np.where(dx > f32(lx * 0.5), dx - f32(lx), dx)
        dx = np.where(dx < -f32(lx * 0.5), dx + f32(lx), dx)
        dy = np.where(dy > f32(ly * 0.5), dy - f32(ly), dy)
        dy = np.where(dy < -f32(ly * 0.5), dy + f32(ly), dy)
        r2 = dx * dx + dy * dy
        g = f32(gamma)
        factor = (g - f32(1.0)) * f32(beta) * f32(beta) / (f32(8.0) * g * two_pi * two_pi)
        Tv = f32(tinf) - factor * np.exp(f32(1.0) - r2)
        e_half = np.exp(f32(0.5) * (f32(1.0) - r2))
        u = f32(u0) - (f32(beta) / two_pi) * dy * e_half
        v = f32(v0) + (f32(beta) / two_pi) * dx * e_half
        rho = Tv ** (f32(1.0) / (g - f32(1.0)))
        p = rho * Tv
        E = p / (g - f32(1.0)) + f32(0.5) * rho * (u * u + v * v)
        z = np.zeros_like(rho)
        return np.stack([rho, rho * u, rho * v, z, E], -1).astype(f32)

    ph = M.Euler(gamma, 1e-6, 1e-6, M.FLUX_HLLEC, False)
    return ph, (int(nx), int(ny), int(nz)), (lx, ly, lz), dt, steps, ic


@pytest.mark.gpu
@pytest.mark.parametrize("P", [2, 3])
def test_product_reproduces_reported_3d_vortex(P):
    """README.md:369-373: rel L2 ~6.8 % over one period at P=2 and P=3."""
    ph, n, L, dt, steps, ic = vortex3d_case(P)
    s = M.Solver(M.Mesh(*n, *L), ph, P=P, precision="f32")
    q0 = ic(s.node_xyz())
    s.upload_state(q0.astype(np.float64))
    s.step_n(dt, steps)
    err = rel_l2(s.download_state(), q0)
    s.close()
    print(f"product 3D vortex P{P}: {steps} steps, rel L2 {100 * err:.3f} % (reported ~6.8 %)")
    assert 0.0675 <= err < 0.0685, err


def maxwell2d_case(name):
    """benchmarks/bench_maxwell_cavity_2d.mojo / bench_maxwell_plane_wave_2d.mojo
    (P2, 16 x 16, c = 1, dt = CFL h / (c (2P+1)) in Float64, rounded to Float32)."""
    P, nx, ny, lx, ly, c, cfl, T = G[f"{name}.config"]
    dt_est = cfl * (lx / nx) / (c * (2 * P + 1))
    steps = int(T / dt_est) + 1
    dt = float(f32(T / steps))
    cavity = name == "maxwell_cavity_2d"
    bcs = (1, 1, 1, 1) if cavity else (0, 0, 0, 0)

    def ic(xy):
        x, y = xy[..., 0].astype(np.float64), xy[..., 1].astype(np.float64)
        q = np.zeros(xy.shape[:-1] + (6,))
        if cavity:
            q[..., 2] = np.sin(np.pi * x) * np.sin(np.pi * y)
        else:
            q[..., 2] = np.cos(2.0 * np.pi * x)
            q[..., 4] = -(1.0 / c) * np.cos(2.0 * np.pi * x)
        return q.astype(f32)

    return M.Maxwell(c), int(P), (int(nx), int(ny)), (lx, ly), bcs, dt, steps, ic


MAXWELL = {"maxwell_cavity_2d": (2.75e-4, 2.85e-4), "maxwell_plane_wave_2d": (5.75e-4, 5.85e-4)}


def leakage(q):
    return float(np.abs(q[..., [0, 1, 3, 5]]).max())


@pytest.mark.parametrize("name", list(MAXWELL))
def test_oracle_reproduces_reported_maxwell_2d(oracle_mod, name):
    ph, P, n, L, bcs, dt, steps, ic = maxwell2d_case(name)
    if name == "maxwell_cavity_2d":
        assert steps == G["reported.maxwell_cavity_2d.steps"]
    o = oracle_mod.Oracle2D(P, n, L, M.physics_dict(ph), bcs=bcs, real="f32")
    q0 = ic(o.node_xy())
    o.set(q0.astype(np.float64))
    o.step(dt, steps)
    q = o.get()
    err = rel_l2(q, q0)
    print(f"oracle {name}: {steps} steps, rel L2 {err:.3e} (reported {G['reported.' + name + '.rel_l2']:g})")
    lo, hi = MAXWELL[name]
    assert lo <= err < hi, err
    if name == "maxwell_plane_wave_2d":
        assert 2.65e-4 <= leakage(q) < 2.75e-4, leakage(q)


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(MAXWELL))
def test_product_reproduces_reported_maxwell_2d(name):
    ph, P, n, L, bcs, dt, steps, ic = maxwell2d_case(name)
    mesh = M.Mesh(n[0], n[1], 1, L[0], L[1], 1.0, bcs=M.BoundaryConditions(*bcs, 0, 0), dim=2)
    s = M.Solver(mesh, ph, P=P, precision="f32")
    q0 = ic(s.node_xyz())
    s.upload_state(q0.astype(np.float64))
    s.step_n(dt, steps)
    q = s.download_state()
    s.close()
    err = rel_l2(q, q0)
    print(f"product {name}: {steps} steps, rel L2 {err:.3e}, leakage {leakage(q):.2e}")
    lo, hi = MAXWELL[name]
    assert lo <= err < hi, err
    if name == "maxwell_plane_wave_2d":
        assert 2.65e-4 <= leakage(q) < 2.75e-4, leakage(q)


@pytest.mark.gpu
def test_product_reproduces_reported_mhd_alfven_3d():
    """benchmarks/bench_mhd_alfven_3d.mojo: 'Measured ~3.6e-3' at P2, 32 x 4 x 4,
    CFL 0.2, dt = CFL h / (max(c_f, c_h) 5) in Float32 (:141-148)."""
    P, nx, ny, nz, lx, ly, lz, cfl = G["mhd_alfven_3d.config"]
    gamma, rho0, b0, p0, amp = G["mhd_alfven_3d_p3.gamma_rho0_b0_p0_amp"]
    c_h, alpha_d = G["mhd_alfven_3d_p3.c_h_alpha_d"]
    cf = np.sqrt(f32(gamma) * f32(p0) / f32(rho0) + (f32(b0) * f32(b0) + f32(amp) * f32(amp)) / f32(rho0))
    wave = max(cf, f32(c_h))
    dt_est = f32(cfl) * (f32(lx) / f32(nx)) / (wave * f32(5.0))
    steps = int(f32(1.0) / dt_est) + 1
    dt = float(f32(1.0) / f32(steps))
    ph = M.IdealMHD(gamma, 1e-6, 1e-6, c_h, alpha_d)
    s = M.Solver(M.Mesh(int(nx), int(ny), int(nz), lx, ly, lz), ph, P=int(P), precision="f32")
    s.fill_ic(M.IC_ALFVEN, [rho0, b0, p0, amp, 1.0])
    q0 = s.download_state()
    s.step_n(dt, steps)
    err = rel_l2(s.download_state(), q0)
    s.close()
    print(f"product 3D MHD Alfven P2: {steps} steps, rel L2 {err:.3e} (reported ~3.6e-3)")
    assert 3.55e-3 <= err < 3.65e-3, err


# ---- further values the benches' comments record for their own runs -----------
def _gauss_ic(L, c, sigma):
    """Periodic Gaussian (the advection benches' IC kernels, Float32)."""
    def ic(x):
        r2 = np.zeros(x.shape[:-1], f32)
        for d in range(x.shape[-1]):
            dd = x[..., d].astype(f32) - f32(c[d])
            dd = np.where(dd > f32(L[d] * 0.5), dd - f32(L[d]), dd)
            dd = np.where(dd < -f32(L[d] * 0.5), dd + f32(L[d]), dd)
            r2 = r2 + dd * dd
        return np.exp(-r2 * (f32(1.0) / (f32(2.0) * f32(sigma) * f32(sigma))))[..., None].astype(f32)
    return ic


def bench_case(name):
    """(physics, P, mesh dims, lengths, BCs, dt, steps, IC, band) of one bench run."""
    if name in ("adv3d_p2_n16", "adv3d_p3_n12"):  # bench_advection_3d(.mojo:37-143), _p3 (:41-148)
        P, N, cfl = (2, 16, 0.2) if name == "adv3d_p2_n16" else (3, 12, 0.1)
        v = np.sqrt(f32(3.0))
        dt_est = f32(cfl) * (f32(1.0) / f32(N)) / (v * f32(2 * P + 1))
        steps = int(f32(1.0) / dt_est) + 1
        band = (9.45e-3, 9.55e-3) if P == 2 else (2.35e-3, 2.45e-3)
        return (M.Advection(1.0, 1.0, 1.0), P, (N, N, N), (1.0, 1.0, 1.0), (0,) * 6, float(f32(1.0) / f32(steps)),
                steps, _gauss_ic((1.0, 1.0, 1.0), (0.5, 0.5, 0.5), 0.12), band)
    if name == "adv2d_translation_n32":  # bench_advection_translation_2d.mojo:38-108
        P, N = 2, 32
        dt_est = f32(0.3) * (f32(1.0) / f32(N)) / (np.sqrt(f32(2.0)) * f32(2 * P + 1))
        steps = int(f32(1.0) / dt_est) + 1
        return (M.Advection(1.0, 1.0, 0.0), P, (N, N), (1.0, 1.0), (0,) * 4, float(f32(1.0) / f32(steps)), steps,
                _gauss_ic((1.0, 1.0), (0.5, 0.5), 0.12), (7.15e-4, 7.25e-4))
    if name == "euler2d_vortex_p3_hllc":  # bench_euler_vortex_2d_p3.mojo:47-133 (HLLC, N=32)
        ph, _, n, L, dt, steps, ic = vortex_case()
        P = 3
        two_pi = 2.0 * np.pi
        wave = np.sqrt(2.0) + np.sqrt(1.4) + 5.0 / two_pi
        dt_est = 0.15 * (10.0 / 32) / (wave * (2 * P + 1))
        steps = int(10.0 / dt_est) + 1
        ph = M.Euler(1.4, 1e-6, 1e-6, M.FLUX_HLLC, False)
        return ph, P, n, L, (0,) * 4, float(f32(10.0 / steps)), steps, ic, (0.06805, 0.06815)
    if name == "maxwell_plane_wave_3d":  # bench_maxwell_plane_wave_3d.mojo:46-140 (P2, 16 x 4 x 4 over [0,1]^3)
        dt_est = f32(0.2) * (f32(1.0) / f32(16)) / (f32(1.0) * f32(5.0))
        steps = int(f32(1.0) / dt_est) + 1
        two_pi = f32(6.28318530717958647692)

        def ic(x):
            q = np.zeros(x.shape[:-1] + (6,), f32)
            q[..., 2] = np.cos(two_pi * x[..., 0].astype(f32))
            q[..., 4] = -np.cos(two_pi * x[..., 0].astype(f32))
            return q
        return (M.Maxwell(1.0), 2, (16, 4, 4), (1.0, 1.0, 1.0), (0,) * 6, float(f32(1.0) / f32(steps)), steps, ic,
                (6.45e-4, 6.55e-4))
    if name == "sw_wave_2d_hll":  # bench_shallow_water_wave_2d.mojo:40-109 (HLL, N=32, square cells)
        P, N, NY = 2, 32, 4
        c = 1.0
        dt_est = 0.15 * (1.0 / N) / (c * (2 * P + 1))
        steps = int(1.0 / dt_est) + 1

        def ic(x):
            q = np.zeros(x.shape[:-1] + (3,))
            q[..., 0] = 1.0 + 0.01 * np.sin(2.0 * np.pi * x[..., 0].astype(np.float64))
            return q.astype(f32)
        return (M.ShallowWater(1.0, 1e-6, flux_type=M.FLUX_HLL), P, (N, NY), (1.0, NY / N), (0,) * 4,
                float(f32(1.0 / steps)), steps, ic, (1.65e-4, 1.75e-4))
    raise KeyError(name)


BENCH = ["adv3d_p2_n16", "adv3d_p3_n12", "adv2d_translation_n32", "euler2d_vortex_p3_hllc", "maxwell_plane_wave_3d",
         "sw_wave_2d_hll"]
ORACLE_CHEAP = ["adv3d_p2_n16", "adv2d_translation_n32", "maxwell_plane_wave_3d", "sw_wave_2d_hll"]


def _check(name, q, q0):
    err = rel_l2(q, q0)
    lo, hi = bench_case(name)[-1]
    print(f"{name}: rel L2 {err:.4e} (reported {G['reported.' + name + '.rel_l2']:g})", end="")
    if name == "maxwell_plane_wave_3d":
        leak = float(np.abs(q[..., [0, 1, 3, 5]]).max())
        print(f", leakage {leak:.2e} (reported ~4.5e-4)", end="")
        assert 4.45e-4 <= leak < 4.55e-4, leak
    print()
    assert lo <= err < hi, err


@pytest.mark.parametrize("name", ORACLE_CHEAP)
def test_oracle_reproduces_bench_values(oracle_mod, name):
    ph, P, n, L, bcs, dt, steps, ic, band = bench_case(name)
    if len(n) == 3:
        o = oracle_mod.Oracle3D(P, n, L, M.physics_dict(ph), bcs=bcs, real="f32")
        q0 = ic(o.node_xyz())
    else:
        o = oracle_mod.Oracle2D(P, n, L, M.physics_dict(ph), bcs=bcs, real="f32")
        q0 = ic(o.node_xy())
    o.set(q0.astype(np.float64))
    o.step(dt, steps)
    _check(name, o.get(), q0)


@pytest.mark.gpu
@pytest.mark.parametrize("name", BENCH)
def test_product_reproduces_bench_values(name):
    ph, P, n, L, bcs, dt, steps, ic, band = bench_case(name)
    if len(n) == 3:
        mesh = M.Mesh(*n, *L, bcs=M.BoundaryConditions(*bcs))
    else:
        mesh = M.Mesh(n[0], n[1], 1, L[0], L[1], 1.0, bcs=M.BoundaryConditions(*bcs, 0, 0), dim=2)
    s = M.Solver(mesh, ph, P=P, precision="f32")
    q0 = ic(s.node_xyz())
    s.upload_state(q0.astype(np.float64))
    s.step_n(dt, steps)
    q = s.download_state()
    s.close()
    _check(name, q, q0)


def langmuir_p2():
    """benchmarks/bench_two_fluid_langmuir_3d.mojo (P2, 8 x 2 x 2, CFL 0.2, dt in Float32)."""
    nx, ny, nz, lx, ly, lz = G["langmuir_3d_p2.mesh"]
    ge, gi, qe, me, qi, mi, eps0, c = G["langmuir_3d_p3.species"]
    n0, pe, pi, a = G["langmuir_3d_p3.n0_pe_pi_upert"]
    c_h, alpha_d, rho_min, p_min = G["langmuir_3d_p3.c_h_alpha_d_rhomin_pmin"]
    ph = M.FiveMomentTwoFluid(ge, gi, qe, me, qi, mi, eps0, c, c_h, alpha_d, rho_min, p_min)
    rho_e, rho_i = me * n0, mi * n0
    state = [rho_e, rho_e * a, 0.0, 0.0, pe / (ge - 1) + 0.5 * rho_e * a * a,
             rho_i, 0.0, 0.0, 0.0, pi / (gi - 1)] + [0.0] * 7
    T = f32(G["langmuir_3d_p3.t_final"])
    dt_est = f32(0.2) * (f32(lx) / f32(nx)) / (max(f32(c), f32(c_h)) * f32(5.0))
    steps = int(T / dt_est) + 1
    wp = np.sqrt(n0 * (qe * qe / me + qi * qi / mi) / eps0)

    def metrics(q):
        drift = abs(q[..., 1].mean() - a * me * n0) / (a * me * n0)
        return drift, abs(q[..., 10].mean()) / (a * me * n0 * wp)

    return ph, (int(nx), int(ny), int(nz)), (lx, ly, lz), np.array(state), float(T / f32(steps)), steps, metrics


def test_oracle_reproduces_langmuir_p2(oracle_mod):
    """The reference records 'rho_e u_e drift = 0.035 %, Ex / E_scale = 6e-5'
    (bench_two_fluid_langmuir_3d.mojo:25).  The oracle keeps the reference's
    FP32 stage combine a q_a + b q_b, whose third-stage weights sum to
    1 + 3e-8: over 14787 steps that bias alone is a 0.04 % momentum drift.
    The oracle lands at 0.043 % (E_x 6.8e-5); the last digit depends on how
    the FP32 products are fused, so the drift is checked for its size, not
    its digits.  (The product, with exact weights, drifts 7e-7.)"""
    ph, n, L, state, dt, steps, metrics = langmuir_p2()
    o = oracle_mod.Oracle3D(2, n, L, M.physics_dict(ph), real="f32")
    o.set(np.broadcast_to(state, (o.Ne, o.NP, 17)).copy())
    o.step(dt, steps)
    drift, ex = metrics(o.get())
    print(f"oracle langmuir P2: {steps} steps, drift {100 * drift:.4f} %, Ex {ex:.2e} (reported 0.035 %, 6e-5)")
    assert 2.5e-4 <= drift < 5e-4, drift
    assert 5e-5 <= ex < 8e-5, ex


@pytest.mark.gpu
def test_product_reproduces_langmuir_p2():
    """E_x as reported (6e-5); the momentum drift is gone (the product's stage
    weights sum to one exactly), so it is bounded instead of matched."""
    ph, n, L, state, dt, steps, metrics = langmuir_p2()
    s = M.Solver(M.Mesh(*n, *L), ph, P=2, precision="f32")
    s.fill_ic(M.IC_CONSTANT, list(state))
    s.step_n(dt, steps)
    drift, ex = metrics(s.download_state().astype(np.float64))
    s.close()
    print(f"product langmuir P2: {steps} steps, drift {100 * drift:.5f} %, Ex {ex:.2e} (reported 0.035 %, 6e-5)")
    assert drift < 1e-5, drift
    assert 5.5e-5 <= ex < 6.5e-5, ex


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["f64", "f32", "mixed"])
def test_smooth_wave_3d_p3_at_or_below_recorded_floor(prec):
    """benchmarks/bench_euler_smooth_wave_3d_p3.mojo (HLLEC, N=12, one period,
    IC and dt in Float32) records '~5.5e-5 at N=12 (Float32 floor)'.  That
    floor is mostly the reference's FP32 stage-weight bias (3e-8 per step
    over 2453 steps, ~4e-5): the product, whose weights sum to one exactly,
    sits at the scheme's own error (~1.8e-5) in every precision, a third of
    the recorded value."""
    gamma, rho0, u0, v0, w0, p0, amp, T, cfl = G["smooth_wave_3d_p3.config"]
    P, N = 3, 12
    wave = np.sqrt(f32(u0) * f32(u0) + f32(v0) * f32(v0) + f32(w0) * f32(w0)) + np.sqrt(f32(gamma) * f32(p0) / f32(rho0))
    dt_est = f32(cfl) * (f32(1.0) / f32(N)) / (wave * f32(2 * P + 1))
    steps = int(f32(T) / dt_est) + 1
    s = M.Solver(M.Mesh(N, N, N), M.Euler(gamma, 1e-6, 1e-6, M.FLUX_HLLEC, False), P=P, precision=prec)
    x = s.node_xyz().astype(f32)
    k = f32(2.0) * f32(np.pi)
    rho = f32(rho0) + f32(amp) * np.sin(k * x[..., 0]) * np.sin(k * x[..., 1]) * np.sin(k * x[..., 2])
    E = f32(p0) / (f32(gamma) - f32(1.0)) + f32(0.5) * rho * f32(u0 * u0 + v0 * v0 + w0 * w0)
    q0 = np.stack([rho, rho * f32(u0), rho * f32(v0), rho * f32(w0), E], -1).astype(f32)
    s.upload_state(q0.astype(np.float64))
    s.step_n(float(f32(T) / f32(steps)), steps)
    err = rel_l2(s.download_state(), q0)
    s.close()
    print(f"smooth wave P3 N=12 {prec}: {steps} steps, rel L2 {err:.3e} (recorded ~5.5e-5, FP32)")
    assert err < G["reported.smooth_wave_3d_p3_n12.rel_l2"] / 2, err
