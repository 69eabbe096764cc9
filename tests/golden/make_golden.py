"""Generate tests/golden/known_answers.json from the reference's own tests.

mojoxm has no CPU path and no golden vectors; what pins its results are the
known answers stated in its test and bench files.  Each entry below is one of
those values, transcribed together with the file, the line range and a
pattern that must occur in that file.  Run in a checkout that has the
reference next to it:

    python tests/golden/make_golden.py /path/to/mojoxm

The script re-reads every cited file and refuses to write the fixture when a
pattern is missing, so the JSON records values that were present verbatim in
the reference.  The tests read only the JSON (the reference is not needed to
run them).
"""
import json
import os
import sys

# (key, value, file, lines, pattern that must appear in that file)
ENTRIES = [
    # reference element (test/reference_element_test.mojo)
    ("refelem.p2_vertex_weight", -1.0 / 20.0, "test/reference_element_test.mojo", "145-170",
     "var v_target = -1.0 / 20.0"),
    ("refelem.p2_edge_weight", 1.0 / 5.0, "test/reference_element_test.mojo", "145-170",
     "var e_target = 1.0 / 5.0"),
    ("refelem.min_node_separation_factor", 0.5, "test/reference_element_test.mojo", "110-117",
     "var expected_d = 0.5 / Float64(P)"),
    ("mat_inv.case_2x2.in", [1.0, 2.0, 3.0, 4.0], "test/reference_element_test.mojo", "193-210",
     "[[1, 2], [3, 4]] -> inverse"),
    ("mat_inv.case_2x2.out", [-2.0, 1.0, 1.5, -0.5], "test/reference_element_test.mojo", "193-210",
     "[[-2, 1], [1.5, -0.5]]"),
    ("mat_inv.case_pivot.in", [0.0, 2.0, 3.0, 4.0], "test/reference_element_test.mojo", "228-248",
     "Pivoting required: [[0, 2], [3, 4]]"),
    ("mat_inv.case_pivot.out", [-2.0 / 3.0, 1.0 / 3.0, 1.0 / 2.0, 0.0], "test/reference_element_test.mojo",
     "228-248", "[[-2/3, 1/3], [1/2, 0]]"),
    ("mat_inv.tol", 1.0e-12, "test/reference_element_test.mojo", "190", "var tol = 1.0e-12"),
    # Sod exact Riemann solver (test/sod_exact_riemann_test.mojo)
    ("sod.eps_tight", 1.0e-4, "test/sod_exact_riemann_test.mojo", "47", "EPS_TIGHT: Float64 = 1.0e-4"),
    ("sod.eps_loose", 5.0e-3, "test/sod_exact_riemann_test.mojo", "48", "EPS_LOOSE: Float64 = 5.0e-3"),
    ("sod.canonical.state", [1.0, 1.0, 0.125, 0.1, 1.4], "test/sod_exact_riemann_test.mojo", "60-64",
     "var rho_R = 0.125"),
    ("sod.canonical.rho_star_L", 0.42632, "test/sod_exact_riemann_test.mojo", "67",
     "rho_star_L_ref: Float64 = 0.42632"),
    ("sod.canonical.rho_star_R", 0.26557, "test/sod_exact_riemann_test.mojo", "68",
     "rho_star_R_ref: Float64 = 0.26557"),
    ("sod.canonical.S_R", 1.7522, "test/sod_exact_riemann_test.mojo", "69", "S_R_ref: Float64 = 1.7522"),
    ("sod.canonical.samples_t", 0.2, "test/sod_exact_riemann_test.mojo", "72-95",
     "sod_exact_rho(0.65, 0.2, gamma"),
    ("sod.canonical.x_star_L", 0.65, "test/sod_exact_riemann_test.mojo", "86", "sod_exact_rho(0.65, 0.2"),
    ("sod.canonical.x_star_R", 0.78, "test/sod_exact_riemann_test.mojo", "93", "sod_exact_rho(0.78, 0.2"),
    ("sod.canonical.fan_x", [0.30 + 0.025 * k for k in range(8)], "test/sod_exact_riemann_test.mojo", "107-113",
     "var x = 0.30 + 0.025 * Float64(k)"),
    ("sod.toro3.state", [1.0, 1000.0, 1.0, 0.01, 1.4], "test/sod_exact_riemann_test.mojo", "137-140",
     "var p_L3: Float64 = 1000.0"),
    ("sod.toro3.t", 0.012, "test/sod_exact_riemann_test.mojo", "145", "sod_exact_rho(0.55, 0.012"),
    ("sod.toro3.rho_star_L", 0.5754, "test/sod_exact_riemann_test.mojo", "141",
     "rho_starL3_ref: Float64 = 0.5754"),
    ("sod.toro3.rho_star_R", 5.999, "test/sod_exact_riemann_test.mojo", "142",
     "rho_starR3_ref: Float64 = 5.999"),
    ("sod.toro3.S_R", 23.5175, "test/sod_exact_riemann_test.mojo", "143", "S_R3_ref: Float64 = 23.5175"),
    ("sod.toro3.x_star_L", 0.55, "test/sod_exact_riemann_test.mojo", "145", "sod_exact_rho(0.55, 0.012"),
    ("sod.toro3.x_star_R", 0.76, "test/sod_exact_riemann_test.mojo", "148", "sod_exact_rho(0.76, 0.012"),
    ("sod.toro3.S_R_tol", 0.01, "test/sod_exact_riemann_test.mojo", "155", "approx_eq(S_R3, S_R3_ref, 0.01)"),
    # SSPRK3 stage plans (test/ssprk3_test.mojo)
    ("ssprk3.coeffs", [[1.0, 0.0, 1.0], [0.75, 0.25, 0.25], [1.0 / 3.0, 2.0 / 3.0, 2.0 / 3.0]],
     "test/ssprk3_test.mojo", "19-22", "stage 2: a=1/3,   b=2/3,   c=2/3"),
    ("ssprk3.routing", [["q", "q", "q", "q1"], ["q1", "q", "q1", "q2"], ["q2", "q", "q2", "q"]],
     "test/ssprk3_test.mojo", "15-18", "stage 1: q_in=q1, q_a=q,  q_b=q1, q_out=q2"),
    # constant-state preservation (test/euler_3d_test.mojo)
    ("euler3d_const.mesh", [4, 4, 4, 1.0], "test/euler_3d_test.mojo", "37-42", "comptime NX = 4"),
    ("euler3d_const.state", [1.5, 0.4, -0.2, 0.3, 0.7, 1.4], "test/euler_3d_test.mojo", "46-51",
     "comptime RHO0: Float32 = 1.5"),
    ("euler3d_const.steps", 5, "test/euler_3d_test.mojo", "44", "comptime NUM_STEPS = 5"),
    ("euler3d_const.cfl", 0.1, "test/euler_3d_test.mojo", "107",
     "var dt = Float32(0.1) * h / (speed * Float32(2 * P + 1))"),
    ("euler3d_const.tol", 1.0e-4, "test/euler_3d_test.mojo", "52", "CONST_TOL: Float32 = Float32(1.0e-4)"),
    # limiter (test/limiter_3d_test.mojo)
    ("limiter3d.P", 2, "test/limiter_3d_test.mojo", "49", "comptime P = 2"),
    ("limiter3d.const_tol", 1.0e-6, "test/limiter_3d_test.mojo", "61", "CONST_TOL: Float32 = Float32(1.0e-6)"),
    ("limiter3d.mean_tol", 1.0e-5, "test/limiter_3d_test.mojo", "62", "MEAN_TOL: Float32 = Float32(1.0e-5)"),
    ("limiter3d.jitter", 0.3, "test/limiter_3d_test.mojo", "97",
     "var jitter = Float32(0.3) if (nn % 2) == 0 else Float32(-0.3)"),
    ("limiter3d.background", [1.0, 0.0, 0.0, 0.0, 2.5], "test/limiter_3d_test.mojo", "98-102",
     "q[base + 4] = Float32(2.5)"),
    ("limiter3d.eps", 0.0, "test/limiter_3d_test.mojo", "131", "solver.enable_cell_limiter(True, Float32(0.0))"),
    ("limiter3d.fired_min", 0.01, "test/limiter_3d_test.mojo", "19-23", "max |q - q_perturbed_ic| > 0.01"),
    # analytic gates of the benches
    ("smooth_wave_p3.l2_max_rel_at_12", 2.0e-4, "benchmarks/bench_euler_smooth_wave_3d_p3.mojo", "64",
     "L2_MAX_REL_AT_12: Float64 = 2.0e-4"),
    ("smooth_wave_p3.rate_min", 2.5, "benchmarks/bench_euler_smooth_wave_3d_p3.mojo", "65",
     "RATE_MIN: Float64 = 2.5"),
    ("smooth_wave_p3.cfl", 0.1, "benchmarks/bench_euler_smooth_wave_3d_p3.mojo", "57", "CFL = Float32(0.1)"),
    ("vortex_3d.l2_max_rel", 0.10, "benchmarks/bench_euler_vortex_3d.mojo", "75",
     "L2_MAX_REL: Float64 = 0.10"),
    # 3D ideal MHD (benchmarks/bench_mhd_alfven_3d_p3.mojo)
    ("mhd_alfven_3d_p3.mesh", [16, 4, 4, 1.0, 0.25, 0.25], "benchmarks/bench_mhd_alfven_3d_p3.mojo", "47-52",
     "comptime LY = Float64(4.0 / 16.0)"),
    ("mhd_alfven_3d_p3.gamma_rho0_b0_p0_amp", [5.0 / 3.0, 1.0, 1.0, 0.1, 0.1], "benchmarks/bench_mhd_alfven_3d_p3.mojo",
     "54-58", "comptime AMPLITUDE = Float32(0.1)"),
    ("mhd_alfven_3d_p3.c_h_alpha_d", [1.5, 0.5], "benchmarks/bench_mhd_alfven_3d_p3.mojo", "59-60",
     "comptime ALPHA_D = Float32(0.5)"),
    ("mhd_alfven_3d_p3.cfl", 0.10, "benchmarks/bench_mhd_alfven_3d_p3.mojo", "65", "comptime CFL = Float32(0.10)"),
    ("mhd_alfven_3d_p3.l2_max_rel", 5.0e-3, "benchmarks/bench_mhd_alfven_3d_p3.mojo", "71",
     "comptime L2_MAX_REL: Float64 = 5.0e-3"),
    # five-moment two-fluid plasma oscillation (benchmarks/bench_two_fluid_langmuir_3d_p3.mojo)
    ("langmuir_3d_p3.mesh", [8, 2, 2, 1.0, 0.25, 0.25], "benchmarks/bench_two_fluid_langmuir_3d_p3.mojo", "60-65",
     "comptime LZ = Float64(2.0 / 8.0)"),
    ("langmuir_3d_p3.species", [5.0 / 3.0, 5.0 / 3.0, -1.0, 1.0, 1.0, 25.0, 1.0, 10.0],
     "benchmarks/bench_two_fluid_langmuir_3d_p3.mojo", "67-74", "comptime M_I: Float32 = 25.0"),
    ("langmuir_3d_p3.n0_pe_pi_upert", [1.0, 0.01, 0.01, 0.01], "benchmarks/bench_two_fluid_langmuir_3d_p3.mojo",
     "75-78", "comptime U_PERTURB: Float32 = 0.01"),
    ("langmuir_3d_p3.c_h_alpha_d_rhomin_pmin", [12.0, 0.5, 1.0e-6, 1.0e-8],
     "benchmarks/bench_two_fluid_langmuir_3d_p3.mojo", "79-82", "comptime MIN_PRESSURE: Float32 = 1.0e-8"),
    ("langmuir_3d_p3.cfl", 0.2, "benchmarks/bench_two_fluid_langmuir_3d_p3.mojo", "84", "comptime CFL = Float32(0.2)"),
    ("langmuir_3d_p3.t_final", 6.1612348, "benchmarks/bench_two_fluid_langmuir_3d_p3.mojo", "90",
     "comptime T_FINAL: Float32 = Float32(6.1612348)"),
    ("langmuir_3d_p3.drift_tol_rel", 0.02, "benchmarks/bench_two_fluid_langmuir_3d_p3.mojo", "92",
     "comptime DRIFT_TOL_REL: Float64 = 0.02"),
    # outputs of the reference itself, as its README reports them for three
    # periodic 2D drivers (relative L2 against the IC after one period)
    ("reported.adv2d_gauss.rel_l2", 0.0007, "README.md", "187-188", "0.07 % rel L2 over one period"),
    ("reported.euler2d_vortex.rel_l2", 0.068, "README.md", "189", "6.8 % rel L2 at P=2 / 32x32"),
    ("reported.mhd2d_alfven.rel_l2", 0.0036, "README.md", "191-192", "0.36 % rel L2 on a one-period"),
    # P, NX, NY, LX, LY, VX, VY, T, frames, CFL, sigma, cx, cy
    ("adv2d_gauss.config", [2, 32, 32, 1.0, 1.0, 1.0, 1.0, 1.0, 20, 0.3, 0.12, 0.5, 0.5],
     "examples/advection_gaussian_2d_gpu.mojo", "29-41", "comptime SIGMA: Float32 = 0.12"),
    # P, NX, NY, LX, LY, T, frames, CFL, gamma, T_inf, u0, v0, beta, cx, cy
    ("euler2d_vortex.config", [2, 32, 32, 10.0, 10.0, 10.0, 20, 0.15, 1.4, 1.0, 1.0, 1.0, 5.0, 5.0, 5.0],
     "examples/euler_vortex_2d_gpu.mojo", "36-51", "comptime BETA = 5.0"),
    # P, NX, NY, LX, LY, gamma, rho0, B0, p0, amplitude, T, frames, CFL
    ("mhd2d_alfven.config", [2, 64, 4, 1.0, 4.0 / 64.0, 5.0 / 3.0, 1.0, 1.0, 0.1, 0.1, 1.0, 20, 0.15],
     "examples/mhd_alfven_2d_gpu.mojo", "39-54", "comptime LY = Float64(4.0 / 64.0)"),
    ("reported.euler3d_vortex.rel_l2", 0.068, "README.md", "369-371", "rel L2 ~6.8 %%"),
    # NX, NY, NZ, LX, LY, T, CFL, gamma, T_inf, u0, v0, beta, cx, cy (LZ = NZ / NX * LX; HLLEC, no fix)
    ("euler3d_vortex.config", [32, 32, 4, 10.0, 10.0, 10.0, 0.15, 1.4, 1.0, 1.0, 1.0, 5.0, 5.0, 5.0],
     "benchmarks/bench_euler_vortex_3d.mojo", "49-64", "comptime LZ = Float64(NZ) / Float64(NX) * LX"),
    ("reported.maxwell_cavity_2d.rel_l2", 2.8e-4, "benchmarks/bench_maxwell_cavity_2d.mojo", "53",
     "Measured 2.8e-4 on current code (NX=NY=16, P=2, 566 SSPRK3 steps)"),
    ("reported.maxwell_cavity_2d.steps", 566, "benchmarks/bench_maxwell_cavity_2d.mojo", "53", "566 SSPRK3 steps"),
    # P, NX, NY, LX, LY, c, CFL, T (PEC walls; Ez = sin(pi x) sin(pi y))
    ("maxwell_cavity_2d.config", [2, 16, 16, 1.0, 1.0, 1.0, 0.2, 1.41421356237],
     "benchmarks/bench_maxwell_cavity_2d.mojo", "42-51", "comptime T_FINAL: Float64 = 1.41421356237"),
    ("reported.maxwell_plane_wave_2d.rel_l2", 5.8e-4, "benchmarks/bench_maxwell_plane_wave_2d.mojo", "64",
     "Empirical: ~5.8e-4 at P=2, NX=NY=16"),
    ("reported.maxwell_plane_wave_2d.leakage", 2.7e-4, "benchmarks/bench_maxwell_plane_wave_2d.mojo", "68",
     "Empirical zero-component leakage ~2.7e-4"),
    # P, NX, NY, LX, LY, c, CFL, T (periodic; Ez = cos(2 pi x), By = -Ez / c)
    ("maxwell_plane_wave_2d.config", [2, 16, 16, 1.0, 1.0, 1.0, 0.2, 1.0],
     "benchmarks/bench_maxwell_plane_wave_2d.mojo", "54-62", "comptime T_FINAL: Float64 = 1.0  # exactly one period"),
    ("reported.mhd_alfven_3d.rel_l2", 3.6e-3, "benchmarks/bench_mhd_alfven_3d.mojo", "59", "Measured ~3.6e-3"),
    # P, NX, NY, NZ, LX, LY, LZ, CFL (physics and IC as mhd_alfven_3d_p3)
    ("mhd_alfven_3d.config", [2, 32, 4, 4, 1.0, 0.125, 0.125, 0.2], "benchmarks/bench_mhd_alfven_3d.mojo", "36-55",
     "comptime LY = Float64(4.0 / 32.0)"),
    # further "Measured" / "Empirical" values in the benches' own comments
    ("reported.adv3d_p2_n16.rel_l2", 9.5e-3, "benchmarks/bench_advection_3d.mojo", "49",
     "Measured rel L2 at N=16 is ~9.5e-3"),
    ("reported.adv3d_p3_n12.rel_l2", 2.4e-3, "benchmarks/bench_advection_3d_p3.mojo", "55", "Measured ~2.4e-3 at N=12"),
    ("reported.adv2d_translation_n32.rel_l2", 7.2e-4, "benchmarks/bench_advection_translation_2d.mojo", "49",
     "Measured ~7.2e-4 at N=32"),
    ("reported.euler2d_vortex_p3_hllc.rel_l2", 0.0681, "benchmarks/bench_euler_vortex_2d_p3.mojo", "61",
     "Empirical 6.81%% at P=3 / HLLC"),
    ("reported.maxwell_plane_wave_3d.rel_l2", 6.5e-4, "benchmarks/bench_maxwell_plane_wave_3d.mojo", "59",
     "Empirical: ~6.5e-4 at NX=16 NY=NZ=4 P=2"),
    ("reported.maxwell_plane_wave_3d.leakage", 4.5e-4, "benchmarks/bench_maxwell_plane_wave_3d.mojo", "61",
     "Empirical leakage ~4.5e-4"),
    ("reported.sw_wave_2d_hll.rel_l2", 1.7e-4, "benchmarks/bench_shallow_water_wave_2d.mojo", "54",
     "Measured ~1.7e-4 across N = 32, 48, 64"),
    ("reported.langmuir_3d_p2.drift_and_ex", [3.5e-4, 6e-5], "benchmarks/bench_two_fluid_langmuir_3d.mojo", "25",
     "Measured values: rho_e u_e drift = 0.035%%, Ex / E_scale = 6e-5"),
    ("langmuir_3d_p2.mesh", [8, 2, 2, 1.0, 0.25, 0.25], "benchmarks/bench_two_fluid_langmuir_3d.mojo", "53-58",
     "comptime LZ = Float64(2.0 / 8.0)"),
    ("reported.smooth_wave_3d_p3_n12.rel_l2", 5.5e-5, "benchmarks/bench_euler_smooth_wave_3d_p3.mojo", "61",
     "Measured ~5.5e-5 at N=12 (Float32 floor)"),
    # gamma, rho0, u, v, w, p0, amplitude, T, CFL (HLLEC, periodic unit cube)
    ("smooth_wave_3d_p3.config", [1.4, 1.0, 1.0, 1.0, 1.0, 1.0, 0.1, 1.0, 0.1],
     "benchmarks/bench_euler_smooth_wave_3d_p3.mojo", "49-57", "comptime AMPLITUDE: Float32 = 0.1"),
]


def main(ref_root):
    out, src = {}, {}
    missing = []
    for key, val, path, lines, pat in ENTRIES:
        full = os.path.join(ref_root, path)
        text = open(full, encoding="utf-8").read()
        if pat not in text:
            missing.append((key, path, pat))
        out[key] = val
        src[key] = f"{path}:{lines}"
    if missing:
        for m in missing:
            print("pattern not found:", m, file=sys.stderr)
        sys.exit(1)
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "known_answers.json"), "w") as f:
        json.dump({"values": out, "source": src}, f, indent=1, sort_keys=True)
    print(f"wrote {len(out)} known answers")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python make_golden.py <root of the mojoxm checkout>")
    main(sys.argv[1])
