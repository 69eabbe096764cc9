#!/usr/bin/env python3
"""Benchmark of the DG RHS + SSPRK3 hot path on B200 (one JSON line on rank 0).

Workload (default): 3D Euler smooth density wave rho = 1 + 0.2 sin(2 pi (x+y+z)),
u = (1,1,1), p = 1 on the periodic [0,1]^3 Kuhn mesh of 32^3 cubes x 6 =
196,608 tets, order P = 3 (NP = 20), Rusanov flux; FP32 state with the
volume/lift contraction as split-BF16 tcgen05 products (--precision mixed,
the default), beside the plain FP64 kernels on the same workload
(`plain_f64` in the JSON line).  A step is one SSPRK3 step = 3 fused stage
kernels over the whole mesh; the metric counts Ne*NP*NC DOF per stage
(Solver.dof_count, src/solver.mojo:757-763).

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

--impl reference times the CPU oracle (the C++ restatement of the reference
algorithm; the Mojo reference itself cannot be built on this image) on the
host cores with all threads, on the same workload (same mesh, order, flux,
initial state and dt; FP32 like the reference's own runs): W warm-up and K
timed SSPRK3 steps.  The `cpu_baseline` object of the product's line is the
same oracle run on the same workload for a few seconds.
Multi-GPU (torchrun): every rank advances its own replica of the workload
(independent solves, no collective on the data path); `value` is the sum of
all ranks' DOF over the max-over-ranks device time.  `--decomp slab` instead
splits one n x n x (n N) mesh into N z-slabs, one per GPU, whose ghost
layers move over NCCL every stage (weak scaling).  Side legs in the same
line: the batched 2D engine, the Maxwell cavity, the 3D MHD Alfven wave, the
served stream, and (`slab`) the headline mesh split into z-slabs on one GPU
with its halo exchange.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

GAMMA = 1.4
METRIC = "DOF·stage/s at fixed L2 err vs plain FP64 on B200"
UNIT = "DOF·stage/s"


# ---- replica bookkeeping (one process per GPU under torchrun) --------------
# The DG hot path exchanges no data between GPUs in replica mode: every rank
# advances its own solve.  What crosses ranks is bookkeeping only -- each
# rank's device time (the job time is the maximum over ranks) and its unit
# counts (summed) -- over the gloo process group the bench opens; without a
# process group the helpers act on the local values.

def _dist():
    try:
        import torch.distributed as dist

        if dist.is_available() and dist.is_initialized():
            return dist
    except ImportError:
        pass
    return None


def rank_world():
    d = _dist()
    return (d.get_rank(), d.get_world_size()) if d else (0, 1)


def shard(items, rank=None, world=None):
    """Items of this rank: every world-th item starting at rank (round robin,
    so ranks get work of similar size when items come from one distribution)."""
    if rank is None or world is None:
        rank, world = rank_world()
    return [it for k, it in enumerate(items) if k % world == rank]


def _reduce(value, op):
    d = _dist()
    if d is None:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64)
    d.all_reduce(t, op=op(d))
    return float(t.item())


def max_over_ranks(value):
    return _reduce(value, lambda d: d.ReduceOp.MAX)


def sum_over_ranks(value):
    return _reduce(value, lambda d: d.ReduceOp.SUM)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", type=int, default=32, help="cubes per axis")
    ap.add_argument("--P", type=int, default=3)
    ap.add_argument("--precision", default="mixed", choices=["f64", "f32", "mixed", "tf32"])
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--l2-steps", type=int, default=100,
                    help="SSPRK3 steps of the accuracy check vs the FP64 path (0 = skip)")
    ap.add_argument("--batch-solves", type=int, default=512, help="batched 2D leg: solves (0 = skip)")
    ap.add_argument("--batch-steps", type=int, default=10)
    ap.add_argument("--batch3d-solves", type=int, default=64, help="batched 3D tensor-core leg: solves (0 = skip)")
    ap.add_argument("--serve-requests", type=int, default=500, help="served leg: requests (0 = skip)")
    ap.add_argument("--serve-lambda", type=float, default=200.0)
    ap.add_argument("--serve-largest", type=int, default=1, help="add the 48^3x6 limited Sod P5 request (1/0)")
    ap.add_argument("--serve-slots", type=int, default=8, help="solves running at once in the served leg")
    ap.add_argument("--serve-low-seconds", type=float, default=25.0,
                    help="served leg at half the measured capacity: seconds of arrivals (0 = skip)")
    ap.add_argument("--serve-f64-requests", type=int, default=100,
                    help="requests of the stream replayed in FP64 for the plain comparison (0 = skip)")
    ap.add_argument("--cavity", type=int, default=1, help="run the 24^3x6 P=4 Maxwell cavity leg (1/0)")
    ap.add_argument("--mhd", type=int, default=1, help="run the 3D ideal-MHD Alfven-wave leg (1/0)")
    ap.add_argument("--slab-parts", type=int, default=4, help="z-slab decomposition leg on one GPU (0 = skip)")
    ap.add_argument("--decomp", default="replicas", choices=["replicas", "slab"],
                    help="under torchrun: independent replicas (default), or one n x n x (n*N) mesh split into "
                         "z-slabs, one per GPU, ghost layers over NCCL (weak scaling)")
    return ap.parse_args()


def accuracy_check(M, a, q0, dt):
    """L2 error of the benchmarked precision after `l2_steps` SSPRK3 steps,
    relative to the FP64 kernels (parity-checked against the FP64 oracle)
    and to the exact translated wave."""
    mesh = M.Mesh(a.n, a.n, a.n, 1.0, 1.0, 1.0)
    phys = M.Euler(GAMMA, 1e-6, 1e-6, M.FLUX_RUSANOV, False)
    ref = M.Solver(mesh, phys, P=a.P, precision="f64")
    ref.upload_state(q0)
    ref.step_n(dt, a.l2_steps)
    q64 = ref.download_state(0)
    xyz = ref.node_xyz()
    ref.close()
    out = {"steps": a.l2_steps}
    if a.precision != "f64":
        s = M.Solver(mesh, phys, P=a.P, precision=a.precision)
        s.upload_state(q0)
        s.step_n(dt, a.l2_steps)
        qp = s.download_state(0).astype(np.float64)
        s.close()
        out["rel_l2_vs_f64"] = float(np.sqrt(((qp - q64) ** 2).sum() / (q64 ** 2).sum()))
    else:
        qp = q64
    t = a.l2_steps * dt
    exact = smooth_wave_state(xyz - t)  # translation with u = (1,1,1)
    out["rel_l2_vs_exact"] = float(np.sqrt(((qp - exact) ** 2).sum() / (exact ** 2).sum()))
    out["rel_l2_f64_vs_exact"] = float(np.sqrt(((q64 - exact) ** 2).sum() / (exact ** 2).sum()))
    return out


def smooth_wave_state(xyz):
    x, y, z = xyz[..., 0], xyz[..., 1], xyz[..., 2]
    rho = 1.0 + 0.2 * np.sin(2 * np.pi * (x + y + z))
    q = np.zeros(xyz.shape[:-1] + (5,))
    q[..., 0] = rho
    q[..., 1] = q[..., 2] = q[..., 3] = rho
    q[..., 4] = 1.0 / (GAMMA - 1.0) + 0.5 * rho * 3.0
    return q


def dt_for(n, P, cfl=0.1):
    # bench_euler_smooth_wave_3d_p3.mojo:131-136: dt = CFL h / ((|u| + c)(2P+1))
    h = 1.0 / n
    return cfl * h / ((np.sqrt(3.0) + np.sqrt(GAMMA)) * (2 * P + 1))


def workload_name(a):
    return (f"3D Euler smooth density wave, periodic [0,1]^3 Kuhn mesh {a.n}^3x6 = {6 * a.n ** 3} tets, "
            f"P={a.P}, Rusanov, " + {"f64": "FP64", "f32": "FP32",
                                     "mixed": "FP32 state + split-BF16 tcgen05 contraction",
                                     "tf32": "FP32 state + split-TF32 tcgen05 contraction"}[a.precision])


DTYPE = {"f64": "f64", "f32": "f32", "mixed": "f32+bf16x3", "tf32": "f32+tf32x3"}


class NvmlClockSampler:
    """SM clock and clock-event reasons sampled through NVML every 2 ms while
    the timed region runs (short timed regions still get samples)."""

    BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40}

    def __init__(self, device):
        import pynvml

        self.nv = pynvml
        pynvml.nvmlInit()
        vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
        idx = device
        if vis:
            parts = [p.strip() for p in vis.split(",")]
            if device < len(parts) and parts[device].isdigit():
                idx = int(parts[device])
        self.h = pynvml.nvmlDeviceGetHandleByIndex(idx)
        self.samples, self.reasons, self.stop = [], set(), threading.Event()
        self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM))

    def _run(self):
        nv = self.nv
        while True:
            try:
                self.samples.append(float(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)))
                get = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                    nv.nvmlDeviceGetCurrentClocksThrottleReasons
                r = int(get(self.h))
                for name, bit in self.BITS.items():
                    if r & bit:
                        self.reasons.add(name)
            except Exception:
                pass
            if self.stop.wait(0.002):
                break

    def __enter__(self):
        self.t = threading.Thread(target=self._run, daemon=True)
        self.t.start()
        return self

    def __exit__(self, *a):
        self.stop.set()
        self.t.join(timeout=2)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples), "source": "nvml"}


def clock_sampler(device):
    try:
        return NvmlClockSampler(device)
    except Exception:
        return ClockSampler(device)


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    def __init__(self, device):
        self.device, self.proc, self.lines = device, None, []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [v.strip() for v in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def fp_peaks(device):
    """FP64 and FP32 (TF32 off) dense GEMM throughput of this GPU through
    torch/cuBLAS (4096^3, best of 5, CUDA events): the denominators of the
    FP64 kernels' contraction-flop fraction (MEASURED_PEAKS.json has only
    the HBM and BF16 figures)."""
    try:
        import torch

        torch.backends.cuda.matmul.allow_tf32 = False
        dev = torch.device("cuda", device)
        out = {}
        for name, dt in (("fp64_tflops", torch.float64), ("fp32_tflops", torch.float32)):
            n = 4096
            x = torch.randn(n, n, device=dev, dtype=dt)
            y = torch.randn(n, n, device=dev, dtype=dt)
            torch.matmul(x, y)
            best = 1e30
            for _ in range(5):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                torch.matmul(x, y)
                e1.record()
                e1.synchronize()
                best = min(best, e0.elapsed_time(e1))
            out[name] = 2 * n ** 3 / (best * 1e-3) / 1e12
            del x, y
        torch.cuda.empty_cache()
        out["how"] = "torch.matmul 4096^3 (cuBLAS), best of 5, CUDA events, TF32 off"
        return out
    except Exception as ex:  # torch without CUDA, etc.
        return {"unavailable": str(ex)[:120]}


def traffic_per_launch(a):
    """DRAM bytes per stage launch from the committed ncu summary, if any."""
    try:
        with open(os.path.join(ROOT, "profiles", "stage3d_traffic.json")) as f:
            d = json.load(f)
        key = f"n{a.n}_P{a.P}_{a.precision}"
        return d.get(key)
    except Exception:
        return None


def cpu_model():
    """The host CPU's model name (first entry of /proc/cpuinfo)."""
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform

    return platform.processor() or "unknown"


def omp_threads():
    """Threads the oracle's OpenMP loops use: OMP_NUM_THREADS if set, else
    the CPUs this process may run on."""
    env = os.environ.get("OMP_NUM_THREADS", "")
    if env.isdigit() and int(env) > 0:
        return int(env)
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_baseline(a, seconds, steps=None, warmup=1):
    """The oracle (C++ restatement of the reference's algorithm, OpenMP over
    elements) on the benchmark's own workload: the same n^3 x 6 mesh, order,
    flux and initial state, in the reference's arithmetic (Float32, or FP64
    for --precision f64).  `steps` SSPRK3 steps are timed after `warmup`;
    without `steps` the count is chosen from one warm step so the timed
    part lasts about `seconds` (at least 3 steps, at most --steps)."""
    import oracle

    oracle.build()
    n = a.n
    o = oracle.Oracle3D(a.P, n, 1.0, dict(kind=1, flux=0, entropy_fix=0, p=[GAMMA, 1e-6, 1e-6, 0, 0, 0, 0, 0, 0, 0, 0]),
                        real="f64" if a.precision == "f64" else "f32")
    o.set(smooth_wave_state(o.node_xyz()))
    dt = dt_for(n, a.P)
    t0 = time.perf_counter()
    o.step(dt, max(1, warmup))
    t_warm = (time.perf_counter() - t0) / max(1, warmup)
    if steps is None:
        steps = int(max(3, min(a.steps, round(seconds / max(t_warm, 1e-9)))))
    t0 = time.perf_counter()
    o.step(dt, steps)
    el = time.perf_counter() - t0
    dof = o.Ne * o.NP * o.NC
    thr = omp_threads()
    return dict(value=3 * dof * steps / el, unit=UNIT, cores=thr, kind="port", cpu_model=cpu_model(),
                ms_per_step=el * 1e3 / steps, steps=steps, warmup=max(1, warmup), same_workload=True,
                sample=f"oracle {'FP64' if a.precision == 'f64' else 'FP32'} restatement on the full workload: "
                       f"{n}^3x6 = {6 * n ** 3} tets P={a.P} Rusanov, same initial state and dt, "
                       f"{steps} timed SSPRK3 steps after {max(1, warmup)} in {el:.1f} s, OpenMP {thr} threads "
                       f"on {cpu_model()}")


def run_reference(a, rank, world):
    """The reference arm: the oracle on the host cores, on the benchmark's own
    workload (same mesh, order, flux, state, dt), W warm-up and K timed
    SSPRK3 steps.  Rank 0 alone runs it; other ranks exit without work."""
    if rank != 0:
        return
    cb = cpu_baseline(a, a.cpu_seconds, steps=a.steps, warmup=max(1, a.warmup))
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": a.gpus,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": cb["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if a.precision == "f64" else "f32", "data": "synthetic",
            "config": {"workload": workload_name(a).split(", FP")[0] + (", FP64" if a.precision == "f64" else ", FP32"),
                       "elements": 6 * a.n ** 3, "sample": cb["sample"]},
            "cpu_baseline": cb, "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                                        "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def batch_member(M, rng, precision):
    """The next member of the batched 2D workload drawn from `rng`: an
    n x n x 2 triangle mesh, n ~ U{16,32,64,128,256}, P ~ U{1..5}, HLLE flux,
    BJ limiter (eps 0.1), and with equal odds an isentropic vortex
    (beta ~ U[2,6], periodic [0,10]^2) or a tanh-smoothed Sod tube (left /
    right rho, p ~ U[0.1,1], width 8h, outflow x, periodic y), filled on the
    device.  Returns (solver, "vortex" | "sod", cell size h)."""
    n = int(rng.choice([16, 32, 64, 128, 256]))
    P = int(rng.integers(1, 6))
    phys = M.Euler(GAMMA, 1e-6, 1e-6, M.FLUX_HLLE, False)
    if rng.random() < 0.5:
        mesh = M.Mesh(n, n, 1, 10.0, 10.0, 1.0, dim=2)
        s = M.Solver(mesh, phys, P=P, precision=precision)
        s.fill_ic(M.IC_VORTEX, [rng.uniform(2, 6), 5.0, 5.0, 1.0, 1.0, 0.0, 1.0])
        kind, h = "vortex", 10.0 / n
    else:
        mesh = M.Mesh(n, n, 1, 1.0, 1.0, 1.0, bcs=M.BoundaryConditions(2, 2, 0, 0), dim=2)
        s = M.Solver(mesh, phys, P=P, precision=precision)
        rl, pl, rr, pr = rng.uniform(0.1, 1.0, 4)
        s.fill_ic(M.IC_SOD, [rl, pl, rr, pr, 0.5, 8.0 / n])
        kind, h = "sod", 1.0 / n
    s.enable_cell_limiter(True, 0.1)
    return s, kind, h


def batched_2d(M, nsolves, steps, seed=2024, precision="f32", loop=True, ref=None, keep=False):
    """Batched 2D Euler on triangles: `nsolves` independent solves, n x n x 2
    tris with n ~ U{16,32,64,128,256}, P ~ U{1..5}, ICs a seeded mix of
    isentropic vortices (beta ~ U[2,6], periodic [0,10]^2) and tanh-smoothed
    Sod tubes (left/right rho, p ~ U[0.1,1], width 8h, outflow x / periodic
    y), HLLE flux, BJ limiter eps 0.1, FP32 (or FP64: the plain comparison),
    dt = 0.3 h / ((2P+1) max|lambda|) per solve from the device wave-speed
    reduction.  `ref`: a kept FP64 run of the same seed; its time steps are
    used and the states are compared after the timed steps (relative L2 per
    IC kind).  `keep`: return the solvers open, for use as `ref`."""
    rng = np.random.default_rng(seed)
    batch = M.Batch()
    solvers, kinds, dts = [], [], []
    for k in range(nsolves):
        s, kind, h = batch_member(M, rng, precision)
        kinds.append(kind)
        dt = ref["dts"][k] if ref else 0.3 * h / ((2 * s.P + 1) * s.max_wavespeed())
        batch.add(s, dt)
        dts.append(dt)
        solvers.append(s)
    dof = batch.dof_count()
    t0 = time.perf_counter()
    batch.step(3)  # autotune + graph capture on the first call, then 3 warm-up steps
    batch.synchronize()
    setup_s = time.perf_counter() - t0
    ms = batch.time_steps(steps)
    batch.synchronize()
    tiles = {}
    for i, s in enumerate(solvers):
        tiles.setdefault(s.P, batch.tile_cells(i))
    launches = batch.launches_per_step()
    value = 3 * dof * steps / (ms * 1e-3)
    out = {"workload": f"{nsolves} independent 2D Euler solves (HLLE, BJ limiter, {precision.upper()}), "
                       "n in {16..256}, P in 1..5",
           "solves": nsolves, "dof": dof, "value": value, "unit": UNIT, "ms_per_step": ms / steps,
           "launches_per_step": launches, "tile_cells_per_P": {str(k): v for k, v in sorted(tiles.items())},
           "setup_s": setup_s, "seed": seed}
    if ref:
        num, den = {}, {}
        for i, s in enumerate(solvers):
            a = s.download_state().astype(np.float64)
            b = ref["solvers"][i].download_state()
            num[kinds[i]] = num.get(kinds[i], 0.0) + float(((a - b) ** 2).sum())
            den[kinds[i]] = den.get(kinds[i], 0.0) + float((b ** 2).sum())
        out["rel_l2_vs_f64"] = {k: float(np.sqrt(num[k] / den[k])) for k in sorted(num)}
        out["rel_l2_vs_f64_steps"] = 3 + steps
    if loop:
        # the same solves advanced one at a time through their own handles
        # (per-solve launches on per-solve streams), 2 steps after an untimed
        # one, wall clock
        for i, s in enumerate(solvers):
            s.step_n(batch.dts[i], 1)
        for s in solvers:
            s.synchronize()
        t0 = time.perf_counter()
        for _ in range(2):
            for i, s in enumerate(solvers):
                s.step_n(batch.dts[i], 1)
        for s in solvers:
            s.synchronize()
        loop_s = (time.perf_counter() - t0) / 2
        out["per_solve_loop_value"] = 3 * dof / loop_s
        out["speedup_vs_per_solve_loop"] = value / (3 * dof / loop_s)
    batch.close()
    if keep:
        out["_keep"] = {"solvers": solvers, "dts": dts}
    else:
        for s in solvers:
            s.close()
    return out


def batched_3d(M, nsolves, steps, seed=2025):
    """Batched 3D Euler on the tensor-core stage: `nsolves` independent solves
    of uneven size and order (n^3 x 6 tets, n ~ U{4..16}, P ~ U{2..5}),
    split-BF16, half smooth density waves (Rusanov, periodic) and half
    limited Sod tubes (HLLEC, BJ limiter, outflow x, walls y/z), advanced
    as one batch (one tensor-core launch per (flux, order) group and stage,
    the limited solves' limiter passes, all in one CUDA graph), against the
    same solves stepped one after another through their own handles."""
    rng = np.random.default_rng(seed)
    batch, solvers = M.Batch(), []
    for _ in range(nsolves):
        n, P = int(rng.integers(4, 17)), int(rng.integers(2, 6))
        if rng.random() < 0.5:
            s = M.Solver(M.Mesh(n, n, n), M.Euler(GAMMA, 1e-6, 1e-6, M.FLUX_RUSANOV, False), P=P, precision="mixed")
            s.fill_ic(M.IC_SINE_WAVE, [1, 0.2, 1, 1, 1, 1, 1, 1, 1])
            lam = np.sqrt(3) + 1.5
        else:
            s = M.Solver(M.Mesh(n, n, n, bcs=M.BoundaryConditions(2, 2, 1, 1, 1, 1)),
                         M.Euler(GAMMA, 1e-6, 1e-6, M.FLUX_HLLEC, False), P=P, precision="mixed")
            rl, pl, rr, pr = rng.uniform(0.1, 1.0, 4)
            s.fill_ic(M.IC_SOD, [rl, pl, rr, pr, 0.5, 1.0 / n])
            s.enable_cell_limiter(True, 0.1)
            lam = np.sqrt(GAMMA * max(pl, pr) / min(rl, rr)) + 1.0
        batch.add(s, 0.1 / n / (lam * (2 * P + 1)))
        solvers.append(s)
    dof = batch.dof_count()
    batch.step(3)
    batch.synchronize()
    ms = batch.time_steps(steps)
    batch.synchronize()
    value = 3 * dof * steps / (ms * 1e-3)
    for i, s in enumerate(solvers):  # one untimed step: the single-solve kernels load
        s.step_n(batch.dts[i], 1)
    for s in solvers:
        s.synchronize()
    t0 = time.perf_counter()
    for _ in range(2):
        for i, s in enumerate(solvers):
            s.step_n(batch.dts[i], 1)
    for s in solvers:
        s.synchronize()
    loop_s = (time.perf_counter() - t0) / 2
    out = {"workload": f"{nsolves} independent 3D Euler solves (split-BF16 tensor-core stage; smooth waves and "
                       "limited Sod tubes), n^3x6 tets with n in 4..16, P in 2..5", "solves": nsolves, "dof": dof,
           "value": value, "unit": UNIT, "ms_per_step": ms / steps, "launches_per_step": batch.launches_per_step(),
           "per_solve_loop_value": 3 * dof / loop_s, "speedup_vs_per_solve_loop": value / (3 * dof / loop_s)}
    batch.close()
    for s in solvers:
        s.close()
    return out


def maxwell_cavity(M, n=24, P=4, cfl=0.2, precision="tf32", compare=("mixed", "f32")):
    """3D vacuum Maxwell PEC cavity standing wave: E_z = sin(pi x) sin(pi y)
    cos(sqrt(2) pi t) on [0,1]^3 (PEC on x and y, periodic z), n^3 x 6 tets,
    order P, Rusanov, one period T = sqrt(2); the field then equals its
    initial value, so the analytic error is |q(T) - q(0)|.  `precision` is
    the config's own (FP32 bulk, split-TF32 tensor-core contraction); the
    `compare` precisions and FP64 run the same period beside it."""
    bcs = M.BoundaryConditions(1, 1, 1, 1, 0, 0)
    phys = M.Maxwell(1.0, *([0.0] * 12))
    T = np.sqrt(2.0)
    dt = cfl * (1.0 / n) / (2 * P + 1)  # bench_maxwell_cavity_3d.mojo:128
    nsteps = int(np.ceil(T / dt))
    dt = T / nsteps
    res = {}
    for prec in (precision, *compare, "f64"):
        s = M.Solver(M.Mesh(n, n, n, bcs=bcs), phys, P=P, precision=prec)
        s.fill_ic(M.IC_CAVITY, [1.0, 1.0, 1.0])
        q0 = s.download_state().astype(np.float64)
        ms = s.time_steps(dt, nsteps)
        res[prec] = (s.download_state().astype(np.float64), ms, s.dof_count())
        s.close()
    qa, ms, dof = res[precision]
    q64, ms64, _ = res["f64"]

    def rl2(a, b):
        return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))

    out = {"workload": f"3D Maxwell PEC cavity, {n}^3x6 = {6 * n ** 3} tets, P={P}, Rusanov, one period "
                       f"({nsteps} SSPRK3 steps)", "precision": precision,
           "value": 3 * dof * nsteps / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms / nsteps,
           "plain_f64_value": 3 * dof * nsteps / (ms64 * 1e-3),
           "speedup_vs_f64": ms64 / ms,
           "rel_l2_vs_f64": rl2(qa, q64), "rel_l2_vs_exact": rl2(qa, q0), "rel_l2_f64_vs_exact": rl2(q64, q0)}
    for prec in compare:
        qc, msc, _ = res[prec]
        out[prec] = {"value": 3 * dof * nsteps / (msc * 1e-3), "rel_l2_vs_f64": rl2(qc, q64),
                     "rel_l2_vs_exact": rl2(qc, q0)}
    return out


def mhd_alfven(M, nx=64, P=3, steps=30, precision="mixed"):
    """3D ideal MHD with GLM cleaning: the right-going Alfven wave of
    benchmarks/bench_mhd_alfven_3d_p3.mojo (gamma 5/3, rho0 = B0 = 1, p0 = 0.1,
    amplitude 0.1, c_h = 1.5, alpha_d = 0.5) on an nx x nx/4 x nx/4 periodic
    slab of [0,1] x [0,1/4]^2, `steps` SSPRK3 steps at CFL 0.1, in
    `precision` and in FP64."""
    ph = M.IdealMHD(5.0 / 3.0, 1e-6, 1e-6, 1.5, 0.5)
    ny = nx // 4
    cf = np.sqrt(5.0 / 3.0 * 0.1 + 1.01)
    dt = 0.1 * (1.0 / nx) / (max(cf, 1.5) * (2 * P + 1))
    res = {}
    for prec in (precision, "f64"):
        s = M.Solver(M.Mesh(nx, ny, ny, 1.0, 0.25, 0.25), ph, P=P, precision=prec)
        s.fill_ic(M.IC_ALFVEN, [1.0, 1.0, 0.1, 0.1, 1.0])
        s.step_n(dt, 3)
        ms = s.time_steps(dt, steps)
        res[prec] = (s.download_state().astype(np.float64), ms, s.dof_count())
        s.close()
    qa, ms, dof = res[precision]
    q64, ms64, _ = res["f64"]
    value = 3 * dof * steps / (ms * 1e-3)
    return {"workload": f"3D ideal MHD + GLM Alfven wave, {nx}x{ny}x{ny}x6 = {6 * nx * ny * ny} tets, P={P}, "
                        f"9 components, Rusanov", "precision": precision, "value": value, "unit": UNIT,
            "ms_per_step": ms / steps, "plain_f64_value": 3 * dof * steps / (ms64 * 1e-3),
            "speedup_vs_f64": value / (3 * dof * steps / (ms64 * 1e-3)),
            "rel_l2_vs_f64": float(np.sqrt(((qa - q64) ** 2).sum() / (q64 ** 2).sum())), "steps": 3 + steps}


def slab_decomposed(M, a, parts, steps=20):
    """The headline mesh split into `parts` z-slabs on this GPU, stepped as one
    in-process group (ghost layers by device copies, ordered by events): the
    cost of the halo exchange against the undecomposed solve, and a check
    that the owned results stay bit-identical to it."""
    mesh = M.Mesh(a.n, a.n, a.n, 1.0, 1.0, 1.0)
    ph = M.Euler(GAMMA, 1e-6, 1e-6, M.FLUX_RUSANOV)
    dt = dt_for(a.n, a.P)
    ic = [1.0, 0.2, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0]
    ps = [M.Solver(mesh, ph, P=a.P, precision=a.precision, nparts=parts, part=r) for r in range(parts)]
    for s in ps:
        s.fill_ic(M.IC_SINE_WAVE, ic)
    grp = M.SlabGroup(ps)
    grp.step_n(dt, 3)
    grp.synchronize()
    el = grp.time_steps(dt, steps) * 1e-3  # CUDA events bracketing every part's work
    one = M.Solver(mesh, ph, P=a.P, precision=a.precision)
    one.fill_ic(M.IC_SINE_WAVE, ic)
    one.step_n(dt, 3)
    one.synchronize()
    el1 = one.time_steps(dt, steps) * 1e-3
    ref = one.download_state().reshape(-1)
    n = one.NP * one.NC
    got = np.concatenate([s.download_state().reshape(-1)[s.owned_e0 * n:(s.owned_e0 + s.owned_ne) * n] for s in ps])
    layer_bytes = ps[0].slab_layout()["layer"] * (8 if a.precision == "f64" else 4)
    ghosts = sum(sum(s.ghosts) for s in ps)
    dof = one.dof_count()
    grp.close()
    for s in ps + [one]:
        s.close()
    return {"workload": f"{workload_name(a)}, split into {parts} z-slabs on one GPU", "parts": parts,
            "value": 3 * dof * steps / el, "unit": UNIT, "ms_per_step": el * 1e3 / steps,
            "single_domain_ms_per_step": el1 * 1e3 / steps, "overhead": el / el1 - 1.0,
            "exchange_bytes_per_stage": ghosts * layer_bytes, "bit_identical_to_single_domain": bool(np.array_equal(got, ref)),
            "timing": "CUDA events (the group's events bracket all parts' streams)"}


SERVED_KINDS = ("euler2d_vortex", "euler3d_wave", "dam_break", "maxwell3d_plane_wave", "euler3d_sod_limited")


def served_requests(M, nreq, seed=7, largest=True, precision=None):
    """The served stream's requests, drawn from `seed`: 2D Euler vortices,
    3D Euler smooth waves, 2D shallow-water dam breaks (h_left ~ U[1,3],
    h_right = 1), 3D Maxwell plane waves and 3D limited Sod tubes (HLLEC,
    BJ limiter, outflow x, walls y/z, left / right rho, p ~ U[0.1, 1]), each
    with 2k-400k elements (log-uniform), P in 2..5 and 50-500 SSPRK3 steps;
    `largest` adds, at a seeded position, the 3D limited Sod at P = 5 on
    48^3 x 6 = 663,552 tets (50 steps).  `precision` replaces every
    request's own (the FP64 comparison).  Returns [(kind, submit args)]."""
    rng = np.random.default_rng(seed)
    reqs = []
    for k in range(nreq):
        kind = int(rng.integers(0, len(SERVED_KINDS)))
        E = float(np.exp(rng.uniform(np.log(2e3), np.log(4e5))))
        P = int(rng.integers(2, 6))
        nsteps = int(rng.integers(50, 501))
        lim = None
        if kind == 0:  # 2D Euler vortex
            n = max(4, int(round(np.sqrt(E / 2))))
            mesh = M.Mesh(n, n, 1, 10.0, 10.0, 1.0, dim=2)
            phys = M.Euler(GAMMA, 1e-6, 1e-6, M.FLUX_HLLE, False)
            ic, prm, lam_est, h = M.IC_VORTEX, [rng.uniform(2, 6), 5, 5, 1, 1, 0, 1], 1.5 + 1.0 + np.sqrt(GAMMA), 10.0 / n
            prec = "f32"
        elif kind == 1:  # 3D Euler smooth wave
            n = max(2, int(round((E / 6) ** (1 / 3))))
            mesh = M.Mesh(n, n, n)
            phys = M.Euler(GAMMA, 1e-6, 1e-6, M.FLUX_RUSANOV, False)
            ic, prm, lam_est, h = M.IC_SINE_WAVE, [1, 0.2, 1, 1, 1, 1, 1, 1, 1], np.sqrt(3) + 1.5, 1.0 / n
            prec = "mixed"  # split-BF16 tensor-core stage (P 2..5)
        elif kind == 2:  # dam break
            n = max(4, int(round(np.sqrt(E / 2))))
            mesh = M.Mesh(n, n, 1, 1.0, 1.0, 1.0, bcs=M.BoundaryConditions(1, 1, 1, 1), dim=2)
            phys = M.ShallowWater(9.81, 1e-6, 1.0, 0.0, 0.0)
            hl = rng.uniform(1, 3)
            ic, prm, lam_est, h = M.IC_DAM_BREAK, [hl, 1.0, 0.5, 2.0 / n], 2 * np.sqrt(9.81 * hl), 1.0 / n
            prec = "f32"
        elif kind == 3:  # 3D Maxwell plane wave
            n = max(2, int(round((E / 6) ** (1 / 3))))
            mesh = M.Mesh(n, n, n)
            phys = M.Maxwell(1.0, *([0.0] * 12))
            ic, prm, lam_est, h = M.IC_PLANE_WAVE, [1.0, 1.0], 1.0, 1.0 / n
            prec = "mixed"
        else:  # 3D limited Sod tube
            n = max(2, int(round((E / 6) ** (1 / 3))))
            mesh = M.Mesh(n, n, n, bcs=M.BoundaryConditions(2, 2, 1, 1, 1, 1))
            phys = M.Euler(GAMMA, 1e-6, 1e-6, M.FLUX_HLLEC, False)
            rl, pl, rr, pr = rng.uniform(0.1, 1.0, 4)
            ic, prm, h = M.IC_SOD, [rl, pl, rr, pr, 0.5, 1.0 / n], 1.0 / n
            lam_est = np.sqrt(GAMMA * max(pl, pr) / min(rl, rr)) + 1.0
            prec, lim = "mixed", 0.1
        dt = 0.1 * h / (lam_est * (2 * P + 1))
        reqs.append((SERVED_KINDS[kind], (mesh, phys, P, precision or prec, ic, prm, dt, nsteps, lim)))
    if largest:
        mesh = M.Mesh(48, 48, 48, bcs=M.BoundaryConditions(2, 2, 1, 1, 1, 1))
        phys = M.Euler(GAMMA, 1e-6, 1e-6, M.FLUX_HLLEC, False)
        big = ("largest_euler3d_sod_limited_P5",
               (mesh, phys, 5, precision or "mixed", M.IC_SOD, [1.0, 1.0, 0.125, 0.1, 0.5, 1.0 / 48],
                0.1 / 48 / (2.5 * 11), 50, 0.1))
        reqs.insert(int(rng.integers(0, len(reqs) + 1)), big)
    return reqs


def _warm_server(M, reqs, slots):
    """One tiny request of every (dim, physics, order, precision, limiter,
    boundaries) the stream uses, so module loading and first-launch set-up
    of each kernel happen before the timed stream."""
    warm, seen, wids = M.Server(hbm_budget_bytes=150e9, max_active=slots, steps_per_chunk=10), set(), []
    for _, (mesh, phys, P, prec, ic, prm, dt, nsteps, lim) in reqs:
        key = (mesh.dim, phys.kind, phys.flux_type, P, prec, lim is not None, tuple(mesh.bcs.as_list()))
        if key in seen:
            continue
        seen.add(key)
        small = M.Mesh(2, 2, 2 if mesh.dim == 3 else 1, mesh.lx, mesh.ly, mesh.lz, bcs=mesh.bcs, dim=mesh.dim)
        wids.append(warm.submit(small, phys, P, prec, ic, prm, dt, 25, lim))
    for i in wids:
        warm.wait(i, timeout_s=300)
    warm.close()


def run_stream(M, reqs, lam, slots, seed=11, warm=True, keep=True):
    """Submit `reqs` with Poisson gaps at `lam`/s to a server with a 150 GB
    HBM budget and `slots` concurrent solves; return the server's latency
    and throughput figures, each kind's latencies, and the slot occupancy and
    admitted bytes sampled every 20 ms from the first submit to the last
    result (time-weighted means, maxima and a series of at most 60 points).
    keep: every result is copied to a host array (released once its
    latency is read); otherwise results stay on the device and the latency
    ends when the solve's last kernel has finished."""
    if warm:
        _warm_server(M, reqs, slots)
    gaps = np.random.default_rng(seed).exponential(1.0 / lam, len(reqs))
    srv = M.Server(hbm_budget_bytes=150e9, max_active=slots, steps_per_chunk=10)
    samples, stop = [], threading.Event()

    def sampler():
        while not stop.is_set():
            st = srv.stats()
            samples.append((time.perf_counter(), st["running"], st["queued"], st["bytes_in_use"]))
            stop.wait(0.02)

    t0 = time.perf_counter()
    th = threading.Thread(target=sampler, daemon=True)
    th.start()
    ids, t_next = [], 0.0
    for (_, r), g in zip(reqs, gaps):
        t_next += g
        delay = t_next - (time.perf_counter() - t0)
        if delay > 0:
            time.sleep(delay)
        ids.append(srv.submit(*r, keep_result=keep))
    lat = []
    for i in ids:
        lat.append(srv.wait(i, timeout_s=1800))
        srv._out.pop(i, None)  # the host copy is not needed past this point
    stop.set()
    th.join(timeout=5)
    st = srv.stats()
    srv.close()
    by_kind = {}
    for (kind, _), l in zip(reqs, lat):
        by_kind.setdefault(kind, []).append(l)
    kinds = {k: {"n": len(v), "p50_ms": float(np.percentile(v, 50)), "max_ms": float(np.max(v))}
             for k, v in sorted(by_kind.items())}
    occ = {}
    if len(samples) > 1:
        t = np.array([x[0] for x in samples]) - t0
        run = np.array([x[1] for x in samples])
        que = np.array([x[2] for x in samples])
        byt = np.array([x[3] for x in samples])
        w = np.diff(t, append=t[-1])
        tw = max(float(w.sum()), 1e-9)
        step = max(1, len(t) // 60)
        occ = {"samples": len(t), "mean_running": float((run * w).sum() / tw), "max_running": float(run.max()),
               "mean_queued": float((que * w).sum() / tw), "max_queued": float(que.max()),
               "mean_admitted_bytes": float((byt * w).sum() / tw), "max_admitted_bytes": float(byt.max()),
               "series_t_s_running_queued_gb": [[round(float(t[i]), 2), int(run[i]), int(que[i]),
                                                 round(float(byt[i]) / 1e9, 3)] for i in range(0, len(t), step)]}
    return {"requests": len(reqs), "lambda_per_s": lam, "results_to_host": keep,
            "solves_per_s": st["solves_per_s"], "p50_ms": st["p50_ms"],
            "p99_ms": st["p99_ms"], "mean_ms": st["mean_ms"], "dof_stage_per_s": st["dof_stage_per_s"],
            "completed": st["completed"], "failed": st["failed"], "peak_concurrent": st["peak_concurrent"],
            "peak_admitted_bytes": st["peak_bytes"], "latency_by_kind": kinds, "occupancy": occ}


def served(M, a):
    """The served configuration: `--serve-requests` requests (+ the largest
    member) at `--serve-lambda`/s, over the server's capacity; the same kinds
    at half the measured capacity (a stable queue; `--serve-low-seconds` of
    arrivals); and the plain FP64 comparison replaying the first
    `--serve-f64-requests` requests of the stream in FP64 beside the same
    subset in the stream's precisions."""
    reqs = served_requests(M, a.serve_requests, seed=7, largest=a.serve_largest)
    # 500 arrivals within a few seconds: results stay on the device so the
    # host does not hold every outstanding request's state at once
    out = run_stream(M, reqs, a.serve_lambda, a.serve_slots, keep=False)
    out["workload"] = (f"{len(reqs)} requests, Poisson arrivals at {a.serve_lambda:g}/s: 2D/3D Euler, 2D dam break, "
                       "3D Maxwell plane wave, 3D limited Sod (HLLEC + limiter); 2k-400k elements, P 2..5, "
                       "50-500 steps" + ("; + 48^3x6 limited Sod P5" if a.serve_largest else "") +
                       "; HBM budget 150 GB")
    out["slots"] = a.serve_slots
    out["hbm_budget_bytes"] = 150e9
    out["over_capacity"] = bool(a.serve_lambda > out["solves_per_s"])
    cap = out["solves_per_s"]
    if a.serve_low_seconds > 0 and cap > 0:
        lam_low = 0.5 * cap
        n_low = max(20, int(lam_low * a.serve_low_seconds))
        low = run_stream(M, served_requests(M, n_low, seed=8, largest=False), lam_low, a.serve_slots, seed=12,
                         warm=False)
        low["note"] = "arrival rate half the capacity measured on the stream above: the queue stays stable"
        out["sub_capacity"] = low
    if a.serve_f64_requests > 0:
        sub = reqs[:a.serve_f64_requests]
        fast = run_stream(M, sub, a.serve_lambda, a.serve_slots, warm=False)
        sub64 = [(k, (r[0], r[1], r[2], "f64") + tuple(r[4:])) for k, r in sub]
        slow = run_stream(M, sub64, a.serve_lambda, a.serve_slots)
        out["plain_f64"] = {"requests": len(sub), "stream_precisions": {k: fast[k] for k in (
            "solves_per_s", "dof_stage_per_s", "p50_ms", "p99_ms")},
            "f64": {k: slow[k] for k in ("solves_per_s", "dof_stage_per_s", "p50_ms", "p99_ms")}}
        out["speedup_vs_f64"] = fast["dof_stage_per_s"] / slow["dof_stage_per_s"]
    return out


def main():
    a = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch.distributed as dist

        dist.init_process_group("gloo", init_method="env://", rank=rank, world_size=world,
                                timeout=__import__("datetime").timedelta(seconds=300))
    if a.impl == "reference":
        run_reference(a, rank, world)
        if dist:
            dist.destroy_process_group()
        return

    import mojoxm_b200 as M

    M.set_device(local)
    phys = M.Euler(GAMMA, 1e-6, 1e-6, M.FLUX_RUSANOV, False)
    slab = a.decomp == "slab" and world > 1

    def make(prec):
        """This rank's solve: a replica of the n^3 mesh, or its z-slab of the
        n x n x (n*world) mesh with the ghost layers connected over NCCL."""
        if not slab:
            return M.Solver(M.Mesh(a.n, a.n, a.n, 1.0, 1.0, 1.0), phys, P=a.P, precision=prec)
        h = M.Solver(M.Mesh(a.n, a.n, a.n * world, 1.0, 1.0, float(world)), phys, P=a.P, precision=prec,
                     nparts=world, part=rank)
        uid = [M.nccl_unique_id() if rank == 0 else None]
        dist.broadcast_object_list(uid, src=0)
        h.connect_nccl(uid[0])
        return h

    s = make(a.precision)
    q0_local = smooth_wave_state(s.node_xyz())  # global positions: the wave is periodic in z with period 1
    s.upload_state(q0_local)
    q0 = q0_local  # the n^3 state of the accuracy check
    if slab:
        tmp = M.Solver(M.Mesh(a.n, a.n, a.n, 1.0, 1.0, 1.0), phys, P=a.P, precision="f64")
        q0 = smooth_wave_state(tmp.node_xyz())
        tmp.close()
    dt = dt_for(a.n, a.P)
    dof = s.owned_ne * s.NP * s.NC  # owned DOF (all of them for a replica)

    def barrier():
        s.synchronize()
        if dist:
            dist.barrier()

    # warm-up (>= 3 SSPRK3 steps)
    s.step_n(dt, max(3, a.warmup))
    barrier()
    with clock_sampler(local) as clk:
        ms = s.time_steps(dt, a.steps)  # CUDA events on the solver's stream
    barrier()
    ms_max = max_over_ranks(ms)  # job time = slowest replica
    value = sum_over_ranks(3 * dof * a.steps) / (ms_max * 1e-3)

    # end to end through the host-buffer entry (pinned in/out, copies timed)
    pin_in = M.PinnedArray(s.shape, s.dtype)
    pin_out = M.PinnedArray(s.shape, s.dtype)
    pin_in.array[:] = s.download_state(0)  # the rank's whole state buffer (ghost layers included)
    # a stream of calls long enough that the pipeline's fill (the first
    # upload) and drain (the last download) are a small part of it
    e2e_steps = max(a.steps, 100)
    s.advance_host_async(pin_in.array, 1, dt, pin_out.array)  # warm (allocates the pipeline)
    s.synchronize()
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):  # pipelined: one step's download beside the next step's upload
        s.advance_host_async(pin_in.array, 1, dt, pin_out.array)
    s.synchronize()
    el = time.perf_counter() - t0
    barrier()
    el = max_over_ranks(el)
    e2e_value = sum_over_ranks(3 * dof * e2e_steps) / el
    qbytes = int(np.prod(s.shape)) * np.dtype(s.dtype).itemsize
    pin_in.free()
    pin_out.free()

    # the plain FP64 kernels on the same workload (the ratio's denominator)
    plain = None
    if a.precision != "f64":
        s64 = make("f64")
        s64.upload_state(q0_local)
        s64.step_n(dt, max(3, a.warmup))
        barrier()
        ms64 = s64.time_steps(dt, a.steps)
        barrier()
        ms64 = max_over_ranks(ms64)
        s64.close()
        v64 = sum_over_ranks(3 * dof * a.steps) / (ms64 * 1e-3)
        plain = {"value": v64, "ms_per_step": ms64 / a.steps, "speedup": value / v64,
                 "contraction_tflops": 2 * (3 * s.NP + 4 * s.NFP) * dof * 3 * a.steps / (ms64 * 1e-3) / 1e12}

    if rank == 0:
        peak, peak_kind = peaks()
        launches = s.launches_per_step()
        avg_launch_s = ms * 1e-3 / (a.steps * launches)
        alg_bytes = (8.0 / 3.0) * dof * np.dtype(s.dtype).itemsize  # per stage launch (state_bytes_per_step / 3)
        achieved = alg_bytes / avg_launch_s / 1e9
        nsm_flops = 2 * (3 * s.NP + 4 * s.NFP) * dof  # contraction flops per stage
        cb = cpu_baseline(a, a.cpu_seconds)
        acc = accuracy_check(M, a, q0, dt) if a.l2_steps > 0 else None
        fpp = fp_peaks(local)
        if plain and "fp64_tflops" in fpp:
            plain["fp64_peak_tflops"] = fpp["fp64_tflops"]
            plain["contraction_frac_of_fp64_peak"] = plain["contraction_tflops"] / fpp["fp64_tflops"]
        bat = None
        if a.batch_solves > 0:  # the same batch in FP64 first: the plain comparison and the accuracy reference
            b64 = batched_2d(M, a.batch_solves, a.batch_steps, precision="f64", loop=False, keep=True)
            keep = b64.pop("_keep")
            bat = batched_2d(M, a.batch_solves, a.batch_steps, ref=keep)
            for s64 in keep["solvers"]:
                s64.close()
            bat["plain_f64_value"] = b64["value"]
            bat["plain_f64_ms_per_step"] = b64["ms_per_step"]
            bat["speedup_vs_f64"] = bat["value"] / b64["value"]
        bat3 = batched_3d(M, a.batch3d_solves, a.batch_steps) if a.batch3d_solves > 0 else None
        cav = maxwell_cavity(M) if a.cavity else None
        mhd = mhd_alfven(M) if a.mhd else None
        slab_leg = slab_decomposed(M, a, a.slab_parts) if a.slab_parts > 0 else None
        srv = served(M, a) if a.serve_requests > 0 else None
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": ms_max / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": DTYPE[a.precision], "data": "synthetic",
            "config": {"workload": workload_name(a) + (f"; one {a.n}x{a.n}x{a.n * world} mesh in {world} z-slabs"
                                                      if slab else ""),
                       "elements": s.owned_ne, "NP": s.NP, "NC": s.NC,
                       "accuracy": acc,
                       "dof_per_stage": dof, "dt": dt,
                       "parallelism": f"z-slabs x{world}, ghost layers over NCCL" if slab else f"replicas x{world}",
                       "l2": "inputs larger than L2: 3 state buffers of "
                             f"{qbytes / 1e6:.0f} MB each (L2 126 MB), no flush"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic_per_launch(a),
                         "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind,
                         "kernel": "stage3d_tc_kernel" if a.precision in ("mixed", "tf32") else "stage3d_kernel",
                         "alg_bytes_per_launch": alg_bytes,
                         "contraction_tflops": nsm_flops / avg_launch_s / 1e12},
            "cpu_baseline": cb,
            "plain_f64": plain,
            "measured_gemm_peaks": fpp,
            "batched": bat, "batched_3d": bat3,
            "maxwell_cavity": cav, "mhd_alfven": mhd, "slab": slab_leg,
            "served": srv,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": qbytes, "d2h_bytes_per_step": qbytes,
                    "calls": e2e_steps, "timing": "wall clock from the first call to the synchronize, max over ranks",
                    "entry": "mxm_dg_advance_host_async (pinned host state in/out every step, 1 SSPRK3 step per "
                             "call, calls pipelined, one synchronize at the end)"},
            "gpu_launches": launches * a.steps,
            "clocks": clk.summary(),
        }
        print(json.dumps(line))
    s.close()
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
