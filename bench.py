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
host cores with all threads, on a bounded sample of the same workload.
Multi-GPU (torchrun): every rank advances its own replica of the workload
(independent solves, no collective on the data path); `value` is the sum of
all ranks' DOF over the max-over-ranks device time.
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


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", type=int, default=32, help="cubes per axis")
    ap.add_argument("--P", type=int, default=3)
    ap.add_argument("--precision", default="mixed", choices=["f64", "f32", "mixed"])
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--l2-steps", type=int, default=100,
                    help="SSPRK3 steps of the accuracy check vs the FP64 path (0 = skip)")
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
                                     "mixed": "FP32 state + split-BF16 tcgen05 contraction"}[a.precision])


DTYPE = {"f64": "f64", "f32": "f32", "mixed": "f32+bf16x3"}


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


def traffic_per_launch(a):
    """DRAM bytes per stage launch from the committed ncu summary, if any."""
    try:
        with open(os.path.join(ROOT, "profiles", "stage3d_traffic.json")) as f:
            d = json.load(f)
        key = f"n{a.n}_P{a.P}_{a.precision}"
        return d.get(key)
    except Exception:
        return None


def cpu_baseline(a, seconds):
    """Oracle (C++ restatement, OpenMP) on a bounded sample of the workload."""
    import oracle

    oracle.build()
    n = 8
    o = oracle.Oracle3D(a.P, n, 1.0, dict(kind=1, flux=0, entropy_fix=0, p=[GAMMA, 1e-6, 1e-6, 0, 0, 0, 0, 0, 0, 0, 0]),
                        real="f64" if a.precision == "f64" else "f32")
    o.set(smooth_wave_state(o.node_xyz()))
    dt = dt_for(n, a.P)
    o.step(dt, 1)
    steps, t0 = 0, time.perf_counter()
    while True:
        o.step(dt, 1)
        steps += 1
        el = time.perf_counter() - t0
        if el >= seconds or steps >= 200:
            break
    dof = o.Ne * o.NP * o.NC
    return dict(value=3 * dof * steps / el, unit=UNIT, cores=os.cpu_count(), kind="port",
                sample=f"oracle FP64 restatement, {n}^3x6 = {6 * n ** 3} tets P={a.P} Rusanov, {steps} SSPRK3 steps "
                       f"in {el:.1f} s, OpenMP {os.cpu_count()} threads")


def run_reference(a, rank, world):
    if rank != 0:
        return
    cb = cpu_baseline(a, a.cpu_seconds)
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": a.gpus,
            "steps": a.steps, "warmup": a.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if a.precision == "f64" else "f32", "data": "synthetic",
            "config": {"workload": workload_name(a), "sample": cb["sample"]},
            "cpu_baseline": cb, "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                                        "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


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
    s = M.Solver(M.Mesh(a.n, a.n, a.n, 1.0, 1.0, 1.0), phys, P=a.P, precision=a.precision)
    q0 = smooth_wave_state(s.node_xyz())
    s.upload_state(q0)
    dt = dt_for(a.n, a.P)
    dof = s.dof_count()

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
    ms_max = ms
    if dist:
        import torch

        t = torch.tensor([ms], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_max = float(t.item())
    value = world * 3 * dof * a.steps / (ms_max * 1e-3)

    # end to end through the host-buffer entry (pinned in/out, copies timed)
    pin_in = M.PinnedArray(s.shape, s.dtype)
    pin_out = M.PinnedArray(s.shape, s.dtype)
    pin_in.array[:] = s.download_state(0)
    e2e_steps = max(2, min(a.steps, 10))
    s.advance_host(pin_in.array, 1, dt, out=pin_out.array)  # warm
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        s.advance_host(pin_in.array, 1, dt, out=pin_out.array)
    el = time.perf_counter() - t0
    barrier()
    if dist:
        import torch

        t = torch.tensor([el], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        el = float(t.item())
    e2e_value = world * 3 * dof * e2e_steps / el
    qbytes = int(np.prod(s.shape)) * np.dtype(s.dtype).itemsize
    pin_in.free()
    pin_out.free()

    # the plain FP64 kernels on the same workload (the ratio's denominator)
    plain = None
    if a.precision != "f64":
        s64 = M.Solver(M.Mesh(a.n, a.n, a.n, 1.0, 1.0, 1.0), phys, P=a.P, precision="f64")
        s64.upload_state(q0)
        s64.step_n(dt, max(3, a.warmup))
        barrier()
        ms64 = s64.time_steps(dt, a.steps)
        barrier()
        if dist:
            import torch

            t = torch.tensor([ms64], dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms64 = float(t.item())
        s64.close()
        v64 = world * 3 * dof * a.steps / (ms64 * 1e-3)
        plain = {"value": v64, "ms_per_step": ms64 / a.steps, "speedup": value / v64}

    if rank == 0:
        peak, peak_kind = peaks()
        launches = s.launches_per_step()
        avg_launch_s = ms * 1e-3 / (a.steps * launches)
        alg_bytes = (8.0 / 3.0) * dof * np.dtype(s.dtype).itemsize  # per stage launch (state_bytes_per_step / 3)
        achieved = alg_bytes / avg_launch_s / 1e9
        nsm_flops = 2 * (3 * s.NP + 4 * s.NFP) * dof  # contraction flops per stage
        cb = cpu_baseline(a, a.cpu_seconds)
        acc = accuracy_check(M, a, q0, dt) if a.l2_steps > 0 else None
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": ms_max / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": DTYPE[a.precision], "data": "synthetic",
            "config": {"workload": workload_name(a), "elements": s.num_elements, "NP": s.NP, "NC": s.NC,
                       "accuracy": acc,
                       "dof_per_stage": dof, "dt": dt, "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2: 3 state buffers of "
                             f"{qbytes / 1e6:.0f} MB each (L2 126 MB), no flush"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic_per_launch(a),
                         "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind,
                         "kernel": "stage3d_tc_kernel" if a.precision == "mixed" else "stage3d_kernel",
                         "alg_bytes_per_launch": alg_bytes,
                         "contraction_tflops": nsm_flops / avg_launch_s / 1e12},
            "cpu_baseline": cb,
            "plain_f64": plain,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": qbytes, "d2h_bytes_per_step": qbytes,
                    "entry": "mxm_dg_advance_host (pinned host state in/out, 1 SSPRK3 step per call)"},
            "gpu_launches": launches * a.steps,
            "clocks": clk.summary(),
        }
        print(json.dumps(line))
    s.close()
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
