"""Benchmark: RHS cell-updates/s per RK stage on B200.

Workload (the configuration the metric is quoted on): viscous LES of the
compressible Taylor-Green vortex, 128^3 unique nodes (DMDA 130^3 with the
periodic boundary layers) on [0, 2*pi]^3, curvilinear grid perturbed by
x_i += 0.05 sin(xi_j) sin(xi_k), Ma 0.1, Re 1600, Pr 0.71, gamma 1.4, constant
viscosity, the reference's LES scheme: MUSCL-minmod + Rusanov upwind blended
with the 4-point skew-symmetric central flux (-central 2, -s_x/y/z 1), constant
Smagorinsky eddy viscosity (CS 0.03) with Yoshizawa term; SSP-RK with
-fluxorder 2 (the reference runs 2 stages per step for MUSCL).  Synthetic
inputs from a formula (no dataset).

A "step" is one physical time step (eddy viscosity + every RK stage with its
periodic boundary/ghost fill).  value = interior nodes x stages x steps x
n_gpus / max-over-ranks device time.  Inputs (state 5 + metrics 10 + nvert +
nu_t planes, ~0.5 GB) exceed the 126 MB L2, so no explicit flush is needed.

Run: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "RHS cell-updates/s per RK3 stage, mixed vs FP64 on 1 B200 at stated L2 error"
UNIT = "cell-updates/s"
N_UNIQUE = 128
B_ALG_LES = 216  # bytes per cell-update: Q in/out/old 120, metrics 72, aj 8, nvert 8, nu_t 8

CFG = dict(les=1, inviscid=0, fluxorder=2, eno_order=2, central=2, s_x=1.0, s_y=1.0, s_z=1.0,
           ren=1600.0, ma=0.1, pr=0.71, gamma=1.4, dt=2e-3)


def workload_config(n):
    return {
        "workload": f"compressible Taylor-Green vortex LES, {n}^3 (DMDA {n + 2}^3), perturbed curvilinear grid, "
                    "MUSCL+Rusanov blended with skew-symmetric central (sigma=1), Smagorinsky CS=0.03, "
                    "viscous Re 1600 Ma 0.1, SSP-RK fluxorder 2 (2 stages/step)",
        "grid": [n + 2, n + 2, n + 2],
        "interior_nodes": n ** 3,
        "stages_per_step": 2,
        "l2_policy": "inputs larger than L2 (~0.5 GB resident per stage vs 126 MB L2); no flush",
        "parallelism": "replicas (one independent block per GPU)",
    }


# ------------------------------------------------------------------ clocks --
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.gpu_id = gpu_id
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", self.gpu_id], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 8:
                continue
            try:
                sm.append(float(p[0]))
                smax.append(float(p[1]))
            except ValueError:
                continue
            for nm, v in zip(names, p[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def gpu_identifier(dev: int) -> str:
    import torch
    try:
        u = torch.cuda.get_device_properties(dev).uuid
        s = str(u)
        return s if s.startswith("GPU-") else "GPU-" + s
    except Exception:
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        if vis:
            return vis.split(",")[dev]
        return str(dev)


def measured_peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic():
    """DRAM bytes per stage-kernel launch from the committed ncu summary (scaled to the bench size)."""
    p = os.path.join(REPO, "profiles", "stage_kernel_traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f)
    return d.get("dram_bytes_per_launch_scaled_to_bench")


# ------------------------------------------------------------------ ranks --
def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, ws, local):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{local}")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ------------------------------------------------------------ reference arm --
def run_reference(args, ws, rank):
    if rank != 0:
        return
    from oracle import cpu_baseline as cb
    n = N_UNIQUE
    r = cb.run(n, steps=args.steps, warmup=args.warmup, cfgkw=CFG)
    line = {
        "metric": METRIC, "value": r["value"], "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * r["seconds"] / max(args.steps, 1), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": workload_config(n),
        "cpu_baseline": {"value": r["value"], "unit": UNIT, "cores": r["cores"], "kind": r["kind"],
                         "sample": r["sample"]},
        "e2e": {"value": r["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ our arm --
def run_ours(args, ws, rank, local):
    import torch

    from chimera_comp_les_b200 import Block
    from chimera_comp_les_b200 import workloads as W

    torch.cuda.set_device(local)
    n = N_UNIQUE
    coords = W.periodic_grid(n, 2 * math.pi, amp=0.05)
    q0 = W.tgv_state(coords, gamma=CFG["gamma"], ma=CFG["ma"])
    nv = np.zeros(coords.shape[:3])
    blk = Block(n + 2, n + 2, n + 2, precision=args.precision, device=local, **CFG)
    blk.FormMetrics(coords)
    blk.set_nvert(nv)
    blk.SetInitialCondition(q0)
    stream = torch.cuda.ExternalStream(blk.stream, device=f"cuda:{local}")
    interior = blk.interior_nodes
    stages = blk.stages

    # warm-up (also captures the CUDA graphs of the buffer rotation)
    blk.RungeKutta(max(args.warmup, 3))

    sampler = ClockSampler(gpu_identifier(local))
    sampler.start()
    time.sleep(0.3)
    barrier(ws)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    blk.RungeKutta(args.steps, sync=False)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(ws)
    clocks = sampler.stop()
    blk.sync()  # device status word: raises on NaN/Inf or rho/p <= 0
    ms = e0.elapsed_time(e1)
    ms = max_over_ranks(ms, ws, local)
    value = ws * interior * stages * args.steps / (ms / 1e3)

    # kernel timing (eager launches, events around every kernel on the library stream)
    blk.timing(True)
    kt_steps = max(3, min(args.steps, 10))
    blk.RungeKutta(kt_steps)
    rhs_ms, rhs_n, other_ms, other_n = blk.timing_read()
    blk.timing(False)
    avg_stage_ms = rhs_ms / max(rhs_n, 1)
    achieved = B_ALG_LES * interior / (avg_stage_ms / 1e3) / 1e9
    peak, peak_kind = measured_peaks()

    # end-to-end through the C-ABI with host buffers: H2D of the step's input
    # state from pinned memory, one time step, D2H of the new state
    e2e_steps = max(3, min(args.steps, 10))
    q_host = torch.empty(q0.shape, dtype=torch.float64, pin_memory=True).numpy()
    q_host[...] = q0
    q_out = torch.empty(q0.shape, dtype=torch.float64, pin_memory=True).numpy()
    blk.SetInitialCondition(q_host)
    blk.RungeKutta(1)
    blk.download(q_out)
    torch.cuda.synchronize()
    barrier(ws)
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(e2e_steps):
        blk.lib.cb_upload_state(blk._ctx, q_host.ctypes.data_as(__import__("ctypes").POINTER(__import__("ctypes").c_double)))
        blk.RungeKutta(1, sync=False)
        blk.download(q_out)
    f1.record(stream)
    torch.cuda.synchronize()
    barrier(ws)
    e2e_ms = max_over_ranks(f0.elapsed_time(f1), ws, local)
    e2e_value = ws * interior * stages * e2e_steps / (e2e_ms / 1e3)
    if not np.isfinite(q_out).all():
        raise RuntimeError("non-finite state after end-to-end steps")

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        from oracle import cpu_baseline as cb
        r = cb.run(n, steps=2, warmup=0, cfgkw=CFG)
        cpu = {"value": r["value"], "unit": UNIT, "cores": r["cores"], "kind": r["kind"], "sample": r["sample"]}

    if rank == 0:
        cfg = workload_config(n)
        cfg["precision_form"] = args.precision
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32-flux/f64-state",
            "data": "synthetic", "config": cfg,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": profile_traffic(),
                         "kernel": "stage_kernel (fused RHS + RK combine)",
                         "kernel_avg_ms": avg_stage_ms, "bytes_per_cell": B_ALG_LES,
                         "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback"},
            "clocks": clocks,
            "e2e": {"value": e2e_value, "unit": UNIT,
                    "h2d_bytes_per_step": int(q0.nbytes), "d2h_bytes_per_step": int(q0.nbytes)},
            "gpu_launches": blk.launches_per_step * args.steps,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    blk.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    ws, rank, local = dist_setup()
    try:
        if args.impl == "reference":
            run_reference(args, ws, rank)
        else:
            run_ours(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
