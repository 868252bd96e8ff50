"""Benchmark: RHS cell-updates/s per RK stage on B200.

Workload (the configuration the metric is quoted on): viscous LES of the
compressible Taylor-Green vortex, 128^3 unique nodes (DMDA 130^3 with the
periodic boundary layers) on [0, 2*pi]^3, curvilinear grid perturbed by
x_i += 0.05 sin(xi_j) sin(xi_k), Ma 0.1, Re 1600, Pr 0.71, gamma 1.4, constant
viscosity, in the reference's flags for MUSCL-minmod upwind with a
Smagorinsky model: -les 1 -fluxorder 2 -s_x 0 -s_y 0 -s_z 0 (MUSCL-minmod
reconstruction, Rusanov flux, hybrid weight 0: pure upwind on every face;
the reference ties the RK stage count to the flux order, so 2 stages per
step), constant Smagorinsky eddy viscosity (CS 0.03), dt 1e-3 (the CFL number
summed over the three directions is 0.67; at 2e-3 it is 1.34 and this purely
upwind RK2 scheme loses positivity within 35 steps).  The same workload with
Roe's flux is reported beside it.  Synthetic inputs from a
formula (no dataset).

A "step" is one physical time step (eddy viscosity + every RK stage with its
periodic boundary/ghost fill).  value = interior nodes x stages x steps x
n_gpus / max-over-ranks device time of the MIXED form (FP32 fluxes, FP64
state); the FP64 parity form is measured the same way and reported beside it,
with the mixed-vs-FP64 per-field error after 100 steps and the kinetic-energy
and enstrophy history deviation.  Inputs (~0.6 GB resident per stage) exceed
the 126 MB L2, so no explicit flush is needed.

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
# algorithmic bytes per cell-update of the stage kernel; the bench's workloads
# have no immersed body, so the kernel runs its no-IBM variant, which reads
# no nvert
B_ALG = {
    "fp64": 208,   # Q in/old/out 120, metrics 72, aj 8, nu_t 8
    "mixed": 200,  # Q in/old/out 120, FP32 metrics 36, aj 8, nu_t 8, FP64 metric divergence 24, FP32 filter width 4
}
ACC_STEPS = 100
# names the headline workload in the committed ncu traffic summaries
WORKLOAD_ID = "tgv128-muscl-rusanov-sigma0-rk2"

# -les 1 -fluxorder 2 -s_x 0 -s_y 0 -s_z 0: MUSCL-minmod + Rusanov, pure upwind
CFG = dict(les=1, inviscid=0, fluxorder=2, eno_order=2, central=2, s_x=0.0, s_y=0.0, s_z=0.0,
           ren=1600.0, ma=0.1, pr=0.71, gamma=1.4, dt=1e-3)
# the reference's default hybrid blend on the same TGV: WENO3 (-fluxorder 3,
# SSP-RK3) blended with the 4-point central flux by the weight sigma, dt 2e-3
CFG_WENO3_BLEND = dict(CFG, fluxorder=3, dt=2e-3)


def workload_config(n):
    return {
        "workload": f"compressible Taylor-Green vortex LES, {n}^3 (DMDA {n + 2}^3), perturbed curvilinear grid, "
                    "MUSCL-minmod + Rusanov upwind (-les 1 -fluxorder 2 -s_x 0 -s_y 0 -s_z 0), Smagorinsky CS=0.03, "
                    "viscous Re 1600 Ma 0.1, RK2 (fluxorder 2: the reference runs 2 stages/step), dt 1e-3",
        "flux_variant": "sigma = 0 on every face (-s_x = -s_y = -s_z = 0, sensor off): the blend (1 - sigma) * "
                        "upwind + sigma * central equals the upwind flux, so the stage kernel forms only that; the "
                        "reference also multiplies the eddy viscosity and Yoshizawa terms by sigma, so the "
                        "Smagorinsky model is inert in this flag set (its kernel still runs every step and the "
                        "stage kernel still forms the SGS terms)",
        "grid": [n + 2, n + 2, n + 2],
        "interior_nodes": n ** 3,
        "stages_per_step": CFG["fluxorder"],
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


def profile_traffic(precision):
    """DRAM bytes per stage-kernel launch from the committed ncu summary of
    this workload (None when no summary for this form is committed)."""
    p = os.path.join(REPO, "profiles", f"stage_kernel_traffic_{precision}.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f)
    if d.get("workload_id") != WORKLOAD_ID:
        return None
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
def _block(precision, local, coords, q0, nv, **over):
    from chimera_comp_les_b200 import Block
    n = coords.shape[0] - 2
    blk = Block(n + 2, n + 2, n + 2, precision=precision, device=local, **dict(CFG, **over))
    blk.FormMetrics(coords)
    blk.set_nvert(nv)
    blk.SetInitialCondition(q0)
    blk.kchunk, _ = blk.autotune()  # k-chunk of the stage kernel by measurement
    return blk


def _timed(blk, steps, warmup, ws, local, sample_clocks=False):
    """Device time of `steps` resident time steps (max over ranks), clocks."""
    import torch
    stream = torch.cuda.ExternalStream(blk.stream, device=f"cuda:{local}")
    blk.RungeKutta(max(warmup, 3))  # also captures the CUDA graphs of the buffer rotation
    sampler = ClockSampler(gpu_identifier(local)) if sample_clocks else None
    if sampler:
        sampler.start()
        time.sleep(0.3)
    barrier(ws)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    blk.RungeKutta(steps, sync=False)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(ws)
    clocks = sampler.stop() if sampler else None
    blk.sync()  # device status word: raises on NaN/Inf or rho/p <= 0
    return max_over_ranks(e0.elapsed_time(e1), ws, local), clocks


def _kernel_ms(blk, steps):
    blk.timing(True)
    blk.RungeKutta(steps)
    rhs_ms, rhs_n, _, _ = blk.timing_read()
    blk.timing(False)
    return rhs_ms / max(rhs_n, 1)


def _accuracy(fp64, mixed, q0):
    """Both forms from the same state for ACC_STEPS steps: per-field error of
    mixed vs FP64 at the end, KE / enstrophy history deviation."""
    from chimera_comp_les_b200 import diagnostics as D
    csi, eta, zet, aj = fp64.metrics()
    hist = {"fp64": [], "mixed": []}
    final = {}
    for name, blk in (("fp64", fp64), ("mixed", mixed)):
        blk.SetInitialCondition(q0)
        for c in range(5):
            if c:
                blk.RungeKutta(ACC_STEPS // 4)
            q = blk.Q()
            hist[name].append((D.kinetic_energy(q, aj), D.enstrophy(q, csi, eta, zet, aj)))
        final[name] = q
    l2, linf = D.field_errors(final["mixed"], final["fp64"])
    ke_dev = max(abs(m[0] - f[0]) / abs(f[0]) for m, f in zip(hist["mixed"], hist["fp64"]))
    en_dev = max(abs(m[1] - f[1]) / abs(f[1]) for m, f in zip(hist["mixed"], hist["fp64"]))
    return {"steps": ACC_STEPS, "rel_l2": l2, "rel_linf": linf, "fields": ["rho", "rhoU", "rhoV", "rhoW", "rhoE"],
            "ke_history_max_rel_dev": ke_dev, "enstrophy_history_max_rel_dev": en_dev,
            "ke": [h[0] for h in hist["fp64"]], "checkpoints_every": ACC_STEPS // 4}


def _batch_timed(bt, steps, warmup, per_block, local):
    import torch
    stream = torch.cuda.ExternalStream(bt.stream, device=f"cuda:{local}")
    bt.RungeKutta(max(warmup, 3), per_block=per_block)  # captures the step graphs of this mode
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    bt.RungeKutta(steps, per_block=per_block, sync=False)
    e1.record(stream)
    torch.cuda.synchronize()
    bt.sync()
    return e0.elapsed_time(e1)


def run_batched(args, local):
    """Uneven multi-block set (24 blocks, sizes drawn from 32..160 x 32..128 x
    32..96 unique points, metric distortion 0.03, von Karman turbulence k_peak 4,
    Mt 0.3, 2-node overlap halos from a seeded donor permutation): the
    persistent work-queue launch against one launch per block, both forms,
    and the mixed-vs-FP64 error after ACC_STEPS steps."""
    from chimera_comp_les_b200 import batch as B
    from chimera_comp_les_b200 import diagnostics as D
    from chimera_comp_les_b200 import workloads as W
    mb = W.multiblock_set(seed=2024, nblocks=24)
    # half upwind (sigma 0.5): the donor halos put jumps at every block face, on
    # which the purely central blend (sigma 1) of the headline loses positivity
    opts = dict(CFG, s_x=0.5, s_y=0.5, s_z=0.5)
    opts["dt"] = mb["dt"]
    maps = B.halo_maps_donor(mb["dims"], mb["perm"])
    out = {"workload": "24 uneven curvilinear blocks (unique points per direction drawn from 32..160 x 32..128 x "
                       "32..96, seed 2024), random smooth metric distortion 0.03, decaying isotropic turbulence "
                       "(von Karman, k_peak 4, Mt 0.3), 2-node overlap halos gathered from a seeded donor "
                       "permutation; LES scheme and RK3 as the headline but sigma 0.5 (half upwind), dt from CFL 0.4",
           "blocks": len(mb["dims"]), "dt": mb["dt"]}
    final, hist = {}, {}
    for prec in ("mixed", "fp64"):
        bt = B.Batch(mb["dims"], precision=prec, device=local, **opts)
        for k in range(len(mb["dims"])):
            bt.FormMetrics(k, mb["coords"][k])
            bt.SetInitialCondition(k, mb["q"][k])
        bt.set_halo_maps(maps)
        kc, tune_ms = bt.autotune()
        interior, stages = bt.interior_nodes, opts["fluxorder"]
        r = {"kchunk": kc, "autotune_stage_ms": tune_ms, "work_items": bt.work_items}
        for name, pb in (("persistent", False), ("per_block", True)):
            ms = _batch_timed(bt, args.steps, args.warmup, pb, local)
            r[name] = {"value": interior * stages * args.steps / (ms / 1e3), "ms_per_step": ms / args.steps}
        r["persistent_vs_per_block"] = r["persistent"]["value"] / r["per_block"]["value"]
        out[prec] = r
        out["interior_nodes"] = interior
        # accuracy run from the initial state
        for k in range(len(mb["dims"])):
            bt.SetInitialCondition(k, mb["q"][k])
        mets = [bt.metrics(k) for k in range(len(mb["dims"]))]
        ke = []
        for c in range(5):
            if c:
                bt.RungeKutta(ACC_STEPS // 4)
            qs = [bt.Q(k) for k in range(len(mb["dims"]))]
            ke.append(sum(D.kinetic_energy(q, m[3]) for q, m in zip(qs, mets)))
        en = sum(D.enstrophy(q, *m) for q, m in zip(qs, mets))
        hist[prec] = (ke, en)
        final[prec] = np.concatenate([q[1:-1, 1:-1, 1:-1].reshape(-1, 5) for q in qs])
        bt.close()
    l2, linf = D.field_errors(final["mixed"], final["fp64"])
    out["speedup_mixed_vs_fp64_persistent"] = out["mixed"]["persistent"]["value"] / out["fp64"]["persistent"]["value"]
    out["mixed_vs_fp64_error"] = {
        "steps": ACC_STEPS, "rel_l2": l2, "rel_linf": linf,
        "ke_history_max_rel_dev": max(abs(a - b) / abs(b) for a, b in zip(hist["mixed"][0], hist["fp64"][0])),
        "enstrophy_final_rel_dev": abs(hist["mixed"][1] - hist["fp64"][1]) / abs(hist["fp64"][1]),
    }
    return out


def _forms(coords, q0, nv, cfg, args, ws, local, clocks_for=None):
    """Both forms of one workload: device-timed steps, per-launch stage-kernel
    time and its HBM rate.  Returns (per-form dict, open blocks)."""
    out, blocks = {}, {}
    for prec in ("fp64", "mixed"):
        blk = _block(prec, local, coords, q0, nv, **cfg)
        blocks[prec] = blk
        ms, clocks = _timed(blk, args.steps, args.warmup, ws, local, sample_clocks=(prec == clocks_for))
        interior, stages = blk.interior_nodes, blk.stages
        kms = _kernel_ms(blk, max(3, min(args.steps, 10)))
        out[prec] = {"value": ws * interior * stages * args.steps / (ms / 1e3), "ms_per_step": ms / args.steps,
                     "kernel_avg_ms": kms, "achieved_gbs": B_ALG[prec] * interior / (kms / 1e3) / 1e9,
                     "launches_per_step": blk.launches_per_step, "kchunk_autotuned": blk.kchunk}
        if clocks is not None:
            out[prec]["clocks"] = clocks
    return out, blocks


def pipe_peaks(local):
    """Measured FP64 / FP32 FMA peaks (TFLOP/s) of this GPU (cb_pipe_peaks)."""
    import ctypes

    from chimera_comp_les_b200 import _lib
    lib = _lib.load()
    f64, f32 = ctypes.c_double(), ctypes.c_double()
    if lib.cb_pipe_peaks(local, ctypes.byref(f64), ctypes.byref(f32)) != 0:
        return None
    return {"fp64_tflops": f64.value, "fp32_tflops": f32.value,
            "source": "measured here by cb_pipe_peaks (dependent-FMA kernel on every SM, 2 flops per FMA)"}


def hbm_copy_gbs(local, nbytes=1 << 31, reps=10):
    """Device-to-device copy bandwidth of this GPU (read + write bytes / time):
    a STREAM-style copy of a 2 GiB buffer, CUDA events around `reps` copies
    after three warm-up copies."""
    import torch
    n = nbytes // 8
    a = torch.ones(n, dtype=torch.float64, device=f"cuda:{local}")
    b = torch.empty_like(a)
    for _ in range(3):
        b.copy_(a)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(reps):
        b.copy_(a)
    e1.record()
    torch.cuda.synchronize()
    gbs = 2 * nbytes * reps / (e0.elapsed_time(e1) / 1e3) / 1e9
    del a, b
    torch.cuda.empty_cache()
    return gbs


def compute_roofline(form, cfgkw, kernel_ms, interior, peaks):
    """Compute-side roofline of the stage kernel: operations per cell-update
    counted on the restatement (oracle/flops.py) x cell-updates per launch /
    launch time, against the measured FMA peak of the form's arithmetic pipe.
    The FP64 form is built without FMA contraction (every add and multiply
    issues alone), so its attainable flop rate is half the FMA peak."""
    from chimera_comp_les_b200 import workloads as W
    from oracle import flops as FL
    n = 16
    coords = W.periodic_grid(n, 2 * math.pi, amp=0.05)
    q = W.tgv_state(coords, gamma=1.4, ma=0.1)
    c = FL.count_per_cell({k: v for k, v in cfgkw.items()}, coords, q)
    fl = c["stage_flops"]
    achieved = fl * interior / (kernel_ms / 1e3) / 1e12
    pk = peaks["fp64_tflops"] if form == "fp64" else peaks["fp32_tflops"]
    ceiling = pk / 2 if form == "fp64" else pk
    return {"flops_per_cell": fl, "ops_per_cell": {k: round(v, 2) for k, v in c["stage"].items()},
            "counted_on": "oracle restatement (operation-counting build) of this scheme, one time step / "
                          "(interior nodes x stages); it forms every flux the reference forms, including "
                          "any the blend multiplies by zero",
            "achieved_tflops": achieved, "pipe": "FP64" if form == "fp64" else "FP32",
            "peak_tflops": pk, "peak_source": peaks["source"], "frac": achieved / pk,
            "attainable_tflops": ceiling, "frac_of_attainable": achieved / ceiling,
            "attainable_note": ("no FMA contraction in the FP64 parity form: one flop per pipe instruction, "
                                "half the FMA peak" if form == "fp64" else "FMA contraction on: FMA peak")}


def _vs_oracle(n, coords, q0, nv, blocks, cfgkw):
    """One full-size step of the oracle restatement against one step of each
    GPU form from the same state."""
    import oracle as O
    from chimera_comp_les_b200 import diagnostics as D
    ocfg = O.Config(mx=n + 2, my=n + 2, mz=n + 2, **{k: v for k, v in cfgkw.items()})
    ora = O.Oracle(ocfg)
    met = ora.metrics(O.to_padded(ocfg, coords))
    nvp = ora.fill_ghosts(O.to_padded(ocfg, nv))
    st = ora.initial_state(q0)
    ora.steps(1, st, met, nvp)
    q_ora = O.from_padded(st["q"])
    out = {"steps": 1, "fields": ["rho", "rhoU", "rhoV", "rhoW", "rhoE"]}
    for prec, blk in blocks.items():
        blk.SetInitialCondition(q0)
        blk.RungeKutta(1)
        l2, linf = D.field_errors(blk.Q(), q_ora)
        out[prec] = {"rel_l2": l2, "rel_linf": linf}
    return out


def config5_case(n):
    """Config 5's inputs and options at n^3: coordinates, state, dt (CFL 0.4)
    and the scheme (WENO5-JS + Roe, pure upwind, Smagorinsky CS 0.17^2,
    SSP-RK3)."""
    from chimera_comp_les_b200 import workloads as W
    coords = W.periodic_grid(n, 2 * math.pi, amp=0.0)
    q0 = W.isotropic_turbulence(n, 5, k_peak=4.0, mach_t=0.4, spectrum="passot_pouquet", u_rms=1.0)
    r = q0[..., 0]
    c = np.sqrt(1.4 * 0.4 * (q0[..., 4] - 0.5 * (q0[..., 1] ** 2 + q0[..., 2] ** 2 + q0[..., 3] ** 2) / r) / r)
    lam = sum(float((np.abs(q0[..., 1 + a] / r) + c).max()) for a in range(3)) * n / (2 * math.pi)
    dt = math.floor(0.4 / lam * 1e6) / 1e6
    opts = dict(CFG, fluxorder=3, weno_order=5, flux="roe", s_x=0.0, s_y=0.0, s_z=0.0, ren=10000.0, ma=0.4,
                cs_const=0.17 ** 2, dt=dt)
    return coords, q0, dt, opts


CONFIG5_SCHEME = "WENO5-JS + Roe, pure upwind (sigma 0), Smagorinsky CS 0.17^2, SSP-RK3, dt from CFL 0.4"


def _ke_enstrophy_device(q, csi, eta, zet, aj, local):
    """diagnostics.kinetic_energy / enstrophy of a host state, evaluated with
    torch on the GPU in FP64 (the same formulas; for the 512^3 box, where the
    host versions take tens of seconds)."""
    import torch
    dev = f"cuda:{local}"
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    s = (slice(1, -1),) * 3
    qd = t(q)
    rho = qd[..., 0]
    ajc = t(aj)[s]
    vol = 1.0 / ajc
    ke = float((0.5 * (qd[s + (1,)] ** 2 + qd[s + (2,)] ** 2 + qd[s + (3,)] ** 2) / rho[s] * vol).sum() / vol.sum())
    u = [qd[..., a] / rho for a in (1, 2, 3)]
    del qd
    m = [t(csi)[s], t(eta)[s], t(zet)[s]]

    def dc(f):
        return (0.5 * (f[1:-1, 1:-1, 2:] - f[1:-1, 1:-1, :-2]), 0.5 * (f[1:-1, 2:, 1:-1] - f[1:-1, :-2, 1:-1]),
                0.5 * (f[2:, 1:-1, 1:-1] - f[:-2, 1:-1, 1:-1]))

    def grad(a, x):
        d = dc(u[a])
        return (d[0] * m[0][..., x] + d[1] * m[1][..., x] + d[2] * m[2][..., x]) * ajc

    w2 = (grad(2, 1) - grad(1, 2)) ** 2
    w2 += (grad(0, 2) - grad(2, 0)) ** 2
    w2 += (grad(1, 0) - grad(0, 1)) ** 2
    en = float((0.5 * rho[s] * w2 * vol).sum() / vol.sum())
    del u, m, w2
    torch.cuda.empty_cache()
    return ke, en


def _histories(blocks, q0, steps, every, diag, keep=None):
    """Both forms from q0 for `steps` steps: (KE, enstrophy) every `every`
    steps and the final states; with `keep` (a dict) also the states after
    the step counts it lists as keys, into keep[step][form]."""
    hist, final = {}, {}
    for name, blk in blocks.items():
        blk.SetInitialCondition(q0)
        h = []
        for c in range(steps // every + 1):
            if c:
                blk.RungeKutta(every)
            q = blk.Q()
            h.append(diag(q))
            if keep is not None and c * every in keep:
                keep[c * every][name] = q
        hist[name], final[name] = h, q
    return hist, final


def _history_devs(hist):
    ke = max(abs(m[0] - f[0]) / abs(f[0]) for m, f in zip(hist["mixed"], hist["fp64"]))
    en = max(abs(m[1] - f[1]) / abs(f[1]) for m, f in zip(hist["mixed"], hist["fp64"]))
    return ke, en


def run_config1(args, local, n=64):
    """3-D inviscid isentropic vortex advection (Shu
    vortex, beta 5, centre (5, 5), free stream rho = p = 1, u = (1, 1, 0)),
    n^3 unique nodes on the periodic box [0, 10]^3 with identity metrics,
    WENO5-JS + Rusanov, SSP-RK3, CFL 0.5, 200 steps, no viscosity, no LES.
    Per form: cell-updates/s and the density error against the vortex
    translated by t (1, 1, 0); mixed vs FP64: per-field error after the 200
    steps and the kinetic-energy / enstrophy history deviation."""
    import torch

    from chimera_comp_les_b200 import diagnostics as D
    from chimera_comp_les_b200 import workloads as W
    torch.cuda.set_device(local)
    L, steps = 10.0, 200
    coords = W.periodic_grid(n, L, amp=0.0)
    q0 = W.vortex_state(coords)
    r = q0[..., 0]
    u = np.abs(q0[..., 1] / r) + np.abs(q0[..., 2] / r)
    c = np.sqrt(1.4 * 0.4 * (q0[..., 4] - 0.5 * (q0[..., 1] ** 2 + q0[..., 2] ** 2 + q0[..., 3] ** 2) / r) / r)
    dt = 0.5 * (L / n) / float((u + c).max())  # CFL 0.5
    opts = dict(les=0, inviscid=1, fluxorder=3, weno_order=5, dt=dt)
    nv = np.zeros(coords.shape[:3])
    out = {"workload": f"isentropic vortex {n}^3 (DMDA {n + 2}^3), periodic [0,10]^3, identity metrics, beta 5, "
                       f"u = (1, 1, 0); WENO5-JS + Rusanov, inviscid, SSP-RK3, CFL 0.5, {steps} steps",
           "grid": [n + 2] * 3, "dt": dt, "steps": steps}
    blocks = {}
    for prec in ("fp64", "mixed"):
        blk = _block(prec, local, coords, q0, nv, **opts)
        ms, _ = _timed(blk, args.steps, args.warmup, 1, local)
        out[prec] = {"value": blk.interior_nodes * blk.stages * args.steps / (ms / 1e3), "ms_per_step": ms / args.steps}
        blocks[prec] = blk
    csi, eta, zet, aj = blocks["fp64"].metrics()
    keep = {100: {}}  # the step count the mixed-vs-FP64 bar is stated at
    hist, final = _histories(blocks, q0, steps, steps // 4,
                             lambda q: (D.kinetic_energy(q, aj), D.enstrophy(q, csi, eta, zet, aj)), keep=keep)
    t_end = steps * dt
    shifted = coords.copy()
    shifted[..., 0] = np.mod(coords[..., 0] - t_end, L)
    shifted[..., 1] = np.mod(coords[..., 1] - t_end, L)
    qe = W.vortex_state(shifted)
    inner = (slice(1, -1),) * 3
    for prec in ("fp64", "mixed"):
        d = final[prec][inner + (0,)] - qe[inner + (0,)]
        out[prec]["rho_error_vs_translated_vortex"] = float(np.linalg.norm(d) / np.linalg.norm(qe[inner + (0,)] - 1.0))
        blocks[prec].close()
    l2, linf = D.field_errors(final["mixed"], final["fp64"])
    ke, en = _history_devs(hist)
    l2h, linfh = D.field_errors(keep[100]["mixed"], keep[100]["fp64"])
    out["mixed_vs_fp64_error"] = {"steps": steps, "rel_l2": l2, "rel_linf": linf,
                                  "fields": ["rho", "rhoU", "rhoV", "rhoW", "rhoE"],
                                  "ke_history_max_rel_dev": ke, "enstrophy_history_max_rel_dev": en,
                                  "checkpoints_every": steps // 4,
                                  "after_100_steps": {"rel_l2": l2h, "rel_linf": linfh}}
    return out


def run_config5(args, local, n=512):
    """BASELINE config 5 at its largest size on one GPU: decaying compressible
    isotropic turbulence on a periodic [0, 2*pi]^3 Cartesian box of n^3 unique
    nodes (DMDA (n+2)^3), Passot-Pouquet spectrum k0 4, u_rms 1, Mt 0.4, seed
    5, rho 1, uniform p; WENO5-JS reconstruction with the Roe flux, pure
    upwind (-les 1 -s_x 0 -s_y 0 -s_z 0), Smagorinsky CS 0.17^2, SSP-RK3, dt
    from CFL 0.4.  Per form: cell-updates/s, stage-kernel GB/s, then the
    per-field mixed-vs-FP64 error after ACC_STEPS steps."""
    import torch

    from chimera_comp_les_b200 import diagnostics as D
    torch.cuda.set_device(local)
    coords, q0, dt, opts = config5_case(n)
    nv = np.zeros(coords.shape[:3])
    out = {"workload": f"decaying isotropic turbulence {n}^3 (DMDA {n + 2}^3), Passot-Pouquet k0 4, u_rms 1, Mt 0.4, "
                       f"seed 5; {CONFIG5_SCHEME}",
           "grid": [n + 2] * 3, "dt": dt, "interior_nodes": n ** 3}
    final, hist = {}, {}
    for prec in ("fp64", "mixed"):
        blk = _block(prec, local, coords, q0, nv, **opts)
        ms, _ = _timed(blk, args.steps, args.warmup, 1, local)
        kms = _kernel_ms(blk, 3)
        interior = blk.interior_nodes
        out[prec] = {"value": interior * blk.stages * args.steps / (ms / 1e3), "ms_per_step": ms / args.steps,
                     "kernel_avg_ms": kms, "achieved_gbs": B_ALG[prec] * interior / (kms / 1e3) / 1e9,
                     "kchunk_autotuned": blk.kchunk}
        if prec == "fp64":
            met = blk.metrics()
        h, f = _histories({prec: blk}, q0, ACC_STEPS, ACC_STEPS // 4,
                          lambda q: _ke_enstrophy_device(q, *met, local))
        hist[prec], final[prec] = h[prec], f[prec]
        blk.close()
    l2, linf = D.field_errors(final["mixed"], final["fp64"])
    ke, en = _history_devs(hist)
    out["speedup_mixed_vs_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    out["mixed_vs_fp64_error"] = {"steps": ACC_STEPS, "rel_l2": l2, "rel_linf": linf,
                                  "fields": ["rho", "rhoU", "rhoV", "rhoW", "rhoE"],
                                  "ke_history_max_rel_dev": ke, "enstrophy_history_max_rel_dev": en,
                                  "checkpoints_every": ACC_STEPS // 4}
    return out


def run_ours(args, ws, rank, local):
    import ctypes
    import torch

    from chimera_comp_les_b200 import workloads as W

    torch.cuda.set_device(local)
    n = N_UNIQUE
    coords = W.periodic_grid(n, 2 * math.pi, amp=0.05)
    q0 = W.tgv_state(coords, gamma=CFG["gamma"], ma=CFG["ma"])
    nv = np.zeros(coords.shape[:3])
    peak, peak_kind = measured_peaks()

    forms, blocks = _forms(coords, q0, nv, {}, args, ws, local, clocks_for=args.precision)
    head = forms[args.precision]
    acc = _accuracy(blocks["fp64"], blocks["mixed"], q0) if rank == 0 else None

    # end-to-end through the C-ABI with host buffers: every step the H2D copy
    # of its input state from pinned memory, the time step, and the D2H copy
    # of its result.  Headline: the streaming calls (cb_upload_state_async /
    # cb_download_state_async: copy streams and double-buffered staging, so one
    # step's download overlaps the next step's upload and compute); beside it
    # the blocking calls one after another (cb_upload_state / cb_download_state).
    blk = blocks[args.precision]
    stream = torch.cuda.ExternalStream(blk.stream, device=f"cuda:{local}")
    # as many steps as the device-timed value, so that the one upload before
    # the first step and the one download after the last (the pipeline's fill
    # and drain) weigh as little as they do in a long run
    e2e_steps = max(3, args.steps)
    q_host = torch.empty(q0.shape, dtype=torch.float64, pin_memory=True).numpy()
    q_host[...] = q0
    q_outs = [torch.empty(q0.shape, dtype=torch.float64, pin_memory=True).numpy() for _ in range(2)]
    qptr = q_host.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    blk.upload_async(q_host)  # first use: allocates the copy streams and staging
    blk.RungeKutta(1, sync=False)
    blk.download_async(q_outs[0])
    blk.join_transfers()
    blk.sync()
    barrier(ws)
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for s_ in range(e2e_steps):
        blk.upload_async(q_host)
        blk.RungeKutta(1, sync=False)
        blk.download_async(q_outs[s_ % 2])
    blk.join_transfers()
    f1.record(stream)
    torch.cuda.synchronize()
    blk.sync()
    barrier(ws)
    e2e_ms = max_over_ranks(f0.elapsed_time(f1), ws, local)
    e2e_value = ws * blk.interior_nodes * blk.stages * e2e_steps / (e2e_ms / 1e3)
    if not (np.isfinite(q_outs[0]).all() and np.isfinite(q_outs[1]).all()):
        raise RuntimeError("non-finite state after end-to-end steps")
    # the blocking calls
    g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    barrier(ws)
    g0.record(stream)
    for _ in range(e2e_steps):
        rc = blk.lib.cb_upload_state(blk._ctx, qptr)  # cb_upload_state: H2D + unpack, stream-ordered
        if rc:
            raise RuntimeError(f"cb_upload_state failed ({rc})")
        blk.RungeKutta(1, sync=False)
        blk.download(q_outs[0])  # cb_download_state: pack + D2H, waits for the stream
    g1.record(stream)
    torch.cuda.synchronize()
    barrier(ws)
    e2e_serial = ws * blk.interior_nodes * blk.stages * e2e_steps / (max_over_ranks(g0.elapsed_time(g1), ws, local) / 1e3)

    cpu = None
    vs_oracle = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        from oracle import cpu_baseline as cb
        r = cb.run(n, steps=1, warmup=0, cfgkw=CFG)
        cpu = {"value": r["value"], "unit": UNIT, "cores": r["cores"], "kind": r["kind"], "sample": r["sample"]}
        # the same slab per process on one core and with the shipped -O0 build
        slab = max(2, n // r["cores"])
        variants = []
        if r["kind"] == "reference":
            for procs, opt in ((1, True), (1, False), (r["cores"], False)):
                v = cb.run(n, steps=1, warmup=0, procs=procs, cfgkw=CFG, optimized=opt, nz=slab)
                variants.append({"value": v["value"], "cores": procs, "build": "-O3" if opt else "-O0 (as shipped)",
                                 "sample": v["sample"]})
        cpu["variants"] = variants
        # the same CPU leg, as the checker
        vs_oracle = _vs_oracle(n, coords, q0, nv, blocks, CFG)
    for b in blocks.values():
        b.close()

    # the same workload with Roe's flux (no counterpart in the reference)
    roe = None
    if not args.no_extras:
        roe_f, roe_b = _forms(coords, q0, nv, {"flux": "roe"}, args, ws, local)
        roe = {"flux": "Roe with Harten's entropy fix, otherwise the headline workload", **roe_f,
               "speedup_mixed_vs_fp64": roe_f["mixed"]["value"] / roe_f["fp64"]["value"]}
        roe["mixed_vs_fp64_error"] = _accuracy(roe_b["fp64"], roe_b["mixed"], q0) if rank == 0 else None
        for b in roe_b.values():
            b.close()

    # the reference's default hybrid scheme on the same TGV: WENO3 + Rusanov
    # blended with the central flux, sigma 1 (central only) and 0.5 (both)
    blends = None
    if not args.no_blend:
        blends = {}
        for name, sig in (("sigma_1", 1.0), ("sigma_half", 0.5)):
            f, bb = _forms(coords, q0, nv, dict(CFG_WENO3_BLEND, s_x=sig, s_y=sig, s_z=sig), args, ws, local)
            blends[name] = {"sigma": sig, **{k: {kk: vv for kk, vv in v.items() if kk != "launches_per_step"}
                                              for k, v in f.items()}}
            for b in bb.values():
                b.close()
        blends["scheme"] = "WENO3 + Rusanov blended with the 4-point skew-symmetric central flux (-fluxorder 3, SSP-RK3)"

    batched = run_batched(args, local) if (ws == 1 and not args.no_batched) else None
    config5 = run_config5(args, local) if (ws == 1 and not args.no_config5) else None
    config1 = run_config1(args, local) if (ws == 1 and not args.no_config1) else None

    if rank == 0:
        peaks = pipe_peaks(local)
        copy_gbs = hbm_copy_gbs(local)
        comp = compute_roofline(args.precision, CFG, head["kernel_avg_ms"], n ** 3, peaks) if peaks else None
        other_comp = (compute_roofline("fp64" if args.precision == "mixed" else "mixed", CFG,
                                       forms["fp64" if args.precision == "mixed" else "mixed"]["kernel_avg_ms"],
                                       n ** 3, peaks) if peaks else None)
        cfg = workload_config(n)
        other = "fp64" if args.precision == "mixed" else "mixed"
        other_d = {k: v for k, v in forms[other].items() if k != "clocks"}
        other_d["roofline_compute"] = other_comp
        line = {
            "metric": METRIC, "value": head["value"], "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32-flux/f64-state" if args.precision == "mixed" else "f64",
            "precision_form": args.precision,
            "data": "synthetic", "config": cfg,
            "roofline": {"bound": "hbm", "achieved": head["achieved_gbs"], "peak": peak, "unit": "GB/s",
                         "frac": head["achieved_gbs"] / peak,
                         "traffic": profile_traffic(args.precision),
                         "kernel": f"stage_kernel ({args.precision} form: fused RHS + RK combine)",
                         "kernel_avg_ms": head["kernel_avg_ms"], "kchunk_autotuned": head["kchunk_autotuned"],
                         "bytes_per_cell": B_ALG[args.precision],
                         "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                         "copy_gbs_measured_here": copy_gbs,
                         "frac_of_copy_measured_here": head["achieved_gbs"] / copy_gbs,
                         "compute": comp},
            "clocks": head.get("clocks"),
            "e2e": {"value": e2e_value, "unit": UNIT,
                    "h2d_bytes_per_step": int(q0.nbytes), "d2h_bytes_per_step": int(q0.nbytes),
                    "api": "cb_upload_state_async + cb_rk_step + cb_download_state_async per step (copies overlap "
                           "the neighbouring steps), cb_join_transfers before the closing event",
                    "steps": e2e_steps, "serial_blocking_calls": e2e_serial},
            "gpu_launches": head["launches_per_step"] * args.steps,
            "cpu_baseline": cpu,
            other: other_d,
            "speedup_mixed_vs_fp64": forms["mixed"]["value"] / forms["fp64"]["value"],
            "mixed_vs_fp64_error": acc,
            "roe": roe,
            "weno3_blend": blends,
            "config5_512": config5,
            "config1_vortex": config1,
            "batched": batched,
            "vs_oracle": vs_oracle,
            "pipe_peaks": peaks,
        }
        print(json.dumps(line), flush=True)


# ------------------------------------------------------------ size sweep --
def run_sweep(args, local):
    """Decaying compressible isotropic turbulence on a periodic [0, 2*pi]^3
    Cartesian box at 128^3 .. 512^3 (Passot-Pouquet spectrum, k0 4, u_rms 1,
    Mt 0.4, seed 5; rho 1, uniform p): per size and form cell-updates/s per
    stage, stage-kernel HBM GB/s, and the mixed-vs-FP64 per-field error after
    ACC_STEPS steps, in config 5's scheme (config5_case).  One JSON line per
    size (not the contract line)."""
    import torch

    from chimera_comp_les_b200 import Block
    from chimera_comp_les_b200 import diagnostics as D
    torch.cuda.set_device(local)
    peak, peak_kind = measured_peaks()
    for n in [int(x) for x in args.sweep.split(",")]:
        coords, q0, dt, opts = config5_case(n)
        nv = np.zeros(coords.shape[:3])
        out = {"sweep": "isotropic turbulence", "scheme": CONFIG5_SCHEME, "n": n, "grid": [n + 2] * 3, "dt": dt}
        final = {}
        for prec in ("fp64", "mixed"):
            blk = Block(n + 2, n + 2, n + 2, precision=prec, device=local, **opts)
            blk.FormMetrics(coords)
            blk.set_nvert(nv)
            blk.SetInitialCondition(q0)
            kc, _ = blk.autotune()
            steps = args.steps
            ms, _ = _timed(blk, steps, args.warmup, 1, local)
            kms = _kernel_ms(blk, 5)
            interior = blk.interior_nodes
            out[prec] = {"value": interior * blk.stages * steps / (ms / 1e3), "ms_per_step": ms / steps,
                         "kernel_avg_ms": kms, "achieved_gbs": B_ALG[prec] * interior / (kms / 1e3) / 1e9,
                         "kchunk_autotuned": kc}
            blk.SetInitialCondition(q0)
            blk.RungeKutta(ACC_STEPS)
            final[prec] = blk.Q()
            blk.close()
        l2, linf = D.field_errors(final["mixed"], final["fp64"])
        out["speedup_mixed_vs_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
        out["mixed_vs_fp64_error"] = {"steps": ACC_STEPS, "rel_l2": l2, "rel_linf": linf}
        out["peak_gbs"] = peak
        out["peak_source"] = peak_kind
        print(json.dumps(out), flush=True)


# -------------------------------------------------------- sphere (IB) --
# algorithmic bytes of one interpolation sweep per list entry: node 16, donor
# offsets 24, weights 88, three donors' Q and P 144, the element's vertex
# velocities now and one step back 144 and its vertex indices 12, the new Q
# and P written 48, then read 48 and stored at the node 48
B_IBM_ENTRY = 16 + 24 + 88 + 144 + 144 + 12 + 48 + 48 + 48
# WENO5-JS + Roe, pure upwind (sigma 0); Smagorinsky Cs 0.1 (CS = Cs^2 = 0.01)
SPHERE_OPTS = dict(les=1, inviscid=0, fluxorder=3, eno_order=2, central=2, s_x=0.0, s_y=0.0, s_z=0.0, ren=300.0,
                   ma=0.3, pr=0.71, gamma=1.4, dt=1e-3, cs_const=0.01, isothermal=0, flux="roe", weno_order=5)


def run_sphere(args, local):
    """Flow past a stationary sphere with the immersed boundary on the device:
    DMDA 192 x 192 x 256 (i, j across, k streamwise on [-5, 15] D), nodes
    clustered toward the sphere (spacing 0.01 D there), slip walls in i and j,
    inflow / outflow 45 in k, Re 300, Ma 0.3, WENO5-JS with the Roe flux (pure
    upwind), Smagorinsky Cs 0.1, dt 1e-3; uniform stream plus seeded 1e-3 white noise.
    The interpolation list comes from workloads.sphere_ibm_list (an analytic
    stand-in for the reference's host search).  Per form: cell-updates/s per
    stage with the interpolation in every step, the interpolation's share of
    the step, one interpolation's device time, and the host round trip
    (download + upload of Q) a host-side interpolation would add per step.
    One JSON line (not the contract line)."""
    import torch

    from chimera_comp_les_b200 import Block
    from chimera_comp_les_b200 import diagnostics as D
    from chimera_comp_les_b200 import workloads as W
    torch.cuda.set_device(local)
    n = tuple(int(x) for x in args.sphere_n.split(","))
    t0 = time.perf_counter()
    case = W.sphere_case(n=n)
    build_s = time.perf_counter() - t0
    info = case["info"]
    out = {"workload": f"sphere D=1, DMDA {n[0]}x{n[1]}x{n[2]}, clustered to 0.01 D, slip i/j, inflow/outflow 45 in k, "
                       "Re 300 Ma 0.3, WENO5-JS + Roe (pure upwind), Smagorinsky Cs 0.1 (CS 0.01), SSP-RK3, dt 1e-3",
           "interface_nodes": int(info.size), "list_build_s": build_s, "unit": UNIT}
    final = {}
    peak, peak_kind = measured_peaks()
    for prec in ("fp64", "mixed"):
        blk = Block(n[0], n[1], n[2], bctype=case["bctype"], precision=prec, device=local, **SPHERE_OPTS)
        blk.FormMetrics(case["coords"])
        blk.set_nvert(case["nvert"])
        blk.SetInitialCondition(case["q"])
        blk.set_ibm_surface(0, case["surface"])
        blk.set_ibm_list(0, info, case["coords"])
        kc, _ = blk.autotune()
        steps = args.steps
        ms_ib, clocks = _timed(blk, steps, args.warmup, 1, local, sample_clocks=(prec == "mixed"))
        # one interpolation (five sweeps), device time on the library's stream
        stream = torch.cuda.ExternalStream(blk.stream, device=f"cuda:{local}")
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(10):
            blk.ibm_interpolation_advanced(0, 1)
        e1.record(stream)
        torch.cuda.synchronize()
        interp_ms = e0.elapsed_time(e1) / 10
        # host round trip per step a host-side interpolation would need
        qh = np.empty(blk.shape + (5,))
        t1 = time.perf_counter()
        for _ in range(3):
            blk.download(qh)
            blk.SetInitialCondition(qh)
        rt_ms = (time.perf_counter() - t1) / 3 * 1e3
        # the same steps without the list
        blk.set_ibm_list(0, info[:0], case["coords"])
        ms_plain, _ = _timed(blk, steps, args.warmup, 1, local)
        interior = blk.interior_nodes
        out[prec] = {"value": interior * blk.stages * steps / (ms_ib / 1e3), "ms_per_step": ms_ib / steps,
                     "ms_per_step_without_ib": ms_plain / steps,
                     "ib_ms_per_step": (ms_ib - ms_plain) / steps,
                     "ib_share_of_step": (ms_ib - ms_plain) / ms_ib,
                     "interpolation_ms": interp_ms,
                     "sweep_gbs": B_IBM_ENTRY * info.size * 5 / (interp_ms / 1e3) / 1e9,
                     "host_roundtrip_ms_per_step": rt_ms, "kchunk_autotuned": kc}
        if clocks:
            out["clocks"] = clocks
        blk.set_ibm_list(0, info, case["coords"])
        blk.SetInitialCondition(case["q"])
        blk.RungeKutta(args.sphere_acc_steps)
        final[prec] = blk.Q()
        blk.close()
    l2, linf = D.field_errors(final["mixed"], final["fp64"])
    out["speedup_mixed_vs_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    out["mixed_vs_fp64_error"] = {"steps": args.sphere_acc_steps, "rel_l2": l2, "rel_linf": linf}
    out["peak_gbs"] = peak
    out["peak_source"] = peak_kind
    print(json.dumps(out), flush=True)


# ------------------------------------------------------- sharded (N > 1) --
def run_sharded(args, ws, rank, local):
    """k-slab decomposition of one periodic TGV box of 128 x 128 x 128N unique
    nodes over N GPUs, one 128^3 slab (DMDA 130^3) per rank: every RK stage
    exchanges the slabs' two-node halos (and the eddy viscosity's once per
    step) with the neighbours through NCCL point-to-point on the library's
    stream.  Weak scaling: per-GPU work equals the N = 1 workload."""
    import torch

    from chimera_comp_les_b200 import batch as B
    from chimera_comp_les_b200 import sharded as S
    from chimera_comp_les_b200 import workloads as W

    torch.cuda.set_device(local)
    n = N_UNIQUE
    gn = (n, n, n * ws)
    glen = (2 * math.pi, 2 * math.pi, 2 * math.pi * ws)
    M = (n + 2, n + 2, n * ws + 2)
    parts = B.decompose(M, [[n], [n], [n] * ws])
    rob = S.slab_ranks(len(parts), ws)
    near = {(rank - 1) % ws, rank, (rank + 1) % ws}
    st, wr = B.halo_maps_decomposed(M, parts, only=near)
    plan = S.exchange_plan(st, wr, rob, rank)
    (b,) = plan.blocks
    off, d = parts[b]
    coords = W.periodic_grid_slab(gn, glen, 0.05, off[2], d[2])
    q0 = W.tgv_state(coords, gamma=CFG["gamma"], ma=CFG["ma"])
    prec = args.precision
    bt = B.Batch([d], precision=prec, device=local, **CFG)
    bt.FormMetrics(0, coords)
    bt.SetInitialCondition(0, q0)
    sh = S.Shard(bt, plan, torch.device("cuda", local))
    tr = S.DistTransport()
    S.fill_ghosts_all([sh], tr)
    S.step_all([sh], tr, max(args.warmup, 3))
    stream = torch.cuda.ExternalStream(bt.stream, device=f"cuda:{local}")
    sampler = ClockSampler(gpu_identifier(local)) if rank == 0 else None
    if sampler:
        sampler.start()
        time.sleep(0.3)
    barrier(ws)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    S.step_all([sh], tr, args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(ws)
    clocks = sampler.stop() if sampler else None
    bt.sync()
    ms = max_over_ranks(e0.elapsed_time(e1), ws, local)
    interior, stages = bt.interior_nodes, CFG["fluxorder"]
    # stage phases alone (stage kernel + local halo gather + pack), on the library stream
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(stages)]
    for s_, (a, c) in enumerate(ev):
        if s_ == 0 and CFG["les"]:
            S._run_phase([sh], tr, S.CB_PHASE_NUT, 0, B.HALO_WRAP, 1, False)
        a.record(stream)
        bt.phase(S.CB_PHASE_STAGE, s_)
        c.record(stream)
        tr.exchange([sh], B.HALO_STAGE, 5)
        bt.phase_unpack(S.CB_PHASE_STAGE)
    torch.cuda.synchronize()
    kms = max_over_ranks(sum(a.elapsed_time(c) for a, c in ev) / stages, ws, local)
    # end to end through the public API with host buffers: upload, ghost exchange, one step, download
    q_host = torch.empty(q0.shape, dtype=torch.float64, pin_memory=True).numpy()
    q_host[...] = q0
    e2e_steps = max(3, args.steps)
    barrier(ws)
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(e2e_steps):
        bt.SetInitialCondition(0, q_host)
        S.fill_ghosts_all([sh], tr)
        S.step_all([sh], tr, 1)
        q_out = bt.Q(0)
    f1.record(stream)
    torch.cuda.synchronize()
    barrier(ws)
    e2e_ms = max_over_ranks(f0.elapsed_time(f1), ws, local)
    if not np.isfinite(q_out).all():
        raise RuntimeError("non-finite state after end-to-end steps")
    if rank == 0:
        peak, peak_kind = measured_peaks()
        achieved = B_ALG[prec] * interior / (kms / 1e3) / 1e9
        cfg = workload_config(n)
        cfg.update({"workload": cfg["workload"].replace(f"{n}^3 (DMDA {n + 2}^3)",
                                                        f"{n}x{n}x{n * ws} box in {ws} k-slabs of {n}^3 (DMDA {n + 2}^3 each)"),
                    "parallelism": f"k-slabs over {ws} GPUs, 2-node halo exchange per stage (NCCL send/recv)",
                    "interior_nodes": interior * ws})
        line = {
            "metric": METRIC, "value": ws * interior * stages * args.steps / (ms / 1e3), "unit": UNIT, "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32-flux/f64-state" if prec == "mixed" else "f64", "precision_form": prec,
            "data": "synthetic", "config": cfg,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": profile_traffic(prec),
                         "kernel": f"stage phase ({prec} form: persistent stage kernel + local halo gather + pack)",
                         "kernel_avg_ms": kms, "bytes_per_cell": B_ALG[prec],
                         "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"},
            "clocks": clocks,
            "e2e": {"value": ws * interior * stages * e2e_steps / (e2e_ms / 1e3), "unit": UNIT,
                    "h2d_bytes_per_step": int(q0.nbytes) * ws, "d2h_bytes_per_step": int(q0.nbytes) * ws},
            "gpu_launches": (stages * 4 + 3) * args.steps,
            "cpu_baseline": None,
            "exchange_entries_per_stage": {"send": int(len(plan.stage.send)), "recv": int(len(plan.stage.recv))},
        }
        print(json.dumps(line), flush=True)
    bt.close()


def run_profile(args, local):
    """The headline workload for a profiler: one form (--precision), the
    k-chunk given by --profile-kchunk (one autotuner candidate: 3 stage
    launches), then --steps time steps; no timing, no other workloads."""
    import torch

    from chimera_comp_les_b200 import workloads as W
    torch.cuda.set_device(local)
    n = N_UNIQUE
    coords = W.periodic_grid(n, 2 * math.pi, amp=0.05)
    q0 = W.tgv_state(coords, gamma=CFG["gamma"], ma=CFG["ma"])
    from chimera_comp_les_b200 import Block
    with Block(n + 2, n + 2, n + 2, precision=args.precision, device=local, **CFG) as blk:
        blk.FormMetrics(coords)
        blk.set_nvert(np.zeros(coords.shape[:3]))
        blk.SetInitialCondition(q0)
        kc, ms = blk.autotune([args.profile_kchunk])
        blk.RungeKutta(args.steps)
        print(json.dumps({"profile_case": workload_config(n)["workload"], "precision_form": args.precision,
                          "kchunk": kc, "stage_ms": ms, "steps": args.steps}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"],
                    help="form reported as the headline value (both are measured)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true", help="skip the multi-block batched measurement")
    ap.add_argument("--no-blend", action="store_true", help="skip the WENO3 blend (sigma 1 and 0.5) on the headline TGV")
    ap.add_argument("--no-extras", action="store_true", help="skip the Roe-flux measurement of the headline workload")
    ap.add_argument("--no-config5", action="store_true", help="skip the 512^3 isotropic-turbulence measurement")
    ap.add_argument("--no-config1", action="store_true", help="skip the 64^3 isentropic-vortex measurement")
    ap.add_argument("--profile", action="store_true",
                    help="run the headline workload in one form for a profiler (no timing, no other workloads)")
    ap.add_argument("--profile-kchunk", type=int, default=10, help="k-chunk of the --profile run")
    ap.add_argument("--sweep", default="", help="comma-separated sizes, e.g. 128,256,384,512: isotropic-turbulence "
                                                  "size sweep, one JSON line per size instead of the bench line")
    ap.add_argument("--workload", default="tgv", choices=["tgv", "sphere"],
                    help="sphere: flow past a sphere with the device immersed boundary, one JSON line of its own")
    ap.add_argument("--sphere-n", default="192,192,256", help="DMDA node counts mx,my,mz of the sphere workload")
    ap.add_argument("--sphere-acc-steps", type=int, default=50, help="steps of the sphere's mixed-vs-FP64 comparison")
    ap.add_argument("--layout", default="auto", choices=["auto", "replicas", "slabs"],
                    help="N GPUs: one TGV box split in k-slabs with halo exchange (default for N > 1), "
                         "or independent replicas")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    ws, rank, local = dist_setup()
    try:
        layout = args.layout if args.layout != "auto" else ("slabs" if ws > 1 else "replicas")
        if args.impl == "reference":
            run_reference(args, ws, rank)
        elif args.profile:
            run_profile(args, local)
        elif args.sweep:
            run_sweep(args, local)
        elif args.workload == "sphere":
            run_sphere(args, local)
        elif layout == "slabs":
            run_sharded(args, ws, rank, local)
        else:
            run_ours(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
