#!/usr/bin/env python
"""Zone-updates/s of the per-stage hot path (reconstruction -> Riemann -> flux
divergence -> SSP-RK stage update with the CFL max-reduction) on B200.

Headline workload: 3D Euler spherical Sod blast, 256^3 cells on [0,1]^3, outflow,
gamma=1.4, kernel-based WENO-AO radius 2 with the KXRCF selector, HLLC, SSP(4,3)
with the adaptive FSAL controller, CFL 0.8, plain FP64.  One "step" is one accepted
time step (4 RHS evaluations + stage updates + error estimate) of the whole grid;
one zone-update is one cell advanced by one accepted step.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload sod3d|kelvin_helmholtz|taylor_green|orszag_tang|isentropic_vortex]
                  [--scale N] [--precision fp64|tf32x3] [--indicator kxrcf|mlp]
                  [--no-forms] [--no-cpu-baseline]

Beside the plain FP64 value the line carries "forms": the same workload with the
3xTF32 tensor-core reconstruction (fp32_3xtf32), and with the learned
troubled-cell indicator (trained untimed on a small grid of the same problem)
with the FP32 and with the FP64 reconstruction.

With N > 1 (torchrun) every rank advances an independent replica of the grid
(the path has no cross-GPU exchange in this scope); value is the total over ranks
divided by the slowest rank's device time.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "kfvm-kokkos_b200"))

import kfvm_abi as abi  # noqa: E402

UNIT = "zone-updates/s"
# workload -> (default cells per axis, dimension, short name, description)
WORKLOADS = {
    "sod3d": (256, 3, "3D Euler Sod blast",
              "3D Euler spherical Sod blast {s}^3, outflow, GP-WENO-AO r=2 + KXRCF, HLLC, SSP(4,3) FSAL "
              "adaptive, CFL 0.8"),
    "kelvin_helmholtz": (1024, 2, "2D Euler Kelvin-Helmholtz",
                         "2D Euler Kelvin-Helmholtz {s}^2 periodic, seeded noise, GP-WENO-AO r=2 + KXRCF, HLLC, "
                         "SSP(4,3) FSAL adaptive, CFL 0.8"),
    "taylor_green": (256, 3, "3D Navier-Stokes Taylor-Green",
                     "3D Navier-Stokes Taylor-Green {s}^3 periodic, Re 1600, Pr 0.71, Mach 0.1, GP-WENO-AO r=2 + "
                     "KXRCF, HLLC + viscous terms, SSP(4,3) FSAL adaptive, CFL 0.8"),
    "orszag_tang": (1024, 2, "2D GLM-MHD Orszag-Tang",
                    "2D GLM-MHD Orszag-Tang {s}^2 periodic, GP-WENO-AO r=2 + KXRCF, HLL, SSP(4,3) FSAL adaptive, "
                    "CFL 0.4, GLM sources"),
    "isentropic_vortex": (128, 2, "2D Euler isentropic vortex",
                          "2D Euler isentropic vortex {s}^2 periodic, GP-WENO-AO r=2 + KXRCF, HLLC, SSP(4,3) FSAL "
                          "adaptive, CFL 0.8"),
    "sr_riemann_2d": (512, 2, "2D SR-hydro four-quadrant Riemann",
                      "2D special-relativistic hydro four-quadrant Riemann problem {s}^2 outflow, GP-WENO-AO r=2 + "
                      "KXRCF, LLF, SSP(4,3) FSAL adaptive, CFL 1.0, Newton pressure recovery"),
}


def metric_name(workload, scale, precision="fp64", indicator="kxrcf"):
    _, dim, short, _ = WORKLOADS[workload]
    form = {("fp64", "kxrcf"): "plain FP64", ("tf32x3", "kxrcf"): "FP32 3xTF32 form",
            ("fp64", "mlp"): "learned indicator + FP64", ("tf32x3", "mlp"): "learned indicator + FP32"}
    return f"zone-updates/s on 1 B200 ({short} {scale}^{dim}, {form[(precision, indicator)]})"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="sod3d", choices=sorted(WORKLOADS))
    p.add_argument("--scale", type=int, default=None, help="grid cells per axis (default: the workload's)")
    p.add_argument("--e2e-steps", type=int, default=4)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--precision", default="fp64", choices=["fp64", "tf32x3"],
                   help="arithmetic of the linear reconstruction contraction")
    p.add_argument("--no-forms", action="store_true", help="skip timing the FP32 and learned forms")
    p.add_argument("--indicator", default="kxrcf", choices=["kxrcf", "mlp"],
                   help="troubled-cell indicator of the timed run (mlp: trained untimed first)")
    a = p.parse_args()
    if a.scale is None:
        a.scale = WORKLOADS[a.workload][0]
    return a


def config_block(workload, scale, extra=None):
    _, dim, _, desc = WORKLOADS[workload]
    c = {"workload": desc.format(s=scale) + ", FP64",
         "grid": [scale] * dim, "cells": scale ** dim,
         "l2": "inputs larger than L2 (state + face arrays ~GBs >> 126 MB)" if scale ** dim >= 2 ** 20
         else "small grid: inputs partly L2 resident"}
    if extra:
        c.update(extra)
    return c


def replica_totals(elapsed, work, world_size, device):
    """Replicas only: every rank advances its own copy of the grid, so the job's
    time is the slowest rank's and its work the sum over ranks."""
    if world_size <= 1:
        return elapsed, work
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(elapsed)], device=device, dtype=torch.float64)
    w = torch.tensor([float(work)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(w, op=dist.ReduceOp.SUM)
    return t.item(), w.item()


def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


# ------------------------------------------------------------------ clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()
        # nvidia-smi's start-up (NVML initialisation) stalls the device for some
        # milliseconds: let it finish before the timed region begins
        t0 = time.time()
        while not self.rows and time.time() - t0 < 3.0 and self.proc.poll() is None:
            time.sleep(0.01)

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.thread is not None:
            self.thread.join(timeout=5)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            for n, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


# ------------------------------------------------------------------ roofline
def _shape(cfg):
    d = cfg.dim
    nv = abi.nvars(cfg)
    nqf = 2 if d == 2 else 4
    nqc = 4 if d == 2 else 8
    ncst = 13 if d == 2 else 33                         # cells of the radius-2 stencil
    src = cfg.eq == abi.KFVM_EQ_MHD_GLM
    return d, nv, nqf, nqc, ncst, src


def algorithmic_bytes(cls, cfg):
    """Algorithmic HBM bytes per launch of each kernel class (8-byte reals; every
    array element read or written once: stencil and halo re-reads are not counted)."""
    n = abi.ncells(cfg)
    d, nv, nqf, nqc, ncst, src = _shape(cfg)
    nf = 2 * d
    nfaces = sum((cfg.nx + (k == 0)) * (cfg.ny + (k == 1)) * ((cfg.nz if d == 3 else 1) + (k == 2))
                 for k in range(d))
    per_cell = {
        # U in; own face states (8-byte reals), KXRCF indicator (4-byte) per own face
        # point, status out
        "recon": nv * 8 + nf * nqf * (nv * 8 + 4) + 1 + ((nqc * nv * 8 + 16) if src else 0),
        # indicators (each face point once), U, theta in; flag out
        "flag": nf * nqf * 4 + nv * 8 + 8 + 1,
        # flag, set, status in; applied out (theta / heavy-list writes are partial)
        "compact": 4,
        # Riemann fluxes, U, Uprev, Uhat in; U', Uhat out
        "stage": (d * nv + 5 * nv) * 8,
        "bc_fill": 0,
    }
    if cls == "riemann":
        return nfaces * (2 * nqf * nv * 8 + nv * 8) / d   # per launch (one direction)
    return per_cell.get(cls, 0) * n


def algorithmic_fma(cls, cfg):
    """FP64 fused multiply-adds per launch of the linear reconstruction contraction:
    every (stencil cell, weight row, variable) triple once per cell."""
    if cls != "recon":
        return None
    d, nv, nqf, nqc, ncst, src = _shape(cfg)
    rows = 2 * d * nqf + (nqc if src else 0)
    return abi.ncells(cfg) * ncst * rows * nv


def load_json(path):
    try:
        with open(path) as f:
            return json.load(f)
    except Exception:
        return None


# ------------------------------------------------------------------ our arm
def train_indicator(workload, seed=1):
    """Weights of the learned indicator for a workload: samples of a plain run of
    the same problem (3D on a 128^3 grid), every 6 steps of 24, all troubled
    cells and 5 % of the others; 800 Adam steps."""
    import kfvm
    dim = WORKLOADS[workload][1]
    cfg, ic = abi.workload(workload, scale=128 if dim == 3 else WORKLOADS[workload][0], steps=40)
    s = kfvm.Solver(cfg)
    s.init_ic(ic)
    s.mlp_reserve(1500000)
    n = npos = 0
    for step in range(25):
        if step % 6 == 0:
            n, npos = s.mlp_collect(tau=0.3, keep=0.05, seed=100 + step)
        s.take_step()
    s.mlp_init(seed)
    l0, l1 = s.mlp_train(800, batch=1024, lr=3e-3, pos_weight=4.0, seed=seed)
    w = s.mlp_weights()
    s.close()
    return w, {"train_grid": [cfg.nx] * dim, "samples": n, "troubled": npos, "loss_first": l0, "loss_last": l1}


def kernel_breakdown(solver, steps):
    """Device time per kernel class (CUDA events around each launch on the solver's
    stream) over `steps` more steps: {class: (ms, launches)}."""
    import torch
    solver.set_timing(True)
    for _ in range(steps):
        solver.take_step()
    torch.cuda.synchronize()
    per_class = solver.timing()
    solver.set_timing(False)
    return per_class


def time_form(cfg, ic, prec, steps, warmup, mlp_weights=None):
    """Zone-updates/s of one arithmetic form: device time of `steps` accepted-step
    attempts after `warmup`, CUDA events on the solver's stream."""
    import torch
    import kfvm
    s = kfvm.Solver(cfg)
    s.set_precision(prec)
    if mlp_weights is not None:
        s.mlp_set_weights(mlp_weights)
        s.set_indicator(abi.KFVM_IND_MLP)
    s.init_ic(ic)
    for _ in range(warmup):
        s.take_step()
    stream = torch.cuda.ExternalStream(s.stream_handle())
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    acc = 0
    for _ in range(steps):
        acc += s.take_step().accepted
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    per_class = kernel_breakdown(s, min(steps, 2))
    out = {"value": acc * abi.ncells(cfg) / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / steps,
           "steps": steps, "accepted_steps": acc,
           "kernel_ms": {k: round(v[0], 3) for k, v in per_class.items() if v[1] > 0}}
    if mlp_weights is not None:
        out["judge"] = s.mlp_stats()
    s.close()
    out["l1_vs_plain"] = form_difference(cfg, ic, prec, mlp_weights)
    return out


def form_difference(cfg, ic, prec, mlp_weights=None, steps=3):
    """Relative L1 difference per conserved variable between a form and plain FP64
    after `steps` accepted steps from the initial condition, the form driven with
    plain FP64's step sizes (so both states are at the same time levels)."""
    import numpy as np
    import kfvm
    a = kfvm.Solver(cfg)
    a.init_ic(ic)
    b = kfvm.Solver(cfg)
    b.set_precision(prec)
    if mlp_weights is not None:
        b.mlp_set_weights(mlp_weights)
        b.set_indicator(abi.KFVM_IND_MLP)
    b.init_ic(ic)
    for _ in range(steps):
        b.set_time(*a.time_dt())
        a.take_step()
        b.take_step()
    ua, ub = a.get_state(), b.get_state()
    a.close()
    b.close()
    den = np.maximum(np.abs(ua).sum(axis=1), 1e-300)
    rel = np.abs(ub - ua).sum(axis=1) / den
    names = ["dens", "momx", "momy", "momz", "etot", "magx", "magy", "magz", "psi"]
    return {"steps": steps, "per_variable": {names[v]: float(rel[v]) for v in range(len(rel))}}


def run_ours(args):
    import numpy as np
    import torch
    import kfvm

    ws, rank, local = dist_init()
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    kfvm.lib()  # raises if the CUDA library is missing: no CPU fallback

    cfg, ic = abi.workload(args.workload, scale=args.scale, steps=args.warmup + args.steps + 10)
    solver = kfvm.Solver(cfg)
    if args.precision == "tf32x3":
        solver.set_precision(abi.KFVM_PREC_TF32X3)
    if args.indicator == "mlp":
        w, _ = train_indicator(args.workload)
        solver.mlp_set_weights(w)
        solver.set_indicator(abi.KFVM_IND_MLP)
    solver.init_ic(ic)
    n = abi.ncells(cfg)
    nv = abi.nvars(cfg)
    rhs0 = 1  # the FSAL priming evaluation
    for _ in range(args.warmup):
        rhs0 = solver.take_step().n_rhs

    stream = torch.cuda.ExternalStream(solver.stream_handle())
    launches0 = solver.launch_count()
    sampler = ClockSampler(local)
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    sampler.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    accepted = 0
    attempts = 0
    nweno = []
    for _ in range(args.steps):
        info = solver.take_step()
        accepted += info.accepted
        attempts += info.attempts
        nweno.append(info.n_weno)
    n_rhs = info.n_rhs - rhs0 if args.steps else 0
    e1.record(stream)
    torch.cuda.synchronize()
    if ws > 1:
        torch.distributed.barrier()
    sampler.stop()
    ms = e0.elapsed_time(e1)
    launches = solver.launch_count() - launches0
    # the per-class breakdown comes from further steps: its events around every
    # launch would take launch slots inside the timed steps
    breakdown_steps = max(1, min(args.steps, 4))
    per_class = kernel_breakdown(solver, breakdown_steps)

    # max over ranks of the device time, sum of the work
    t_max, work = replica_totals(ms, accepted * n, ws, "cuda")
    value = work / (t_max / 1e3)

    # end to end through the public API with host buffers: per step upload the
    # state from pinned host memory (set_state primes the FSAL stage), one
    # TakeStep, read the state back
    host = torch.empty((nv, n), dtype=torch.float64, pin_memory=True).numpy()
    solver.get_state(host)
    torch.cuda.synchronize()
    if ws > 1:
        torch.distributed.barrier()
    t0 = time.perf_counter()
    e2e_acc = 0
    for _ in range(args.e2e_steps):
        solver.set_state(host)
        info = solver.take_step()
        e2e_acc += info.accepted
        solver.get_state(host)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    e2e_s, e2e_work = replica_totals(e2e_s, e2e_acc * n, ws, "cuda")
    e2e = {"value": e2e_work / e2e_s, "unit": UNIT, "h2d_bytes_per_step": int(nv * n * 8),
           "d2h_bytes_per_step": int(nv * n * 8),
           "how": "per step: kfvm_set_state from pinned host (re-primes FSAL), kfvm_take_step, "
                  "kfvm_get_state to pinned host; wall clock"}

    # roofline of the dominant kernel class
    peaks = load_json(os.path.join(ROOT, "MEASURED_PEAKS.json"))
    hbm_peak = peaks.get("hbm_gbs") if peaks else 6650.0
    peak_src = "measured" if peaks else "fallback"
    dom = max((k for k in per_class if per_class[k][1] > 0), key=lambda k: per_class[k][0])
    dom_ms, dom_n = per_class[dom]
    tf32_recon = args.precision == "tf32x3" and dom == "recon"
    # the FP32 form's reconstruction is two launches per evaluation (the limiter
    # bounds, then the tensor-core contraction): time per evaluation
    avg_ms = dom_ms / max(dom_n // 2 if tf32_recon else dom_n, 1)
    algo = algorithmic_bytes(dom, cfg)
    achieved = algo / (avg_ms / 1e3) / 1e9
    # DRAM bytes per cell of each kernel class from one ncu capture (profiles/),
    # scaled by the cells one launch processes
    traffic_tbl = load_json(os.path.join(ROOT, "profiles", "dram_traffic.json")) or {}
    case = f"{cfg.dim}d_{('hydro', 'ns', 'glm', 'sr')[cfg.eq]}"
    per_cell = traffic_tbl.get("cases", {}).get(case, {}).get("bytes_per_cell", {}).get(
        "recon_tc" if args.precision == "tf32x3" and dom == "recon" else dom)
    traffic = per_cell * n if per_cell is not None else None
    hbm = {"achieved": achieved, "peak": hbm_peak, "unit": "GB/s", "frac": achieved / hbm_peak,
           "algorithmic_bytes": algo,
           "peak_source": f"{peak_src} (MEASURED_PEAKS.json hbm_gbs)" if peaks else "fallback"}
    fma = algorithmic_fma(dom, cfg)
    if fma is not None and tf32_recon:
        # 3xTF32 on tcgen05: three MMAs per product (hi hi, hi lo, lo hi); TF32 runs at
        # half the dense bf16 rate, so its peak is half the measured bf16 GEMM
        tf32_peak = (peaks.get("bf16_tflops") if peaks else 1590.0) / 2
        tf = 3 * 2 * fma / (avg_ms / 1e3) / 1e12
        roofline = {"bound": "tensor", "kernel": "recon (bounds + recon_tc_tma)", "achieved": tf, "peak": tf32_peak,
                    "unit": "TFLOP/s", "frac": tf / tf32_peak, "traffic": traffic, "tf32_mma_flop_per_launch": 6 * fma,
                    "launch_ms": avg_ms,
                    "peak_source": ("half of the measured dense bf16 GEMM (MEASURED_PEAKS.json bf16_tflops)" if peaks
                                    else "half of the fallback bf16 1.59 PFLOP/s"),
                    "hbm": hbm}
    elif fma is not None:
        # the FP64 reconstruction runs on the FP64 tensor pipe (m8n8k4 DMMA): its bound
        # is that pipe's throughput, measured on this GPU by back-to-back MMAs
        fp64_peak = kfvm.measure_fp64_mma()
        fp64 = 2 * fma / (avg_ms / 1e3) / 1e12
        roofline = {"bound": "tensor", "kernel": dom, "achieved": fp64, "peak": fp64_peak, "unit": "TFLOP/s",
                    "frac": fp64 / fp64_peak, "traffic": traffic, "fma_per_launch": fma, "launch_ms": avg_ms,
                    "peak_source": "measured on this GPU: FP64 m8n8k4 MMAs back to back on every SM "
                                   "(kfvm_measure_fp64_mma); FP64, so not the bf16 figure of MEASURED_PEAKS.json",
                    "hbm": hbm}
    else:
        roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                    "frac": achieved / hbm_peak, "traffic": traffic, "algorithmic_bytes": algo, "launch_ms": avg_ms,
                    "peak_source": hbm["peak_source"]}
    # the whole path: attainable zone-updates/s = min(HBM / B_zu, FP64 / F_zu)
    # B_zu: per stage U, Uprev, Utmp, Uhat in and U', Utmp, Uhat out (7 NV reals),
    #       plus the error pass (2 NV reals); F_zu: per RHS evaluation and cell the
    #       linear contraction (2 rows C NV), d NQF Riemann solves at ~200 flops and
    #       ~300 flops of divergence / update, 4 evaluations per step (WENO cells extra)
    d_, nv_, nqf_, nqc_, ncst_, src_ = _shape(cfg)
    rows_ = 2 * d_ * nqf_ + (nqc_ if src_ else 0)
    b_zu = 4 * 7 * nv_ * 8 + 2 * nv_ * 8
    f_zu = 4 * (2 * rows_ * ncst_ * nv_ + d_ * nqf_ * 200 + 300)
    fp64_peak_ = (roofline["peak"] * 1e12 if roofline["unit"] == "TFLOP/s" and not tf32_recon
                  else kfvm.measure_fp64_mma() * 1e12)
    att_hbm, att_fp64 = hbm_peak * 1e9 / b_zu, fp64_peak_ / f_zu
    path_roofline = {"bytes_per_zone_update": b_zu, "flops_per_zone_update": f_zu,
                     "attainable_hbm": att_hbm, "attainable_fp64": att_fp64,
                     "binding": "fp64" if att_fp64 < att_hbm else "hbm",
                     "frac_hbm": value / att_hbm, "frac_fp64": value / att_fp64,
                     "frac_binding": value / min(att_hbm, att_fp64), "unit": UNIT}
    share = {k: round(v[0] / max(sum(x[0] for x in per_class.values()), 1e-9), 4)
             for k, v in per_class.items() if v[1] > 0}

    out = {"metric": metric_name(args.workload, args.scale, args.precision, args.indicator), "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic (analytic initial condition)",
           "config": config_block(args.workload, args.scale, {"parallelism": f"replicas x{ws}",
                                               "accepted_steps": accepted, "attempts": attempts,
                                               "weno_cells_last": nweno[-1] if nweno else None}),
           "rhs_evals": int(n_rhs), "rhs_cell_rate": n_rhs * n / (t_max / 1e3) if n_rhs else None,
           "e2e": e2e, "gpu_launches": int(launches), "roofline": roofline, "path_roofline": path_roofline,
           "kernel_share": share,
           "kernel_ms": {k: round(v[0], 3) for k, v in per_class.items() if v[1] > 0},
           "kernel_breakdown_steps": breakdown_steps}
    out["clocks"] = sampler.summary()

    solver.close()
    if not args.no_forms and cfg.eq != abi.KFVM_EQ_SRHYDRO:
        # the FP32 form (3xTF32 tensor-core reconstruction) and the learned + FP32
        # form (network trained untimed on a small grid of the same problem)
        fs = max(2, args.steps // 2)
        form = time_form(cfg, ic, abi.KFVM_PREC_TF32X3, steps=fs, warmup=2)
        form["vs_plain"] = form["value"] / value
        w, info = train_indicator(args.workload)
        lf = time_form(cfg, ic, abi.KFVM_PREC_TF32X3, steps=fs, warmup=2, mlp_weights=w)
        lf["vs_plain"] = lf["value"] / value
        lf["training"] = info
        lf64 = time_form(cfg, ic, abi.KFVM_PREC_FP64, steps=fs, warmup=2, mlp_weights=w)
        lf64["vs_plain"] = lf64["value"] / value
        out["forms"] = {"fp32_3xtf32": form, "learned_fp32": lf, "learned_fp64": lf64}
    if not args.no_forms and ws == 1 and cfg.eq != abi.KFVM_EQ_SRHYDRO:
        # the target's own workloads: Taylor-Green 256^3 and Kelvin-Helmholtz 1024^2,
        # plain FP64 against the FP32 and the learned + FP32 forms (short runs)
        out["target_forms"] = {}
        for wl, sc in (("taylor_green", 256), ("kelvin_helmholtz", 1024)):
            tcfg, tic = abi.workload(wl, scale=sc, steps=40)
            plain = time_form(tcfg, tic, abi.KFVM_PREC_FP64, steps=3, warmup=2)
            f32 = time_form(tcfg, tic, abi.KFVM_PREC_TF32X3, steps=3, warmup=2)
            w, info = train_indicator(wl)
            lf32 = time_form(tcfg, tic, abi.KFVM_PREC_TF32X3, steps=3, warmup=2, mlp_weights=w)
            entry = {"grid": [sc] * WORKLOADS[wl][1], "plain_fp64": plain["value"], "unit": UNIT}
            for name, r in (("fp32_3xtf32", f32), ("learned_fp32", lf32)):
                entry[name] = {"value": r["value"], "vs_plain": r["value"] / plain["value"],
                               "l1_vs_plain": r["l1_vs_plain"], "kernel_ms": r["kernel_ms"]}
            entry["plain_kernel_ms"] = plain["kernel_ms"]
            out["target_forms"][f"{wl}_{sc}"] = entry
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(args.workload, sample_scale=cpu_sample_scale(args.workload),
                                           sample_steps=3)
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)


# ------------------------------------------------------------------ CPU arms
def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    oracle.lib()
    return oracle


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def cpu_sample_scale(workload):
    """Grid of the bounded CPU sample (about 10-30 s of host work for 3 steps)."""
    return 64 if WORKLOADS[workload][1] == 3 else 512


def _refrun():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import refrun
    return refrun


def reference_build_rate(workload, sample_scale, steps, cores, warmup=0):
    """The reference's own CPU code, timed: its src/ compiled unchanged against the
    host stand-ins of oracle/refshim (OpenMP over cells), one process per run.
    Seconds per accepted step = (wall time of a run of `steps` steps - wall time of
    a run of 0 steps) / steps: both runs pay the same set-up (weights, initial
    condition, FSAL priming evaluation) and write no files.  Returns
    (zone-updates/s, seconds per step) or None where no build exists."""
    refrun = _refrun()
    if refrun.binary(workload) is None:
        return None
    cfg, _ = abi.workload(workload, scale=sample_scale, steps=steps)
    if warmup:
        refrun.run(workload, cfg, warmup, threads=cores, ckpt=False)
    sec = refrun.time_steps(workload, cfg, steps, threads=cores)
    return abi.ncells(cfg) / sec, sec


def oracle_rate(workload, sample_scale, steps, cores, warmup=0):
    """The oracle (this repository's CPU restatement of the path, OpenMP over cells)."""
    oracle = _oracle()
    oracle.set_threads(cores)
    cfg, ic = abi.workload(workload, scale=sample_scale, steps=steps + warmup + 2)
    s = oracle.OracleSolver(cfg)
    s.init_ic(ic)
    for _ in range(warmup):
        s.take_step()
    t0 = time.perf_counter()
    acc = 0
    for _ in range(steps):
        acc += s.take_step().accepted
    dt = time.perf_counter() - t0
    return acc * abi.ncells(cfg) / dt, dt / max(steps, 1)


def cpu_rate(workload, sample_scale, steps, cores, warmup=0):
    """(value, seconds per step, kind, what): the reference build where it exists
    (kind "reference"), else the oracle port (kind "port")."""
    dim = WORKLOADS[workload][1]
    r = reference_build_rate(workload, sample_scale, steps, cores, warmup)
    if r is not None:
        return r[0], r[1], "reference", (
            f"the reference's own CPU code (its src/ compiled unchanged against host-only Kokkos/MPI/PDI "
            f"stand-ins, OpenMP on {cores} threads), {steps} accepted steps of the same problem on a "
            f"{sample_scale}^{dim} grid, stepping loop only (run of {steps} steps minus run of 0 steps)")
    v, sec = oracle_rate(workload, sample_scale, steps, cores, warmup)
    return v, sec, "port", (
        f"the oracle (CPU restatement of the reference path, OpenMP on {cores} threads; no reference build "
        f"present), {steps} accepted steps of the same problem on a {sample_scale}^{dim} grid")


def cpu_baseline(workload, sample_scale, sample_steps=3):
    """The reference's CPU code timed on the host cores on a bounded sample of the workload."""
    cores = os.cpu_count() or 1
    v, sec, kind, what = cpu_rate(workload, sample_scale, sample_steps, cores)
    return {"value": v, "unit": UNIT, "cores": cores, "cpu": cpu_model(), "kind": kind, "sample": what}


def run_reference(args):
    ws, rank, local = dist_init()
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    sample = cpu_sample_scale(args.workload)
    dim = WORKLOADS[args.workload][1]
    value, sec, kind, what = cpu_rate(args.workload, sample, args.steps, cores, warmup=args.warmup)
    out = {"impl": "reference", "metric": metric_name(args.workload, args.scale), "value": value, "unit": UNIT,
           "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic (analytic initial condition)",
           "config": config_block(args.workload, args.scale, {"sample_grid": [sample] * dim}),
           "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "cpu": cpu_model(), "kind": kind,
                            "sample": "each step: " + what},
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
