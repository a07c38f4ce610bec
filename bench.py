#!/usr/bin/env python
"""Headline benchmark: Gcell-updates/s of the split finite-volume update.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload euler4096]

A step is one full time step (x sweep + y sweep + wave-speed reduction + dt)
over the whole grid of the workload.  The default workload is the 4096 x 4096
Euler shock/bubble problem (gamma 1.4, 32 seeded bubbles, Mach-2 shock,
reflective top/bottom, transmissive left/right, CFL 0.8) in the plain FP64
form, which matches the reference to the bit.  Its state (537 MB per buffer)
is larger than the 126 MB L2, so no flush is needed between steps.

value      device-resident throughput, CUDA events on the solver's stream,
           max over ranks (N>1 runs independent replicas: the single grid is
           not sharded; scaling "weak").
e2e        the same metric through the C ABI with host buffers: upload of the
           initial grid from pinned memory, the reference-shaped host loop
           (compute_dt -> step per step, a device->host read of the wave speeds
           each step), download of the final grid to pinned memory.
roofline   dominant sweep kernel: algorithmic bytes (nx*ny*nvar*8 read + write)
           over its mean CUDA-event duration, against MEASURED_PEAKS.json.
cpu_baseline  the reference's own CPU code (oracle/_ref, all host threads) on a
           1024x1024 instance of the same workload for a bounded number of steps.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import re
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "cfd-art_b200"))

METRIC = "Gcell-updates/s + p50/p99 latency: served mixed vs plain FP64, L1 err ≤1e-4"
UNIT = "Gcell-updates/s"
SEED = 20261203

WORKLOADS = {
    # name: (recipe, nx, ny, nbubbles)
    "euler4096": ("shock_bubbles", 4096, 4096, 32),
    "euler2048": ("shock_bubbles", 2048, 2048, 32),  # smaller case for ncu captures
}


def _peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def _profile_traffic(kernel: str) -> float | None:
    """DRAM bytes per launch of `kernel` from the committed ncu summary."""
    for f in sorted((ROOT / "profiles").glob("*.md")):
        m = re.search(rf"traffic_bytes_per_launch\[{re.escape(kernel)}\]\s*[:=]\s*([0-9.eE+]+)",
                      f.read_text())
        if m:
            return float(m.group(1))
    return None


class ClockSampler:
    """nvidia-smi sampling of SM clock and throttle reasons during a region."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_id: str | None):
        self.dev = device_id
        self.rows: list[list[str]] = []
        self.proc = None
        self.thread = None

    def start(self):
        cmd = ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms", "200"]
        if self.dev:
            cmd += ["-i", self.dev]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                                         text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self) -> dict:
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread:
            self.thread.join(timeout=5)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            if len(r) < 7:
                continue
            try:
                sm.append(float(r[0]))
                mx = float(r[1])
            except ValueError:
                continue
            for k, name in enumerate(names):
                if r[3 + k].lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def _gpu_id(torch, dev: int) -> str | None:
    try:
        u = str(torch.cuda.get_device_properties(dev).uuid)
        return u if u.startswith("GPU-") else "GPU-" + u
    except Exception:
        return None


def cpu_baseline(recipe: str, nbub: int, budget_s: float = 15.0) -> dict:
    """The reference's own CPU path (oracle/_ref, all host threads) on a
    1024 x 1024 instance of the workload, steps bounded to ~budget_s."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import cfdgpu as G
    import oracle_py as O

    if not O.ref_available("euler"):
        return {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                "sample": "unavailable: oracle/_ref/libref_euler.so not built"}
    cores = os.cpu_count() or 1
    n = 1024
    cfg = G.recipe_config(recipe, n, n)
    ic = G.recipe_ic(cfg, recipe, seed=SEED, nbubbles=nbub)
    p = O.make_params(n, n, cfg.dx, cfg.dy, cfg.gamma1, cfg.pinf1, bc=tuple(cfg.bc), cfl=cfg.cfl,
                      T=cfg.T, limiter=cfg.limiter)
    lib = O.ref_lib("euler")
    lib.ref_euler_last_loop_seconds.restype = __import__("ctypes").c_double
    g = ic.copy()
    O.ref_run("euler", p, g, 1, threads=cores)  # first step: calibrate
    t1 = lib.ref_euler_last_loop_seconds()
    steps = max(2, min(50, int(budget_s / max(t1, 1e-3))))
    taken, nn, tt, _ = O.ref_run("euler", p, g, steps, n=1, t=0.0, threads=cores)
    sec = lib.ref_euler_last_loop_seconds()
    val = n * n * taken / sec / 1e9
    return {"value": val, "unit": UNIT, "cores": cores, "kind": "reference",
            "sample": f"{n}x{n} shock-bubble grid (same recipe), {taken} steps, "
                      f"{cores} OpenMP threads, time loop only ({sec:.1f} s)"}


def run_reference(args) -> None:
    """Reference arm: the reference's CPU implementation on a bounded sample
    of the workload (512 x 512 instance, one time step per step)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle_py as O

    recipe, nx, ny, nbub = WORKLOADS[args.workload]
    base = {"impl": "reference", "metric": METRIC, "unit": UNIT}
    if not O.ref_available("euler"):
        print(json.dumps({**base, "unavailable": "oracle/_ref/libref_euler.so (reference build) absent"}))
        return
    import ctypes

    import cfdgpu as G

    cores = os.cpu_count() or 1
    n = 512
    cfg = G.recipe_config(recipe, n, n)
    ic = G.recipe_ic(cfg, recipe, seed=SEED, nbubbles=nbub)
    p = O.make_params(n, n, cfg.dx, cfg.dy, cfg.gamma1, cfg.pinf1, bc=tuple(cfg.bc), cfl=cfg.cfl,
                      T=cfg.T, limiter=cfg.limiter)
    lib = O.ref_lib("euler")
    lib.ref_euler_last_loop_seconds.restype = ctypes.c_double
    g = ic.copy()
    if args.warmup:
        O.ref_run("euler", p, g, args.warmup, threads=cores)
    taken, nn, tt, _ = O.ref_run("euler", p, g, args.steps, n=args.warmup, t=0.0, threads=cores)
    sec = lib.ref_euler_last_loop_seconds()
    val = n * n * taken / sec / 1e9
    sample = (f"{n}x{n} instance of the {nx}x{ny} shock-bubble workload, one time step per step, "
              f"{cores} OpenMP threads")
    print(json.dumps({
        **base, "value": val, "n_gpus": args.gpus, "steps": taken, "warmup": args.warmup,
        "ms_per_step": 1e3 * sec / max(taken, 1), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "grid": [n, n], "model": "euler",
                   "precision": "fp64", "sample_of": [nx, ny]},
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def end_to_end(G, torch, cfg, ic, K, W, barrier, max_over_ranks, world, cells) -> dict:
    """Same metric through the C ABI with host buffers: upload from pinned
    memory, the reference-shaped host loop (compute_dt -> step), download."""
    pinned_ic = torch.empty(ic.size, dtype=torch.float64, pin_memory=True)
    pinned_ic.numpy()[:] = ic.ravel()
    ic_pinned = pinned_ic.numpy().reshape(ic.shape)
    pinned_out = torch.empty(ic.size, dtype=torch.float64, pin_memory=True)
    out_pinned = pinned_out.numpy().reshape(ic.shape)
    s2 = G.Solver(cfg)
    s2.upload(ic_pinned)
    s2.run_reference_loop(W)
    s2.download(out=out_pinned)
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    s2.upload(ic_pinned)
    taken, n2, t2 = s2.run_reference_loop(K)
    s2.download(out=out_pinned)
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    s2.close()
    state_bytes = ic.size * 8
    status_bytes = 96  # DevState read by compute_dt
    return {"value": world * cells * taken / e2e_s / 1e9, "unit": UNIT,
            "h2d_bytes_per_step": state_bytes / K,
            "d2h_bytes_per_step": status_bytes + state_bytes / K, "seconds": e2e_s}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="euler4096", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end pass (profiling)")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
        return

    import torch
    import torch.distributed as dist

    import cfdgpu as G

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    recipe, nx, ny, nbub = WORKLOADS[args.workload]
    cfg = G.recipe_config(recipe, nx, ny)
    ic = G.recipe_ic(cfg, recipe, seed=SEED + rank, nbubbles=nbub)
    stream = torch.cuda.Stream()  # a real stream: the library must not fall back to its own
    torch.cuda.set_stream(stream)
    cfg.stream = stream.cuda_stream
    cells = nx * ny
    nv = cfg.nvar
    K, W = args.steps, args.warmup

    # ---- device-resident throughput --------------------------------------
    s = G.Solver(cfg)
    s.upload(ic)
    s.advance(W)
    s.synchronize()
    s.set_kernel_timing(True)
    s.reset_kernel_times()
    clocks = ClockSampler(_gpu_id(torch, local))
    clocks.start()
    time.sleep(0.3)
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    s.advance(K)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    ck = clocks.stop()
    ms = e0.elapsed_time(e1)
    kms, kn = s.kernel_times()
    st = s.status()
    s.set_kernel_timing(False)
    ms_max = max_over_ranks(ms)
    value = world * cells * K / (ms_max / 1e3) / 1e9

    # ---- roofline of the dominant sweep ----------------------------------
    peak, peak_kind = _peaks()
    dom = 0 if kms[0] >= kms[1] else 1
    kname = ["sweep_x", "sweep_y"][dom]
    avg_s = kms[dom] / max(kn[dom], 1) / 1e3
    bytes_launch = cells * nv * 8 * 2
    achieved = bytes_launch / avg_s / 1e9
    traffic = _profile_traffic(f"euler_{kname}")

    # ---- end to end through the C ABI with host buffers ------------------
    e2e = None
    if not args.no_e2e:
        e2e = end_to_end(G, torch, cfg, ic, K, W, barrier, max_over_ranks, world, cells)
    s.close()
    
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(recipe, nbub)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K,
            "warmup": W, "ms_per_step": ms_max / K, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": args.workload, "model": "euler", "precision": "fp64 (plain)",
                       "grid": [nx, ny], "bubbles": nbub, "seed": SEED, "cfl": cfg.cfl,
                       "limiter": "minmod", "flux": "MUSCL-Hancock + HLLC",
                       "splitting": "naive", "l2": "state 537 MB/buffer > 126 MB L2, no flush",
                       "parallelism": f"replicas x{world}"},
            "clocks": ck,
            "gpu_launches": int(kn[0] + kn[1]),
            "roofline": {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic,
                         "algorithmic_bytes_per_launch": bytes_launch,
                         "mean_launch_ms": [kms[0] / max(kn[0], 1), kms[1] / max(kn[1], 1)]},
            "e2e": e2e,
            "cpu_baseline": cpu,
            "sim": {"n": st.n, "t": st.t, "counters": st.counter_dict()},
        }
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
