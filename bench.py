#!/usr/bin/env python
"""Headline benchmark: Gcell-updates/s of the split finite-volume update.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload served|batch256|euler4096[_mixed]|allaire2048[_mixed]|...]

Default workload ("served", the configuration the headline metric is quoted
on): a seeded Poisson stream (mean 50 requests/s) of solves, 70 % Euler
(shock + bubbles recipe) and 30 % Allaire two-material (water shock on an air
bubble, PVRS speeds, alpha clipped to [1e-6, 1-1e-6]), cells log-uniform in
[128^2, 2048^2], steps uniform in [100, 2000], admitted against 80 % of the
free HBM.  K = --steps requests are timed after W = --warmup requests.

  value      device-resident throughput of the mixed form on that request
             set: every request resident in one batch, each advancing to its
             own step count (CUDA events on the batch's stream).
  e2e        the served run through the C ABI: requests submitted from host
             buffers at their arrival times, continuous batching, results back
             in host memory; cell-updates of all requests / makespan.  p50/p99
             completion latency come from this run.
  plain_fp64 the same served run in the plain FP64 form at its best: fast
             FP64 members of one batch (relative L1 density error against
             the bit-identical form stated beside it), for the "mixed vs
             plain" ratio; plain_fp64_bit_exact the same run in the
             bit-identical form (one solver per request).  l1_vs_fp64 and
             linf_vs_fp64 are the largest (and median) relative L1 and L-inf
             density errors of a mixed result against its bit-identical FP64
             result.
  roofline   the dominant mixed sweep kernel on a resident sample of the
             requests: algorithmic bytes (cells x nvar x (4+4) B read + write)
             over its mean CUDA-event launch time, against MEASURED_PEAKS.json.

Other workloads are the single-grid and batched configurations: euler4096
(4096^2 shock/bubbles, K steps timed), allaire2048 (2048x1024 water shock),
each in the bit-identical FP64 form, with _fast (the fast FP64 form) or with
_mixed, and batch256 (256 uneven Euler instances, 64..1024 per side, 500
steps each).
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

# single-grid workloads: (recipe, nx, ny, nbubbles, precision)
SINGLE = {
    "euler4096": ("shock_bubbles", 4096, 4096, 32, "fp64"),
    "euler4096_mixed": ("shock_bubbles", 4096, 4096, 32, "mixed"),
    "euler2048": ("shock_bubbles", 2048, 2048, 32, "fp64"),
    "euler2048_mixed": ("shock_bubbles", 2048, 2048, 32, "mixed"),
    "euler2048_fast": ("shock_bubbles", 2048, 2048, 32, "fp64_fast"),
    "euler4096_fast": ("shock_bubbles", 4096, 4096, 32, "fp64_fast"),
    "allaire2048": ("water_shock_air_bubble", 2048, 1024, 1, "fp64"),
    "allaire2048_fast": ("water_shock_air_bubble", 2048, 1024, 1, "fp64_fast"),
    "allaire2048_mixed": ("water_shock_air_bubble", 2048, 1024, 1, "mixed"),
    "allaire1024_mixed": ("water_shock_air_bubble", 1024, 512, 1, "mixed"),
}
WORKLOADS = ["served", "batch256", *SINGLE]


# ----------------------------------------------------------------- helpers --

def _peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def _profile_traffic(kernel: str) -> float | None:
    """DRAM bytes per launch of `kernel` from the committed ncu summaries."""
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


def _interior_density(a: np.ndarray, model: int) -> np.ndarray:
    return a[2:-2, 2:-2, 0] if model == 0 else a[2:-2, 2:-2, 0] + a[2:-2, 2:-2, 1]


def _rel_l1_density(a: np.ndarray, b: np.ndarray, model: int) -> float:
    ra, rb = _interior_density(a, model), _interior_density(b, model)
    return float(np.abs(ra - rb).sum() / np.abs(rb).sum())


def _rel_linf_density(a: np.ndarray, b: np.ndarray, model: int) -> float:
    """max |rho_a - rho_b| / max |rho_b| over the interior cells."""
    ra, rb = _interior_density(a, model), _interior_density(b, model)
    return float(np.abs(ra - rb).max() / np.abs(rb).max())


def _errors(a: np.ndarray, b: np.ndarray, model: int) -> tuple[float, float]:
    return _rel_l1_density(a, b, model), _rel_linf_density(a, b, model)


def _error_summary(pairs, basis: str) -> dict:
    """Relative L1 and L-inf density errors of a set of results: largest and
    median, with what they were measured against."""
    l1 = [a for a, _ in pairs]
    li = [b for _, b in pairs]
    return {"l1": {"max": max(l1), "median": float(np.median(l1)), "bound": 1e-4},
            "linf": {"max": max(li), "median": float(np.median(li))}, "results": len(pairs),
            "basis": basis}


# ------------------------------------------------------- request streams --

def served_requests(n: int, seed: int):
    """The served mix: (arrival_s, recipe, nx, ny, steps, seed, nbubbles)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for k in range(n):
        t += rng.exponential(1.0 / 50.0)
        euler = rng.uniform() < 0.7
        cells = math.exp(rng.uniform(math.log(128 ** 2), math.log(2048 ** 2)))
        steps = int(rng.integers(100, 2001))
        if euler:
            nx = ny = max(16, int(round(math.sqrt(cells))))
            out.append((t, "shock_bubbles", nx, ny, steps, seed + k, int(rng.integers(4, 33))))
        else:
            ny = max(16, int(round(math.sqrt(cells / 2))))
            out.append((t, "water_shock_air_bubble", 2 * ny, ny, steps, seed + k, 1))
    return out


# The batched instances take the y sweep's MUSCL-Hancock half step on dy.
# Their cells are up to 16 times longer one way than the other, and the
# reference's half step on dx in the y sweep (E/sourcecode/euler_colsweep.cpp:43)
# makes those runs ill-conditioned where dx is several times dy: round-off
# grows until even two FP64 forms of the same scheme (bit-identical and fast)
# differ by a few per cent after 500 steps, while with the dy half step
# every form agrees with the others to about 1e-6.  Every other workload has
# square cells, where the two half steps are the same.
BATCH_FIX_DY = 1


def batch_instances(n: int, seed: int):
    """Batched config: Euler instances with nx, ny log-uniform in [64, 1024]
    and 4-16 bubbles each, 500 steps."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        nx = int(round(math.exp(rng.uniform(math.log(64), math.log(1024)))))
        ny = int(round(math.exp(rng.uniform(math.log(64), math.log(1024)))))
        out.append(("shock_bubbles", nx, ny, 500, seed + k, int(rng.integers(4, 17))))
    return out


def build_ic(G, recipe, nx, ny, seed, nbub):
    cfg = G.recipe_config(recipe, nx, ny)
    return cfg, G.recipe_ic(cfg, recipe, seed=seed, nbubbles=nbub)


# ------------------------------------------------------------ CPU baseline --

def _host_threads() -> int:
    """Host CPUs this process may run on (its affinity mask, which a container
    or a scheduler may narrow below the machine's count)."""
    try:
        return max(1, len(os.sched_getaffinity(0)))
    except (AttributeError, OSError):
        return os.cpu_count() or 1


def _cpu_model() -> str:
    """The host CPU's model name (first entry of /proc/cpuinfo)."""
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform

    return platform.processor() or "unknown"


# Cell-updates per reference-arm unit: a request or instance runs at most
# this many cell-updates (its own step count, truncated), so one unit takes
# a few seconds of host time.
REF_UNIT_CELLS = {"euler": 1.6e7, "allaire": 6e6}


def reference_units(workload: str, count: int):
    """The workload's units as the reference's CPU code runs them:
    (recipe, nx, ny, seed, nbubbles, steps, fix_dy_halfstep).  served: the
    repo arm's request stream (same seeds; warm-up requests first);
    batch256: its instances; single-grid workloads: the grid itself,
    `steps` = 1 per unit."""
    if workload == "served":
        return [(rec, nx, ny, sd, nb, steps, 0)
                for (_, rec, nx, ny, steps, sd, nb) in served_requests(count, SEED)]
    if workload == "batch256":
        return [(r, nx, ny, sd, nb, steps, BATCH_FIX_DY)
                for r, nx, ny, steps, sd, nb in batch_instances(256, SEED)][:count]
    recipe, nx, ny, nbub, _prec = SINGLE[workload]
    return [(recipe, nx, ny, SEED, nbub, 1, 0)]


class RefRunner:
    """The reference's own CPU implementation of the path (oracle/_ref: its
    sources built here) driven through its time loop on grids that the
    CPU-side recipe builder makes (oracle/oracle_recipes.c), so the shipped
    library is never loaded on this arm.  Returns cell-updates and the loop's
    own seconds (the reference's omp_get_wtime around the loop)."""

    def __init__(self, threads: int):
        import ctypes

        sys.path.insert(0, str(ROOT / "oracle"))
        import oracle_py as O

        self.O, self.threads = O, threads
        self.secs = {}
        for model in ("euler", "allaire"):
            f = getattr(O.ref_lib(model), f"ref_{model}_last_loop_seconds")
            f.restype = ctypes.c_double
            self.secs[model] = f

    def unit(self, recipe, nx, ny, seed, nb, steps, fix_dy=0, cap=True):
        grid, p, model = self.O.port_recipe_ic(recipe, nx, ny, seed, nb)
        p.fix_dy_halfstep = fix_dy
        if cap:
            steps = max(2, min(steps, int(REF_UNIT_CELLS[model] // (nx * ny))))
        taken, _, _, _ = self.O.ref_run(model, p, grid, steps, threads=self.threads)
        return nx * ny * taken, self.secs[model](), taken, model

    def grid_steps(self, recipe, nx, ny, seed, nb, warm, steps):
        """Single-grid workloads: `warm` steps, then `steps` timed ones, one
        timing per step."""
        grid, p, model = self.O.port_recipe_ic(recipe, nx, ny, seed, nb)
        if warm:
            self.O.ref_run(model, p, grid, warm, threads=self.threads)
        out, n = [], warm
        for _ in range(steps):
            taken, n, _, _ = self.O.ref_run(model, p, grid, 1, n=n, threads=self.threads)
            out.append((nx * ny * taken, self.secs[model]()))
        return out


def _ref_available() -> bool:
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle_py as O

    return O.ref_available("euler") and O.ref_available("allaire") and O.port_available()


def cpu_baseline(workload: str, budget_s: float = 16.0, single_thread_s: float = 5.0) -> dict:
    """The reference's own CPU code (oracle/_ref, all host threads) on a
    bounded sample of the workload's units, plus a one-thread run
    (`single_thread`, deterministic: with more threads the reference's
    compute_dt races on its maxima) on units cut to a quarter of the size."""
    if not _ref_available():
        return {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                "sample": "unavailable: oracle/_ref (reference build) absent"}
    cores = _host_threads()
    out = {}
    for threads, budget, shrink in ((cores, budget_s, 1), (1, single_thread_s, 4)):
        R = RefRunner(threads)
        cells = secs = 0.0
        units = taken_steps = 0
        for (rec, nx, ny, sd, nb, steps, fix) in reference_units(workload, 64):
            nx, ny = max(16, nx // shrink), max(16, ny // shrink)
            if workload in SINGLE:
                c, s, k, _ = R.unit(rec, nx, ny, sd, nb, 1 << 30, fix)
            else:
                c, s, k, _ = R.unit(rec, nx, ny, sd, nb, steps, fix)
            cells += c
            secs += s
            units += 1
            taken_steps += k
            if secs >= budget:
                break
        what = ("requests" if workload == "served" else
                "instances" if workload == "batch256" else "grid runs")
        desc = (f"first {units} {what} of the {workload} workload"
                + (f" at 1/{shrink} size per side" if shrink > 1 else "")
                + f", each truncated to <= {REF_UNIT_CELLS['euler']:.2g} (Euler) / "
                  f"{REF_UNIT_CELLS['allaire']:.2g} (Allaire) cell-updates, {taken_steps} steps "
                  f"in all ({threads} OpenMP thread{'s' if threads > 1 else ''}, time loop only, "
                  f"{secs:.1f} s)")
        rec = {"value": cells / secs / 1e9, "unit": UNIT, "cores": threads, "sample": desc}
        if threads == cores:
            out = {**rec, "kind": "reference", "cpu_model": _cpu_model()}
        else:
            out["single_thread"] = rec
    return out


def run_reference(args) -> None:
    """Reference arm: the reference's CPU implementation (oracle/_ref: its
    own sources built here) with all host threads, on the repo arm's
    workload, with the shipped library never loaded.  One bench step is one
    unit of the workload: served, a request of the same seeded stream (its
    own step count, truncated to a few seconds of host work); batch256, an
    instance; single-grid workloads, one time step of the full grid."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    base = {"impl": "reference", "metric": METRIC, "unit": UNIT}
    if not _ref_available():
        print(json.dumps({**base, "unavailable": "oracle/_ref (reference build) absent"}))
        return
    cores = _host_threads()
    R = RefRunner(cores)
    w, K, W = args.workload, args.steps, args.warmup
    cells = secs = 0.0
    if w in SINGLE:
        rec, nx, ny, sd, nb, _, _ = reference_units(w, 1)[0]
        for c, s in R.grid_steps(rec, nx, ny, sd, nb, W, K):
            cells += c
            secs += s
        sample = f"{rec} {nx}x{ny}: {W} warm-up steps, then {K} timed steps"
    else:
        units = reference_units(w, W + K)
        for u in units[:W]:
            R.unit(*u)
        taken_steps = 0
        for u in units[W:W + K]:
            c, s, k, _ = R.unit(*u)
            cells += c
            secs += s
            taken_steps += k
        sample = (f"{'requests' if w == 'served' else 'instances'} {W + 1}-{W + K} of the "
                  f"{w} workload's seeded list (after {W} warm-up ones), each run from its "
                  f"initial grid for its own step count truncated to <= "
                  f"{REF_UNIT_CELLS['euler']:.2g} (Euler) / {REF_UNIT_CELLS['allaire']:.2g} "
                  f"(Allaire) cell-updates: {taken_steps} steps in all")
    val = cells / secs / 1e9
    sample += f"; {cores} OpenMP threads, the reference's time loop only ({secs:.1f} s)"
    print(json.dumps({
        **base, "value": val, "n_gpus": args.gpus, "steps": K, "warmup": W,
        "ms_per_step": 1e3 * secs / max(K, 1), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": w, "step": "one request" if w == "served" else
                   "one instance" if w == "batch256" else "one time step", "sample": sample},
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": cores, "kind": "reference",
                         "cpu_model": _cpu_model(), "sample": sample},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


# ---------------------------------------------------------------- GPU arms --

class Ctx:
    """Ranks of one job: barrier, and max / sum over ranks (one process per
    GPU, NCCL; the tests run the same code on CPU ranks over gloo)."""

    def __init__(self, torch, dist, world, rank, local, device="cuda"):
        self.torch, self.dist, self.world, self.rank, self.local = torch, dist, world, rank, local
        self.device = device

    def barrier(self):
        if self.world > 1:
            self.dist.barrier()

    def max(self, x: float) -> float:
        if self.world == 1:
            return x
        t = self.torch.tensor([x], device=self.device, dtype=self.torch.float64)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x: float) -> float:
        if self.world == 1:
            return x
        t = self.torch.tensor([x], device=self.device, dtype=self.torch.float64)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return float(t.item())


def job_throughput(ctx, cell_updates: float, ms: float) -> float:
    """Whole-job Gcell-updates/s of N replicas: the updates of all ranks over
    the slowest rank's device time."""
    return ctx.sum(cell_updates) / (ctx.max(ms) / 1e3) / 1e9


def roofline(kernel: str, ms: float, launches: int, bytes_per_launch: float, traffic_key: str):
    peak, kind = _peaks()
    avg_s = ms / max(launches, 1) / 1e3
    achieved = bytes_per_launch / avg_s / 1e9 if avg_s > 0 else 0.0
    return {"bound": "hbm", "kernel": kernel, "achieved": achieved, "peak": peak,
            "peak_kind": kind, "unit": "GB/s", "frac": achieved / peak,
            "traffic": _profile_traffic(traffic_key),
            "algorithmic_bytes_per_launch": bytes_per_launch, "mean_launch_ms": avg_s * 1e3}


def bench_single(args, ctx, G, stream, clocks):
    torch = ctx.torch
    recipe, nx, ny, nbub, prec = SINGLE[args.workload]
    cfg, ic = build_ic(G, recipe, nx, ny, SEED + ctx.rank, nbub)
    cfg.stream = stream.cuda_stream
    if prec == "fp64_fast":
        cfg.precision = G.FP64_FAST  # a batch member of the fast FP64 form
    cells, nv, K, W = nx * ny, cfg.nvar, args.steps, args.warmup
    model = "euler" if cfg.model == G.EULER else "allaire"
    if prec == "fp64":
        s = G.Solver(cfg)
        s.upload(ic)
        s.advance(W)
        s.synchronize()
        s.set_kernel_timing(True)
        s.reset_kernel_times()
        run = lambda: s.advance(K)
    else:
        s = G.Batch(stream=stream.cuda_stream)
        mid = s.add(cfg, ic, 0)
        s.autotune(1)
        s.step(max(W, 8))  # at least one CUDA-graph replay: the graph is captured here
        torch.cuda.synchronize()
        run = lambda: s.step(K)
    clocks.start()
    time.sleep(0.3)
    ctx.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    run()
    e1.record(stream)
    torch.cuda.synchronize()
    ctx.barrier()
    ck = clocks.stop()
    ms = ctx.max(e0.elapsed_time(e1))
    if prec == "fp64":
        kms, kn = s.kernel_times()
        st = s.status()
        launches = kn[0] + kn[1]
        dom = 0 if kms[0] >= kms[1] else 1
        rl = roofline(["sweep_x", "sweep_y"][dom], kms[dom], kn[dom], cells * nv * 8 * 2,
                      f"{model}_sweep_{'xy'[dom]}_{nx}")
    else:
        mx, my, n = s.step_timed(4)
        st = s.status(mid)
        launches = 2 * K
        dom = 0 if mx >= my else 1
        kname = "fast_sweep" if prec == "fp64_fast" else "mixed_sweep"
        rl = roofline([f"{kname}_x", f"{kname}_y"][dom], [mx, my][dom], 4,
                      cells * nv * 8 * 2, f"{model}_{kname}_{'xy'[dom]}_{nx}")
    s.close()
    e2e = None
    if not args.no_e2e:
        e2e = e2e_single(G, torch, cfg, ic, K, W, ctx, prec)
    acc = None
    if prec != "fp64" and not args.no_accuracy:
        acc = accuracy_single(G, cfg, ic, STATED_STEPS.get(recipe, K))
    value = job_throughput(ctx, cells * K, ms)
    config = {"workload": args.workload, "model": model, "precision": prec, "grid": [nx, ny],
              "bubbles": nbub, "seed": SEED, "cfl": cfg.cfl,
              "l2": f"state {cells * nv * 8 / 1e6:.0f} MB per buffer vs 126 MB L2"
                    + (", no flush" if cells * nv * 8 > 126e6 else ""),
              "parallelism": f"replicas x{ctx.world}"}
    return {"value": value, "ms_per_step": ms / K,
            "dtype": "f32+f32comp" if prec == "mixed" else "f64", "config": config, "clocks": ck,
            "gpu_launches": launches, "roofline": rl, "e2e": e2e, "sim": {"n": st.n, "t": st.t},
            **({"accuracy_vs_fp64": acc} if acc else
               {"accuracy_vs_fp64": {"l1": {"max": 0.0}, "linf": {"max": 0.0},
                                     "basis": "bit-identical to the oracle and the reference "
                                              "build (tests/test_gpu_parity.py)"}}
               if prec == "fp64" else {})}


# the stated step counts of the benchmarked configurations
STATED_STEPS = {"shock_bubbles": 2000, "water_shock_air_bubble": 1500}


def accuracy_single(G, cfg, ic, steps) -> dict:
    """A batch form (mixed or fast FP64, cfg.precision) vs the bit-identical
    FP64 form (= the reference) on the bench's grid over the configuration's
    stated step count, outside the timed region."""
    plain = cfg.copy()
    plain.precision = G.FP64
    with G.Solver(plain) as s:
        s.upload(ic)
        s.advance(steps)
        ref = s.download()
    with G.Batch(stream=cfg.stream) as b:
        i = b.add(cfg, ic, steps)
        b.step(steps)
        out = b.download(i)
        n = b.status(i).n
    acc = _error_summary([_errors(out, ref, cfg.model)],
                         "plain FP64 form, bit-identical to the reference")
    if cfg.precision == G.FP64_FAST:
        acc["l1"]["bound"] = 1e-12  # the plain form's bound
    return {**acc, "steps": n}


def e2e_single(G, torch, cfg, ic, K, W, ctx, prec) -> dict:
    """Same metric through the C ABI with pinned host buffers: upload, K
    steps (FP64: the reference-shaped compute_dt -> step loop), download."""
    pin_in = torch.empty(ic.size, dtype=torch.float64, pin_memory=True).numpy().reshape(ic.shape)
    pin_in[:] = ic
    pin_out = torch.empty(ic.size, dtype=torch.float64, pin_memory=True).numpy().reshape(ic.shape)

    def run(steps):
        if prec == "fp64":
            s = G.Solver(cfg)
            s.upload(pin_in)
            taken, _, _ = s.run_reference_loop(steps)
            s.download(out=pin_out)
        else:
            s = G.Batch(stream=cfg.stream)
            mid = s.add(cfg, pin_in, 0)
            s.step(steps)
            s.download(mid, out=pin_out)
            taken = steps
        return s, taken

    # one untimed pass first (W steps): loads the conversion kernels and
    # warms the device pool, as the warm-up steps do for the device timing
    s, _ = run(max(W, 1))
    torch.cuda.synchronize()
    s.close()
    ctx.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    s, taken = run(K)
    torch.cuda.synchronize()
    secs = ctx.max(time.perf_counter() - t0)
    s.close()
    d2h_step = 96 if prec == "fp64" else 0
    cells = cfg.nx * cfg.ny
    return {"value": ctx.world * cells * taken / secs / 1e9, "unit": UNIT,
            "h2d_bytes_per_step": ic.size * 8 / K, "d2h_bytes_per_step": d2h_step + ic.size * 8 / K,
            "seconds": secs}


def bench_batch(args, ctx, G, stream, clocks):
    torch = ctx.torch
    insts = batch_instances(256, SEED + 1000 * ctx.rank)
    ics = [build_ic(G, r, nx, ny, sd, nb) for r, nx, ny, steps, sd, nb in insts]
    for c, _ in ics:
        c.fix_dy_halfstep = BATCH_FIX_DY
    cells = sum(c.nx * c.ny for c, _ in ics)
    K, W = args.steps, args.warmup
    b = G.Batch(stream=stream.cuda_stream)
    for (c, ic), inst in zip(ics, insts):
        b.add(c, ic, inst[3])
    tune_ms = b.autotune(1)
    pre = {i: s for i, s, _, _ in b.poll()}
    b.step(max(W, 8))  # at least one CUDA-graph replay: the graph is captured here
    torch.cuda.synchronize()
    clocks.start()
    time.sleep(0.3)
    ctx.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start = {i: s for i, s, _, _ in b.poll()}
    e0.record(stream)
    b.step(K)
    e1.record(stream)
    torch.cuda.synchronize()
    ctx.barrier()
    ck = clocks.stop()
    ms = ctx.max(e0.elapsed_time(e1))
    end = {i: s for i, s, _, _ in b.poll()}
    upd = sum(b.cfgs[i].nx * b.cfgs[i].ny * (end[i] - start[i]) for i in end)
    mx, my, n = b.step_timed(4)
    dom = 0 if mx >= my else 1
    rl = roofline(["mixed_sweep_x", "mixed_sweep_y"][dom], [mx, my][dom], 4, cells * 4 * 8 * 2,
                  f"batch_mixed_sweep_{'xy'[dom]}")
    shapes = b.get_shapes(0)
    b.close()
    value = job_throughput(ctx, upd, ms)
    e2e = None
    if not args.no_e2e:
        # pinned host buffers: the initial grids and the results
        pins = []
        for _, ic in ics:
            a = torch.empty(ic.size, dtype=torch.float64, pin_memory=True).numpy().reshape(ic.shape)
            a[:] = ic
            pins.append(a)
        outs = [torch.empty(ic.size, dtype=torch.float64, pin_memory=True).numpy().reshape(ic.shape)
                for _, ic in ics]
        ctx.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        b2 = G.Batch(stream=stream.cuda_stream)
        ids = [b2.add(c, a, inst[3]) for (c, _), a, inst in zip(ics, pins, insts)]
        b2.step(K)
        for i, o in zip(ids, outs):
            b2.download(i, out=o)
        torch.cuda.synchronize()
        secs = ctx.max(time.perf_counter() - t0)
        b2.close()
        upd2 = sum(c.nx * c.ny * min(i[3], K) for (c, _), i in zip(ics, insts))
        nbytes = sum(ic.size * 8 for _, ic in ics)
        e2e = {"value": ctx.sum(upd2) / secs / 1e9, "unit": UNIT,
               "h2d_bytes_per_step": nbytes / K, "d2h_bytes_per_step": nbytes / K, "seconds": secs}
        del outs, pins
    acc = None
    if not args.no_accuracy:
        # every instance to its 500 steps, mixed vs plain FP64
        outs = {}
        with G.Batch(stream=stream.cuda_stream) as b3:
            ids = [b3.add(c, ic, inst[3]) for (c, ic), inst in zip(ics, insts)]
            b3.step(max(i[3] for i in insts))
            for k, i in enumerate(ids):
                outs[k] = b3.download(i)
        pairs = []
        for k, ((c, ic), inst) in enumerate(zip(ics, insts)):
            with G.Solver(c) as s1:
                s1.upload(ic)
                s1.advance(inst[3])
                pairs.append(_errors(outs[k], s1.download(), c.model))
        acc = {**_error_summary(pairs, "plain FP64 form, bit-identical to the reference"),
               "steps": insts[0][3]}
    return {"value": value, "ms_per_step": ms / K, "dtype": "f32+f32comp",
            "accuracy_vs_fp64": acc,
            "config": {"workload": "batch256", "model": "euler", "precision": "mixed",
                       "instances": 256, "cells": cells, "sizes": "nx, ny log-uniform [64, 1024]",
                       "y_half_step": "dy (fix_dy_halfstep; see BATCH_FIX_DY)",
                       "bubbles": "4-16 per instance", "steps_per_instance": 500,
                       "tile_shapes": list(shapes), "autotune_tick_ms": tune_ms,
                       "autotune_steps": sum(pre.values()), "graph": "8 ticks per CUDA graph",
                       "l2": f"state {cells * 32 / 1e6:.0f} MB > 126 MB L2, no flush",
                       "parallelism": f"replicas x{ctx.world}"},
            "clocks": ck, "gpu_launches": 2 * K, "roofline": rl, "e2e": e2e,
            "sim": {"cell_updates_timed": upd}}


def _serve(G, reqs, ics, precision, ticks, stream):
    """Submits the requests at their arrival times; returns per-request
    (info, result), server statistics and the makespan."""
    # request grids in pinned host memory (pinned once, when the server starts)
    pinned = sum(ic.nbytes for _, ic in ics) + len(ics) * 256 + (1 << 20)
    srv = G.Server(precision, budget_fraction=0.8, ticks_per_round=ticks,
                   stream=stream.cuda_stream if stream is not None else None,
                   host_pinned_bytes=pinned)
    ids = [None] * len(reqs)
    # the clients' result buffers, allocated and written once before the clock
    # starts (np.zeros would leave the pages unmapped until the result lands)
    outs = [np.empty(cfg.ghosted_shape()) for cfg, _ in ics]
    for o in outs:
        o.fill(0.0)
    t0 = time.perf_counter()

    def submitter():
        for k, r in enumerate(reqs):
            delay = r[0] - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
            cfg, ic = ics[k]
            ids[k] = srv.submit(cfg, ic, r[4])

    th = threading.Thread(target=submitter)
    th.start()
    th.join()
    res = [srv.wait(i, out=o) for i, o in zip(ids, outs)]
    makespan = time.perf_counter() - t0
    st = srv.stats()
    srv.close()
    return res, st, makespan


def bench_served(args, ctx, G, stream, clocks):
    torch = ctx.torch
    K, W = max(args.steps, 1), args.warmup
    reqs = served_requests(W + K, SEED + 7919 * ctx.rank)
    t_ic = time.perf_counter()
    ics = [build_ic(G, rec, nx, ny, sd, nb) for (_, rec, nx, ny, steps, sd, nb) in reqs]
    t_ic = time.perf_counter() - t_ic
    warm, timed = reqs[:W], reqs[W:]
    warm_ics, timed_ics = ics[:W], ics[W:]
    base = timed[0][0]
    timed = [(r[0] - base, *r[1:]) for r in timed]
    upd = sum(r[2] * r[3] * r[4] for r in timed)
    if warm:
        _serve(G, [(0.0, *r[1:]) for r in warm], warm_ics, G.MIXED, 16, stream)

    # device-resident throughput of the mixed form on the timed request set
    b = G.Batch(stream=stream.cuda_stream)
    ids = [b.add(c, ic, r[4]) for (c, ic), r in zip(timed_ics, timed)]
    b.autotune(1)  # trial steps are real steps; they are not counted below
    b.step(8)  # captures the tick graph outside the timed region (not counted either)
    before = {i: s for i, s, _, _ in b.poll()}
    max_steps = max(r[4] for r in timed)
    clocks.start()
    time.sleep(0.3)
    ctx.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    b.step(max_steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ck = clocks.stop()
    ms = ctx.max(e0.elapsed_time(e1))
    res_upd = sum(b.cfgs[i].nx * b.cfgs[i].ny * (r[4] - before[i]) for i, r in zip(ids, timed))
    value = job_throughput(ctx, res_upd, ms)
    b.close()
    # roofline of the mixed sweeps on a resident sample (16 requests)
    b = G.Batch(stream=stream.cuda_stream)
    sample = list(zip(timed_ics, timed))[:16]
    for (c, ic), r in sample:
        b.add(c, ic, r[4])
    b.step(2)
    mx, my, _n = b.step_timed(4)
    b.close()
    dom = 0 if mx >= my else 1
    byts = sum(c.nx * c.ny * c.nvar * 8 * 2 for (c, _), _r in sample)
    rl = roofline(["mixed_sweep_x", "mixed_sweep_y"][dom], [mx, my][dom], 4, byts,
                  f"served_mixed_sweep_{'xy'[dom]}")
    rl["note"] = ("16-request resident sample, one launch per model and direction per tick; "
                  "bytes summed over the requests of a tick, time summed over its launches")

    # served runs (host buffers, arrivals, continuous batching)
    ctx.barrier()
    res_m, st_m, mk_m = _serve(G, timed, timed_ics, G.MIXED, 16, stream)
    # the plain FP64 form at its best: fast FP64 members of one batch (relative
    # L1 density error far below 1e-12); and the bit-identical form, one solver
    # per request
    res_q, st_q, mk_q = _serve(G, timed, timed_ics, G.FP64_FAST, 16, stream)
    res_f, st_f, mk_f = _serve(G, timed, timed_ics, G.FP64, 16, stream)
    lat_m = [i.latency_s for i, _ in res_m]
    lat_q = [i.latency_s for i, _ in res_q]
    lat_f = [i.latency_s for i, _ in res_f]
    pct = lambda v, q: float(np.percentile(v, q))
    l1 = [_rel_l1_density(a, f, c.model) for (_, a), (_, f), (c, _) in zip(res_m, res_f, timed_ics)]
    linf = [_rel_linf_density(a, f, c.model)
            for (_, a), (_, f), (c, _) in zip(res_m, res_f, timed_ics)]
    acc_q = _error_summary([_errors(a, f, c.model) for (_, a), (_, f), (c, _)
                            in zip(res_q, res_f, timed_ics)],
                           "bit-identical FP64 form (= the reference)")
    acc_q["l1"]["bound"] = 1e-12
    nbytes = sum(ic.size * 8 for _, ic in timed_ics)
    e2e_val = ctx.sum(upd) / ctx.max(mk_m) / 1e9
    fast_val = ctx.sum(upd) / ctx.max(mk_q) / 1e9
    fp64_val = ctx.sum(upd) / ctx.max(mk_f) / 1e9
    models = 1 + any(r[1] != "shock_bubbles" for r in timed)
    return {
        "value": value, "ms_per_step": ms / len(timed), "dtype": "f32+f32comp",
        "config": {"workload": "served", "step": "one request (ms_per_step: device ms of the "
                   "resident run per timed request)", "requests": len(timed), "warmup_requests": W,
                   "arrivals": "Poisson, mean 50/s, seeded",
                   "mix": "70% Euler shock_bubbles, 30% Allaire water_shock_air_bubble "
                          "(PVRS, alpha clip 1e-6)",
                   "cells": "log-uniform [128^2, 2048^2]", "steps": "uniform [100, 2000]",
                   "budget": "80% of free HBM", "ticks_per_round": 16, "seed": SEED,
                   "cell_updates": upd, "ic_build_s": t_ic,
                   "value_def": "all timed requests resident in one batch, device time",
                   "l2": "resident set >> 126 MB L2, no flush",
                   "parallelism": f"replicas x{ctx.world}"},
        "p50_ms": 1e3 * pct(lat_m, 50), "p99_ms": 1e3 * pct(lat_m, 99),
        "plain_fp64": {"value": fast_val, "unit": UNIT, "form": "fast FP64, batched",
                       "p50_ms": 1e3 * pct(lat_q, 50), "p99_ms": 1e3 * pct(lat_q, 99),
                       "makespan_s": mk_q, "device_s": st_q.device_s,
                       "max_resident": st_q.max_running, "accuracy_vs_bit_exact": acc_q},
        "plain_fp64_bit_exact": {"value": fp64_val, "unit": UNIT,
                                 "form": "bit-identical FP64, one solver per request",
                                 "p50_ms": 1e3 * pct(lat_f, 50), "p99_ms": 1e3 * pct(lat_f, 99),
                                 "makespan_s": mk_f, "device_s": st_f.device_s,
                                 "max_resident": st_f.max_running},
        "mixed_vs_plain": e2e_val / fast_val,
        "mixed_vs_bit_exact": e2e_val / fp64_val,
        "l1_vs_fp64": {"max": max(l1), "median": float(np.median(l1)), "bound": 1e-4},
        "linf_vs_fp64": {"max": max(linf), "median": float(np.median(linf))},
        "clocks": ck, "gpu_launches": 2 * models * max_steps,
        "roofline": rl,
        "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": nbytes / len(timed),
                "d2h_bytes_per_step": nbytes / len(timed), "step": "one request",
                "host_buffers": "client arrays copied into the server's pinned arena at submit",
                "makespan_s": mk_m, "device_s": st_m.device_s, "max_resident": st_m.max_running},
        "sim": {"max_steps": max_steps},
    }


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--warmup", type=int, default=None)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="served", choices=WORKLOADS)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end pass (profiling)")
    ap.add_argument("--no-accuracy", action="store_true",
                    help="skip the mixed-vs-FP64 error runs (profiling)")
    args = ap.parse_args()
    if args.steps is None:
        args.steps = 48 if args.workload == "served" else 50
    if args.warmup is None:
        args.warmup = 4 if args.workload == "served" else 5
    if args.impl == "ours" and args.warmup < 3:
        args.warmup = 3
    world = int(os.environ.get("WORLD_SIZE", "0"))
    if world == 0 and args.gpus > 1:
        # one process per GPU: relaunch under torchrun with the same arguments
        port = 29500 + os.getpid() % 2000
        cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
               f"--nproc-per-node={args.gpus}", "--master-addr", "127.0.0.1",
               "--master-port", str(port), str(Path(__file__).resolve()), *sys.argv[1:]]
        os.execv(sys.executable, cmd)
    world = max(world, 1)
    if world != args.gpus:
        sys.exit(f"bench.py: --gpus {args.gpus} but WORLD_SIZE={world}; launch one rank per GPU")
    if args.impl == "reference":
        run_reference(args)
        return

    import torch
    import torch.distributed as dist

    import cfdgpu as G

    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    ctx = Ctx(torch, dist, world, rank, local)
    stream = torch.cuda.Stream()  # a real stream: the library runs on it
    torch.cuda.set_stream(stream)
    clocks = ClockSampler(_gpu_id(torch, local))
    if args.workload == "served":
        r = bench_served(args, ctx, G, stream, clocks)
    elif args.workload == "batch256":
        r = bench_batch(args, ctx, G, stream, clocks)
    else:
        r = bench_single(args, ctx, G, stream, clocks)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args.workload)
    if rank == 0:
        line = {"metric": METRIC, "value": r.pop("value"), "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": r.pop("ms_per_step"),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": r.pop("dtype"), "data": "synthetic", "config": r.pop("config")}
        line.update(r)
        line["cpu_baseline"] = cpu
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
