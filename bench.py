#!/usr/bin/env python
"""Benchmark of the Pearl FP64 time-step hot path on B200.

Workload (the large FP64 configuration): nx=2048 periodic x 4096 growth rows,
dx=2 nm, 64 lamellar pairs (spacing 32 cells with seeded +-10% jitter, ferrite
fraction 0.875), per-column fronts at row 32+U{-1,0,1}, 20 K undercooling,
adaptive dt (dt=4e-12 s, dt_max=8e-12 s), moving window enabled, implicit
diffusion on.  Synthetic, seeded data; the 336 MB state is larger than L2.

One step = one accepted pearl::advance (pearl_serial.cpp:1119) of the whole
domain, including rejected attempts.  Metric: cell-updates/s = nx*ny*steps/time.

  value    device-resident throughput: K steps in one persistent launch
           (pearl_gpu_run), CUDA events on the launching stream.
  e2e      the same through the public C ABI with host buffers: every output
           interval uploads the state from pinned host memory, runs, applies
           the moving window, reduces the diagnostics and downloads the state.
  roofline algorithmic bytes per cell-update 80 + 64*n_CG (read+write of the
           5-double state, plus per CG iteration read p,K,chi,x,r and write
           x,r,p) over the kernel's event time, against the measured HBM copy
           bandwidth.
  cpu_baseline / --impl reference: the reference solver compiled from its own
           source (oracle/_ref), else the C restatement, on host cores.

Other workloads (same JSON contract, not the default line):
  --precision mixed     the same domain in the mixed form: FP32 propose forces and
                        FP32 inner-solve rounds closed by FP64 residuals
  --workload sweep      256 independent instances in one batched launch, with
                        the autotuner and an all-cores CPU baseline
  --workload adjoint    gradient of a 256x512, --steps-step run w.r.t. mobility,
                        sigma and D_gamma (--checkpoint-every K), checked against
                        central differences and the CPU reference gradient

Profiling aids (no bench line): --probe propose | diffusion launches one phase
of the step on its own; --probe fp64-peak measures the FP64 roofline.

Multi-GPU: the path does not shard (one resident domain per GPU), so N GPUs run
N independent replicas ("scaling": "weak"); time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
PKG = ROOT / "fe-c_eutectoid_phase-field_simulation_b200"
for _p in (str(ROOT), str(PKG)):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "cell-updates/s"
UNIT = "cell-updates/s"
FALLBACK_HBM_GBS = 6650.0


def parse_args(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["pearl_gpu", "reference"], default="pearl_gpu")
    ap.add_argument("--nx", type=int, default=2048)
    ap.add_argument("--ny", type=int, default=4096)
    ap.add_argument("--output-every", type=int, default=50, help="accepted steps per e2e output interval")
    ap.add_argument("--cpu-seconds", type=float, default=20.0, help="bound of the CPU-baseline sample")
    ap.add_argument("--ref-seconds", type=float, default=60.0, help="bound of the reference arm's timed work")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", choices=["plain_large", "sweep", "adjoint"], default="plain_large",
                    help="plain_large (default): one 2048x4096 domain; sweep: 256 small independent "
                         "instances in one batched persistent launch; adjoint: gradient of a 256x512, "
                         "1000-step run (--steps sets the step count of that run)")
    ap.add_argument("--checkpoint-every", type=int, default=50, help="adjoint: steps per checkpoint segment")
    ap.add_argument("--cpu-gradient-steps", type=int, default=100,
                    help="adjoint: steps of the run the CPU reference gradient covers (bounded CPU time)")
    ap.add_argument("--precision", choices=["fp64", "mixed", "mixed_propose", "mixed_solve"], default="fp64",
                    help="fp64 (default): the reference's arithmetic; mixed: FP32 propose forces and FP32 "
                         "inner-solve rounds with FP64 refinement; mixed_propose / mixed_solve: one of the two")
    ap.add_argument("--probe", choices=["propose", "diffusion", "fp64-peak"], default=None,
                    help="profiling aid instead of the bench line: launch one phase of the hot path on its own "
                         "(propose: propose_phi + mixture; diffusion: one proposal, then the FP64 implicit solve) "
                         "--steps times on the --nx x --ny large workload, or measure the FP64 peak")
    ap.add_argument("--instances", type=int, default=256, help="sweep: number of instances")
    ap.add_argument("--group-blocks", type=int, default=0,
                    help="sweep: blocks per instance group (0 = autotune, -1 = sized per instance)")
    return ap.parse_args(argv)


def workload(nx: int, ny: int, seed: int = 0):
    from pearl_gpu import workloads

    return workloads.plain_large(seed=seed, nx=nx, ny=ny, pairs=max(1, nx // 32))


def config_dict(w, args) -> dict:
    return {
        "workload": f"plain FP64 large: {w.nx}x{w.ny} (x periodic, y growth), {max(1, w.nx // 32)} pairs "
                    f"spacing 32+-10%, "
                    f"f_alpha 0.875, T_E-20K, adaptive dt, moving window, implicit diffusion",
        "nx": w.nx, "ny": w.ny, "cells": w.cells, "dx_m": w.params["dx"],
        "dt": w.params["dt_max"] / 2, "dt_max": w.params["dt_max"],
        "l2": "inputs larger than L2 (state 40 B/cell = %.0f MB)" % (40 * w.cells / 1e6),
        "parallelism": f"replicas x{args.gpus}",
        "bytes_per_cell_update": "80 + 64*n_CG",
        "precision": args.precision,
    }


# ------------------------------------------------------------------ helpers
def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            d = json.loads(p.read_text())
            return float(d["hbm_gbs"]), "measured"
        except Exception:  # noqa: BLE001
            pass
    return FALLBACK_HBM_GBS, "fallback"


# B200 HBM3e specification (the measured copy bandwidth in MEASURED_PEAKS.json is
# the roofline's denominator; the fraction of this figure is reported beside it)
SPEC_HBM_GBS = 8000.0

# Bytes each pass of the persistent step reads and writes per cell (float64):
# PROPOSE phi x3 + mu in, trial phi x3, K, chi, c(mu_ref) out; SETUP K, mu, chi,
# c(mu_ref), c in, faces x2, x, r, z, diag out; APPLY faces x2, z, chi (+ p_old
# after the first iteration) in, p, Ap out; UPDATE x, p, r, Ap, diag in, x, r, z
# out; FINAL faces x2, x, trial phi x3, c, chi, c(mu_ref) in, r, c, mu out.
PHASE_BYTES = {"propose": 80, "setup": 88, "apply_first": 48, "apply": 56, "update": 64, "final": 96}


def phase_hbm_fracs(phase_ms: dict, phase_n: dict, cells: int, peak_gbs: float) -> dict:
    """Per phase: its bytes over its clocked time (the phase clock includes the
    phase's closing reduction), as a fraction of the HBM peak.  An APPLY after
    SETUP or RESET starts a solve and reads no previous direction."""
    out = {}
    for k in ("propose", "setup", "apply", "update", "final"):
        ms, n = phase_ms.get(k, 0.0), phase_n.get(k, 0)
        if not ms or not n:
            continue
        if k == "apply":
            first = min(n, phase_n.get("setup", 0) + phase_n.get("reset", 0))
            nbytes = cells * (first * PHASE_BYTES["apply_first"] + (n - first) * PHASE_BYTES["apply"])
        else:
            nbytes = cells * n * PHASE_BYTES[k]
        out[k] = round(nbytes / (ms / 1e3) / 1e9 / peak_gbs, 4)
    return out


def ncu_traffic_per_cell():
    """DRAM bytes per cell-update of pearl_kernel from the committed ncu summary, or None."""
    p = ROOT / "profiles" / "pearl_kernel_fp64_plain_large.md"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.startswith("dram_bytes_per_cell_update:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


class ClockSampler:
    """SM clock and throttle reasons sampled during the timed region.

    Uses NVML from a background thread every few milliseconds (read-only
    queries), so even a short timed region yields many samples; falls back to
    `nvidia-smi -lms` when NVML is unavailable."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
               "sw_power_cap": 0x4}

    def __init__(self, index: int, period_s: float = 0.005):
        self.index = index
        self.period = period_s
        self.samples: list[tuple[float, float, int]] = []
        self._stop = None
        self._thread = None
        self._nvml = None

    def start(self):
        import threading

        try:
            import pynvml

            pynvml.nvmlInit()
            self._nvml = pynvml
            handle = pynvml.nvmlDeviceGetHandleByIndex(self.index)
        except Exception:  # noqa: BLE001 - no NVML: nothing sampled
            self._nvml = None
            return
        self._stop = threading.Event()
        first = threading.Event()

        def run():
            P = self._nvml
            get_reasons = getattr(P, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                P.nvmlDeviceGetCurrentClocksThrottleReasons
            max_mhz = float(P.nvmlDeviceGetMaxClockInfo(handle, P.NVML_CLOCK_SM))
            while True:
                try:
                    sm = float(P.nvmlDeviceGetClockInfo(handle, P.NVML_CLOCK_SM))
                    reasons = int(get_reasons(handle))
                except Exception:  # noqa: BLE001
                    break
                self.samples.append((sm, max_mhz, reasons))
                first.set()
                # one more sample after stop() is called: the end of the timed region
                if self._stop.is_set():
                    break
                self._stop.wait(self.period)
            first.set()

        self._thread = threading.Thread(target=run, daemon=True)
        self._thread.start()
        # the sampler is running before the timed region starts
        first.wait(timeout=2.0)

    def stop(self) -> dict | None:
        if self._thread is None:
            return None
        self._stop.set()
        self._thread.join(timeout=5)
        try:
            self._nvml.nvmlShutdown()
        except Exception:  # noqa: BLE001
            pass
        if not self.samples:
            return None
        reasons = sorted(name for name, bit in self.REASONS.items() if any(r & bit for _, _, r in self.samples))
        sm = [s for s, _, _ in self.samples]
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(m for _, m, _ in self.samples),
                "reasons": reasons, "samples": len(self.samples), "source": "nvml"}


def reduce_over_ranks(dist, x: float, op: str, device: str) -> float:
    """Max or sum of a per-rank scalar (replicas: throughput is the sum of cells over the
    slowest rank's time).  Identity without a process group."""
    if dist is None:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def replica_throughput(dist, cells: float, seconds: float, device: str) -> tuple[float, float]:
    """(whole-job cell-updates/s, max time over ranks) for independent replicas."""
    t_max = reduce_over_ranks(dist, seconds, "max", device)
    return reduce_over_ranks(dist, cells, "sum", device) / t_max, t_max


# ------------------------------------------------------------------ CPU sides
def cpu_sample(w, seconds: float, max_steps: int | None = None):
    """Time the reference (or the C restatement) on one host core over whole steps of the
    same workload, stopping once `seconds` have elapsed.  Returns (rate, kind, steps, secs)."""
    from oracle import pyoracle

    ref = pyoracle.reference()
    lib, kind = (ref, "reference") if ref is not None else (pyoracle.port(), "port")
    phi, c, mu = w.phi.copy(), w.carbon.copy(), w.mu.copy()
    s = pyoracle.scalars_from(w.scalars)
    steps, t_total = 0, 0.0
    while t_total < seconds and (max_steps is None or steps < max_steps):
        t0 = time.perf_counter()
        out = lib.advance_n(w.params, phi, c, mu, s, 1)
        t_total += time.perf_counter() - t0
        if out[0] != 0:
            raise RuntimeError(f"CPU baseline failed: {out[1]}")
        steps += 1
    return w.cells * steps / t_total, kind, steps, t_total


def reference_arm(args, rank: int, world: int) -> None:
    if rank != 0:
        return
    w = workload(args.nx, args.ny)
    from oracle import pyoracle

    ref = pyoracle.reference()
    lib, kind = (ref, "reference") if ref is not None else (pyoracle.port(), "port")
    # Bounded: up to three whole warm-up steps, then whole steps until
    # --ref-seconds of timed work (a few seconds per step of the full domain on
    # one core) or K steps.
    warm = min(args.warmup, 3)
    phi, c, mu = w.phi.copy(), w.carbon.copy(), w.mu.copy()
    s = pyoracle.scalars_from(w.scalars)
    rc = lib.advance_n(w.params, phi, c, mu, s, warm)
    if rc[0]:
        raise RuntimeError(rc[1])
    timed, dt = 0, 0.0
    while timed < args.steps and (timed == 0 or dt < args.ref_seconds):
        t0 = time.perf_counter()
        rc = lib.advance_n(w.params, phi, c, mu, s, 1)
        dt += time.perf_counter() - t0
        if rc[0]:
            raise RuntimeError(rc[1])
        timed += 1
    value = w.cells * timed / dt
    sample = (f"{timed} timed whole steps after {warm} warm-up steps of the full {w.nx}x{w.ny} workload "
              f"(requested {args.steps}+{args.warmup}; bounded to about {args.ref_seconds:.0f} s)")
    cores = 1
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": timed, "warmup": warm,
        "ms_per_step": dt / timed * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic", "config": config_dict(w, args), "impl": "reference",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample,
                         "cpu": _cpu_model()},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def _cpu_model() -> str:
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


# ------------------------------------------------------------------ GPU arm
def gpu_arm(args, rank: int, world: int, dist) -> None:
    import numpy as np
    import torch

    import pearl_gpu

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    stream = torch.cuda.current_stream()
    w = workload(args.nx, args.ny, seed=rank)
    ctx = pearl_gpu.Context(w.params, w.nx, w.ny, device=local, stream=stream.cuda_stream)
    ctx.set_precision(args.precision)
    # pinned host buffers for the end-to-end leg
    phi_h = torch.from_numpy(w.phi).pin_memory().numpy()
    c_h = torch.from_numpy(w.carbon).pin_memory().numpy()
    mu_h = torch.from_numpy(w.mu).pin_memory().numpy()
    ctx.upload(phi_h, c_h, mu_h, w.scalars)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x: float) -> float:
        return reduce_over_ranks(dist, x, "max", "cuda")

    def sum_over_ranks(x: float) -> float:
        return reduce_over_ranks(dist, x, "sum", "cuda")

    # warm-up (also fills the step-energy cache)
    ctx.run(max(args.warmup, 1))
    meta = w.meta

    # ---- device-resident timed region: K accepted steps in one persistent launch
    clocks = ClockSampler(local)
    barrier()
    launches0 = ctx.stats()["launches"]
    rejected0 = ctx.scalars().rejected
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    rep = ctx.run(args.steps)
    ev1.record(stream)
    barrier()
    clock_info = clocks.stop()
    launches = ctx.stats()["launches"] - launches0
    kernel_ms = ctx.stats()["last_ms"]
    phase_ms = {k: round(v[0], 3) for k, v in ctx.phase_times().items()}
    phase_n = {k: v[1] for k, v in ctx.phase_times().items()}
    rejected = ctx.scalars().rejected - rejected0
    elapsed = ev0.elapsed_time(ev1) / 1e3
    assert rep.steps == args.steps, "run stopped early"
    value, t_max = replica_throughput(dist, float(w.cells * rep.steps), elapsed, "cuda")

    # roofline of the persistent kernel: algorithmic bytes of its launch over its event time
    algo_bytes = w.cells * (80.0 * rep.steps + 64.0 * rep.cg_total)
    achieved = algo_bytes / (kernel_ms / 1e3) / 1e9
    peak, peak_kind = measured_peak()
    tpc = ncu_traffic_per_cell()
    traffic = tpc * w.cells * rep.steps if tpc is not None else None

    # ---- end-to-end through the C ABI with host buffers
    m = max(1, min(args.output_every, args.steps))
    intervals = max(1, math.ceil(args.steps / m))
    phi_o = torch.empty(w.phi.shape, dtype=torch.float64).pin_memory().numpy()
    c_o = torch.empty(w.carbon.shape, dtype=torch.float64).pin_memory().numpy()
    mu_o = torch.empty(w.mu.shape, dtype=torch.float64).pin_memory().numpy()
    phi_h[...], c_h[...], mu_h[...], s_h = ctx.download()
    barrier()
    t0 = time.perf_counter()
    e2e_steps = 0
    for _ in range(intervals):
        ctx.upload(phi_h, c_h, mu_h, s_h)
        r = ctx.run(m)
        e2e_steps += r.steps
        ctx.maybe_shift(meta["shift_trigger"], meta["shift_target"], meta["shift_gamma_carbon"])
        ctx.snapshot()
        _, _, _, s_h = ctx.download(out=(phi_o, c_o, mu_o))
        phi_h, phi_o = phi_o, phi_h
        c_h, c_o = c_o, c_h
        mu_h, mu_o = mu_o, mu_h
    barrier()
    e2e_t = max_over_ranks(time.perf_counter() - t0)
    e2e_value = sum_over_ranks(float(w.cells * e2e_steps)) / e2e_t
    bytes_state = 40 * w.cells

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, kind, steps, secs = cpu_sample(w, args.cpu_seconds)
        cpu = {"value": rate, "unit": UNIT, "cores": 1, "kind": kind,
               "sample": f"{steps} whole steps of the same {w.nx}x{w.ny} workload in {secs:.1f} s "
                         f"(single-threaded serial solver)", "cpu": _cpu_model()}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32+f64",
            "data": "synthetic", "config": config_dict(w, args),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "spec_gbs": SPEC_HBM_GBS, "frac_of_spec": achieved / SPEC_HBM_GBS,
                         "peak_source": f"{peak_kind} HBM copy bandwidth",
                         "kernel": "pearl_kernel (persistent FP64 step)",
                         # 148 on B200: one 512-thread block per SM (32x32 tiles); 296: two 256-thread blocks
                         "grid_blocks": ctx.stats()["grid"],
                         "algorithmic_bytes_per_launch": algo_bytes, "cg_iterations": rep.cg_total,
                         "rejected_attempts": rejected, "phase_ms": phase_ms, "phase_count": phase_n,
                         "phase_hbm_frac": phase_hbm_fracs(phase_ms, phase_n, w.cells, peak),
                         "phase_bytes_per_cell": PHASE_BYTES},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": bytes_state / m,
                    "d2h_bytes_per_step": bytes_state / m,
                    "step": f"one output interval of {m} accepted steps: upload state, run, maybe_shift, "
                            f"snapshot, download state"},
            "clocks": clock_info,
            "gpu_launches": launches,
        }
        print(json.dumps(line), flush=True)
    ctx.close()


def _cpu_sweep_task(task):
    """One sweep instance on one host core: `steps` whole steps of the reference solver
    (oracle/_ref, else the C restatement).  Returns (cell-updates, kind)."""
    i, seed, steps = task
    from oracle import pyoracle
    from pearl_gpu import workloads

    w = workloads.sweep_one(i, seed)
    ref = pyoracle.reference()
    lib, kind = (ref, "reference") if ref is not None else (pyoracle.port(), "port")
    phi, c, mu = w.phi.copy(), w.carbon.copy(), w.mu.copy()
    s = pyoracle.scalars_from(w.scalars)
    out = lib.advance_n(w.params, phi, c, mu, s, steps)
    if out[0] != 0:
        raise RuntimeError(f"CPU sweep instance {i} failed: {out[1]}")
    return w.cells * steps, kind


def cpu_sweep_sample(n: int, seed: int, steps: int):
    """The sweep on all host cores: one process per core, each running whole
    instances (`steps` steps each) of the same n instances.  Processes are
    spawned (the parent holds a CUDA context).  Returns (rate, kind, cores, secs)."""
    import multiprocessing as mp

    cores = max(1, os.cpu_count() or 1)
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        pool.map(_cpu_sweep_task, [(0, seed, 1)] * cores)  # start-up (imports, oracle load) untimed
        t0 = time.perf_counter()
        res = pool.map(_cpu_sweep_task, [(i, seed, steps) for i in range(n)], chunksize=1)
        secs = time.perf_counter() - t0
    return sum(r[0] for r in res) / secs, res[0][1], cores, secs


def sweep_arm(args, rank: int, world: int, dist) -> None:
    """Batched parameter sweep: --instances independent domains (2 lamellar pairs of
    spacing U{16..96} across x, growth length U{64..1024}, ferrite fraction
    U(0.85,0.90), undercooling U(5,40) K, adaptive dt) advanced K steps each in one
    persistent launch.  Metric: cell-updates/s summed over instances."""
    import numpy as np
    import torch

    import pearl_gpu
    from pearl_gpu import workloads

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    ws = workloads.sweep(args.instances, seed=rank)
    cells = sum(w.cells for w in ws)
    b = pearl_gpu.Batch([(w.params, w.nx, w.ny) for w in ws], device=local,
                        group_blocks=max(args.group_blocks, -1))
    b.set_precision(args.precision)
    pinned = []
    for i, w in enumerate(ws):
        hp = [torch.from_numpy(a).pin_memory().numpy() for a in (w.phi, w.carbon, w.mu)]
        pinned.append(hp)
        b.upload(i, *hp, w.scalars)
    tuned = None
    if args.group_blocks == 0:
        tuned = b.autotune(steps=10)
    b.run(max(args.warmup, 1))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    clocks = ClockSampler(local)
    barrier()
    l0 = b.stats()["launches"]
    rej0 = [b.download(i)[3].rejected for i in range(len(ws))]
    clocks.start()
    t0 = time.perf_counter()
    reps, st = b.run(args.steps)
    barrier()
    wall = time.perf_counter() - t0
    clock_info = clocks.stop()
    st_ = b.stats()
    kernel_ms = st_["last_ms"]
    if any(st):
        raise RuntimeError(f"sweep instance failed: {[pearl_gpu.STATUS.get(x, x) for x in st if x]}")
    steps = [r.steps for r in reps]
    cell_updates = float(sum(w.cells * n for w, n in zip(ws, steps)))
    rejected = [b.download(i)[3].rejected - r0 for i, r0 in enumerate(rej0)]
    rejected_cell_attempts = float(sum(w.cells * r for w, r in zip(ws, rejected)))
    value, t_max = replica_throughput(dist, cell_updates, kernel_ms / 1e3, "cuda")
    cg = sum(r.cg_total * w.cells for r, w in zip(reps, ws))
    algo_bytes = 80.0 * cell_updates + 64.0 * cg
    achieved = algo_bytes / (kernel_ms / 1e3) / 1e9
    peak, peak_kind = measured_peak()

    # end to end: upload every instance from pinned host memory, run, download every instance
    outs = [[torch.empty(a.shape, dtype=torch.float64).pin_memory().numpy() for a in hp] for hp in pinned]
    scal = [b.download(i)[3] for i in range(len(ws))]
    barrier()
    t0 = time.perf_counter()
    for i in range(len(ws)):
        b.upload(i, *pinned[i], scal[i])
    reps2, _ = b.run(args.steps)
    for i in range(len(ws)):
        scal[i] = b.download(i, out=outs[i])[3]
    barrier()
    e2e_t = reduce_over_ranks(dist, time.perf_counter() - t0, "max", "cuda")
    e2e_cells = reduce_over_ranks(dist, float(sum(w.cells * r.steps for w, r in zip(ws, reps2))), "sum", "cuda")
    state_bytes = 40 * cells
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, kind, cores, secs = cpu_sweep_sample(len(ws), rank, 10)
        cpu = {"value": rate, "unit": UNIT, "cores": cores, "kind": kind,
               "sample": f"all {len(ws)} instances, 10 whole steps each, one process per host core "
                         f"({secs:.1f} s wall)", "cpu": _cpu_model()}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32+f64",
            "data": "synthetic",
            "config": {"workload": f"batched sweep: {len(ws)} instances, nx=2*spacing (spacing U{{16..96}}), "
                                   f"ny U{{64..1024}}, f_alpha U(0.85,0.90), T_E-U(5,40)K, adaptive dt, "
                                   f"{args.precision}",
                       "instances": len(ws), "cells": cells, "group_blocks": st_["group_blocks"],
                       "grid_blocks": st_["grid"], "autotuned": tuned is not None,
                       "tma": None if tuned is None else tuned[1],
                       "tile": None if tuned is None else f"{32 * tuned[2]}x{16 // tuned[2]}",
                       "l2": "inputs larger than L2 (state 40 B/cell = %.0f MB)" % (40 * cells / 1e6),
                       "parallelism": f"replicas x{world}", "bytes_per_cell_update": "80 + 64*n_CG"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None,
                         "spec_gbs": SPEC_HBM_GBS, "frac_of_spec": achieved / SPEC_HBM_GBS,
                         "peak_source": f"{peak_kind} HBM copy bandwidth",
                         "kernel": "pearl_batch_kernel (persistent FP64 step, block groups)",
                         "algorithmic_bytes_per_launch": algo_bytes,
                         "rejected_attempts": int(sum(rejected)),
                         "cg_per_step": sum(r.cg_total for r in reps) / max(1, sum(steps)),
                         "rejected_share_of_cell_attempts": rejected_cell_attempts
                         / (rejected_cell_attempts + cell_updates)},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_cells / e2e_t, "unit": UNIT, "h2d_bytes_per_step": state_bytes / args.steps,
                    "d2h_bytes_per_step": state_bytes / args.steps,
                    "step": f"upload all instances, {args.steps} steps each in one launch, download all"},
            "clocks": clock_info,
            "gpu_launches": st_["launches"] - l0,
            "wall_s": wall,
        }
        print(json.dumps(line), flush=True)
    b.close()


def adjoint_arm(args, rank: int, world: int, dist) -> None:
    """Gradient of J = sum (phi_alpha - target)^2 after K fixed-dt steps of a 256x512
    domain (4 lamellar pairs of spacing 64, ferrite fraction 0.875, T_E-15 K, dt 2e-12 s)
    w.r.t. (mobility scale, sigma, D_gamma); the target comes from a forward run with
    the three parameters perturbed by seeded U(-5%, 5%).  One timed step = one whole
    gradient (forward with checkpoints, recomputation, adjoint sweep).  Metric:
    gradient cell-steps/s = cells * K / gradient time."""
    import numpy as np
    import torch

    import pearl_gpu
    from pearl_gpu import workloads as W

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    K = args.steps
    w = W.adjoint_case(steps=K, seed=rank)
    every = args.checkpoint_every

    def ctx_for(params):
        c = pearl_gpu.Context(params, w.nx, w.ny, device=local)
        c.upload(w.phi, w.carbon, w.mu, w.scalars)
        return c

    with ctx_for(W.perturb(w.params, w.meta["target_rel"])) as c:
        c.run(K)
        target = np.ascontiguousarray(c.download()[0][..., 0])
    phi_h = torch.from_numpy(w.phi).pin_memory().numpy()
    c_h = torch.from_numpy(w.carbon).pin_memory().numpy()
    mu_h = torch.from_numpy(w.mu).pin_memory().numpy()
    ctx = pearl_gpu.Context(w.params, w.nx, w.ny, device=local)
    for _ in range(max(args.warmup, 1)):
        ctx.upload(phi_h, c_h, mu_h, w.scalars)
        ctx.adjoint_gradient(K, every, target)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    clocks = ClockSampler(local)
    barrier()
    l0 = ctx.stats()["launches"]
    clocks.start()
    t0 = time.perf_counter()
    ctx.upload(phi_h, c_h, mu_h, w.scalars)
    rep = ctx.adjoint_gradient(K, every, target)
    out = ctx.download()
    barrier()
    wall = time.perf_counter() - t0
    clock_info = clocks.stop()
    launches = ctx.stats()["launches"] - l0
    dev_ms = rep.forward_ms + rep.recompute_ms + rep.adjoint_ms
    cell_steps = float(w.cells * K)
    value, t_max = replica_throughput(dist, cell_steps, dev_ms / 1e3, "cuda")
    e2e_value, _ = replica_throughput(dist, cell_steps, wall, "cuda")
    # central differences of the device forward (h = 1e-6 relative)
    h = 1e-6
    base = [1.0, w.params["sigma"], w.params["D"][2]]
    fd_err = {}
    for k in range(3):
        J = []
        for sign in (1, -1):
            rel = [0.0, 0.0, 0.0]
            rel[k] = sign * h
            with ctx_for(W.perturb(w.params, rel)) as c:
                c.run(K)
                J.append(float(((c.download()[0][..., 0] - target) ** 2).sum()))
        fd = (J[0] - J[1]) / (2 * h * base[k])
        fd_err[W.ADJOINT_PARAMETERS[k]] = abs(rep.grad[k] - fd) / abs(fd)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the CPU reference gradient (oracle/pearl_adjoint.c, one core) on a bounded
        # prefix of the same run, and the device gradient of that prefix beside it
        from oracle import pyoracle

        port = pyoracle.port()
        kp = min(K, max(1, args.cpu_gradient_steps))
        phi, c, mu = w.phi.copy(), w.carbon.copy(), w.mu.copy()
        s = pyoracle.scalars_from(w.scalars)
        tc = time.perf_counter()
        rc, orep = port.adjoint_gradient(w.params, phi, c, mu, s, kp, min(every, kp), target)
        secs = time.perf_counter() - tc
        if rc:
            raise RuntimeError("CPU reference gradient failed")
        ctx.upload(phi_h, c_h, mu_h, w.scalars)
        prep = ctx.adjoint_gradient(kp, min(every, kp), target)
        cpu = {"value": w.cells * kp / secs, "unit": "gradient cell-steps/s", "cores": 1, "kind": "port",
               "sample": f"CPU reference gradient of the first {kp} steps ({secs:.1f} s, single thread)",
               "gpu_vs_cpu_gradient_rel_err": {W.ADJOINT_PARAMETERS[k]: abs(prep.grad[k] - orep.grad[k])
                                               / abs(orep.grad[k]) for k in range(3)},
               "cpu": _cpu_model()}
    ctx.close()
    if rank == 0:
        # forward, recomputation of every segment but the last, tape, adjoint
        nseg = -(-K // every)
        recomputed = (nseg - 1) / nseg
        per_step = (1.0 + recomputed) * (80.0 + 64.0 * rep.cg_forward / K) + 48.0 + 160.0 + 64.0 * rep.cg_adjoint / K
        algo = per_step * cell_steps
        peak, peak_kind = measured_peak()
        line = {
            "metric": "gradient cell-steps/s", "value": value, "unit": "gradient cell-steps/s", "n_gpus": world,
            "steps": K, "warmup": args.warmup, "ms_per_step": t_max / K * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"adjoint: {w.nx}x{w.ny}, 4 pairs spacing 64, f_alpha 0.875, T_E-15K, "
                                   f"dt 2e-12 s fixed, {K} steps, checkpoint every {every}",
                       "parameters": list(W.ADJOINT_PARAMETERS), "target_rel": w.meta["target_rel"],
                       "objective": rep.objective, "gradient": list(rep.grad),
                       "fd_rel_err": fd_err, "cg_forward": rep.cg_forward, "cg_adjoint": rep.cg_adjoint,
                       "forward_ms": rep.forward_ms, "recompute_ms": rep.recompute_ms,
                       "adjoint_ms": rep.adjoint_ms,
                       "l2": f"state {40 * w.cells / 1e6:.0f} MB, tape {48 * w.cells * min(K, every) / 1e6:.0f} MB",
                       "parallelism": f"replicas x{world}"},
            "roofline": {"bound": "hbm", "achieved": algo / (dev_ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": algo / (dev_ms / 1e3) / 1e9 / peak, "traffic": None,
                         "spec_gbs": SPEC_HBM_GBS, "frac_of_spec": algo / (dev_ms / 1e3) / 1e9 / SPEC_HBM_GBS,
                         "peak_source": f"{peak_kind} HBM copy bandwidth",
                         "kernel": "pearl_kernel (forward, recompute with tape) + pearl_adjoint_kernel",
                         "bytes_per_cell_step": "(1 + recomputed fraction)*(80+64*n_CG) + 48 tape + 160 adjoint "
                                                "+ 64*n_CG_adjoint"},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "gradient cell-steps/s", "h2d_bytes_per_step": 48 * w.cells / K,
                    "d2h_bytes_per_step": 40 * w.cells / K,
                    "step": "upload state and target, whole gradient, download final state"},
            "clocks": clock_info,
            "gpu_launches": launches,
        }
        print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ single-phase probes
def probe_arm(args) -> None:
    """One phase of the time step as its own launch, so that a profiler sees it
    alone (the step itself is one persistent kernel), or the FP64 peak of the
    device.  Prints one JSON line per launch; not a bench line."""
    import pearl_gpu

    if args.probe == "fp64-peak":
        print(json.dumps({"probe": "fp64-peak", "fp64_tflops": pearl_gpu.fp64_peak_tflops(0)}), flush=True)
        return
    w = workload(args.nx, args.ny)
    dt = w.meta["dt"]
    with pearl_gpu.Context(w.params, w.nx, w.ny) as ctx:
        ctx.set_precision(args.precision)
        ctx.upload(w.phi, w.carbon, w.mu, w.scalars)
        for _ in range(max(1, args.steps)):
            if args.probe == "propose":
                change = ctx.propose_phi(dt)
                out = {"probe": "propose", "max_phase_change": change}
            else:
                ctx.propose_phi(dt)
                d = ctx.implicit_diffusion(dt)
                out = {"probe": "diffusion", "ok": d["ok"], "cg_iterations": d["it"]}
            out.update(nx=w.nx, ny=w.ny, precision=args.precision, kernel_ms=ctx.stats()["last_ms"],
                       geometry=ctx.geometry(),
                       phase_ms={k: round(v[0], 4) for k, v in ctx.phase_times().items()})
            print(json.dumps(out), flush=True)


def main(argv=None) -> int:
    args = parse_args(argv)
    if args.probe:
        probe_arm(args)
        return 0
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as tdist

        backend = "nccl" if args.impl == "pearl_gpu" else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        tdist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
        dist = tdist
    try:
        if args.impl == "reference":
            reference_arm(args, rank, world)
        elif args.workload == "sweep":
            sweep_arm(args, rank, world, dist)
        elif args.workload == "adjoint":
            adjoint_arm(args, rank, world, dist)
        else:
            gpu_arm(args, rank, world, dist)
    finally:
        if dist is not None:
            dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
