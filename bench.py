#!/usr/bin/env python
"""Benchmark: 3D Taylor-Green 256^3 projection steps per second on B200.

Workload (the reference's headline path): 3D periodic Taylor-Green on
[0, 2 pi]^3 at 256^3, nu = 1/1600, CFL 0.5 (fixed dt = 0.5 / sum(1/h)),
u = sin x cos y cos z, v = -cos x sin y cos z, w = 0, MG-PCG pressure solve to
relative residual 1e-12, FP64 (``--precision mixed``: FP32 V-cycle inside the
FP64 CG).  One bench "step" is one full projection time step (TVD advection,
ADI Helmholtz predictor, MG-PCG Poisson, divergence/gradient correction) on
the resident state.  Every field of the 256^3 state (138 MB) is larger than
the 126 MB L2, so no L2 flush is needed between steps.

Arms:
  --impl b200 (default)   this repository's CUDA path through its C ABI;
  --impl reference        the reference's own CPU implementation of the same
                          step (oracle/_ref, the reference's sources compiled
                          in place; the plain-C oracle port if that build is
                          absent): the K timed 256^3 steps run as concurrent
                          single-thread replicas on the host cores.

The FP64 1-GPU line also carries two measurements of the rest of the
headline metric (skip with --no-extras): "mixed" -- the mixed path's steps/s
on the same workload, its speed-up, and its max-norm relative velocity
difference from the FP64 path after 200 steps; "adjoint" -- the adjoint check
workload (128^3, nu = 0.01, perturbed Taylor-Green, 100 steps, checkpoint
every 10): adjoint/forward device-time ratio and a central-difference check.

``--adjoint-long`` runs, instead of the step benchmark, the long-horizon
adjoint workload (512^3, Re 1600, 400 steps, mixed forward and adjoint with
the binomial checkpoint schedule sized to the device memory; the gradient's
mixed-vs-FP64 error checked at 256^3) and prints its own JSON line.

Multi-GPU: the path does not shard (replicas only): each rank runs its own
independent 256^3 simulation; value = total steps/s over ranks, time = max
over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_DEFAULT = 256
NU = 1.0 / 1600.0
CFL = 0.5
TOL = 1e-12
MAX_IT = 400
METRIC = "TGV 256^3 steps/s (FP64 projection step)"


def tg_dt(n, cfl=CFL):
    h = 2.0 * math.pi / n
    return cfl / (3.0 / h)


# ---------------------------------------------------------------------------
# algorithmic bytes per launch of each kernel class (compulsory traffic: each
# distinct input read once, each output written once), N = active cells
# ---------------------------------------------------------------------------

def bytes_per_launch(n, precision):
    """Compulsory bytes per launch of each kernel class.  FP64 path: every
    pressure-solve vector is FP64.  Mixed path (defect correction): the inner
    MG-PCG -- V-cycle and CG vectors alike -- is FP32 (s = 4); the outer FP64
    kernels are the defect_correction class (three launches per correction:
    rhs scaling 16 B, x update 20 B and residual 24 B per cell, 20 B average)."""
    N = n ** 3
    d = 8
    s = 4 if precision == "mixed" else 8  # inner solve vectors
    out = {
        "predictor_rhs": 5 * d * N,  # per component: read f, p, prev, adv; write rhs
        "advection": 4 * d * N,      # per component: read u, v, w; write adv
        "adi_sweep": 2 * d * N,
        "divergence_rhs": 5 * d * N,
        "pcg_initial_residual": 3 * d * N,
        "pcg_apply_ap": 2 * s * N,
        "pcg_update_xr": 6 * s * N,
        "pcg_update_p": 3 * s * N,
        "vcycle_smooth_first_fine": 2 * s * N,        # read b, write x
        "vcycle_smooth_fine": 3 * s * N,              # read a, b; write x
        "vcycle_restrict_fine": (2 + 1 / 8) * s * N,  # read b, x; write coarse b
        "vcycle_prolong_smooth_fine": (3 + 1 / 8) * s * N,  # read x, b, coarse x; write a
        "correct_velocity": (1 + 3 + 3) * d * N / 3 + d * N,  # per component launch
        "cell_pass": 7 * d * N,
    }
    if precision == "mixed":
        # the FP32 inner CG fuses the p update, A p and the deferred x update
        # into one plane-pipelined launch (read z, p_old, x; write p, A p, x)
        # and updates r alone (read r, A p; write r)
        out["pcg_apply_ap"] = 6 * s * N
        out["pcg_update_xr"] = 3 * s * N
        out["defect_correction"] = 20 * N
    return out


def read_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def read_traffic():
    """Per-launch DRAM bytes of kernel classes (FP64, 256^3) from the committed
    ncu summary (profiles/ncu_traffic.txt)."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    out = {}
    if os.path.exists(p):
        with open(p) as f:
            for line in f:
                line = line.strip()
                if not line or line.startswith("#"):
                    continue
                parts = line.split()
                if len(parts) >= 2:
                    try:
                        out[parts[0]] = float(parts[1])
                    except ValueError:
                        pass
    return out


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(prefix="clocks_", suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        if self.proc is None:
            return out
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax.append(float(parts[2]))
                except ValueError:
                    continue
                for name, val in zip(names, parts[5:9]):
                    if val.lower() == "active":
                        reasons.add(name)
        os.unlink(self.path)
        if sm:
            out = {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax),
                   "reasons": sorted(reasons), "samples": len(sm)}
        return out


def reduce_max(x, dist, device=None):
    """Max of a per-rank scalar over all ranks (identity without a process group)."""
    if dist is None or not dist.is_initialized():
        return x
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(steps_per_rank, elapsed_ms_max, world):
    """Whole-job steps/s of `world` independent replicas timed as the max over ranks."""
    return world * steps_per_rank / (elapsed_ms_max / 1000.0)


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


# ---------------------------------------------------------------------------
# CPU baseline (reference build or oracle port), bounded sample
# ---------------------------------------------------------------------------

def cpu_lib_path():
    ref = os.path.join(ROOT, "oracle", "_ref", "liborchard_ref.so")
    if os.path.exists(ref):
        return ref, "reference"
    return os.path.join(ROOT, "oracle", "liborchard_oracle.so"), "port"


def cpu_step_seconds(n_sample, steps=1):
    """Seconds per projection step of the CPU implementation at n_sample^3."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    path, kind = cpu_lib_path()
    lib = pyoracle.Oracle(path)
    cfg = pyoracle.steps_config(n_sample, n_sample, n_sample, NU, CFL, steps, TOL, MAX_IT)
    s = lib.tg_init(cfg, 0)
    t0 = time.perf_counter()
    lib.tg_steps(cfg, steps, s)
    return (time.perf_counter() - t0) / steps, kind


def cpu_baseline(n, n_sample=128):
    """A bounded sample (one step at n_sample^3, ~15 s on one core), extrapolated to
    n^3 by cell count.  The reference arm (--impl reference) measures n^3 itself."""
    sec, kind = cpu_step_seconds(n_sample, 1)
    scale = (n_sample / n) ** 3
    return {"value": scale / sec, "unit": "steps/s", "cores": 1, "kind": kind,
            "sample": f"1 FP64 step of Taylor-Green {n_sample}^3 (nu=1/1600, CFL 0.5, tol 1e-12) "
                      f"on 1 core took {sec:.2f} s; value EXTRAPOLATED to {n}^3 by cell count "
                      f"(x{(n / n_sample) ** 3:g}); bench.py --impl reference measures {n}^3 steps",
            "seconds_per_sample_step": sec, "extrapolated": True}


# Resident memory of one reference replica at 256^3 (the reference's state,
# its step's work fields and the MG hierarchy, plus this driver's copy of the
# state): 7.8 GB measured, scaled by cell count for other sizes.
REF_REPLICA_BYTES_256 = 7.9e9


def host_available_bytes():
    """Host memory this process may use: MemAvailable, capped by the cgroup limit."""
    avail = None
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    avail = int(line.split()[1]) * 1024
    except OSError:
        pass
    try:
        with open("/sys/fs/cgroup/memory.max") as f:
            lim = f.read().strip()
        if lim != "max":
            avail = min(avail or int(lim), int(lim))
    except OSError:
        pass
    return avail if avail is not None else 16 * 2 ** 30


def reference_config(n):
    """The workload's TaylorGreenConfig for the reference: the 200-step final time of
    the shipped 256^3 case, whose dt (the reference's T / ceil(T / dt_max) rule) is
    exactly the B200 arm's dt."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    return pyoracle.tg_config(n, n, n, NU, CFL, 200 * tg_dt(n), MAX_IT, TOL)


def _ref_replica(n, warm, timed, barrier, out):
    """One reference replica (spawned process): its own Taylor-Green state, `warm`
    untimed steps, then -- after every replica is ready -- `timed` steps of the
    reference's run_taylor_green_steps, one call per step."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    path, _ = cpu_lib_path()
    lib = pyoracle.Oracle(path)
    cfg = reference_config(n)
    assert lib.tg_dt(cfg) == tg_dt(n)
    s = lib.tg_init(cfg, 0)
    for _ in range(warm):
        s = lib.tg_steps(cfg, 1, s)
    barrier.wait()
    t0 = time.perf_counter()
    for _ in range(timed):
        s = lib.tg_steps(cfg, 1, s)
    t1 = time.perf_counter()
    out.put((t0, t1, timed, s.metrics["pressure_iterations"]))


def run_reference_arm(args, world, rank):
    """The reference's own CPU step of the same 256^3 workload on the host cores.

    The reference is single-threaded, so the K timed steps run as P independent
    replicas in parallel (P = K when memory allows, else as many as fit in half of
    the host's available memory, each replica taking its share of the K steps).
    Each replica first runs its own untimed warm-up steps (the first, Euler step
    included; together at least W), then all start their timed steps together;
    the timed region ends when the last replica finishes.  value = K / that wall
    time, so ms_per_step * K is the measured wall time of the K steps."""
    if rank != 0:
        return 0
    import multiprocessing as mp
    cores = os.cpu_count() or 1
    n = args.n
    per_replica = REF_REPLICA_BYTES_256 * (n / 256.0) ** 3
    fit = max(1, int(0.5 * host_available_bytes() // per_replica))
    P = max(1, min(args.steps, fit))
    timed = [args.steps // P + (1 if i < args.steps % P else 0) for i in range(P)]
    warm = max(1, -(-args.warmup // P))
    ctx = mp.get_context("spawn")
    barrier = ctx.Barrier(P)
    out = ctx.Queue()
    procs = [ctx.Process(target=_ref_replica, args=(n, warm, timed[i], barrier, out)) for i in range(P)]
    for p in procs:
        p.start()
    results = [out.get() for _ in range(P)]
    for p in procs:
        p.join()
    t0 = min(r[0] for r in results)
    t1 = max(r[1] for r in results)
    wall = t1 - t0
    value = args.steps / wall
    _, kind = cpu_lib_path()
    sample = (f"{args.steps} FP64 steps of Taylor-Green {n}^3 (nu=1/1600, CFL 0.5, dt = "
              f"{tg_dt(n):.17g}, tol 1e-12; the reference's own run_taylor_green_steps) as {P} "
              f"concurrent single-thread replicas on {cores} host cores "
              f"({max(timed)} timed steps on the busiest; {warm} warm-up step(s) each); "
              f"measured wall time of the {args.steps} steps {wall:.1f} s")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "steps/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * wall / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (analytic Taylor-Green initial state)",
        "config": workload_config(n, "fp64"),
        "pressure_iterations_last_step": results[0][3],
        "cpu_baseline": {"value": value, "unit": "steps/s", "cores": min(P, cores), "kind": kind,
                         "sample": sample},
        "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def workload_config(n, precision):
    """The `config` object of both arms' lines (the workload, not the implementation)."""
    return {"workload": f"taylor_green_3d_{n}", "n": n, "viscosity": NU, "cfl": CFL,
            "dt": tg_dt(n), "poisson_tolerance": TOL, "precision": precision,
            "parallelism": "replicas1", "l2": "every field > 126 MB L2; no flush"}


# ---------------------------------------------------------------------------
# B200 arm
# ---------------------------------------------------------------------------

def run_b200_arm(args, world, rank, local):
    import numpy as np
    import torch
    import solver_b200 as sb

    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    device = local

    n = args.n
    h = 2.0 * math.pi / n
    grid = sb.Grid(n, n, n, h, h, h)
    dt = tg_dt(n)
    precision = sb.OF_MIXED if args.precision == "mixed" else sb.OF_FP64
    ctx = sb.Context(grid, [sb.PERIODIC] * 6, device=device, precision=precision)
    prm = sb.step_params(NU, dt, MAX_IT, TOL)
    ctx.tg_init(NU, dt, mode=1)
    stream = torch.cuda.ExternalStream(sb.context_stream(ctx), device=device)

    def barrier():
        if dist is not None:
            t = torch.zeros(1, device=f"cuda:{device}")
            dist.all_reduce(t)
            torch.cuda.synchronize()

    def max_over_ranks(x):
        return reduce_max(x, dist, f"cuda:{device}")

    for _ in range(args.warmup):
        ctx.run_steps(prm, 1)

    # ---- timed region: K steps on the resident state (no instrumentation) ----
    sampler = ClockSampler(device)
    sb.profile_reset()
    barrier()
    torch.cuda.synchronize()
    sampler.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    metrics = ctx.run_steps(prm, args.steps)
    ev1.record(stream)
    ev1.synchronize()
    torch.cuda.synchronize()
    barrier()
    clocks = sampler.stop()
    counted = sb.profile_read()
    launches = sum(v[0] for v in counted.values())
    elapsed_ms = max_over_ranks(ev0.elapsed_time(ev1))
    value = replica_throughput(args.steps, elapsed_ms, world)

    # ---- per-kernel device times: the same steps replayed with every launch
    # bracketed by CUDA events on the context stream (kernels launched one by
    # one, so the event pairs see each kernel alone) ----
    replay_steps = max(1, min(args.steps, args.profile_steps))
    sb.profile_reset()
    sb.profile_enable(True)
    pr0 = torch.cuda.Event(enable_timing=True)
    pr1 = torch.cuda.Event(enable_timing=True)
    pr0.record(stream)
    ctx.run_steps(prm, replay_steps)
    pr1.record(stream)
    pr1.synchronize()
    sb.profile_enable(False)
    prof = sb.profile_read()
    replay_ms = pr0.elapsed_time(pr1)

    # ---- roofline of the dominant kernel class ----
    bpl = bytes_per_launch(n, args.precision)
    timed = {k: v for k, v in prof.items() if v[1] > 0 and k in bpl}
    dom = max(timed, key=lambda k: timed[k][2])
    dom_launches, dom_timed, dom_ms = timed[dom]
    avg_s = dom_ms / dom_timed / 1000.0
    achieved = bpl[dom] / avg_s / 1e9
    peak, peak_kind = read_peaks()
    # the committed ncu figures are for the FP64 256^3 workload
    traffic = read_traffic().get(dom) if (args.precision == "fp64" and n == 256) else None
    step_bytes = sum(bpl[k] * v[0] for k, v in prof.items() if k in bpl) / replay_steps
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                "traffic": traffic, "algorithmic_bytes_per_launch": bpl[dom],
                "avg_launch_us": avg_s * 1e6, "launches_per_step": dom_launches / replay_steps,
                "share_of_replay": dom_ms / replay_ms,
                "timing": "CUDA events around each launch, instrumented replay of "
                          f"{replay_steps} of the timed steps"}
    step_hbm = {"algorithmic_bytes_per_step": step_bytes,
                "achieved_gbs": step_bytes / (elapsed_ms / args.steps / 1000.0) / 1e9,
                "frac": step_bytes / (elapsed_ms / args.steps / 1000.0) / 1e9 / peak}
    kernels = {k: {"launches_per_step": v[0] / replay_steps, "ms_per_step": round(v[2] / replay_steps, 4)}
               for k, v in prof.items() if v[0]}
    # The coarse levels are ~13 kernels of a few microseconds per V-cycle: in
    # the host-driven replay their time is set by the host's launch rate, so
    # they are timed as the product runs them, a CUDA graph of the chain
    # replayed on the device (of_profile_coarse_chain).
    coarse = kernels.get("vcycle_coarse_levels")
    if coarse and args.chain_reps > 0:
        chain_us, chain_launches = sb.profile_coarse_chain(ctx, reps=args.chain_reps)
        if chain_launches:
            vcycles = coarse["launches_per_step"] / chain_launches
            coarse["ms_per_step_host_loop"] = coarse["ms_per_step"]
            coarse["ms_per_step"] = round(chain_us * vcycles / 1000.0, 4)
            coarse["us_per_vcycle"] = round(chain_us, 2)
            coarse["launches_per_vcycle"] = chain_launches
            coarse["timing"] = (f"CUDA graph of one coarse-level chain replayed {args.chain_reps} times, "
                                "times the V-cycles per step; ms_per_step_host_loop is the "
                                "per-launch event timing of the host-driven replay")

    # ---- e2e: the C-ABI step call with host state in pinned memory ----
    st = ctx.download_state()
    pinned = {}
    for k in ("u", "v", "w", "adv_u", "adv_v", "adv_w", "p"):
        t = torch.empty(st[k].shape, dtype=torch.float64, pin_memory=True)
        t.numpy()[...] = st[k]
        pinned[k] = t.numpy()
    state_bytes = sum(a.nbytes for a in pinned.values())
    e2e_steps = max(1, min(args.steps, args.e2e_steps))
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    pinned["has_previous_advection"] = 1
    pinned["metrics"] = st["metrics"]
    for _ in range(e2e_steps):
        ctx.step_host(prm, pinned)
    e1.record(stream)
    e1.synchronize()
    barrier()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1))
    e2e_value = replica_throughput(e2e_steps, e2e_ms, world)

    line = {
        "metric": METRIC if args.precision == "fp64" else METRIC.replace("FP64", "mixed FP32/FP64"),
        "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": elapsed_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f64+f32",
        "data": "synthetic (analytic Taylor-Green initial state)",
        "config": dict(workload_config(n, args.precision), parallelism=f"replicas{world}"),
        "pressure_iterations_last_step": metrics["pressure_iterations"],
        "roofline": roofline,
        "step_hbm": step_hbm,
        "e2e": {"value": e2e_value, "unit": "steps/s", "h2d_bytes_per_step": state_bytes,
                "d2h_bytes_per_step": state_bytes,
                "note": "per step: of_step_host on pinned host state (upload, one step, download; "
                        "the AB2 history is copied back while the pressure solve runs)"},
        "gpu_launches": launches,
        "clocks": clocks,
        "kernels": kernels,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(n, args.cpu_sample_n)
    if world == 1 and args.precision == "fp64" and not args.no_extras:
        ctx.close()
        line["mixed"] = mixed_extra(n, dt, args, value)
        line["adjoint"] = adjoint_extra()
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist is not None:
        barrier()
        dist.destroy_process_group()
    return 0


def timed_steps(ctx, prm, steps, stream):
    """Device time (ms) of `steps` resident steps, CUDA events on the context stream."""
    import torch
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    ctx.run_steps(prm, steps)
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1)


def mixed_extra(n, dt, args, fp64_value, error_steps=200):
    """The mixed path on the same workload: steps/s (same timing as the main
    line), the speed-up over the FP64 value, and the max-norm relative
    velocity difference from the FP64 path after `error_steps` steps from the
    same initial state."""
    import numpy as np
    import torch
    import solver_b200 as sb
    h = 2.0 * math.pi / n
    grid = sb.Grid(n, n, n, h, h, h)
    prm = sb.step_params(NU, dt, MAX_IT, TOL)
    out = {}
    with sb.Context(grid, [sb.PERIODIC] * 6, precision=sb.OF_MIXED) as ctx:
        stream = torch.cuda.ExternalStream(sb.context_stream(ctx))
        ctx.tg_init(NU, dt, mode=1)
        for _ in range(args.warmup):
            ctx.run_steps(prm, 1)
        ms = timed_steps(ctx, prm, args.steps, stream)
        out["value"] = args.steps / (ms / 1000.0)
        out["unit"] = "steps/s"
        out["speedup_vs_fp64"] = out["value"] / fp64_value
        ctx.tg_init(NU, dt, mode=1)
        ctx.run_steps(prm, error_steps)
        mixed = ctx.download_state()
    with sb.Context(grid, [sb.PERIODIC] * 6) as ctx:
        ctx.tg_init(NU, dt, mode=1)
        ctx.run_steps(prm, error_steps)
        ref = ctx.download_state()
    err = max(float(np.max(np.abs(mixed[c][1:-1, 1:-1, 1:-1] - ref[c][1:-1, 1:-1, 1:-1])))
              for c in "uvw") / max(float(np.max(np.abs(ref[c][1:-1, 1:-1, 1:-1]))) for c in "uvw")
    out["rel_velocity_error_vs_fp64"] = err
    out["error_steps"] = error_steps
    out["precision"] = "FP64 defect correction (residual, update, convergence, mean removal) around an FP32 MG-PCG (V-cycle and CG vectors: FP32 storage and arithmetic)"
    return out


def adjoint_extra(n=128, steps=100, every=10, viscosity=0.01):
    """The adjoint check workload: Taylor-Green plus a seeded solenoidal
    perturbation (Fourier modes |k| <= 4, RMS 1e-2, projected), loss
    1/2 |u(T) - u_target|^2 with the target from another seed's forward run,
    `steps` steps, checkpoint every `every`.  Reports the adjoint/forward
    device-time ratio and a central-difference check of the gradient along a
    smooth direction (eps = 1e-8)."""
    import numpy as np
    import torch
    import solver_b200 as sb
    from solver_b200.adjoint import perturbed_taylor_green, smooth_field, unique_loss, upload_initial
    h = 2.0 * math.pi / n
    grid = sb.Grid(n, n, n, h, h, h)
    dt = tg_dt(n)
    prm = sb.step_params(viscosity, dt, MAX_IT, TOL)
    with sb.Context(grid, [sb.PERIODIC] * 6) as ctx:
        stream = torch.cuda.ExternalStream(sb.context_stream(ctx))
        state = perturbed_taylor_green(ctx, viscosity, dt, seed=1)
        other = perturbed_taylor_green(ctx, viscosity, dt, seed=2)
        upload_initial(ctx, other)
        ctx.run_steps(prm, steps)
        tst = ctx.download_state()
        target = [tst[c] for c in "uvw"]
        upload_initial(ctx, state)
        ctx.run_steps(prm, 2)
        upload_initial(ctx, state)
        fwd_ms = timed_steps(ctx, prm, steps, stream)
        upload_initial(ctx, state)
        grad, info = ctx.adjoint_gradient(prm, steps, target, checkpoint_every=every)
        d = smooth_field(grid, 5)
        eps = 1e-8
        loss = []
        for sgn in (1.0, -1.0):
            upload_initial(ctx, (state[0] + sgn * eps * d[0], state[1] + sgn * eps * d[1],
                                 state[2] + sgn * eps * d[2], state[3]))
            ctx.run_steps(prm, steps)
            st = ctx.download_state()
            loss.append(unique_loss([st[c] for c in "uvw"], target))
        fd = (loss[0] - loss[1]) / (2 * eps)
        ad = sum(float(np.sum(d[i][1:-1, 1:-1, 1:-1] * grad[i][1:-1, 1:-1, 1:-1])) for i in range(3))
    return {"workload": f"taylor_green_3d_{n}_perturbed", "steps": steps, "checkpoint_every": every,
            "viscosity": viscosity, "forward_ms": fwd_ms,
            "adjoint_ms": info["forward_ms"] + info["backward_ms"],
            "ratio_adjoint_over_forward": (info["forward_ms"] + info["backward_ms"]) / fwd_ms,
            "forward_steps_run": info["forward_steps"], "loss": info["loss"],
            "grad_viscosity": info["grad_viscosity"],
            "fd_check": {"direction": "smooth, |k| <= 4", "eps": eps, "fd": fd, "adjoint": ad,
                         "rel_error": abs(fd - ad) / abs(fd)},
            "device_bytes": info["device_bytes"],
            "timing": "CUDA events; adjoint = first forward pass + segment recomputation + reverse steps"}


def adjoint_long(n=512, steps=400, check_n=256, viscosity=NU, snapshots=0):
    """The long-horizon adjoint workload: Taylor-Green at Re 1600 on n^3 plus
    the seeded solenoidal perturbation (seed 1; |k| <= 4, RMS 1e-2,
    projected), `steps` steps at CFL 0.5, loss 1/2 |u(T) - u_target|^2 with the
    target from the seed-2 forward run; mixed-precision forward and adjoint
    with the binomial checkpoint schedule sized to the device memory.  Reports
    forward steps/s, the adjoint/forward device-time ratio, the snapshots and
    the device memory in use; then, on check_n^3 over the same final time,
    the mixed-precision gradient against the FP64 adjoint gradient."""
    import numpy as np
    import psutil
    import solver_b200 as sb
    from solver_b200.adjoint import perturbed_taylor_green, upload_initial

    # the host side holds about 30 padded fields at the largest size
    need = 30 * 8 * (n + 3) ** 3
    avail = psutil.virtual_memory().available
    if avail < 2 * need:
        raise RuntimeError(f"adjoint_long: {avail / 1e9:.0f} GB of host memory available, "
                           f"{2 * need / 1e9:.0f} GB wanted")

    def case(size, nsteps, precision):
        h = 2.0 * math.pi / size
        ctx = sb.Context(sb.Grid(size, size, size, h, h, h), [sb.PERIODIC] * 6, precision=precision)
        dt = tg_dt(size)
        prm = sb.step_params(viscosity, dt, MAX_IT, TOL)
        state = perturbed_taylor_green(ctx, viscosity, dt, seed=1)
        other = perturbed_taylor_green(ctx, viscosity, dt, seed=2)
        upload_initial(ctx, other)
        t0 = time.perf_counter()
        ctx.run_steps(prm, nsteps)
        target_s = time.perf_counter() - t0
        tst = ctx.download_state()
        target = [tst[c] for c in "uvw"]
        del tst, other
        return ctx, prm, state, target, target_s

    ctx, prm, state, target, target_s = case(n, steps, sb.OF_MIXED)
    upload_initial(ctx, state)
    del state
    _, info = ctx.adjoint_gradient_binomial(prm, steps, target, snapshots=snapshots)
    ctx_bytes = ctx.device_bytes()
    ctx.close()
    del target
    fwd_ms = info["forward_ms"]
    total_ms = info["forward_ms"] + info["backward_ms"]
    dt = prm.dt
    check_steps = steps * check_n // n
    ctx, prm, state, target, _ = case(check_n, check_steps, sb.OF_FP64)
    upload_initial(ctx, state)
    g64, i64 = ctx.adjoint_gradient_binomial(prm, check_steps, target)
    ctx.set_precision(sb.OF_MIXED)
    upload_initial(ctx, state)
    g32, i32 = ctx.adjoint_gradient_binomial(prm, check_steps, target)
    ctx.close()
    gmax = max(float(np.max(np.abs(a))) for a in g64)
    gerr = max(float(np.max(np.abs(a - b))) for a, b in zip(g32, g64)) / gmax
    return {
        "metric": f"adjoint/forward time ratio, Taylor-Green {n}^3 Re 1600, {steps} steps, mixed",
        "value": total_ms / fwd_ms, "unit": "x", "higher_is_better": False, "n_gpus": 1,
        "dtype": "f64+f32", "data": "synthetic (Taylor-Green + seeded solenoidal perturbation)",
        "config": {"workload": f"taylor_green_3d_{n}_adjoint", "n": n, "steps": steps,
                   "viscosity": viscosity, "dt": dt, "poisson_tolerance": TOL,
                   "perturbation": "seed 1, |k| <= 4, RMS 1e-2; target: seed 2 forward run",
                   "schedule": "binomial (optimal revolve), snapshots sized to device memory"},
        "forward_steps_per_s": steps / (fwd_ms / 1000.0),
        "forward_ms": fwd_ms, "adjoint_total_ms": total_ms,
        "target_run_wall_s": target_s,
        "snapshots": info["snapshots"], "forward_steps_run": info["forward_steps"],
        "loss": info["loss"], "grad_viscosity": info["grad_viscosity"],
        "device_bytes_context": ctx_bytes, "device_bytes_adjoint": info["device_bytes"],
        "device_bytes_in_use": info["device_bytes_in_use"],
        "check": {"n": check_n, "steps": check_steps,
                  "mixed_vs_fp64_gradient_rel_maxnorm": gerr,
                  "mixed_vs_fp64_grad_viscosity_rel": abs(i32["grad_viscosity"] - i64["grad_viscosity"])
                  / abs(i64["grad_viscosity"]),
                  "fp64_snapshots": i64["snapshots"], "fp64_forward_steps_run": i64["forward_steps"],
                  "fp64_ratio": (i64["forward_ms"] + i64["backward_ms"]) / i64["forward_ms"]},
        "timing": "CUDA events inside the adjoint call: forward = its first pass over the steps "
                  "(plain steps plus snapshot copies); total = that pass + recomputation + reverse steps",
    }


def main():
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--n", type=int, default=N_DEFAULT)
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--profile-steps", type=int, default=2)
    ap.add_argument("--chain-reps", type=int, default=200,
                    help="graph replays of the coarse-level chain for its device time (0: skip)")
    ap.add_argument("--cpu-sample-n", type=int, default=None)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the mixed-precision and adjoint measurements of the FP64 1-GPU line")
    ap.add_argument("--adjoint-long", action="store_true",
                    help="run the long-horizon adjoint workload (512^3, 400 steps, mixed; "
                         "minutes of GPU time) instead of the step benchmark")
    args = ap.parse_args()
    if args.adjoint_long:
        print(json.dumps(adjoint_long()), flush=True)
        return 0
    if args.warmup < 3:
        ap.error("--warmup must be at least 3")
    if args.cpu_sample_n is None:
        args.cpu_sample_n = 128
    world, rank, local = dist_setup()
    if args.impl == "reference":
        return run_reference_arm(args, world, rank)
    return run_b200_arm(args, world, rank, local)


if __name__ == "__main__":
    sys.exit(main())
