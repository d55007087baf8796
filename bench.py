#!/usr/bin/env python3
"""Benchmark of the ocean-core time step on B200.

Workload: the seeded seamount basin (512 x 512 x 50 cells, 2000 km square,
closed, stretched levels 10 -> 250 m, double-gyre wind, TKE closure, TVD3
advection, polyTEOS10 EOS, theta = 0.6 with the multigrid Helmholtz solver,
dt = 600 s). A "step" is one model time step over the whole grid.

Prints one JSON line. ``value`` is cell-steps/s of the device-resident state
(all ranks, max-over-ranks device time, CUDA events on the launching stream,
the steps replayed as recorded two-step CUDA graphs). ``kernels`` and
``roofline`` come from a second timed region of plain launches with CUDA
events around every launch: the dominant kernel's algorithmic bandwidth
against the measured HBM peak. ``e2e`` is the same metric through the C ABI
with pinned host buffers: every step uploads a full state, steps it and
downloads it, three independent states taking turns so that copies overlap
steps (``e2e.sequential``: one state, every copy waiting). ``cpu_baseline``
times the CPU oracle (a NumPy port, bit-identical to the reference's NumPy
stepper) on a bounded sample of the same recipe.

Multi-GPU: replicas only (the theta step does not shard); each rank advances
its own replica, ``scaling`` is "weak".

``--impl reference`` times the reference's own CPU implementation of the path
(its NumPy stepper, as the bit-identical port) on the host's cores instead: one
single-threaded replica per usable core, started together, on a bounded sample.
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
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "cell-steps/s fp64 vs mixed (≤1e-6 rel L2 vs fp64); adjoint/forward time ratio"
UNIT = "cell-steps/s"
HBM_FALLBACK_GBS = 6650.0


# ------------------------------------------------------------------ helpers
def env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


def record_dir():
    """Directory for the raw clock samples (OCEAN_B200_RECORD_DIR), if it names one."""
    d = os.environ.get("OCEAN_B200_RECORD_DIR")
    return Path(d) if d and Path(d).is_dir() else None


def measured_hbm_peak():
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        try:
            return float(json.loads(path.read_text())["hbm_gbs"]), "measured"
        except (KeyError, ValueError):
            pass
    return HBM_FALLBACK_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int, path: Path | None = None):
        self.gpu = gpu_index
        self.rows: list[list[str]] = []
        self.proc = None
        self.path = path

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", str(self.gpu)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (FileNotFoundError, OSError):
            self.proc = None
        time.sleep(0.3)

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.2)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        if self.path is not None:
            self.path.write_text("\n".join(",".join(r) for r in self.rows) + "\n")
        sm, smax, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                smax.append(float(r[2]))
                power.append(float(r[3]))
            except ValueError:
                continue
            for n, flag in zip(names, r[5:9]):
                if flag.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "power_w_max": max(power) if power else None,
                "samples": len(sm), "reasons": sorted(reasons)}


# ------------------------------------------------------------------ algorithmic bytes
# Per-launch algorithmic bytes of each kernel class: every logical array access
# counted once (fp64, 8 B), static geometry excluded.
ACCESSES_PER_CELL = {
    "closure": 10,          # reads u, v, b, e, K_m, K_h; writes e, K_m, K_h, q
    "mom_explicit": 14,     # reads u, v, b, phi, w, K_m; writes 8 explicit-term fields
    "predictor_rhs": 14,    # reads u, v, u_it, v_it, 8 explicit terms; writes r_u, r_v
    "momentum_solve": 5,    # reads r_u, r_v, K_m; writes gh_u, gh_v
    "tracer_rhs": 8,        # reads T, S, u, v, w, K_h; writes r_T, r_S
    "tracer_solve": 6,      # reads r_T, r_S, K_h; writes T, S, b
    "backsub": 5,           # reads gh_u, gh_v, q; writes u, v
    "wcol": 3,              # reads u, v; writes w
    "phi": 2,               # reads b; writes phi
    "transport": 2,         # reads u, v
    "kukv": 1,              # reads q
}


def mg_level_cells(nx, ny, min_size=8):
    cells = [nx * ny]
    while nx % 2 == 0 and ny % 2 == 0 and nx // 2 >= min_size and ny // 2 >= min_size:
        nx, ny = nx // 2, ny // 2
        cells.append(nx * ny)
    return cells


def helm_bytes_per_iteration(p):
    """Algorithmic bytes of one Helmholtz iteration: PCG-Jacobi 15 arrays per
    column, MG V(2,2) 32 arrays per cell of every level plus 4 fine arrays for the
    residual check, MG-preconditioned CG the V-cycle plus 13 fine arrays (A p, the
    updates of x, r, p and the copies around the cycle)."""
    n0 = p.nx * p.ny
    if p.solver_kind == "multigrid":
        return 8 * (32 * sum(mg_level_cells(p.nx, p.ny)) + 4 * n0)
    if p.solver_kind == "pcg_mg":
        return 8 * (32 * sum(mg_level_cells(p.nx, p.ny)) + 13 * n0)
    return 8 * 15 * n0


def step_algorithmic_bytes(p, iterations_per_step, word=8):
    """Minimal-pass bytes of one step (44 or 29 accesses per cell + the solver).

    word = 4 counts the mixed-precision step: its 3D fields are FP32, except the
    buoyancy b, whose accesses (read by the closure and both predictor passes,
    written by the tracer pass; 3 without the closure) stay 8 B, as do the
    solver's 2D arrays."""
    n3 = p.nx * p.ny * p.nz
    a3 = 44 if p.closure == "tke" else 29
    nb = 0 if word == 8 else (4 if p.closure == "tke" else 3)
    return (word * (a3 - nb) + 8 * nb) * n3 + helm_bytes_per_iteration(p) * iterations_per_step


def dram_traffic_from_profiles(kernel: str):
    """DRAM bytes per launch of `kernel` from the committed ncu summary, if any."""
    for path in sorted((ROOT / "profiles").glob("*.md")):
        for line in path.read_text().splitlines():
            key = f"dram_bytes_per_launch[{kernel}]"
            if line.strip().startswith(key):
                try:
                    return float(line.split("=", 1)[1].split()[0])
                except (IndexError, ValueError):
                    return None
    return None


# ------------------------------------------------------------------ workloads
def workload(args):
    from hydrostatic_ocean_core_benchmark_b200 import cases
    over = {} if args.rtol is None else {"rtol": args.rtol}
    return cases.seamount_basin(nx=args.nx, ny=args.ny, nz=args.nz, seed=args.seed, dt=args.dt, **over)


def cpu_oracle_rate(args, steps: int, warmup: int):
    """cell-steps/s of the CPU oracle on a bounded sample of the same recipe."""
    import numpy as np

    from hydrostatic_ocean_core_benchmark_b200 import cases
    from oracle import ocean_oracle as orc
    s = cases.seamount_basin(nx=args.cpu_nx, ny=args.cpu_nx, nz=args.nz, seed=args.seed)
    p = s.params
    geo = orc.Geometry(p, s.H, s.mask, s.dzr)
    b = orc.buoyancy(p.eos, s.T, s.S, geo.zc, p.g, p.rho0, p.alpha_t, p.beta_s, p.t0, p.s0) * geo.mask3
    st = orc.OracleStepper(p, s.H, s.mask, dzr=s.dzr, taux_c=s.taux_c, tauy_c=s.tauy_c)
    state = orc.OracleState(s.u, s.v, b, s.eta, s.T, s.S)
    for _ in range(warmup):
        state = st.step(state)
    t0 = time.perf_counter()
    for _ in range(steps):
        state = st.step(state)
    dt = time.perf_counter() - t0
    cells = p.nx * p.ny * p.nz
    assert np.all(np.isfinite(state.eta))
    return cells * steps / dt, dt, p


def host_cpu() -> dict:
    """The host's logical core count and CPU model, recorded beside a CPU rate."""
    model = "unknown"
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.lower().startswith("model name"):
                model = ln.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    try:
        usable = len(os.sched_getaffinity(0))
    except AttributeError:
        usable = os.cpu_count()
    return {"nproc": os.cpu_count(), "usable": usable, "cpu_model": model}


def reference_sample_nx(args, budget_s=150.0) -> int:
    """Largest sample (columns per side) whose W + K oracle steps fit the budget."""
    per_step_64 = 1.1 * args.nz / 50.0          # seconds per step at 64 x 64 columns
    for nx in (128, 96, 64, 48, 32, 16):
        if per_step_64 * (nx / 64.0) ** 2 * (args.steps + args.warmup) <= budget_s:
            return nx
    return 16


def _oracle_replica(cpu_nx, nz, seed, steps, warmup, barrier, out):
    """One replica of the CPU oracle, in a process of its own: the warm-up steps,
    a start common to all replicas, then the timed steps on the host's monotonic
    clock (the same clock in every process)."""
    import numpy as np

    from hydrostatic_ocean_core_benchmark_b200 import cases
    from oracle import ocean_oracle as orc
    s = cases.seamount_basin(nx=cpu_nx, ny=cpu_nx, nz=nz, seed=seed)
    p = s.params
    geo = orc.Geometry(p, s.H, s.mask, s.dzr)
    b = orc.buoyancy(p.eos, s.T, s.S, geo.zc, p.g, p.rho0, p.alpha_t, p.beta_s, p.t0, p.s0) * geo.mask3
    st = orc.OracleStepper(p, s.H, s.mask, dzr=s.dzr, taux_c=s.taux_c, tauy_c=s.tauy_c)
    state = orc.OracleState(s.u, s.v, b, s.eta, s.T, s.S)
    for _ in range(warmup):
        state = st.step(state)
    try:
        barrier.wait(timeout=1800)
    except Exception:  # another replica failed before the start
        out.put(None)
        return
    t0 = time.monotonic()
    for _ in range(steps):
        state = st.step(state)
    t1 = time.monotonic()
    out.put((t0, t1, bool(np.all(np.isfinite(state.eta)))))


def oracle_replicas(args) -> int:
    """Replicas of the CPU oracle the host can run at once: one per usable core,
    within half the available memory (about 200 MB per 64 x 64 x 50 sample)."""
    cores = host_cpu()["usable"] or 1
    per_replica = 200e6 * (args.cpu_nx / 64.0) ** 2 * args.nz / 50.0
    avail = None
    try:
        for ln in open("/proc/meminfo"):
            if ln.startswith("MemAvailable:"):
                avail = float(ln.split()[1]) * 1024.0
                break
    except OSError:
        pass
    by_mem = int(0.5 * avail / per_replica) if avail else cores
    return max(1, min(cores, by_mem, 128))


def cpu_oracle_rate_parallel(args, steps: int, warmup: int, replicas: int):
    """cell-steps/s of `replicas` independent CPU oracles on the same bounded sample,
    each single-threaded in a spawned process, timed from the common start to the
    last replica's end. Returns (aggregate rate, seconds, median replica rate)."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    barrier = ctx.Barrier(replicas)
    out = ctx.Queue()
    keys = ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS")
    saved = {k: os.environ.get(k) for k in keys}
    os.environ.update({k: "1" for k in keys})  # one thread per replica (the children inherit it)
    procs = [ctx.Process(target=_oracle_replica, args=(args.cpu_nx, args.nz, args.seed, steps, warmup, barrier, out))
             for _ in range(replicas)]
    try:
        for pr in procs:
            pr.start()
    finally:
        for k, v in saved.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    res = []
    while len(res) < replicas:
        try:
            res.append(out.get(timeout=10))
        except Exception:  # queue.Empty: every replica still alive keeps the wait going
            if not any(pr.is_alive() for pr in procs):
                break
    for pr in procs:
        pr.join(timeout=60)
    if len(res) < replicas or any(r is None or not r[2] for r in res):
        raise RuntimeError(f"CPU oracle replicas failed ({len(res)} of {replicas} reported)")
    span = max(r[1] for r in res) - min(r[0] for r in res)
    cells = args.cpu_nx * args.cpu_nx * args.nz
    single = statistics.median(cells * steps / (r[1] - r[0]) for r in res)
    return replicas * cells * steps / span, span, single


def run_reference_arm(args, rank):
    """The reference arm: the CPU oracle (a bit-identical NumPy port of the
    reference's stepper) on every usable host core, one single-threaded replica
    per core, on a bounded sample of the workload."""
    if rank != 0:
        return 0
    # a single replica's W + K steps fit ~90 s; sharing the host's memory bandwidth
    # slows each replica (1.4x with 8 replicas on an 8-core host)
    args.cpu_nx = min(args.cpu_nx, reference_sample_nx(args, budget_s=90.0))
    replicas = oracle_replicas(args)
    rate, secs, single = cpu_oracle_rate_parallel(args, args.steps, args.warmup, replicas)
    n = args.cpu_nx
    sample = (f"{replicas} replicas (one per usable host core, single-threaded NumPy each) of the "
              f"seamount-basin recipe at {n}x{n}x{args.nz} (same physics, solver and seed as the "
              f"{args.nx}x{args.ny}x{args.nz} workload), {args.warmup} warm-up + {args.steps} timed "
              f"steps each; {secs:.1f} s from the common start to the last replica's end; "
              f"{single:.4g} cell-steps/s per replica (median)")
    line = {"impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * secs / max(1, args.steps), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"seamount_basin {args.nx}x{args.ny}x{args.nz}",
                       "sample": f"{n}x{n}x{args.nz}", "replicas": replicas},
            "cpu_baseline": {"value": rate, "unit": UNIT, "cores": replicas, "kind": "port",
                             "sample": sample, "host": host_cpu(), "per_core_value": single},
            "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ mixed precision
MIXED_FIELDS = ("eta", "u", "v", "b", "T", "S", "e", "km", "kh")


def precision_leg(s, local_rank, steps, warmup, time_fp64=False, mixed_solver="configured"):
    """The mixed-precision step beside the fp64 one on the same initial state.

    Both advance warmup + steps steps (two-step CUDA graphs) from the state of
    the seeded recipe; the mixed path's last `steps` are timed with CUDA events
    on the launching stream (and the fp64 path's too with time_fp64). Returns
    the rates, the relative L2 error of every field against the fp64 path (which
    is bit-identical to the reference), and the multigrid cycle counts."""
    import torch

    from hydrostatic_ocean_core_benchmark_b200.stepper import OceanStepper
    p = s.params
    n3 = p.nx * p.ny * p.nz
    out, rate, ms, logs = {}, {}, {}, {}
    stream = torch.cuda.Stream(device=local_rank)
    for prec in ("fp64", "mixed"):
        pp = p if prec == "fp64" or mixed_solver == "configured" else p.replace(solver_kind=mixed_solver)
        st = OceanStepper(pp, s.H, s.mask, dzr=s.dzr, taux_c=s.taux_c, tauy_c=s.tauy_c, device=local_rank,
                          precision=prec)
        st.set_state(eta=s.eta, u=s.u, v=s.v, T=s.T, S=s.S)
        st.step(warmup, stream=stream, graph=True)
        stream.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        st.step(steps, stream=stream, graph=True)
        e1.record(stream)
        e1.synchronize()
        ms[prec] = e0.elapsed_time(e1) / steps
        rate[prec] = n3 / (ms[prec] / 1e3)
        stats = st.stats()
        if stats["solver_failures"] or stats["diverged"]:
            raise RuntimeError(f"{prec} run failed: {stats}")
        logs[prec] = st.solve_log()
        shapes = {"eta": st.shape2, "e": st.shapei, "km": st.shapei, "kh": st.shapei}
        o = {f: torch.empty(shapes.get(f, st.shape3), dtype=torch.float64, device=f"cuda:{local_rank}")
             for f in MIXED_FIELDS}
        st.get_state(out=o)
        out[prec] = o
        st.close()
    rel = {}
    for f in MIXED_FIELDS:
        a, b = out["mixed"][f], out["fp64"][f]
        den = float(torch.linalg.vector_norm(b))
        rel[f] = float(torch.linalg.vector_norm(a - b)) / den if den > 0 else float(torch.linalg.vector_norm(a))
    la, lb = logs["fp64"], logs["mixed"]
    msolver = p.solver_kind if mixed_solver == "configured" else mixed_solver
    leg = {"steps": warmup + steps, "timed_steps": steps, "ms_per_step": ms["mixed"], "value": rate["mixed"],
           "unit": UNIT, "rel_l2_vs_fp64": rel, "worst_field": max(rel, key=rel.get),
           "solvers": {"fp64": p.solver_kind, "mixed": msolver},
           "solver_iterations": {"fp64": sum(la), "mixed": sum(lb), "solves": len(lb)}}
    if msolver == p.solver_kind:
        leg["solver_iterations"]["max_per_solve_difference"] = max((abs(x - y) for x, y in zip(la, lb)), default=0)
    # minimal-pass bytes of a step over its measured time, the solve's iterations
    # averaged over every step of the run (FP32 3D fields on the mixed path)
    peak, src = measured_hbm_peak()

    def step_roofline(pp, log, step_ms, word):
        bstep = step_algorithmic_bytes(pp, sum(log) / (warmup + steps), word=word)
        gbs = bstep / (step_ms / 1e3) / 1e9
        return {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s", "frac": gbs / peak,
                "peak_source": src, "algorithmic_bytes_per_step": bstep}

    if time_fp64:
        leg["fp64"] = {"ms_per_step": ms["fp64"], "value": rate["fp64"],
                       "step_roofline": step_roofline(p, la, ms["fp64"], 8)}
        leg["speedup_vs_fp64"] = ms["fp64"] / ms["mixed"]
    if msolver in ("multigrid", "pcg_mg", "pcg_jacobi"):
        pm = p if msolver == p.solver_kind else p.replace(solver_kind=msolver)
        leg["step_roofline"] = step_roofline(pm, lb, ms["mixed"], 4)
    del out
    torch.cuda.empty_cache()
    return leg


def run_precision(args, rank, world, local_rank):
    """--workload precision: the benchmark's precision form (the seamount recipe
    at 1024 x 1024 x 64, 100 steps), fp64 beside mixed on one GPU."""
    import torch
    torch.cuda.set_device(local_rank)
    if rank != 0:
        return 0
    s = workload(args)
    p = s.params
    leg = precision_leg(s, local_rank, args.steps, args.warmup, time_fp64=True, mixed_solver=args.mixed_solver)
    line = {"metric": "cell-steps/s, mixed FP32/FP64 step vs fp64 (rel L2 vs fp64 per field)",
            "value": leg["value"], "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": leg["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 (3D state and stencils) + f64 (b, pressure gradient, EOS, eta, Helmholtz)",
            "data": "synthetic (seeded seamount-basin recipe)",
            "config": {"workload": f"seamount_basin {p.nx}x{p.ny}x{p.nz}, TKE + TVD3 + polyTEOS10, "
                                   f"theta={p.theta:g} + {p.solver_kind} at rtol {p.rtol:g}, dt={p.dt:g} s",
                       "cells": p.nx * p.ny * p.nz, "rtol": p.rtol, "variant": "precision form (mixed vs fp64)"},
            "fp64": leg["fp64"], "speedup_vs_fp64": leg["speedup_vs_fp64"],
            "step_roofline": leg.get("step_roofline"),
            "rel_l2_vs_fp64": leg["rel_l2_vs_fp64"], "solvers": leg["solvers"],
            "solver_iterations": leg["solver_iterations"]}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ our arm
def run_ours(args, rank, world, local_rank):
    import numpy as np
    import torch

    from hydrostatic_ocean_core_benchmark_b200.stepper import OceanStepper

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device(f"cuda:{local_rank}"))

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if dist is None:
            return x
        t = torch.tensor([x], device=f"cuda:{local_rank}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    s = workload(args)
    p = s.params
    n3 = p.nx * p.ny * p.nz
    n2 = p.nx * p.ny
    n3i = n2 * (p.nz + 1)
    st = OceanStepper(p, s.H, s.mask, dzr=s.dzr, taux_c=s.taux_c, tauy_c=s.tauy_c,
                      device=local_rank)
    st.set_state(eta=s.eta, u=s.u, v=s.v, T=s.T, S=s.S)
    stream = torch.cuda.Stream(device=local_rank)
    graph = not args.no_graph
    # warm-up; with graphs, two more steps record the graph of the buffer the
    # timed region starts from, so no recording happens inside it
    st.step(args.warmup, stream=stream, graph=graph)
    if graph:
        st.step(2, stream=stream, graph=True)
    stream.synchronize()
    st.stats()
    log0 = len(st.solve_log())
    launches0 = st.stats()["kernel_launches"]
    # timed region: device-resident state, events on the launching stream; the
    # steps replay the recorded two-step CUDA graphs (oc_step_graph)
    out_dir = record_dir()
    clocks = ClockSampler(local_rank, out_dir / f"clocks_rank{rank}.csv" if out_dir else None)
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    ev0.record(stream)
    st.step(args.steps, stream=stream, graph=graph)
    ev1.record(stream)
    ev1.synchronize()
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    ms_max = max_over_ranks(ms)
    launches = st.stats()["kernel_launches"] - launches0
    # per-kernel timed region: the same steps launched one by one with CUDA events
    # around every launch on the launching stream (oc_set_profiling); these give
    # the kernel shares and the roofline's per-launch durations
    st.kernel_times()
    st.set_profiling(True)
    pv0 = torch.cuda.Event(enable_timing=True)
    pv1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    pv0.record(stream)
    st.step(args.profile_steps, stream=stream)
    pv1.record(stream)
    pv1.synchronize()
    st.set_profiling(False)
    ms_prof = max_over_ranks(pv0.elapsed_time(pv1))
    ktimes = st.kernel_times()
    stats = st.stats()
    log = st.solve_log()[log0:]
    if stats["solver_failures"] or stats["diverged"]:
        raise RuntimeError(f"the timed run failed: {stats}")
    value = world * n3 * args.steps / (ms_max / 1e3)

    # end to end through the C ABI with pinned host buffers, every step. Each of
    # `members` independent model states (an ensemble; member 0 is the timed
    # state) round-trips through its own pinned host buffers every step: upload
    # (oc_set_state_async) on one stream, the step on the compute stream, download
    # (oc_get_state_async) on a third, ordered per member with events, so one
    # member's copies overlap another's step. All steps share one compute stream,
    # so the multigrid solves never run concurrently.
    e2e = None
    if args.e2e_steps > 0:
        fields = ("eta", "u", "v", "b", "T", "S", "e")
        host = st.get_state()
        members = max(1, args.e2e_members)
        steppers = [st] + [OceanStepper(p, s.H, s.mask, dzr=s.dzr, taux_c=s.taux_c, tauy_c=s.tauy_c,
                                        device=local_rank) for _ in range(members - 1)]
        bufs = [{k: torch.from_numpy(np.ascontiguousarray(host[k])).pin_memory() for k in fields}
                for _ in range(members)]
        for m in range(1, members):
            steppers[m].set_state(**{k: host[k] for k in fields})
        h2d = sum(v.numel() * 8 for v in bufs[0].values())
        d2h = h2d
        s_in = torch.cuda.Stream(device=local_rank)
        s_cmp = torch.cuda.Stream(device=local_rank)
        s_out = torch.cuda.Stream(device=local_rank)
        ev_out = [None] * members

        def round_trip(n):
            m = n % members
            if ev_out[m] is not None:
                s_in.wait_event(ev_out[m])
            steppers[m].set_state_async(s_in, **bufs[m])
            e_in = torch.cuda.Event()
            e_in.record(s_in)
            s_cmp.wait_event(e_in)
            steppers[m].step(1, stream=s_cmp)
            e_c = torch.cuda.Event()
            e_c.record(s_cmp)
            s_out.wait_event(e_c)
            steppers[m].get_state_async(s_out, bufs[m])
            ev_out[m] = torch.cuda.Event()
            ev_out[m].record(s_out)

        for n in range(members):  # warm-up round
            round_trip(n)
        torch.cuda.synchronize()
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(s_in)
        for n in range(args.e2e_steps):
            round_trip(n)
        for ev in ev_out:
            s_in.wait_event(ev)
        e1.record(s_in)
        e1.synchronize()
        torch.cuda.synchronize()
        barrier()
        e_ms = max_over_ranks(e0.elapsed_time(e1))
        for m in range(members):
            stm = steppers[m].stats()
            if stm["solver_failures"] or stm["diverged"]:
                raise RuntimeError(f"end-to-end member {m} failed: {stm}")
        # the same protocol with one state, every step waiting for the previous one
        seq_steps = max(1, args.e2e_steps // members)
        pinned = bufs[0]
        torch.cuda.synchronize()
        q0 = torch.cuda.Event(enable_timing=True)
        q1 = torch.cuda.Event(enable_timing=True)
        q0.record(torch.cuda.default_stream())
        for _ in range(seq_steps):
            st.set_state(**pinned)
            st.step(1)
            st.get_state(out=pinned)
        q1.record(torch.cuda.default_stream())
        q1.synchronize()
        q_ms = max_over_ranks(q0.elapsed_time(q1))
        for m in range(1, members):
            steppers[m].close()
        e2e = {"value": world * n3 * args.e2e_steps / (e_ms / 1e3), "unit": UNIT,
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "steps": args.e2e_steps, "ms_per_step": e_ms / args.e2e_steps, "members": members,
               "path": "OceanStepper.set_state_async/step/get_state_async (oc_set_state_async, "
                       "oc_step, oc_get_state_async), pinned host buffers, one round trip of the "
                       "full state per step",
               "sequential": {"value": world * n3 * seq_steps / (q_ms / 1e3), "unit": UNIT,
                              "steps": seq_steps, "ms_per_step": q_ms / seq_steps,
                              "path": "OceanStepper.set_state/step/get_state (synchronous, one state)"}}

    # roofline of the dominant kernel
    peak, peak_kind = measured_hbm_peak()
    top = max(ktimes.items(), key=lambda kv: kv[1][1])
    name, (nlaunch, tot_ms) = top
    iters_per_solve = (sum(log) / len(log)) if log else 0.0

    def alg_bytes(kernel):
        if kernel == "helm_solve":
            return helm_bytes_per_iteration(p) * iters_per_solve
        return 8 * ACCESSES_PER_CELL.get(kernel, 0) * n3

    alg = alg_bytes(name)
    per_launch_ms = tot_ms / max(1, nlaunch)
    achieved = alg / (per_launch_ms / 1e3) / 1e9
    traffic = dram_traffic_from_profiles(name)
    roofline = {"kernel": name, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                "algorithmic_bytes_per_launch": alg, "launch_ms": per_launch_ms}
    iters_per_step = sum(log) / (args.steps + args.profile_steps)  # both timed regions
    bstep = step_algorithmic_bytes(p, iters_per_step)
    step_gbs = bstep / (ms / args.steps / 1e3) / 1e9
    kernel_share = {}
    for k, (nl, kms) in sorted(ktimes.items(), key=lambda kv: -kv[1][1]):
        row = {"launches": nl, "ms": kms, "share": kms / max(1e-12, sum(x[1] for x in ktimes.values()))}
        kb = alg_bytes(k)
        if kb > 0 and nl > 0 and kms > 0:
            # algorithmic bytes per launch over the launch's average duration, against the HBM peak
            gbs = kb / (kms / nl / 1e3) / 1e9
            row.update({"algorithmic_bytes_per_launch": kb, "achieved_gbs": gbs, "frac": gbs / peak,
                        "dram_bytes_per_launch": dram_traffic_from_profiles(k)})
        kernel_share[k] = row

    # the mixed-precision step on the same recipe and grid, beside a fresh fp64
    # run from the same initial state (errors per field against the fp64 path)
    mixed = None
    if args.mixed_steps > 0:
        mixed = precision_leg(s, local_rank, args.mixed_steps, args.warmup, mixed_solver=args.mixed_solver)
        mixed["speedup_vs_fp64"] = (ms_max / args.steps) / mixed["ms_per_step"]
        mixed["fp64_ms_per_step"] = ms_max / args.steps

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        rate, secs, cp = cpu_oracle_rate(args, args.cpu_steps, 1)
        cpu = {"value": rate, "unit": UNIT, "cores": 1, "kind": "port", "host": host_cpu(),
               "sample": f"CPU oracle (NumPy, bit-identical port of the reference stepper) on the "
                         f"same recipe at {cp.nx}x{cp.ny}x{cp.nz}, 1 warm-up + {args.cpu_steps} "
                         f"steps, {secs:.1f} s"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded seamount-basin recipe; inputs generated on the host)",
            "config": {"workload": f"seamount_basin {p.nx}x{p.ny}x{p.nz}, TKE + TVD3 + polyTEOS10, "
                                   f"theta={p.theta:g} + {p.solver_kind}, dt={p.dt:g} s, stretched levels, "
                                   f"double-gyre wind",
                       "cells": n3, "rtol": p.rtol, "parallelism": f"replicas x{world}", "variant": "fp64 plain path",
                       "l2": "working set of several GB per replica, far above the 126 MB L2"},
            "roofline": roofline,
            "step_roofline": {"bound": "hbm", "achieved": step_gbs, "peak": peak, "unit": "GB/s",
                              "frac": step_gbs / peak, "algorithmic_bytes_per_step": bstep,
                              "solver_iterations_per_step": iters_per_step},
            "cpu_baseline": cpu,
            "mixed": mixed,
            "e2e": e2e,
            "gpu_launches": launches,
            "launch_mode": "two-step CUDA graphs (oc_step_graph)" if graph else "one launch per kernel",
            "clocks": clk,
            "kernels": kernel_share,
            "kernels_region": {"steps": args.profile_steps, "ms_per_step": ms_prof / args.profile_steps,
                               "note": "per-kernel CUDA events around every launch (plain launches)"},
            "solver_iterations_per_solve": iters_per_solve,
        }
        print(json.dumps(line), flush=True)
    st.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


def run_ensemble(args, rank, world, local_rank):
    """Batched-ensemble form: members with seeded uneven grids (nx, ny drawn from the
    multiples of 32 in 128..384, nz in {24, 32, 48}: the multigrid halves a grid only
    while its sizes are even, and on sizes with an odd factor above 8 the stationary
    multigrid -- the reference's algorithm -- falls back to smoothing and needs
    thousands of cycles), each the seamount-basin recipe with its own seed, tuned by
    oc_autotune, advanced together by one recorded graph per two steps
    (oc_ensemble_step); beside it the same members stepped one after another, each
    with its own recorded graphs."""
    import numpy as np
    import torch

    from hydrostatic_ocean_core_benchmark_b200 import cases
    from hydrostatic_ocean_core_benchmark_b200.stepper import OceanEnsemble, OceanStepper

    torch.cuda.set_device(local_rank)
    rng = np.random.default_rng(args.seed + 5)
    members, shapes, solvers, twins = [], [], [], []
    prec = args.ens_precision
    for m in range(args.ens_members):
        if args.ens_sizes == "any":
            nx, ny = (int(x) for x in rng.integers(128, 385, 2))
        else:
            nx, ny = (32 * int(x) for x in rng.integers(4, 13, 2))
        nz = int(rng.choice([24, 32, 48]))
        # the stationary multigrid halves a grid only while its sizes are even, and on
        # a large odd coarsest level it needs thousands of cycles: other sizes take CG
        # preconditioned by the same V-cycle (pcg_mg)
        solver = "multigrid" if nx % 32 == 0 and ny % 32 == 0 else "pcg_mg"
        s = cases.seamount_basin(nx=nx, ny=ny, nz=nz, seed=args.seed + 1000 * (rank + 1) + m, solver_kind=solver)
        st = OceanStepper(s.params, s.H, s.mask, dzr=s.dzr, taux_c=s.taux_c, tauy_c=s.tauy_c,
                          device=local_rank, precision=prec)
        st.set_state(eta=s.eta, u=s.u, v=s.v, T=s.T, S=s.S)
        members.append(st)
        shapes.append((nx, ny, nz))
        solvers.append(solver)
        if prec == "mixed" and len(twins) < args.ens_check:
            # an fp64 twin of the member, stepped as often, for the per-member error
            tw = OceanStepper(s.params, s.H, s.mask, dzr=s.dzr, taux_c=s.taux_c, tauy_c=s.tauy_c,
                              device=local_rank)
            tw.set_state(eta=s.eta, u=s.u, v=s.v, T=s.T, S=s.S)
            twins.append((m, tw))
    cells = sum(nx * ny * nz for nx, ny, nz in shapes)
    # each member's tile shapes timed on its own kernels (FP32 ones for mixed members)
    tiling = [st.autotune() for st in members]
    stream = torch.cuda.Stream(device=local_rank)
    steps = args.steps + (args.steps % 2)
    warm = max(args.warmup, 3)
    warm += warm % 2
    ens = OceanEnsemble(members)
    ens.step(warm, stream=stream)
    ens.step(2, stream=stream)          # the graph of the timed region's starting buffers
    stream.synchronize()
    out_dir = record_dir()
    clocks = ClockSampler(local_rank, out_dir / f"clocks_ens_rank{rank}.csv" if out_dir else None)
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    ens.step(steps, stream=stream)
    ev1.record(stream)
    ev1.synchronize()
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    # the same members one after another, each replaying its own recorded graphs
    for st in members:
        st.step(2, stream=stream, graph=True)
    stream.synchronize()
    ev0.record(stream)
    for st in members:
        st.step(steps, stream=stream, graph=True)
    ev1.record(stream)
    ev1.synchronize()
    ms_seq = ev0.elapsed_time(ev1)
    failures = sum(st.stats()["solver_failures"] for st in members)
    diverged = sum(st.stats()["diverged"] for st in members)
    if failures or diverged:
        raise RuntimeError(f"ensemble run failed: {failures} solver failures, {diverged} diverged members")
    # HBM roofline of the ensemble step: every member's minimal-pass bytes (fp64
    # accounting) over the batched step's time
    hbm = None
    if prec == "fp64":
        alg = 0.0
        for st, (nx, ny, nz) in zip(members, shapes):
            sts = st.stats()
            alg += step_algorithmic_bytes(st.p, sts["solver_iterations"] / max(sts["steps"], 1))
        peak, src = measured_hbm_peak()
        achieved = alg / (ms / steps / 1e3) / 1e9
        hbm = {"achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
               "algorithmic_bytes_per_step": alg, "peak_source": src}
    errors = None
    if twins:
        total = warm + 2 + steps + 2 + steps
        errors = []
        for m, tw in twins:
            tw.step(total, stream=stream, graph=True)
            stream.synchronize()
            a = members[m].get_state(fields=("eta", "u", "v", "T", "S"))
            b = tw.get_state(fields=("eta", "u", "v", "T", "S"))
            rel = {f: float(np.linalg.norm(a[f] - b[f]) / max(np.linalg.norm(b[f]), 1e-300)) for f in a}
            errors.append({"member": m, "grid": list(shapes[m]), "rel_l2_vs_fp64": rel})
            tw.close()
    line = {"metric": METRIC, "value": world * cells * steps / (ms / 1e3), "unit": UNIT, "n_gpus": world,
            "steps": steps, "warmup": warm, "ms_per_step": ms / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded seamount-basin recipe per member; inputs generated on the host)",
            "config": {"workload": f"ensemble of {len(members)} seamount basins, nx, ny "
                                   + ("uniform in 128..384" if args.ens_sizes == "any" else "multiples of 32 in 128..384")
                                   + ", nz in {24, 32, 48}, theta=0.6 + multigrid (MG-preconditioned CG on sizes the "
                                   "multigrid cannot halve to 8), TKE, TVD3, polyTEOS10",
                       "members": len(members), "cells": cells, "precision": prec,
                       "solvers": {k: solvers.count(k) for k in sorted(set(solvers))},
                       "grids": [list(g) for g in shapes[:8]] + (["..."] if len(shapes) > 8 else []),
                       "parallelism": "replicas x1"},
            "sequential": {"value": world * cells * steps / (ms_seq / 1e3), "unit": UNIT,
                           "ms_per_step": ms_seq / steps,
                           "path": "members one after another, each with its own recorded graphs"},
            "tiling": {"levels_per_cta_momentum": sorted(set(t[0] for t in tiling)),
                       "levels_per_cta_tracers": sorted(set(t[1] for t in tiling))} if tiling else "default",
            "clocks": clk}
    if hbm:
        line["roofline"] = hbm
    if errors:
        line["member_errors"] = errors
        line["worst_member_rel_l2"] = {f: max(e["rel_l2_vs_fp64"][f] for e in errors) for f in errors[0]["rel_l2_vs_fp64"]}
    if prec == "mixed":
        line["dtype"] = "f32 (3D state and stencils) + f64 (b, pressure gradient, EOS, eta, Helmholtz)"
    if rank == 0:
        print(json.dumps(line), flush=True)
    ens.close()
    for st in members:
        st.close()
    return 0


def helmholtz_system(n, seed):
    """A seeded n x n free-surface system of the reference cases' conditioning
    (c K / dx^2 between 0.25 and 0.5; the reference-written cases reach 0.49): face
    coefficients in [0.5, 1], a rectangular island whose faces are closed, a
    normal right-hand side on the wet cells."""
    import numpy as np
    rng = np.random.default_rng(seed)
    dx = 4.0e6 / n
    mask = np.ones((n, n))
    mask[n // 4:n // 3, n // 5:n // 2] = 0.0
    ku = (0.5 + 0.5 * rng.random((n, n))) * mask * np.roll(mask, -1, 1)
    kv = (0.5 + 0.5 * rng.random((n, n))) * mask * np.roll(mask, -1, 0)
    rhs = rng.standard_normal((n, n)) * mask
    return dx, 0.5 * dx * dx, ku, kv, mask, rhs


def refined_bytes_per_cell(inner, outer):
    """Minimal-pass bytes per cell of one FP32-inner / FP64-refined solve: the
    start (rhs, mask, 1/diag in; x, r, z, d out: 40 B), every inner iteration
    (the direction and A p: z, p_old, wet, ax, ay, diag in, p, Ap out, 29 B, no
    p_old in an inner solve's first iteration; the update: p, d, r, Ap, 1/diag
    in, d, r, z out, 32 B) and every refinement step (x += d: 20 B; the FP64
    residual: x, mask, Ku, Kv, rhs, 1/diag in, r, z, d out: 56 B)."""
    return 40 + 61 * inner - 4 * outer + 76 * outer


def run_helmholtz(args, rank, world, local_rank):
    """The free-surface Helmholtz solve alone: the FP64 PCG-Jacobi solver (the
    step's, bit-identical to NumPy) beside the FP32-inner / FP64-refined solver,
    on seeded synthetic systems of growing size, both through oc_helm_solve with
    the data on the device, timed by CUDA events on the call's stream."""
    import ctypes as C

    import numpy as np
    import torch

    from hydrostatic_ocean_core_benchmark_b200 import _lib

    torch.cuda.set_device(local_rank)
    lib = _lib.load()
    stream = torch.cuda.Stream(device=local_rank)
    peak, peak_kind = measured_hbm_peak()
    rtol, reps = 1e-10, max(args.steps, 1)
    sizes = [int(s) for s in args.helm_sizes.split(",")]
    rows = []
    for n in sizes:
        dx, coef, ku, kv, mask, rhs = helmholtz_system(n, args.seed + n)
        d_rhs = torch.from_numpy(rhs).to(f"cuda:{local_rank}")
        row = {"n": n}
        xs = {}
        for name, kind in (("fp64_pcg_jacobi", 0), ("pcg_refined", 4)):
            cfg = _lib.OcHelmConfig(nx=n, ny=n, dx=dx, dy=dx, coef=coef, solver=kind, rtol=rtol, max_iter=20000,
                                    device=local_rank)
            h = C.c_void_p()
            rc = lib.oc_helm_create(C.byref(cfg), ku.ctypes.data, kv.ctypes.data, mask.ctypes.data, C.byref(h))
            if rc:
                row[name] = {"unavailable": f"{_lib.ERRORS.get(rc, rc)}: {lib.oc_helm_last_error(h).decode()}"
                             if h else _lib.ERRORS.get(rc, rc)}
                continue
            x = torch.zeros_like(d_rhs)
            its, conv = C.c_int32(), C.c_int32()

            def solve():
                _lib.check(lib.oc_helm_solve(h, C.c_void_p(d_rhs.data_ptr()), C.c_void_p(x.data_ptr()), 1,
                                             C.byref(its), C.byref(conv), C.c_void_p(stream.cuda_stream)),
                           None, name)

            for _ in range(max(args.warmup, 3)):
                solve()
            times = []
            for _ in range(reps):
                ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                ev0.record(stream)
                solve()
                ev1.record(stream)
                ev1.synchronize()
                times.append(ev0.elapsed_time(ev1))
            ms = statistics.median(times)
            r = {"ms": ms, "iterations": its.value, "converged": bool(conv.value)}
            if kind == 4:
                outer, rel = C.c_int32(), C.c_double()
                _lib.check(lib.oc_helm_refine_report(h, C.byref(outer), C.byref(rel)), None, name)
                r["refinement_steps"], r["relative_residual_fp64"] = outer.value, rel.value
                byt = refined_bytes_per_cell(its.value, outer.value) * n * n
            else:
                byt = helm_bytes_per_iteration(type("P", (), {"nx": n, "ny": n, "solver_kind": "pcg_jacobi"})) \
                    * its.value
            r["algorithmic_gbs"] = byt / (ms * 1e-3) / 1e9
            r["frac"] = r["algorithmic_gbs"] / peak
            xs[name] = x.cpu().numpy()
            lib.oc_helm_destroy(h)
            row[name] = r
        if len(xs) == 2:
            a, b = xs["fp64_pcg_jacobi"], xs["pcg_refined"]
            row["rel_l2_refined_vs_fp64"] = float(np.linalg.norm(b - a) / np.linalg.norm(a))
            row["speedup"] = row["fp64_pcg_jacobi"]["ms"] / row["pcg_refined"]["ms"]
        rows.append(row)
    top = rows[-1]["pcg_refined"]
    line = {"metric": "helmholtz_solve_time", "value": top["ms"], "unit": "ms", "n_gpus": world,
            "steps": reps, "warmup": max(args.warmup, 3), "ms_per_step": top["ms"], "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 inner, f64 refinement",
            "data": "synthetic (seeded face coefficients, island, normal right-hand side)",
            "config": {"workload": f"free-surface Helmholtz solve, {sizes[-1]}x{sizes[-1]}, rtol {rtol:g}",
                       "sizes": sizes, "rtol": rtol,
                       "l2": "working sets from 10 MB (512^2, L2-resident) to 2.6 GB (4096^2)"},
            "roofline": {"bound": "hbm", "peak": peak, "peak_kind": peak_kind, "unit": "GB/s"},
            "sizes": rows}
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def run_adjoint(args, rank, world, local_rank):
    """--workload adjoint: the gradient form. The seamount recipe with the
    closure off (the adjoint's scope) at 256 x 256 x 32, 20 steps with a
    checkpoint every 5: the forward run (steps back to back, the state fetched
    at the checkpoints), the gradient of the mean temperature of the top three
    levels with respect to the initial temperature and the x-stress field
    (segments recomputed from their checkpoints, then walked back with
    oc_adjoint_step), their ratio and the peak device memory."""
    import numpy as np
    import torch

    from hydrostatic_ocean_core_benchmark_b200 import cases
    from hydrostatic_ocean_core_benchmark_b200.adjoint import OceanRollout, rollout_apply
    torch.cuda.set_device(local_rank)
    if rank != 0:
        return 0
    nx, ny, nz = (args.nx, args.ny, args.nz) if "--nx" in sys.argv else (256, 256, 32)
    n_steps = args.steps if "--steps" in sys.argv else 20
    every = 5
    s = cases.seamount_basin(nx=nx, ny=ny, nz=nz, seed=args.seed, closure="none", advection="up3_tvd")
    dev = f"cuda:{local_rank}"
    T = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)  # noqa: E731
    fixed = {"eta": T(s.eta), "u": T(s.u), "v": T(s.v), "S": T(s.S)}
    T0, taux = T(s.T), T(s.taux_c)
    w = torch.zeros(s.params.nz, ny, nx, dtype=torch.float64, device=dev)
    w[:3] = 1.0 / (3 * nx * ny)
    ro = OceanRollout(s.params, s.H, s.mask, dzr=s.dzr, n_steps=n_steps, every=every, device=local_rank)
    state0 = {"eta": fixed["eta"], "u": fixed["u"], "v": fixed["v"], "T": T0, "S": fixed["S"]}
    fwd, bwd = [], []
    torch.cuda.reset_peak_memory_stats(local_rank)
    free0 = torch.cuda.mem_get_info(local_rank)[0]
    low = free0
    for it in range(args.warmup + 3):
        t0 = T0.clone().requires_grad_(True)
        tx = taux.clone().requires_grad_(True)
        out = rollout_apply(ro, t0, tx, fixed)
        low = min(low, torch.cuda.mem_get_info(local_rank)[0])
        (w * out["T"]).sum().backward()
        if it >= args.warmup:
            fwd.append(ro.timing["forward_s"])
            bwd.append(ro.timing["backward_s"])
        del out, t0, tx
    plain = []
    for _ in range(3):
        ro.forward(state0, taux)
        plain.append(ro.timing["forward_s"])
    lib_bytes = int(ro.st.stats()["device_bytes"])
    peak = int(torch.cuda.max_memory_allocated(local_rank))
    ro.close()
    cells = nx * ny * s.params.nz
    f_s, b_s = float(np.median(fwd)), float(np.median(bwd))
    line = {"metric": "adjoint / forward wall time of the gradient of a 20-step run",
            "value": b_s / f_s, "unit": "x", "n_gpus": 1, "steps": n_steps, "warmup": args.warmup,
            "ms_per_step": b_s / n_steps * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded seamount-basin recipe, closure off)",
            "config": {"workload": f"seamount_basin {nx}x{ny}x{s.params.nz}, TVD3 + polyTEOS10, closure off, "
                                   f"theta={s.params.theta:g} + {s.params.solver_kind}, {n_steps} steps, "
                                   f"checkpoint every {every}",
                       "cells": cells, "variant": "gradient form (hand-written adjoint)"},
            "forward_ms": f_s * 1e3, "adjoint_ms": b_s * 1e3, "forward_alone_ms": float(np.median(plain)) * 1e3,
            "forward_cell_steps_per_s": cells * n_steps / f_s,
            "adjoint_includes": "segment recomputation from the checkpoints + adjoint steps + EOS adjoint",
            "peak_device_bytes": {"torch_tensors": peak, "library_handle": lib_bytes,
                                  "process_delta_at_forward_end": int(free0 - low)}}
    print(json.dumps(line), flush=True)
    return 0

def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--nx", type=int, default=512)
    ap.add_argument("--ny", type=int, default=512)
    ap.add_argument("--nz", type=int, default=50)
    ap.add_argument("--seed", type=int, default=20261203)
    ap.add_argument("--dt", type=float, default=None,
                    help="time step in s (default 600; the precision workload's 1024x1024 grid takes 300)")
    ap.add_argument("--rtol", type=float, default=None,
                    help="Helmholtz stopping tolerance of the seamount and precision workloads (default: the "
                         "recipe's 1e-12; the reference's precision study runs both precisions at 1e-6)")
    ap.add_argument("--e2e-steps", type=int, default=12)
    ap.add_argument("--profile-steps", type=int, default=20,
                    help="steps of the per-kernel event region (kernel shares, roofline)")
    ap.add_argument("--no-graph", action="store_true", help="launch the timed steps one by one")
    ap.add_argument("--e2e-members", type=int, default=3,
                    help="independent states round-tripped through the host in turn (overlap)")
    ap.add_argument("--cpu-steps", type=int, default=2)
    ap.add_argument("--cpu-nx", type=int, default=128)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--workload", choices=["seamount", "ensemble", "helmholtz", "precision", "adjoint"], default="seamount",
                    help="seamount: the 512x512x50 basin (the headline line); ensemble: the "
                         "batched-ensemble form (its own line); helmholtz: the FP64 and the "
                         "FP32-inner/FP64-refined Helmholtz solvers alone (its own line); precision: "
                         "the mixed FP32/FP64 step beside the fp64 one (default grid 1024x1024x64); "
                         "adjoint: gradient of a run through the hand-written adjoint (256x256x32, "
                         "--steps steps)")
    ap.add_argument("--mixed-steps", type=int, default=100,
                    help="timed steps of the mixed-precision leg of the headline line (0: skip it)")
    ap.add_argument("--mixed-solver", choices=["configured", "pcg_refined", "pcg_mg"], default="configured",
                    help="Helmholtz solver of the mixed-precision step (configured: the recipe's multigrid; "
                         "pcg_refined needs ~600 inner iterations per solve on the recipe's systems)")
    ap.add_argument("--ens-members", type=int, default=64)
    ap.add_argument("--ens-sizes", choices=["mult32", "any"], default="mult32",
                    help="member nx, ny: multiples of 32 in 128..384, or any integer in 128..384")
    ap.add_argument("--ens-precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--ens-check", type=int, default=8,
                    help="mixed members checked against an fp64 twin")
    ap.add_argument("--helm-sizes", default="512,1024,2048,4096",
                    help="grid sizes n of the n x n Helmholtz systems")
    args = ap.parse_args()
    if args.workload == "precision" and "--nx" not in sys.argv:
        args.nx, args.ny, args.nz = 1024, 1024, 64
    if args.dt is None:
        # at dx = 1.95 km (1024 x 1024) the explicit baroclinic terms take dt <= ~400 s:
        # the recipe's 600 s grows u threefold per step there; 768^2 and 512^2 run 600 s
        args.dt = 300.0 if args.nx >= 1024 else 600.0
    rank = env_int("RANK", 0)
    world = env_int("WORLD_SIZE", 1)
    local_rank = env_int("LOCAL_RANK", 0)
    if args.impl == "reference":
        return run_reference_arm(args, rank)
    if args.workload == "ensemble":
        return run_ensemble(args, rank, world, local_rank)
    if args.workload == "helmholtz":
        return run_helmholtz(args, rank, world, local_rank)
    if args.workload == "adjoint":
        return run_adjoint(args, rank, world, local_rank)
    if args.workload == "precision":
        return run_precision(args, rank, world, local_rank)
    return run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    raise SystemExit(main())
