"""Experiment driver of the B200 ocean core: the v0.5 subcommands over the TOML tree.

    python -m hydrostatic_ocean_core_benchmark_b200.main bundle|run|verify|bench
        [--config DIR] [--set KEY=VALUE ...] [--case NAME] [--nx N] [--ny N] [--nz N]
        [--cfl X] [--steps N] [--precision fp64|mixed] [--prefix PATH] [--reference DIR]

The reference's driver (main.py:55-99,121-291) runs its run/verify/bench
subcommands on the 2D model only; its v0.5 core is reached through
tools/toml2nml.py (bundle) and tools/compare_backends3d5.py (the R2 gate).
These subcommands give the v0.5 core the same driver, reading the same TOML
tree (``toml_front``) with the same ``--set`` rules:

  bundle  write <prefix>.nml + _domain.bin + _init.bin for the compiled
          binaries (the reference's ``toml2nml.py --v05``);
  run     integrate the case on the GPU; write <prefix>_state3d5.bin and
          <prefix>_metrics.json (the binaries' output files and keys);
  verify  the reference's R2 gate (tools/compare_backends3d5.py:28-99): the
          GPU run against the reference's own NumPy stepper, imported from the
          reference checkout named by --reference (or OCEAN_REFERENCE), after
          one step (relative L2 < 1e-12) and after the run (< 1e-9), field by
          field, with the state-scale fallback for near-zero fields;
  bench   cell-steps/s of the case on one GPU (CUDA events, graph replay).
"""

from __future__ import annotations

import argparse
import json
import os
import sys
import time
from pathlib import Path

import numpy as np

from . import toml_front as tf
from .bundle import write_bundle

FIELDS = ("eta", "u", "v", "b", "T", "S")
DEFAULT_CONFIG = Path(__file__).resolve().parent / "config"


def field_error(a, b, scale: float) -> float:
    """Relative L2 error, or L2 error over the state scale for a field near zero
    (the reference gate's metric, tools/compare_backends3d.py:52-67)."""
    num = float(np.sqrt(np.sum((np.asarray(a) - np.asarray(b)) ** 2)))
    den = float(np.sqrt(np.sum(np.asarray(b) ** 2)))
    if den > 1e-11 * scale:
        return num / den
    return num / scale if scale > 0.0 else num


def _setup(args) -> tf.RunSetup:
    config = tf.apply_overrides(tf.load_config(args.config), args.set)
    return tf.resolve_run(config, nx=args.nx, nz=args.nz, case=args.case, cfl=args.cfl, n_steps=args.steps,
                          ny=args.ny)


def _stepper(run: tf.RunSetup, precision: str):
    from .stepper import OceanStepper
    s = run.state
    st = OceanStepper(run.params, run.H, run.mask, dzr=run.dzr, taux_c=run.taux_c, tauy_c=run.tauy_c,
                      precision=precision)
    ts = run.params.tracers == "TS"
    st.set_state(eta=s.eta, u=s.u, v=s.v, b=s.b, T=s.T if ts else None, S=s.S if ts else None)
    return st


def cmd_bundle(args) -> int:
    run = _setup(args)
    nml = write_bundle(args.prefix, run.params.replace(out_prefix=args.prefix, n_repeat=args.n_repeat,
                                                       n_warmup=args.n_warmup),
                       run.H, run.mask, run.state, dzr=run.dzr, taux_c=run.taux_c, tauy_c=run.tauy_c)
    print(f"{nml}  (dt={run.dt:.6f}s, n_steps={run.n_steps}, cfl={run.dt / run.dt_max:.3f}, v0.5 bundle)")
    return 0


def cmd_run(args) -> int:
    import torch
    run = _setup(args)
    st = _stepper(run, args.precision)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    st.step(run.n_steps, graph=True)
    out = st.get_state(fields=FIELDS if run.params.tracers == "TS" else FIELDS[:4])
    wall = time.perf_counter() - t0
    stats = st.stats()
    st.close()
    p = run.params
    prefix = args.prefix
    Path(prefix).parent.mkdir(parents=True, exist_ok=True)
    with open(prefix + "_state3d5.bin", "wb") as fh:
        for f in FIELDS:
            if f in out:
                fh.write(np.ascontiguousarray(out[f], np.float64).tobytes())
    cells = p.nx * p.ny * p.nz
    metrics = {"backend": "ocean_b200 (python)", "precision": args.precision, "nx": p.nx, "ny": p.ny, "nz": p.nz,
               "cells": cells, "n_steps": run.n_steps, "scheme": p.scheme_name, "solver": p.solver_kind,
               "eos": p.eos, "advection": p.advection, "tracers": p.tracers, "theta": p.theta, "dt": run.dt,
               "solver_iterations": stats["solver_iterations"], "solver_failures": stats["solver_failures"],
               "tridiagonal_solves": stats["tridiagonal_solves"], "solver_rebuilds": stats["solver_rebuilds"],
               "n_split": stats["n_split"], "barotropic_substeps": stats["barotropic_substeps"],
               "device_bytes": stats["device_bytes"], "diverged": bool(stats["diverged"]), "wall_s": wall,
               "cell_steps_per_s": cells * run.n_steps / wall}
    Path(prefix + "_metrics.json").write_text(json.dumps(metrics, indent=1) + "\n")
    print(f"case={p.case_name} nx={p.nx} ny={p.ny} nz={p.nz} steps={run.n_steps} dt={run.dt:.3f}s "
          f"solver_iterations={stats['solver_iterations']} diverged={bool(stats['diverged'])} wall={wall:.3f}s")
    return 1 if stats["diverged"] or stats["solver_failures"] else 0


def reference_stepper_factory(reference_dir: str | Path, config: tf.Config, run: tf.RunSetup):
    """A builder of the reference's own NumPy stepper (model3d_v05.py Stepper3DV05)
    for the run, from the reference checkout, as tools/compare_backends3d5.py
    builds it; returns (stepper, initial State3D)."""
    import types
    sys.path.insert(0, str(reference_dir))
    nc = types.ModuleType("netCDF4")
    nc.Dataset = object
    sys.modules.setdefault("netCDF4", nc)
    from libs.core.domain import Domain
    from libs.core.grid import CGrid
    from libs.core.model3d import State3D
    from libs.core.driver3d_v05 import physics_v05_from_config
    from libs.core.model3d_v05 import Stepper3DV05
    from libs.core.schemes import scheme_params_from_config
    from libs.utils.config import Config as RefConfig

    p = run.params
    rc = RefConfig(config.data, Path(config.source_dir or "."))
    grid = CGrid(nx=p.nx, ny=p.ny, Lx=p.lx, Ly=p.ly, nz=p.nz, depth=p.h0)
    domain = Domain(grid=grid, H=run.H, mask=run.mask, vcoord=p.vcoord, bc_x=p.bc_x, bc_y=p.bc_y,
                    min_partial=p.min_partial, face_rule=p.face_rule)
    stepper = Stepper3DV05(domain, physics_v05_from_config(rc), scheme_params_from_config(rc), run.dt)
    s = run.state
    s0 = State3D(u=s.u, v=s.v, b=s.b, eta=s.eta, t=0.0, T=s.T, S=s.S)
    return stepper, s0


def verify_run(run: tf.RunSetup, reference, precision: str = "fp64", gate_one: float = 1e-12,
               gate_run: float = 1e-9) -> dict:
    """The R2 gate (compare_backends3d5.py:28-99) of the GPU run against a
    reference stepper: `reference` is (stepper, initial state) with
    ``stepper.step(state)`` and ``stepper.solve_log`` (or ``solver_iterations``)."""
    stepper, s_ref = reference
    st = _stepper(run, precision)
    fields = [f for f in FIELDS if getattr(s_ref, f, None) is not None]
    report = {"steps": run.n_steps, "precision": precision, "per_step": []}
    worst = 0.0
    for n in range(run.n_steps):
        s_ref = stepper.step(s_ref)
        st.step(1)
        got = st.get_state(fields=tuple(fields))
        scale = max(float(np.sqrt(np.sum(np.asarray(getattr(s_ref, f)) ** 2))) for f in fields)
        errs = {f: field_error(got[f], getattr(s_ref, f), scale) for f in fields}
        report["per_step"].append(errs)
        worst = max(worst, max(errs.values()))
        if n == 0:
            report["one_step"] = {"errors": errs, "pass": max(errs.values()) < gate_one}
    report["full_run"] = {"errors": report["per_step"][-1], "pass": max(report["per_step"][-1].values()) < gate_run}
    report["worst_step_error"] = worst
    log = list(getattr(stepper, "solve_log", []))
    if log:
        report["solve_log_equal"] = st.solve_log() == log
    st.close()
    report["pass"] = report["one_step"]["pass"] and report["full_run"]["pass"] and report.get("solve_log_equal", True)
    return report


def cmd_verify(args) -> int:
    ref_dir = args.reference or os.environ.get("OCEAN_REFERENCE")
    if not ref_dir or not (Path(ref_dir) / "libs" / "core" / "model3d_v05.py").exists():
        print("FATAL: verify needs the reference checkout (--reference DIR or OCEAN_REFERENCE)", file=sys.stderr)
        return 2
    config = tf.apply_overrides(tf.load_config(args.config), args.set)
    run = tf.resolve_run(config, nx=args.nx, nz=args.nz, case=args.case, cfl=args.cfl, n_steps=args.steps,
                         ny=args.ny)
    report = verify_run(run, reference_stepper_factory(ref_dir, config, run), args.precision)
    print(json.dumps({k: v for k, v in report.items() if k != "per_step"}, indent=1))
    return 0 if report["pass"] else 1


def cmd_bench(args) -> int:
    import torch
    run = _setup(args)
    st = _stepper(run, args.precision)
    st.step(max(2, args.n_warmup), graph=True)
    torch.cuda.synchronize()
    times = []
    for _ in range(max(1, args.n_repeat)):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        st.step(run.n_steps, graph=True)
        e1.record()
        e1.synchronize()
        times.append(e0.elapsed_time(e1) / 1e3)
    stats = st.stats()
    st.close()
    p = run.params
    cells = p.nx * p.ny * p.nz
    med = float(np.median(times))
    print(json.dumps({"case": p.case_name, "precision": args.precision, "nx": p.nx, "ny": p.ny, "nz": p.nz,
                      "n_steps": run.n_steps, "wall_s": med, "cell_steps_per_s": cells * run.n_steps / med,
                      "solver_iterations": stats["solver_iterations"], "diverged": bool(stats["diverged"])}))
    return 0


def build_parser() -> argparse.ArgumentParser:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("command", choices=["bundle", "run", "verify", "bench"])
    ap.add_argument("--config", default=str(DEFAULT_CONFIG), help="TOML tree (the reference's config/ works too)")
    ap.add_argument("--set", action="append", default=[], metavar="KEY=VALUE")
    ap.add_argument("--case", default=None)
    ap.add_argument("--nx", type=int, default=None)
    ap.add_argument("--ny", type=int, default=None)
    ap.add_argument("--nz", type=int, default=None)
    ap.add_argument("--cfl", type=float, default=None)
    ap.add_argument("--steps", type=int, default=None, help="pin the step count instead of reaching t_final")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--prefix", default="output/b200/run")
    ap.add_argument("--n-repeat", type=int, default=1)
    ap.add_argument("--n-warmup", type=int, default=0)
    ap.add_argument("--reference", default=None, help="reference checkout for verify")
    return ap


def main(argv=None) -> int:
    args = build_parser().parse_args(argv)
    return {"bundle": cmd_bundle, "run": cmd_run, "verify": cmd_verify, "bench": cmd_bench}[args.command](args)


if __name__ == "__main__":
    raise SystemExit(main())
