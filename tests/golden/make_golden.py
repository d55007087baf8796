#!/usr/bin/env python3
"""Generate the golden vectors that pin the CPU oracle to the unmodified reference.

Run in a container that has the reference checked out (``OCEAN_REFERENCE``, or a
checkout named ``reference`` beside this repository); the fixtures it writes
under ``tests/golden/*.npz`` are what travels. It imports the reference's own
NumPy stepper (``libs/core/model3d_v05.py`` ``Stepper3DV05``), its bundle
writer (``tools/toml2nml.py`` ``write_v05_bundle``), its case generators and
its config tree, runs each case, and records per step a fingerprint of every
state field, the per-solve Helmholtz iteration counts and the counters.

Cases:
* ``lock_exchange_channel``: the 128x4x32 lock-exchange channel, 200 steps at
  dt = 0.05 s (initial state from the reference's ``LockExchange.initial``).
* ``seamount_basin_ref_mg`` / ``seamount_basin_ref_pcg``: small seamount basins
  with the wind-driven TKE/TVD3/EOS physics in the form the reference can
  express (uniform levels, scalar stress); the first also pins the oracle's
  stretched-level and stress-field extensions on their special case.
* ``gate_*``: the reference's twelve R2 gate combinations
  (``tools/gate3d5.sh:20-31``) at nx = 16, nz = 6, 6 steps.
"""

from __future__ import annotations

import os
import shutil
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
REF = Path(os.environ.get("OCEAN_REFERENCE", str(Path(__file__).resolve().parents[3] / "reference")))
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(REPO))
sys.path.insert(0, str(REF))

from golden_io import fhash, save_fixture  # noqa: E402

from hydrostatic_ocean_core_benchmark_b200 import cases as oc_cases  # noqa: E402
from hydrostatic_ocean_core_benchmark_b200.params import params_from_reference  # noqa: E402

from libs.core import solvers_var  # noqa: E402
from libs.core.cases3d_v05 import LockExchange  # noqa: E402
from libs.core.domain import Domain  # noqa: E402
from libs.core.eos import buoyancy as ref_buoyancy  # noqa: E402
from libs.core.grid import CGrid  # noqa: E402
from libs.core.model3d import Physics3D, State3D  # noqa: E402
from libs.core.model3d_v05 import PhysicsV05, Stepper3DV05  # noqa: E402
from libs.core.schemes import SchemeParams  # noqa: E402
from libs.utils.config import load_config  # noqa: E402
from tools.toml2nml import write_v05_bundle  # noqa: E402

GATE_NX, GATE_NZ, GATE_STEPS = 16, 6, 6

# tools/gate3d5.sh:16-31, verbatim overrides of the reference gate matrix
GATE_BASE = ["grid.Lx=4.0e5", "grid.Ly=4.0e5", "physics3d.N2=0.0", "physics3d_v05.pgf=keep",
             "physics3d.nu=1e-3", "physics3d.kappa=1e-3"]
GATE_CASES = {
    "flat.theta.pcg": "--case seamount_rest --set bathymetry.kind=flat --set solver.kind=pcg_jacobi",
    "seamount.theta.mg.closed": "--case seamount_rest --set bathymetry.kind=seamount --set solver.kind=multigrid --set domain.bc_x=closed --set domain.bc_y=closed",
    "seamount.split.closed": "--case seamount_rest --set bathymetry.kind=seamount --set scheme.name=split_explicit --set domain.bc_x=closed",
    "seamount.theta1.rbgs": "--case seamount_rest --set bathymetry.kind=seamount --set scheme.theta=1.0 --set solver.kind=pcg_rbgs",
    "rough.TS.teos10.mg": "--case lock_exchange --set bathymetry.kind=rough --set physics3d_v04.tracers=TS --set scheme.advection=centered2 --set physics3d_v05.eos=teos10 --set solver.kind=multigrid --set physics3d_v04.A_h=10.0 --set physics3d_v04.K_h=10.0 --set physics.f0=0.0",
    "rough.TS.fb.upwind": "--case lock_exchange --set bathymetry.kind=rough --set physics3d_v04.tracers=TS --set scheme.advection=upwind1 --set scheme.name=fb --set physics.f0=0.0",
    "v06.rough.TS.up3.mg": "--case lock_exchange --set bathymetry.kind=rough --set physics3d_v04.tracers=TS --set scheme.advection=up3 --set physics3d_v05.eos=teos10 --set solver.kind=multigrid --set physics.f0=0.0 --set domain.bc_x=closed",
    "v06.seamount.tvd.tke.theta": "--case lock_exchange --set bathymetry.kind=seamount --set physics3d_v04.tracers=TS --set scheme.advection=up3_tvd --set physics3d_v06.closure=tke --set physics3d.tau_x=0.1 --set solver.kind=multigrid --set physics3d.nu=1e-5 --set physics3d.kappa=1e-6",
    "v06.seamount.tke.split": "--case lock_exchange --set bathymetry.kind=seamount --set physics3d_v04.tracers=TS --set scheme.advection=up3 --set physics3d_v06.closure=tke --set scheme.name=split_explicit --set physics3d.tau_x=0.1 --set physics3d.nu=1e-5 --set physics3d.kappa=1e-6 --set domain.bc_x=closed",
    "v06.mxl_rec.tke.theta": "--case lock_exchange --set bathymetry.kind=seamount --set physics3d_v04.tracers=TS --set scheme.advection=up3_tvd --set physics3d_v06.closure=tke --set physics3d_v06.mxl=recursive --set physics3d.tau_x=0.1 --set solver.kind=multigrid --set physics3d.nu=1e-5 --set physics3d.kappa=1e-6",
    "v06.mxl_rec.tke.fb": "--case lock_exchange --set bathymetry.kind=rough --set physics3d_v04.tracers=TS --set scheme.advection=up3 --set physics3d_v06.closure=tke --set physics3d_v06.mxl=recursive --set scheme.name=fb --set physics3d.tau_x=0.1 --set physics3d.nu=1e-5 --set physics3d.kappa=1e-6 --set physics.f0=0.0",
    "seamount.split.seos.forcing": "--case lock_exchange --set bathymetry.kind=seamount --set physics3d_v04.tracers=TS --set scheme.advection=centered2 --set scheme.name=split_explicit --set physics3d_v05.eos=seos --set physics3d.tau_x=0.1 --set physics3d_v04.q_heat=100.0 --set physics3d.bottom_drag=1e-3 --set domain.bc_x=closed",
}


def parse_value(raw: str):
    """Value parsing of the reference driver's --set (main.py:335-349)."""
    try:
        return int(raw)
    except ValueError:
        try:
            return float(raw)
        except ValueError:
            return {"true": True, "false": False}.get(raw.lower(), raw)


def state_hashes(s, stepper) -> dict:
    return {"eta": fhash(s.eta), "u": fhash(s.u), "v": fhash(s.v), "b": fhash(s.b),
            "T": fhash(s.T), "S": fhash(s.S), "e": fhash(s.e), "Km": fhash(stepper.nu),
            "Kh": fhash(stepper.kappa)}


def run_reference(stepper, s0, n_steps):
    """Step the reference, recording per-step fingerprints and per-solve iterations."""
    log: list[int] = []
    orig = solvers_var.HelmholtzVar.solve

    def recording_solve(self, rhs):
        x, rep = orig(self, rhs)
        log.append(int(rep.iterations))
        return x, rep

    solvers_var.HelmholtzVar.solve = recording_solve
    try:
        s = s0
        hashes = []
        for _ in range(n_steps):
            s = stepper.step(s)
            hashes.append(state_hashes(s, stepper))
    finally:
        solvers_var.HelmholtzVar.solve = orig
    counters = {k: int(getattr(stepper, k)) for k in
                ("solver_iterations", "solver_failures", "solver_rebuilds",
                 "tridiagonal_solves", "barotropic_substeps")}
    counters["n_split"] = int(stepper.n_split)
    return s, hashes, log, counters


def params_dict(domain, physics, scheme, dt):
    from dataclasses import asdict
    return asdict(params_from_reference(domain, physics, scheme, dt))


def final_norms(s) -> dict:
    out = {}
    for f in ("eta", "u", "v", "b", "T", "S", "e"):
        a = getattr(s, f)
        if a is not None:
            out[f] = float(np.sqrt(np.sum(a * a)))
    return out


def make_lock_exchange_channel(n_steps=200):
    setup = oc_cases.lock_exchange_channel()
    p = setup.params
    grid = CGrid(nx=p.nx, ny=p.ny, Lx=p.lx, Ly=p.ly, nz=p.nz, depth=p.h0)
    dom = Domain(grid=grid, H=setup.H, mask=setup.mask, vcoord="zlevel", bc_x="closed",
                 bc_y="closed")
    base = Physics3D(g=p.g, f=p.f0, H=p.h0, N2=p.n2, nu=p.nu, kappa=p.kappa, rho0=p.rho0,
                     tracers="TS", alpha_T=p.alpha_t, beta_S=p.beta_s, T0=p.t0, S0=p.s0)
    phys = PhysicsV05(base=base, eos="linear", pgf=p.pgf)
    scheme = SchemeParams(name="theta", theta=0.5, theta_cor=0.5, n_picard=2, theta_v=0.5,
                          advection="up3_tvd", solver="pcg_jacobi", rtol=1e-12, max_iter=2000)
    case = LockExchange(dom, phys, delta_T=10.0, n_hours=1.0)
    s0 = case.initial()
    stepper = Stepper3DV05(dom, phys, scheme, p.dt)
    init = {"eta": fhash(s0.eta), "u": fhash(s0.u), "v": fhash(s0.v), "b": fhash(s0.b),
            "T": fhash(s0.T), "S": fhash(s0.S)}
    s, hashes, log, counters = run_reference(stepper, s0, n_steps)
    meta = {"name": "lock_exchange_channel", "params": params_dict(dom, phys, scheme, p.dt),
            "n_steps": n_steps, "hashes": hashes, "solve_log": log, "counters": counters,
            "init_hashes": init, "init_regenerate": "lock_exchange_channel",
            "final_norms": final_norms(s)}
    save_fixture("lock_exchange_channel", meta, H=setup.H, mask=setup.mask,
                 final_eta=s.eta, final_T=s.T)


def make_seamount_basin(name, n_steps, **over):
    setup = oc_cases.seamount_basin(stretched=False, wind_field=False, **over)
    p = setup.params
    grid = CGrid(nx=p.nx, ny=p.ny, Lx=p.lx, Ly=p.ly, nz=p.nz, depth=p.h0)
    dom = Domain(grid=grid, H=setup.H, mask=setup.mask, vcoord="zlevel", bc_x=p.bc_x,
                 bc_y=p.bc_y)
    base = Physics3D(g=p.g, f=p.f0, H=p.h0, N2=p.n2, nu=p.nu, kappa=p.kappa, rho0=p.rho0,
                     tau_x=p.tau_x, tau_y=p.tau_y, tracers="TS", alpha_T=p.alpha_t,
                     beta_S=p.beta_s, T0=p.t0, S0=p.s0)
    phys = PhysicsV05(base=base, eos=p.eos, pgf=p.pgf, closure=p.closure, mxl=p.mxl)
    scheme = SchemeParams(name=p.scheme_name, theta=p.theta, theta_cor=p.theta_cor,
                          n_picard=p.n_picard, theta_v=p.theta_v, advection=p.advection,
                          solver=p.solver_kind, rtol=p.rtol, max_iter=p.max_iter)
    stepper = Stepper3DV05(dom, phys, scheme, p.dt)
    z = dom.depth_at_centres()
    b0 = ref_buoyancy(p.eos, setup.T, setup.S, z, g=p.g, rho0=p.rho0, alpha_T=p.alpha_t,
                      beta_S=p.beta_s, T0=p.t0, S0=p.s0) * dom.mask3
    s0 = State3D(u=setup.u, v=setup.v, b=b0, eta=setup.eta, T=setup.T, S=setup.S)
    init = {"H": fhash(setup.H), "T": fhash(setup.T), "S": fhash(setup.S), "b": fhash(b0)}
    s, hashes, log, counters = run_reference(stepper, s0, n_steps)
    meta = {"name": name, "params": params_dict(dom, phys, scheme, p.dt), "n_steps": n_steps,
            "hashes": hashes, "solve_log": log, "counters": counters, "init_hashes": init,
            "init_regenerate": "seamount_basin", "regenerate_kwargs": over,
            "final_norms": final_norms(s)}
    save_fixture(name, meta, H=setup.H, mask=setup.mask)


def make_gate_case(label, args, workdir):
    tokens = args.split()
    case_name = tokens[tokens.index("--case") + 1]
    sets = GATE_BASE + [tokens[i + 1] for i, t in enumerate(tokens) if t == "--set"]
    config = load_config(REF / "config").with_overrides(
        {k: parse_value(v) for k, v in (s.split("=", 1) for s in sets)})
    prefix = str(Path(workdir) / label.replace(".", "_"))
    r = write_v05_bundle(prefix, config, GATE_NX, GATE_NZ, case_name, 0.5, GATE_STEPS, 1, 0)
    nml_text = Path(r["nml"]).read_text(encoding="utf-8")
    dom, phys, scheme, dt = r["domain"], r["physics"], r["params"], r["dt"]
    s0 = r["state0"]
    stepper = Stepper3DV05(dom, phys, scheme, dt)
    s, hashes, log, counters = run_reference(stepper, s0, GATE_STEPS)
    name = "gate_" + label.replace(".", "_")
    meta = {"name": name, "label": label, "params": params_dict(dom, phys, scheme, dt),
            "n_steps": GATE_STEPS, "hashes": hashes, "solve_log": log, "counters": counters,
            "nml_text": nml_text, "final_norms": final_norms(s)}
    save_fixture(name, meta, H=dom.H, mask=dom.mask, init_eta=s0.eta, init_u=s0.u,
                 init_v=s0.v, init_b=s0.b, init_T=s0.T, init_S=s0.S)


def main() -> int:
    if not (REF / "libs" / "core" / "model3d_v05.py").exists():
        print(f"reference not found at {REF}", file=sys.stderr)
        return 2
    make_lock_exchange_channel()
    make_seamount_basin("seamount_basin_ref_mg", 8, nx=32, ny=32, nz=12)
    make_seamount_basin("seamount_basin_ref_pcg", 6, nx=24, ny=16, nz=10,
                        solver_kind="pcg_jacobi", mxl="recursive", eos="seos")
    work = tempfile.mkdtemp(prefix="ocean_golden_")
    try:
        for label, args in GATE_CASES.items():
            make_gate_case(label, args, work)
    finally:
        shutil.rmtree(work, ignore_errors=True)
    print("fixtures written to", HERE)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
