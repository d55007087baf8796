#!/usr/bin/env python3
"""Golden bundles of the reference's hardware-ladder case, written by the
reference's own tool on the reference's own TOML tree.

The reference times its v0.5 core on `lock_exchange` at N^2 x 30, theta = 0.5,
50 steps, with the case flags of its sweep script (tools/tier2_sweep.sh:87,95 and
its solver flag). This script runs the reference's bundle writer
(tools/toml2nml.py `write_v05_bundle`, `--set` parsing from main.py) on the
reference's `config/` tree with those flags at two small sizes and stores the
namelist and the SHA-256 of the domain and initial-state files, together with
the flags this package's own tree needs on top (`EXTRA`) to describe the same
case. tests/test_toml_front.py resolves this package's tree with both flag sets
and compares, so `main.py run|bench` with them runs the reference's ladder case
at any size. Run where the reference is checked out (OCEAN_REFERENCE, or a
checkout named `reference` beside this repository).
"""

from __future__ import annotations

import hashlib
import json
import os
import sys
import tempfile
import types
from pathlib import Path

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
REF = Path(os.environ.get("OCEAN_REFERENCE", str(Path(__file__).resolve().parents[3] / "reference")))
sys.path.insert(0, str(REPO))
sys.path.insert(0, str(REF))
_nc = types.ModuleType("netCDF4")  # the reference driver imports its NetCDF writer; no file is written here
_nc.Dataset = object
sys.modules.setdefault("netCDF4", _nc)

from hydrostatic_ocean_core_benchmark_b200.params import parse_namelist_text  # noqa: E402

from libs.utils.config import load_config  # noqa: E402
from main import _apply_overrides  # noqa: E402
from tools.toml2nml import write_v05_bundle  # noqa: E402

# the sweep's flags for the lock_exchange case and the theta 0.5 scheme
LADDER = ["bathymetry.kind=rough", "physics3d_v04.tracers=TS", "scheme.advection=centered2",
          "physics3d_v05.eos=teos10", "physics3d_v04.A_h=10.0", "physics3d_v04.K_h=10.0", "physics.f0=0.0",
          "physics3d.N2=0.0", "physics3d.nu=1e-3", "physics3d.kappa=1e-3", "physics3d_v05.pgf=keep",
          "grid.Lx=6.4e4", "grid.Ly=6.4e3", "physics.H=20.0", "scheme.name=theta", "scheme.theta=0.5"]
# where this package's default tree differs from the reference's for that case
EXTRA = ["physics3d.tau_x=0.0", "domain.bc_x=periodic", "domain.bc_y=periodic", "physics3d_v06.closure=none",
         "bathymetry.h_rel=0.9", "bathymetry.seed=20260911", "case.lock_exchange.delta_T=2.0"]
# (name, nx, cfl, solver)
SIZES = [("ladder_64_cfl2_mg", 64, 2.0, "multigrid"), ("ladder_100_cfl4_pcg", 100, 4.0, "pcg_jacobi")]


def sha(path):
    return hashlib.sha256(Path(path).read_bytes()).hexdigest()


def main():
    out = []
    with tempfile.TemporaryDirectory() as tmp:
        for name, nx, cfl, solver in SIZES:
            over = LADDER + [f"solver.kind={solver}"]
            config = _apply_overrides(load_config(REF / "config"), list(over))
            prefix = str(Path(tmp) / name)
            r = write_v05_bundle(prefix, config, nx, 30, "lock_exchange", cfl, 50, 1, 0)
            kv = parse_namelist_text(Path(r["nml"]).read_text())
            out.append({"name": name, "case": "lock_exchange", "nx": nx, "nz": 30, "cfl": cfl, "steps": 50,
                        "overrides": over, "extra": EXTRA, "namelist": kv,
                        "domain_sha256": sha(prefix + "_domain.bin"), "init_sha256": sha(prefix + "_init.bin")})
    (HERE / "ladder_case.json").write_text(json.dumps(out, indent=1) + "\n")
    print(f"wrote {len(out)} cases")


if __name__ == "__main__":
    main()
