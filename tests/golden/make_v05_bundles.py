#!/usr/bin/env python3
"""Golden bundles of the TOML front end, written by the reference's own tool.

Runs the reference's v0.5 bundle writer (``tools/toml2nml.py``
``write_v05_bundle``, with its ``--set`` parsing, ``main.py`` ``_apply_overrides``)
on this package's default TOML tree (``hydrostatic_ocean_core_benchmark_b200/config``)
under each override set below, and stores per case the namelist it writes
(every key and raw value) and the SHA-256 of its domain and initial-state
files. ``tests/test_toml_front.py`` resolves the same tree and overrides with
the package's front end and compares. Run where the reference is checked out
(``OCEAN_REFERENCE``, or a checkout named ``reference`` beside this repository).
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
CONFIG = REPO / "hydrostatic_ocean_core_benchmark_b200" / "config"
sys.path.insert(0, str(REPO))
sys.path.insert(0, str(REF))
_nc = types.ModuleType("netCDF4")  # the reference driver imports its NetCDF writer; no file is written here
_nc.Dataset = object
sys.modules.setdefault("netCDF4", _nc)

from hydrostatic_ocean_core_benchmark_b200.params import parse_namelist_text  # noqa: E402

from libs.utils.config import load_config  # noqa: E402
from main import _apply_overrides  # noqa: E402
from tools.toml2nml import write_v05_bundle  # noqa: E402

# (name, case, nx, nz, cfl, steps, overrides)
CASES = [
    ("lock_exchange.seamount.tke", "lock_exchange", 24, 8, 2.0, 4, []),
    ("lock_exchange.rough.up3.fb", "lock_exchange", 32, 6, 0.8, None,
     ["bathymetry.kind=rough", "scheme.name=fb", "scheme.advection=up3", "physics3d_v06.closure=none",
      "case.lock_exchange.n_hours=2.0"]),
    ("lock_exchange.ridge.seos.split", "lock_exchange", 20, 5, 1.0, 3,
     ["bathymetry.kind=ridge", "scheme.name=split_explicit", "physics3d_v05.eos=seos", "domain.bc_x=periodic"]),
    ("seamount_rest.flat.pcg", "seamount_rest", 16, 6, 2.0, 6,
     ["bathymetry.kind=flat", "solver.kind=pcg_jacobi", "physics3d_v04.tracers=buoyancy",
      "physics3d_v06.closure=none"]),
    ("seamount_rest.slope.island", "seamount_rest", 20, 4, 1.5, 2,
     ["bathymetry.kind=slope", "bathymetry.island=true", "physics3d_v04.tracers=buoyancy",
      "solver.kind=pcg_rbgs", "domain.face_rule=mean"]),
    ("basin_seiche.rough.kmax", "basin_seiche", 24, 4, 1.0, None,
     ["bathymetry.kind=rough", "bathymetry.spectrum_kmax=5", "physics3d_v04.tracers=buoyancy",
      "physics3d_v06.closure=none", "scheme.advection=none"]),
]


def sha(path):
    return hashlib.sha256(Path(path).read_bytes()).hexdigest()


def main():
    out = []
    with tempfile.TemporaryDirectory() as tmp:
        for name, case, nx, nz, cfl, steps, over in CASES:
            config = _apply_overrides(load_config(CONFIG), list(over))
            prefix = str(Path(tmp) / name.replace(".", "_"))
            r = write_v05_bundle(prefix, config, nx, nz, case, cfl, steps, 1, 0)
            kv = parse_namelist_text(Path(r["nml"]).read_text())
            out.append({"name": name, "case": case, "nx": nx, "nz": nz, "cfl": cfl, "steps": steps,
                        "overrides": over, "namelist": kv, "domain_sha256": sha(prefix + "_domain.bin"),
                        "init_sha256": sha(prefix + "_init.bin")})
    (HERE / "v05_bundles.json").write_text(json.dumps(out, indent=1) + "\n")
    print(f"wrote {len(out)} cases")


if __name__ == "__main__":
    main()
