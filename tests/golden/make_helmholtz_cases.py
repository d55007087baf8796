#!/usr/bin/env python3
"""Generate the standalone-Helmholtz golden cases with the reference's own tool.

Runs the reference's ``tools/write_helmholtz_case.py --reference`` (from the
reference tree: ``OCEAN_REFERENCE``, or a checkout named ``reference`` beside
this repository)
for a 64 x 64 and a 96 x 96 rough-topography case, and stores per case the
face coefficients, mask, right-hand side, the reference's PCG solution at
rtol 1e-13 (``eta_ref``) and its metadata, which carries NumPy's
``HelmholtzVar`` iteration count for each of the four solvers at rtol 1e-10.
The domain length (the reference config's ``grid.Lx``) is added so the spacing
of every multigrid level can be formed as the reference forms it.
"""

from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF = Path(os.environ.get("OCEAN_REFERENCE", str(Path(__file__).resolve().parents[3] / "reference")))
CASES = {64: dict(nz=10, seed=20260911), 96: dict(nz=12, seed=20261203)}


def main() -> int:
    sys.path.insert(0, str(REF))
    from libs.utils.config import load_config
    lx = float(load_config(REF / "config").get("grid.Lx"))
    env = dict(os.environ, PYTHONDONTWRITEBYTECODE="1")
    for nx, kw in CASES.items():
        with tempfile.TemporaryDirectory() as tmp:
            out = Path(tmp) / "case"
            subprocess.run([sys.executable, str(REF / "tools" / "write_helmholtz_case.py"), "--nx", str(nx),
                            "--nz", str(kw["nz"]), "--seed", str(kw["seed"]), "--out", str(out),
                            "--reference"], cwd=REF, env=env, check=True, capture_output=True)
            meta = json.loads((out / "case.json").read_text())
            meta["lx"] = lx
            arrays = {name: np.fromfile(out / f"{name}.bin", dtype=np.float64).reshape(nx, nx)
                      for name in ("ku", "kv", "mask", "rhs", "eta_ref")}
        (HERE / "helmholtz").mkdir(exist_ok=True)
        np.savez_compressed(HERE / "helmholtz" / f"case_{nx}.npz", meta=json.dumps(meta), **arrays)
        print(nx, {k: v for k, v in meta.items() if k.startswith("numpy_iters") or k == "reference_iterations"})
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
