"""Cross-check against the reference's own CUDA backend, built from its source for
sm_100a into oracle/_ref (make -C oracle): both binaries run the same bundle
through the same file protocol; their final states must agree under the
reference's gate (tools/compare_backends3d5.py:28-29, 1e-9 after a full run),
and their same-box wall times are recorded (the reference's own GPU path is
the bar the B200 path has to beat).
"""

import json
import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

from harness import case_inputs, load_fixture
from oracle import ocean_oracle as orc

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]
REF_BIN = ROOT / "oracle" / "_ref" / "cfd_exp3d5_cuda"
OUR_BIN = ROOT / "hydrostatic_ocean_core_benchmark_b200" / "bin" / "ocean3d5_b200"

if not REF_BIN.exists():
    pytest.skip("reference CUDA backend not built (make -C oracle)", allow_module_level=True)


def run(binary, nml, timeout=900):
    proc = subprocess.run([str(binary), str(nml)], capture_output=True, text=True, timeout=timeout)
    assert proc.returncode == 0, proc.stderr[-2000:]
    return proc


def test_reference_cuda_agrees_on_a_gate_case(tmp_path):
    from hydrostatic_ocean_core_benchmark_b200 import bundle
    meta, arrays = load_fixture("gate_v06_seamount_tvd_tke_theta")
    p, H, mask, _, _, _, s = case_inputs(meta, arrays)
    p = p.replace(n_steps=6, n_repeat=1, n_warmup=0)
    fields = ("eta", "u", "v", "b", "T", "S")
    ref_oracle = orc.OracleStepper(p, H, mask).integrate(s, 6)
    got = {}
    for tag, exe in (("ref", REF_BIN), ("b200", OUR_BIN)):
        prefix = str(tmp_path / tag)
        nml = bundle.write_bundle(prefix, p.replace(out_prefix=prefix), H, mask, s)
        run(exe, nml)
        got[tag] = bundle.read_state(prefix + "_state3d5.bin", p.nx, p.ny, p.nz, True)
    scale = max(float(np.sqrt(np.sum(getattr(ref_oracle, f) ** 2))) for f in fields)
    for f in fields:
        # ours is bit-identical to the NumPy reference; the reference CUDA is within its gate
        assert np.array_equal(got["b200"][f], getattr(ref_oracle, f)), f
        assert orc.field_error(got["ref"][f], getattr(ref_oracle, f), scale) < 1e-9, f


def test_same_box_timing_against_reference_cuda(tmp_path):
    """512x512x50 seamount basin in the form the reference can express (uniform
    levels, scalar stress), 10 steps, both binaries; records the timings."""
    from hydrostatic_ocean_core_benchmark_b200 import bundle, cases
    s = cases.seamount_basin(stretched=False, wind_field=False)
    p = s.params.replace(n_steps=10, n_repeat=3, n_warmup=1)
    geo = orc.Geometry(p, s.H, s.mask)
    b = orc.buoyancy(p.eos, s.T, s.S, geo.zc, p.g, p.rho0, p.alpha_t, p.beta_s, p.t0, p.s0) * geo.mask3
    state = orc.OracleState(s.u, s.v, b, s.eta, s.T, s.S)
    out, states = {}, {}
    for tag, exe in (("reference_cuda", REF_BIN), ("b200", OUR_BIN)):
        prefix = str(tmp_path / tag)
        nml = bundle.write_bundle(prefix, p.replace(out_prefix=prefix), s.H, s.mask, state)
        run(exe, nml, timeout=1800)
        m = json.loads(Path(prefix + "_metrics.json").read_text())
        out[tag] = {"wall_s": m["wall_s"], "ms_per_step": 1e3 * m["wall_s"] / p.n_steps,
                    "cell_steps_per_s": m["cells"] * p.n_steps / m["wall_s"],
                    "solver_iterations": m["solver_iterations"], "diverged": m["diverged"]}
        states[tag] = bundle.read_state(prefix + "_state3d5.bin", p.nx, p.ny, p.nz, True)
    scale = max(float(np.sqrt(np.sum(states["b200"][f] ** 2))) for f in ("eta", "u", "v", "b", "T", "S"))
    errs = {f: orc.field_error(states["reference_cuda"][f], states["b200"][f], scale)
            for f in ("eta", "u", "v", "b", "T", "S")}
    out["rel_l2_reference_cuda_vs_b200"] = errs
    out["speedup"] = out["reference_cuda"]["wall_s"] / out["b200"]["wall_s"]
    print(json.dumps(out))
    dest = os.environ.get("OCEAN_B200_RECORD_DIR")
    if dest and os.path.isdir(dest):
        (Path(dest) / "reference_cuda_vs_b200.json").write_text(json.dumps(out, indent=2))
    assert not out["reference_cuda"]["diverged"] and not out["b200"]["diverged"]
    assert max(errs.values()) < 1e-9
