"""GPU-side helpers of the parity tests (import only inside gpu-marked tests)."""

from __future__ import annotations

import numpy as np

from golden_io import fhash
from harness import case_inputs
from hydrostatic_ocean_core_benchmark_b200.stepper import OceanStepper


def gpu_case(meta, arrays, **ext):
    p, H, mask, dzr, taux, tauy, s = case_inputs(meta, arrays, **ext)
    st = OceanStepper(p, H, mask, dzr=dzr, taux_c=taux, tauy_c=tauy, device=0)
    ts = p.tracers == "TS"
    st.set_state(eta=s.eta, u=s.u, v=s.v, b=s.b, T=s.T if ts else None, S=s.S if ts else None)
    return p, st


def gpu_hashes(p, out: dict) -> dict:
    ts = p.tracers == "TS"
    return {"eta": fhash(out["eta"]), "u": fhash(out["u"]), "v": fhash(out["v"]),
            "b": fhash(out["b"]), "T": fhash(out["T"]) if ts else None,
            "S": fhash(out["S"]) if ts else None,
            "e": fhash(out["e"]) if p.closure == "tke" else None,
            "Km": fhash(out["km"]), "Kh": fhash(out["kh"])}


FIELDS = ("eta", "u", "v", "b", "T", "S")


def state_errors(p, got: dict, want) -> dict:
    """The reference gate's per-field error (tools/compare_backends3d5.py:82-89)."""
    from oracle.ocean_oracle import field_error
    fields = [f for f in FIELDS if getattr(want, f) is not None]
    scale = max(float(np.sqrt(np.sum(getattr(want, f) ** 2))) for f in fields)
    return {f: field_error(got[f], getattr(want, f), scale) for f in fields}
