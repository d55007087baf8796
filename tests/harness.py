"""Shared test helpers: rebuild a golden case, run the CPU oracle, compare states."""

from __future__ import annotations

import sys
from dataclasses import fields
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT, ROOT / "tests" / "golden"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))

from golden_io import fhash, fixture_names, load_fixture  # noqa: E402,F401
from hydrostatic_ocean_core_benchmark_b200 import cases  # noqa: E402
from hydrostatic_ocean_core_benchmark_b200.params import OceanParams  # noqa: E402
from oracle import ocean_oracle as orc  # noqa: E402


def params_from_meta(meta) -> OceanParams:
    names = {f.name for f in fields(OceanParams)}
    return OceanParams(**{k: v for k, v in meta["params"].items() if k in names})


def case_inputs(meta, arrays, dzr=None, taux=None, tauy=None):
    """(params, H, mask, dzr, taux, tauy, initial OracleState) of a fixture."""
    p = params_from_meta(meta)
    kind = meta.get("init_regenerate")
    if kind == "lock_exchange_channel":
        s = cases.lock_exchange_channel()
        H, mask = s.H, s.mask
        geo = orc.Geometry(p, H, mask)
        b = orc.buoyancy(p.eos, s.T, s.S, geo.zc, p.g, p.rho0, p.alpha_t, p.beta_s, p.t0,
                         p.s0) * geo.mask3
        st = orc.OracleState(s.u, s.v, b, s.eta, s.T * geo.mask3, s.S * geo.mask3)
    elif kind == "seamount_basin":
        s = cases.seamount_basin(stretched=False, wind_field=False, **meta["regenerate_kwargs"])
        H, mask = s.H, s.mask
        geo = orc.Geometry(p, H, mask)
        b = orc.buoyancy(p.eos, s.T, s.S, geo.zc, p.g, p.rho0, p.alpha_t, p.beta_s, p.t0,
                         p.s0) * geo.mask3
        st = orc.OracleState(s.u, s.v, b, s.eta, s.T, s.S)
    else:
        H, mask = arrays["H"], arrays["mask"]
        ts = p.tracers == "TS"
        st = orc.OracleState(arrays["init_u"], arrays["init_v"], arrays["init_b"],
                             arrays["init_eta"], arrays["init_T"] if ts else None,
                             arrays["init_S"] if ts else None)
    return p, H, mask, dzr, taux, tauy, st


def state_hashes(s, Km, Kh) -> dict:
    return {"eta": fhash(s.eta), "u": fhash(s.u), "v": fhash(s.v), "b": fhash(s.b),
            "T": fhash(s.T), "S": fhash(s.S), "e": fhash(s.e), "Km": fhash(Km),
            "Kh": fhash(Kh)}


def run_oracle(meta, arrays, n_steps=None, **ext):
    p, H, mask, dzr, taux, tauy, s = case_inputs(meta, arrays, **ext)
    st = orc.OracleStepper(p, H, mask, dzr=dzr, taux_c=taux, tauy_c=tauy)
    n = meta["n_steps"] if n_steps is None else n_steps
    hashes = []
    for _ in range(n):
        s = st.step(s)
        hashes.append(state_hashes(s, st.Km, st.Kh))
    return st, s, hashes


def max_rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = float(np.sqrt(np.sum(b * b)))
    num = float(np.sqrt(np.sum((a - b) ** 2)))
    return num / den if den > 0 else num
