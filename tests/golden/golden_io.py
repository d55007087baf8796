"""Helpers shared by the golden-vector generator and the tests that read its fixtures.

A field is fingerprinted by the SHA-256 of its fp64 bytes after ``+ 0.0`` (which
maps -0.0 to +0.0, so only the sign of zero is ignored); two fingerprints are
equal exactly when the arrays are bit-identical up to signed zeros.
"""

from __future__ import annotations

import hashlib
import json
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
STATE_FIELDS = ("eta", "u", "v", "b", "T", "S", "e", "Km", "Kh")


def fhash(a) -> str | None:
    if a is None:
        return None
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float64) + 0.0)
    return hashlib.sha256(a.tobytes()).hexdigest()[:16]


def save_fixture(name: str, meta: dict, **arrays) -> Path:
    path = HERE / f"{name}.npz"
    clean = {k: np.asarray(v, dtype=np.float64) for k, v in arrays.items() if v is not None}
    np.savez_compressed(path, meta=np.array(json.dumps(meta, sort_keys=True)), **clean)
    return path


def load_fixture(name: str):
    with np.load(HERE / f"{name}.npz", allow_pickle=False) as z:
        meta = json.loads(str(z["meta"]))
        arrays = {k: np.array(z[k]) for k in z.files if k != "meta"}
    return meta, arrays


def fixture_names() -> list[str]:
    return sorted(p.stem for p in HERE.glob("*.npz"))
