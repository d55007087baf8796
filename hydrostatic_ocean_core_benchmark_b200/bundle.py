"""The bundle files of the backend protocol (reference tools/toml2nml.py:143-273 and
tools/compare_backends3d5.py:32-43).

``<prefix>_domain.bin``  H then mask, fp64 [ny, nx] C order
``<prefix>_init.bin``    eta [ny, nx]; u, v, b [nz, ny, nx]; then T, S when tracers = TS
``<prefix>_levels.bin``  (new, optional) nz level thicknesses
``<prefix>_forcing.bin`` (new, optional) taux, tauy at cell centres [ny, nx]
``<prefix>.nml``         the namelist (params.write_namelist)

and the output ``<prefix>_state3d5.bin``: eta, u, v, b[, T, S].
"""

from __future__ import annotations

from pathlib import Path

import numpy as np

from .params import OceanParams, write_namelist


def _f64(a) -> bytes:
    return np.ascontiguousarray(a, dtype=np.float64).tobytes()


def write_bundle(prefix: str, p: OceanParams, H, mask, state, dzr=None, taux_c=None,
                 tauy_c=None) -> Path:
    """Write namelist + binaries for ``state`` (any object with eta, u, v, b, T, S)."""
    out = Path(prefix)
    out.parent.mkdir(parents=True, exist_ok=True)
    p = p.replace(domain_file=f"{prefix}_domain.bin", init_file=f"{prefix}_init.bin")
    with open(p.domain_file, "wb") as fh:
        fh.write(_f64(H))
        fh.write(_f64(mask))
    ts = p.tracers == "TS"
    b = getattr(state, "b", None)
    if b is None:
        raise ValueError("the init bundle needs b")
    with open(p.init_file, "wb") as fh:
        for a in (state.eta, state.u, state.v, b):
            fh.write(_f64(a))
        if ts:
            fh.write(_f64(state.T))
            fh.write(_f64(state.S))
    if dzr is not None:
        p = p.replace(levels_file=f"{prefix}_levels.bin")
        Path(p.levels_file).write_bytes(_f64(dzr))
    if taux_c is not None or tauy_c is not None:
        p = p.replace(forcing_file=f"{prefix}_forcing.bin")
        zero = np.zeros((p.ny, p.nx))
        with open(p.forcing_file, "wb") as fh:
            fh.write(_f64(zero if taux_c is None else taux_c))
            fh.write(_f64(zero if tauy_c is None else tauy_c))
    return write_namelist(f"{prefix}.nml", p)


def read_state(path, nx: int, ny: int, nz: int, ts: bool) -> dict:
    """Read ``<prefix>_state3d5.bin`` (layout of compare_backends3d5.py:32-43)."""
    raw = np.fromfile(path, dtype=np.float64)
    n2, n3 = nx * ny, nx * ny * nz
    names = ["u", "v", "b"] + (["T", "S"] if ts else [])
    if raw.size != n2 + len(names) * n3:
        raise ValueError(f"{path}: expected {n2 + len(names) * n3} doubles, got {raw.size}")
    out = {"eta": raw[:n2].reshape(ny, nx)}
    off = n2
    for name in names:
        out[name] = raw[off:off + n3].reshape(nz, ny, nx)
        off += n3
    return out


def read_domain(path, nx: int, ny: int):
    raw = np.fromfile(path, dtype=np.float64)
    n2 = nx * ny
    if raw.size < 2 * n2:
        raise ValueError(f"{path}: expected {2 * n2} doubles, got {raw.size}")
    return raw[:n2].reshape(ny, nx), raw[n2:2 * n2].reshape(ny, nx)
