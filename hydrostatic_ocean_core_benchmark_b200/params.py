"""Run parameters of the ocean-core time step and the namelist bundle contract.

``OceanParams`` carries every key the reference's bundle writer puts in the
namelist (reference ``tools/toml2nml.py:188-268``) plus the two optional files
this backend adds (stretched levels, surface-stress field), in a new
``&b200_nml`` group that the reference's own parser ignores.

``read_namelist`` follows the reference parser's rules
(``libs/cuda/src/config.hpp:62-93``): ``!`` comments, ``&group``/``/`` lines
skipped, ``key = value`` pairs, Fortran ``d`` exponents, quoted strings.
"""

from __future__ import annotations

import dataclasses
import math
from dataclasses import dataclass, fields
from pathlib import Path
from typing import Any


@dataclass
class OceanParams:
    """Every scalar of the v0.5/v0.6 core step, keyed like the reference namelist."""

    # &grid_nml
    nx: int = 32
    ny: int = 32
    nz: int = 10
    lx: float = 1.0e7
    ly: float = 1.0e7
    # &physics_nml
    g: float = 9.80616
    f0: float = 1.0e-4
    h0: float = 1000.0
    n2: float = 1.0e-4
    nu: float = 1.0e-3
    kappa: float = 1.0e-3
    rho0: float = 1025.0
    tau_x: float = 0.0
    tau_y: float = 0.0
    bottom_drag: float = 0.0
    # &scheme_nml
    scheme_name: str = "theta"
    theta: float = 0.5
    theta_cor: float = 0.5
    theta_v: float = 0.5
    n_picard: int = 2
    n_split: int = 0
    barotropic_average: str = "none"
    solver_kind: str = "pcg_jacobi"
    rtol: float = 1.0e-12
    max_iter: int = 2000
    # &case_nml
    case_name: str = ""
    # &run_nml
    dt: float = 0.0
    t_final: float = 0.0
    n_steps: int = 1
    n_repeat: int = 1
    n_warmup: int = 0
    out_prefix: str = "run"
    # &v05_nml
    vcoord: str = "zlevel"
    bc_x: str = "periodic"
    bc_y: str = "periodic"
    face_rule: str = "min"
    min_partial: float = 0.1
    eos: str = "linear"
    pgf: str = "remove"
    pgf_correction: bool = True
    advection: str = "none"
    tracers: str = "buoyancy"
    alpha_t: float = 2.0e-4
    beta_s: float = 7.4e-4
    t0: float = 10.0
    s0: float = 35.0
    cp: float = 3990.0
    a_h: float = 0.0
    k_h: float = 0.0
    q_heat: float = 0.0
    q_salt: float = 0.0
    closure: str = "none"
    c_k: float = 0.1
    c_eps: float = 0.7
    pr_t: float = 1.0
    z_0: float = 0.1
    e_min: float = 1.0e-6
    l_min: float = 0.01
    e_bb: float = 3.75
    n2_min: float = 1.0e-8
    mxl: str = "integral"
    domain_file: str = ""
    init_file: str = ""
    # &b200_nml (new; absent means the reference's uniform levels / scalar stress)
    levels_file: str = ""
    forcing_file: str = ""

    # ------------------------------------------------------------------ checks
    def validate(self) -> None:
        """Refuse what the step cannot do, never change it silently.

        Mirrors ``SchemeParams.validate`` (reference ``libs/core/schemes.py:69-81``)
        and the compiled backend's refusals (``cfd_exp3d5_cuda.cu:110-114``).
        """
        bad = []
        if self.scheme_name not in ("fb", "theta", "split_explicit"):
            bad.append(f"unknown scheme {self.scheme_name!r} (expected fb|theta|split_explicit)")
        if self.scheme_name == "theta" and not (0.0 < self.theta <= 1.0):
            bad.append(f"theta must lie in (0,1]; got {self.theta}")
        if self.n_picard < 1:
            bad.append("n_picard must be >= 1")
        if self.dt <= 0.0:
            bad.append("dt must be > 0")
        # only the theta scheme owns an elliptic solve (reference model3d_v05.py:99-101);
        # pcg_mg (CG preconditioned by one V(2,2) cycle) and pcg_refined (FP32 inner
        # PCG inside FP64 refinement, mixed-precision step only) have no reference counterpart
        if self.scheme_name == "theta" and self.solver_kind not in (
                "pcg_jacobi", "pcg_rbgs", "rbgs", "multigrid", "pcg_mg", "pcg_refined"):
            bad.append(f"unknown variable-coefficient solver {self.solver_kind!r} "
                       "(expected pcg_jacobi|pcg_rbgs|rbgs|multigrid|pcg_mg|pcg_refined)")
        if self.vcoord != "zlevel":
            bad.append("vcoord must be zlevel")
        for name in ("bc_x", "bc_y"):
            if getattr(self, name) not in ("periodic", "closed"):
                bad.append(f"{name} must be periodic|closed")
        if self.face_rule not in ("min", "mean", "harmonic"):
            bad.append("face_rule must be min|mean|harmonic")
        if self.eos not in ("linear", "seos", "teos10"):
            bad.append(f"unknown eos {self.eos!r} (expected linear|seos|teos10)")
        if self.pgf not in ("remove", "keep"):
            bad.append("pgf must be remove|keep")
        if self.advection not in ("none", "centered2", "upwind1", "up3", "up3_tvd"):
            bad.append(f"unknown advection {self.advection!r}")
        if self.tracers not in ("buoyancy", "TS"):
            bad.append("tracers must be buoyancy|TS")
        if self.closure not in ("none", "tke"):
            bad.append("closure must be none|tke")
        if self.mxl not in ("integral", "recursive"):
            bad.append("mxl must be integral|recursive")
        if self.barotropic_average not in ("none", "mean"):
            bad.append("barotropic_average must be none|mean")
        if min(self.nx, self.ny, self.nz) < 1:
            bad.append("nx, ny, nz must be >= 1")
        if bad:
            raise ValueError("; ".join(bad))

    @property
    def dx(self) -> float:
        return self.lx / self.nx

    @property
    def dy(self) -> float:
        return self.ly / self.ny

    def replace(self, **kw) -> "OceanParams":
        return dataclasses.replace(self, **kw)


# ----------------------------------------------------------------------------
# conversion from the reference's own objects (duck-typed: Domain, PhysicsV05,
# SchemeParams of libs/core), so that a reference user can hand them over as is


def params_from_reference(domain, physics, scheme, dt) -> OceanParams:
    """Build ``OceanParams`` from reference-style objects.

    ``domain`` needs ``grid`` (nx, ny, nz, Lx, Ly), ``vcoord``, ``bc_x``,
    ``bc_y``, ``min_partial``, ``face_rule``; ``physics`` the ``PhysicsV05``
    attributes (reference ``model3d_v05.py:40-75``); ``scheme`` the
    ``SchemeParams`` attributes (reference ``schemes.py:53-67``).
    """
    g = domain.grid
    get = lambda o, k, d: getattr(o, k, d)  # noqa: E731
    p = OceanParams(
        nx=int(g.nx), ny=int(g.ny), nz=int(g.nz), lx=float(g.Lx), ly=float(g.Ly),
        g=float(physics.g), f0=float(physics.f), h0=float(physics.H),
        n2=float(get(physics, "N2", 0.0)), nu=float(get(physics, "nu", 0.0)),
        kappa=float(get(physics, "kappa", 0.0)), rho0=float(get(physics, "rho0", 1025.0)),
        tau_x=float(get(physics, "tau_x", 0.0)), tau_y=float(get(physics, "tau_y", 0.0)),
        bottom_drag=float(get(physics, "bottom_drag", 0.0)),
        scheme_name=str(scheme.name), theta=float(scheme.theta),
        theta_cor=float(scheme.theta_cor), theta_v=float(get(scheme, "theta_v", 0.5)),
        n_picard=int(scheme.n_picard), n_split=int(get(scheme, "n_split", 0)),
        barotropic_average=str(get(scheme, "barotropic_average", "none")),
        solver_kind=str(scheme.solver), rtol=float(scheme.rtol),
        max_iter=int(scheme.max_iter), dt=float(dt),
        vcoord=str(get(domain, "vcoord", "zlevel")), bc_x=str(get(domain, "bc_x", "periodic")),
        bc_y=str(get(domain, "bc_y", "periodic")), face_rule=str(get(domain, "face_rule", "min")),
        min_partial=float(get(domain, "min_partial", 0.1)),
        eos=str(get(physics, "eos", "linear")), pgf=str(get(physics, "pgf", "remove")),
        pgf_correction=bool(get(physics, "pgf_correction", True)),
        advection=str(get(scheme, "advection", "none")),
        tracers=str(get(physics, "tracers", "buoyancy")),
        alpha_t=float(get(physics, "alpha_T", 2.0e-4)), beta_s=float(get(physics, "beta_S", 7.4e-4)),
        t0=float(get(physics, "T0", 10.0)), s0=float(get(physics, "S0", 35.0)),
        cp=float(get(physics, "cp", 3990.0)), a_h=float(get(physics, "A_h", 0.0)),
        k_h=float(get(physics, "K_h", 0.0)), q_heat=float(get(physics, "q_heat", 0.0)),
        q_salt=float(get(physics, "q_salt", 0.0)),
        closure=str(get(physics, "closure", "none")), c_k=float(get(physics, "c_k", 0.1)),
        c_eps=float(get(physics, "c_eps", 0.7)), pr_t=float(get(physics, "pr_t", 1.0)),
        z_0=float(get(physics, "z_0", 0.1)), e_min=float(get(physics, "e_min", 1.0e-6)),
        l_min=float(get(physics, "l_min", 0.01)), e_bb=float(get(physics, "e_bb", 3.75)),
        n2_min=float(get(physics, "n2_min", 1.0e-8)), mxl=str(get(physics, "mxl", "integral")),
    )
    return p


# ----------------------------------------------------------------------------
# namelist I/O (the format of reference tools/toml2nml.py:27-34,188-268)

_GROUPS = {
    "grid_nml": ("nx", "ny", "nz", "lx", "ly"),
    "physics_nml": ("g", "f0", "h0", "n2", "nu", "kappa", "rho0", "tau_x", "tau_y",
                    "bottom_drag"),
    "scheme_nml": ("scheme_name", "theta", "theta_cor", "theta_v", "n_picard", "n_split",
                   "solver_kind", "rtol", "max_iter"),
    "case_nml": ("case_name",),
    "run_nml": ("dt", "t_final", "n_steps", "n_repeat", "n_warmup", "out_prefix"),
    "v05_nml": ("vcoord", "bc_x", "bc_y", "face_rule", "min_partial", "eos", "pgf",
                "pgf_correction", "advection", "tracers", "alpha_t", "beta_s", "t0", "s0", "cp",
                "a_h", "k_h", "q_heat", "q_salt", "closure", "c_k", "c_eps", "pr_t", "z_0",
                "e_min", "l_min", "e_bb", "n2_min", "mxl", "domain_file", "init_file"),
    "b200_nml": ("levels_file", "forcing_file", "barotropic_average"),
}


def fortran_double(value: float) -> str:
    """Full-precision Fortran double literal (reference toml2nml.py:27-34)."""
    return f"{float(value):.17e}".replace("e", "d")


def _format(value: Any) -> str:
    if isinstance(value, bool):
        return ".true." if value else ".false."
    if isinstance(value, int):
        return str(value)
    if isinstance(value, float):
        return fortran_double(value)
    return f"'{value}'"


def write_namelist(path: str | Path, p: OceanParams) -> Path:
    lines = ["! ocean-core bundle namelist (reference v05 layout plus &b200_nml)"]
    for group, keys in _GROUPS.items():
        lines.append(f"&{group}")
        for k in keys:
            lines.append(f"  {k} = {_format(getattr(p, k))}")
        lines.append("/")
    path = Path(path)
    path.write_text("\n".join(lines) + "\n", encoding="utf-8")
    return path


def parse_namelist_text(text: str) -> dict[str, str]:
    """name -> raw value of a Fortran namelist file as the bundle writer emits it
    (reference tools/toml2nml.py:27-34, 188-268): ``&group`` opens a group and
    ``/`` (or ``&end``) closes it; items are ``name = value`` separated by
    newlines or commas; character values are quoted, a doubled quote standing
    for itself; ``!`` outside quotes starts a comment; names are
    case-insensitive. Quoted values come back without their quotes. The same
    scanner as the compiled protocol's (csrc/protocol.cpp)."""
    items: dict[str, str] = {}
    i, n = 0, len(text)
    in_group = False

    def name_char(ch):
        return ch.isalnum() or ch in "_%"

    def skip_line():
        nonlocal i
        while i < n and text[i] != "\n":
            i += 1

    while i < n:
        ch = text[i]
        if ch == "!":
            skip_line()
            continue
        if not in_group:
            i += 1
            if ch in "&$":
                in_group = True
                while i < n and name_char(text[i]):
                    i += 1
            continue
        if ch.isspace() or ch == ",":
            i += 1
            continue
        if ch in "/&$":
            in_group = False
            i += 1
            while i < n and name_char(text[i]):
                i += 1
            continue
        n0 = i
        while i < n and name_char(text[i]):
            i += 1
        name = text[n0:i].lower()
        while i < n and text[i] in " \t":
            i += 1
        if not name or i >= n or text[i] != "=":
            skip_line()
            continue
        i += 1
        while i < n and text[i] in " \t":
            i += 1
        if i < n and text[i] in "'\"":
            q = text[i]
            i += 1
            out = []
            while i < n:
                if text[i] == q:
                    if i + 1 < n and text[i + 1] == q:
                        out.append(q)
                        i += 2
                        continue
                    i += 1
                    break
                out.append(text[i])
                i += 1
            items[name] = "".join(out)
        else:
            v0 = i
            while i < n and not text[i].isspace() and text[i] not in ",/!":
                i += 1
            items[name] = text[v0:i]
    return items


def _to_double(raw: str) -> float:
    """A Fortran real literal: the exponent letter d/D/q/Q read as e."""
    out, mantissa = [], False
    for ch in raw:
        if mantissa and ch in "dDqQ":
            ch = "e"
        if ch.isdigit() or ch == ".":
            mantissa = True
        out.append(ch)
    return float("".join(out))


def _logical(raw: str) -> bool:
    r = raw[1:] if raw.startswith(".") else raw
    return r[:1].lower() == "t"


def read_namelist(path: str | Path) -> OceanParams:
    """Read a bundle namelist into ``OceanParams`` (missing keys keep defaults)."""
    path = Path(path)
    if not path.exists():
        raise FileNotFoundError(f"cannot open namelist {path}")
    kv = parse_namelist_text(path.read_text(encoding="utf-8"))
    p = OceanParams()
    for f in fields(OceanParams):
        if f.name not in kv:
            continue
        raw = kv[f.name]
        if f.type in ("int", int):
            setattr(p, f.name, int(_to_double(raw)))
        elif f.type in ("float", float):
            setattr(p, f.name, _to_double(raw))
        elif f.type in ("bool", bool):
            setattr(p, f.name, _logical(raw))
        else:
            setattr(p, f.name, raw)
    return p


def split_n_substeps(p: OceanParams, h_max: float) -> int:
    """Barotropic substep count of the split-explicit scheme (model3d_v05.py:111-123)."""
    c = math.sqrt(p.g * h_max)
    dt_baro = 1.0 / (c * math.sqrt(1.0 / p.dx ** 2 + 1.0 / p.dy ** 2))
    n = p.n_split if p.n_split > 0 else max(1, int(math.ceil(1.2 * p.dt / dt_baro)))
    if p.dt / n > dt_baro:
        raise ValueError(f"n_split={n} leaves a barotropic substep of {p.dt / n:.1f}s "
                         f"above the limit {dt_baro:.1f}s")
    return n
