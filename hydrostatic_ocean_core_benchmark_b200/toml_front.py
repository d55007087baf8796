"""The reference's TOML configuration tree, read as the front end of the step.

The reference drives its compiled backends from one TOML tree (``settings``,
``grid``, ``schemes``, ``cases`` and ``backends`` files merged in that order,
reference ``libs/utils/config.py:22-98``), from which its bundle writer
resolves the domain, physics, scheme, case, time step and step count of a
v0.5 run (reference ``tools/toml2nml.py:143-273`` over
``libs/core/driver3d_v05.py:25-94``, ``libs/core/bathymetry.py:85-139``,
``libs/core/cases3d_v05.py`` and ``libs/core/schemes.py:180-196``). This
module reads the same tree with the same key names and resolves the same
run; ``main.py`` writes it as a bundle or runs it on the GPU.

Cases: ``seamount_rest``, ``lock_exchange`` and ``basin_seiche`` (the
reference's ``zstar_constancy`` and ``flather_radiate`` need moving
coordinates and open boundaries, which the step refuses; ``baroclinic_igw``
is not carried), plus ``seamount_basin``, the benchmark's own recipe
(``cases.seamount_basin``). Bathymetries: flat, slope, seamount, ridge, rough.
"""

from __future__ import annotations

import copy
import tomllib
from dataclasses import dataclass
from pathlib import Path
from types import SimpleNamespace
from typing import Any

import numpy as np

from . import cases as _cases
from .params import OceanParams

CONFIG_FILES = ("settings.toml", "grid.toml", "schemes.toml", "cases.toml", "backends.toml")
_MISSING = object()


class ConfigError(KeyError):
    pass


class Config:
    """The merged tree, with dotted-key lookup."""

    def __init__(self, data: dict, source_dir: Path | None = None):
        self.data = data
        self.source_dir = source_dir

    def get(self, dotted: str, default: Any = _MISSING) -> Any:
        node: Any = self.data
        for part in dotted.split("."):
            if not isinstance(node, dict) or part not in node:
                if default is _MISSING:
                    raise ConfigError(f"missing config key '{dotted}'")
                return default
            node = node[part]
        return node

    def section(self, dotted: str) -> dict:
        node = self.get(dotted)
        if not isinstance(node, dict):
            raise ConfigError(f"config key '{dotted}' is not a table")
        return dict(node)

    def with_overrides(self, overrides: dict) -> "Config":
        data = copy.deepcopy(self.data)
        for dotted, value in overrides.items():
            node = data
            parts = dotted.split(".")
            for part in parts[:-1]:
                node = node.setdefault(part, {})
            node[parts[-1]] = value
        return Config(data, self.source_dir)


def _merge(base: dict, extra: dict) -> dict:
    for k, v in extra.items():
        if isinstance(v, dict) and isinstance(base.get(k), dict):
            _merge(base[k], v)
        else:
            base[k] = v
    return base


def load_config(config_dir: str | Path) -> Config:
    """Merge the five files of the tree, later files over earlier ones."""
    d = Path(config_dir)
    if not d.is_dir():
        raise FileNotFoundError(f"config directory not found: {d}")
    merged: dict = {}
    for name in CONFIG_FILES:
        path = d / name
        if not path.exists():
            raise FileNotFoundError(f"required config file missing: {path}")
        with path.open("rb") as fh:
            _merge(merged, tomllib.load(fh))
    return Config(merged, d)


def parse_override(raw: str) -> Any:
    """A ``--set`` value: an integer, else a float, else true/false, else the text
    (the reference driver's rule, main.py:335-349)."""
    try:
        return int(raw)
    except ValueError:
        pass
    try:
        return float(raw)
    except ValueError:
        pass
    return {"true": True, "false": False}.get(raw.lower(), raw)


def apply_overrides(config: Config, items: list[str]) -> Config:
    parsed = {}
    for item in items:
        if "=" not in item:
            raise SystemExit(f"--set expects KEY=VALUE, got '{item}'")
        key, raw = item.split("=", 1)
        parsed[key] = parse_override(raw)
    return config.with_overrides(parsed) if parsed else config


# ---------------------------------------------------------------- bathymetry
def _spectral_field(nx: int, ny: int, slope: float, seed: int, kmax: int = 0) -> np.ndarray:
    """Zero-mean periodic random field with amplitude spectrum |k|^-slope and
    seeded random phases; with kmax > 0 band-limited to |k| <= kmax, the phases
    drawn on the (2 kmax + 1)^2 lattice of the retained modes so the same modes
    get the same phases at any grid size (reference bathymetry.py:47-82)."""
    rng = np.random.default_rng(seed)
    kx = np.fft.fftfreq(nx) * nx
    ky = np.fft.fftfreq(ny) * ny
    KX, KY = np.meshgrid(kx, ky, indexing="xy")
    kk = np.hypot(KX, KY)
    amp = np.zeros_like(kk)
    pos = kk > 0
    amp[pos] = kk[pos] ** (-slope)
    if kmax > 0:
        amp[kk > kmax] = 0.0
        phase = np.zeros_like(kk)
        m = int(kmax)
        lattice = rng.uniform(0.0, 2.0 * np.pi, size=(2 * m + 1, 2 * m + 1))
        ix = np.round(KX).astype(int)
        iy = np.round(KY).astype(int)
        sel = (np.abs(ix) <= m) & (np.abs(iy) <= m)
        phase[sel] = lattice[iy[sel] + m, ix[sel] + m]
    else:
        phase = rng.uniform(0.0, 2.0 * np.pi, size=kk.shape)
    field = np.fft.ifft2(amp * np.exp(1j * phase)).real
    return field - field.mean()


def bathymetry(p: OceanParams, kind: str, H0: float, *, h_rel=0.9, length=0.0, slope=0.5, spectrum_slope=1.5,
               spectrum_kmax=0, r_target=0.1, seed=20260911, island=False):
    """(H, mask) of the named topography (reference bathymetry.py:85-124)."""
    x, y = _cases.centre_coords(p)
    Lx, Ly = p.lx, p.ly
    L = length if length > 0.0 else 0.1 * Lx
    if kind == "flat":
        H = np.full((p.ny, p.nx), H0)
    elif kind == "slope":
        H = H0 * (1.0 - slope * x / Lx)
    elif kind == "seamount":
        H = H0 * (1.0 - h_rel * np.exp(-((x - 0.5 * Lx) ** 2 + (y - 0.5 * Ly) ** 2) / L ** 2))
    elif kind == "ridge":
        H = H0 * (1.0 - h_rel * np.exp(-((x - 0.5 * Lx) / L) ** 2))
    elif kind == "rough":
        f = _spectral_field(p.nx, p.ny, spectrum_slope, seed, spectrum_kmax)
        f = f / np.std(f)
        H = np.maximum(H0 * (1.0 + r_target * f), 0.1 * H0)
    else:
        raise ValueError(f"unknown bathymetry '{kind}' (expected flat|slope|seamount|ridge|rough)")
    mask = np.ones((p.ny, p.nx))
    if island:
        mask[(np.abs(x - 0.5 * Lx) < 0.1 * Lx) & (np.abs(y - 0.5 * Ly) < 0.1 * Ly)] = 0.0
    return H, mask


# ---------------------------------------------------------------- the run
@dataclass
class RunSetup:
    params: OceanParams
    H: np.ndarray
    mask: np.ndarray
    dzr: np.ndarray | None
    taux_c: np.ndarray | None
    tauy_c: np.ndarray | None
    state: SimpleNamespace      # eta, u, v, b, T, S (T, S None with buoyancy tracers)
    dt: float
    n_steps: int
    t_final: float
    dt_max: float


def params_from_config(config: Config, nx: int, nz: int, ny: int | None = None) -> OceanParams:
    """The namelist parameters of the tree (driver3d_v05.py:25-94, schemes.py:180-196);
    dt and the step count are resolved by ``resolve_run``."""
    g = config.get
    v6 = g("physics3d_v06", {}) or {}
    return OceanParams(
        nx=int(nx), ny=int(ny if ny is not None else nx), nz=int(nz),
        lx=float(g("grid.Lx")), ly=float(g("grid.Ly")),
        g=float(g("physics.g")), f0=float(g("physics.f0")), h0=float(g("physics.H")),
        n2=float(g("physics3d.N2")), nu=float(g("physics3d.nu")), kappa=float(g("physics3d.kappa")),
        rho0=float(g("physics.rho0")), tau_x=float(g("physics3d.tau_x")), tau_y=float(g("physics3d.tau_y")),
        bottom_drag=float(g("physics3d.bottom_drag")),
        scheme_name=str(g("scheme.name")), theta=float(g("scheme.theta")),
        theta_cor=float(g("scheme.theta_cor")), theta_v=float(g("scheme.theta_v", 0.5)),
        n_picard=int(g("scheme.n_picard")), n_split=int(g("scheme.n_split", 0)),
        barotropic_average=str(g("scheme.barotropic_average", "none")),
        solver_kind=str(g("solver.kind")), rtol=float(g("solver.rtol")), max_iter=int(g("solver.max_iter")),
        vcoord=str(g("domain.vcoord")), bc_x=str(g("domain.bc_x")), bc_y=str(g("domain.bc_y")),
        face_rule=str(g("domain.face_rule", "min")), min_partial=float(g("domain.min_partial", 0.1)),
        eos=str(g("physics3d_v05.eos")), pgf=str(g("physics3d_v05.pgf")),
        pgf_correction=bool(g("physics3d_v05.pgf_correction", True)),
        advection=str(g("scheme.advection", "none")), tracers=str(g("physics3d_v04.tracers")),
        alpha_t=float(g("physics3d_v04.alpha_T")), beta_s=float(g("physics3d_v04.beta_S")),
        t0=float(g("physics3d_v04.T0")), s0=float(g("physics3d_v04.S0")), cp=float(g("physics3d_v04.cp")),
        a_h=float(g("physics3d_v04.A_h")), k_h=float(g("physics3d_v04.K_h")),
        q_heat=float(g("physics3d_v04.q_heat")), q_salt=float(g("physics3d_v04.q_salt")),
        closure=str(v6.get("closure", "none")), mxl=str(v6.get("mxl", "integral")),
        c_k=float(v6.get("c_k", 0.1)), c_eps=float(v6.get("c_eps", 0.7)), pr_t=float(v6.get("pr_t", 1.0)),
        z_0=float(v6.get("z_0", 0.1)), e_min=float(v6.get("e_min", 1.0e-6)), l_min=float(v6.get("l_min", 0.01)),
        e_bb=float(v6.get("e_bb", 3.75)), n2_min=float(v6.get("n2_min", 1.0e-8)),
    )


def barotropic_dt_max(p: OceanParams, H, mask) -> float:
    """Surface gravity-wave limit of the deepest wet column (driver3d_v05.py:97-101)."""
    c = np.sqrt(p.g * float(np.max(H[mask > 0])))
    return 1.0 / (c * np.sqrt(1.0 / p.dx ** 2 + 1.0 / p.dy ** 2))


def _eos_b(p, T, S, z):
    from .eos_host import buoyancy
    return buoyancy(p, T, S, z)


def _case_state(config: Config, name: str, p: OceanParams, H, mask):
    """(state, t_final) of a v0.5 case (cases3d_v05.py:32-400)."""
    nz, ny, nx = p.nz, p.ny, p.nx
    s = config.section(f"case.{name}")
    _, m3, zc = _cases.resting_layers(H, mask, None, nz, p.min_partial)
    zero3 = np.zeros((nz, ny, nx))
    if name == "seamount_rest":
        b = -p.g * (float(s["delta_rho"]) * np.exp(-zc / 500.0)) / p.rho0 * m3
        st = SimpleNamespace(eta=np.zeros((ny, nx)), u=zero3, v=zero3.copy(), b=b, T=None, S=None)
        return st, float(s["n_days"]) * 86400.0
    if name == "lock_exchange":
        x, _ = _cases.centre_coords(p)
        warm = (x > 0.5 * p.lx).astype(np.float64)
        T = (p.t0 + float(s["delta_T"]) * warm)[None, :, :] * np.ones((nz, ny, nx))
        S = np.full((nz, ny, nx), p.s0)
        b = _eos_b(p, T, S, zc) * m3
        st = SimpleNamespace(eta=np.zeros((ny, nx)), u=zero3, v=zero3.copy(), b=b, T=T * m3, S=S * m3)
        return st, float(s["n_hours"]) * 3600.0
    if name == "basin_seiche":
        x, _ = _cases.centre_coords(p)
        eta = float(s["eta0"]) * np.cos(np.pi * x / p.lx) * mask
        eta -= np.sum(eta) / max(1.0, float(np.sum(mask)))
        eta *= mask
        h_mean = float(np.mean(H[mask > 0]))
        period = 2.0 * p.lx / np.sqrt(p.g * h_mean)
        st = SimpleNamespace(eta=eta, u=zero3, v=zero3.copy(), b=zero3.copy(), T=None, S=None)
        return st, float(s["n_periods"]) * period
    raise ValueError(f"case '{name}' is not carried by this front end "
                     "(seamount_rest|lock_exchange|basin_seiche|seamount_basin)")


def resolve_run(config: Config, nx: int | None = None, nz: int | None = None, case: str | None = None,
                cfl: float | None = None, n_steps: int | None = None, ny: int | None = None) -> RunSetup:
    """Domain, parameters, initial state, dt and step count of a v0.5 run
    (tools/toml2nml.py:143-186): dt = cfl x the barotropic limit, and the step
    count lands on the case's t_final unless pinned."""
    case = case or str(config.get("case.name"))
    nx = int(nx or config.get("grid.nx"))
    nz = int(nz or config.get("grid.nz"))
    cfl = float(cfl if cfl is not None else config.get("time.cfl_factor"))
    if case == "seamount_basin":
        s = _cases.seamount_basin(nx=nx, ny=ny or nx, nz=nz)
        p = s.params
        st = SimpleNamespace(eta=s.eta, u=s.u, v=s.v, b=None, T=s.T, S=s.S)
        steps = n_steps if n_steps is not None else 100
        return RunSetup(p, s.H, s.mask, s.dzr, s.taux_c, s.tauy_c, st, p.dt, steps, p.dt * steps,
                        barotropic_dt_max(p, s.H, s.mask))
    p = params_from_config(config, nx, nz, ny)
    g = lambda k, d: config.get(f"bathymetry.{k}", d)  # noqa: E731
    H, mask = bathymetry(p, str(g("kind", "flat")), p.h0, h_rel=float(g("h_rel", 0.9)),
                         length=float(g("length", 0.0)), slope=float(g("slope", 0.5)),
                         spectrum_slope=float(g("spectrum_slope", 1.5)), spectrum_kmax=int(g("spectrum_kmax", 0)),
                         r_target=float(g("r_target", 0.1)), seed=int(g("seed", 20260911)),
                         island=bool(g("island", False)))
    state, t_final = _case_state(config, case, p, H, mask)
    dt_max = barotropic_dt_max(p, H, mask)
    dt_req = cfl * dt_max
    if n_steps is not None:
        steps, dt = int(n_steps), dt_req
    else:
        steps = max(1, int(round(t_final / dt_req)))
        dt = t_final / steps
    p = p.replace(dt=dt, n_steps=steps, t_final=dt * steps, case_name=case)
    return RunSetup(p, H, mask, None, None, None, state, dt, steps, dt * steps, dt_max)
