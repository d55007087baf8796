"""Seeded synthetic workloads for the ocean-core step (host-side set-up only).

Two recipes, with the sizes and value distributions the benchmark names:

* ``lock_exchange_channel``: the reference's lock-exchange initial state
  (reference ``libs/core/cases3d_v05.py:245-258``) in a flat closed channel,
  T = T0 | T0 + delta_T split at x = Lx/2, S = S0, at rest.
* ``seamount_basin``: a closed basin over depth ``h0`` minus a seeded sum of
  Gaussian seamounts (clipped to a minimum depth), stretched levels growing
  geometrically from ``dz_top`` to ``dz_bottom``, a stratified T/S profile with
  seeded noise and a double-gyre zonal wind stress 0.1 cos(2 pi y / Ly).

Nothing here is on the timed path; every array is fp64 [k, j, i].
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .params import OceanParams


@dataclass
class CaseSetup:
    params: OceanParams
    H: np.ndarray                  # [ny, nx] positive depth
    mask: np.ndarray               # [ny, nx] 1 ocean / 0 land
    dzr: np.ndarray | None         # [nz] reference level thicknesses, None = uniform
    taux_c: np.ndarray | None      # [ny, nx] surface stress at centres, None = scalar
    tauy_c: np.ndarray | None
    T: np.ndarray | None           # initial T/S at cell centres before masking
    S: np.ndarray | None
    u: np.ndarray
    v: np.ndarray
    eta: np.ndarray
    b: np.ndarray | None = None    # None = diagnose from T/S with the EOS
    seed: int = 0
    name: str = ""


def centre_coords(p: OceanParams):
    x = (np.arange(p.nx) + 0.5) * p.dx
    y = (np.arange(p.ny) + 0.5) * p.dy
    return np.meshgrid(x, y, indexing="xy")


def resting_layers(H, mask, dzr, nz, min_partial):
    """Resting thickness per cell and the centre depth (z-level partial cells).

    Same rule as the reference's ``Domain._resting_thickness`` and
    ``depth_at_centres`` (``libs/core/domain.py:113-154``); used here only to
    place the initial T/S profiles.
    """
    if dzr is None:
        dzr = np.full(nz, float(np.max(H[mask > 0])) / nz)
    edges = np.concatenate([[0.0], np.cumsum(dzr)])
    dz3 = np.clip(H[None] - edges[:-1, None, None], 0.0, dzr[:, None, None])
    dz3 = np.where((dz3 > 0.0) & (dz3 < min_partial * dzr[:, None, None]), 0.0, dz3)
    m3 = (dz3 > 0.0).astype(np.float64) * mask[None]
    dz3 = dz3 * m3
    above = np.concatenate([np.zeros((1,) + H.shape), np.cumsum(dz3[:-1], axis=0)], axis=0)
    return dz3, m3, above + 0.5 * dz3


def lock_exchange_channel(nx=128, ny=4, nz=32, lx=0.8, ly=0.025, depth=0.1, delta_T=10.0,
                          dt=0.05, **over) -> CaseSetup:
    """Flat closed channel, linear EOS, TVD3, TKE off, theta + PCG-Jacobi."""
    p = OceanParams(nx=nx, ny=ny, nz=nz, lx=lx, ly=ly, h0=depth, nu=1.0e-6, kappa=1.0e-6,
                    scheme_name="theta", theta=0.5, n_picard=2, solver_kind="pcg_jacobi",
                    rtol=1.0e-12, max_iter=2000, dt=dt, bc_x="closed", bc_y="closed",
                    eos="linear", advection="up3_tvd", tracers="TS", closure="none",
                    case_name="lock_exchange")
    p = p.replace(**over)
    H = np.full((ny, nx), depth)
    mask = np.ones((ny, nx))
    x, _ = centre_coords(p)
    warm = (x > 0.5 * p.lx).astype(np.float64)
    T = (p.t0 + delta_T * warm)[None, :, :] * np.ones((nz, ny, nx))
    S = np.full((nz, ny, nx), p.s0)
    zero3 = np.zeros((nz, ny, nx))
    return CaseSetup(p, H, mask, None, None, None, T, S, zero3, zero3.copy(),
                     np.zeros((ny, nx)), name="lock_exchange_channel")


def seamount_bathymetry(p: OceanParams, rng, n_seamounts=8, h_lo=500.0, h_hi=2500.0,
                        r_lo=5.0e4, r_hi=2.0e5, h_min=200.0):
    x, y = centre_coords(p)
    H = np.full((p.ny, p.nx), p.h0)
    for _ in range(n_seamounts):
        x0, y0 = rng.uniform(0.0, p.lx), rng.uniform(0.0, p.ly)
        h, r = rng.uniform(h_lo, h_hi), rng.uniform(r_lo, r_hi)
        H = H - h * np.exp(-((x - x0) ** 2 + (y - y0) ** 2) / r ** 2)
    return np.maximum(H, h_min)


def stretched_levels(nz, h_max, dz_top=10.0, dz_bottom=250.0):
    """Thicknesses growing geometrically from dz_top to dz_bottom, summing to h_max."""
    if nz == 1:
        return np.array([h_max])
    dz = dz_top * (dz_bottom / dz_top) ** (np.arange(nz) / (nz - 1))
    return dz * (h_max / np.sum(dz))


def seamount_basin(nx=512, ny=512, nz=50, seed=20261203, stretched=True, wind_field=True,
                   lx=2.0e6, ly=2.0e6, depth=4000.0, dt=600.0, **over) -> CaseSetup:
    """Closed seamount basin: TKE, TVD3, polyTEOS10, theta + multigrid, wind-driven.

    theta = 0.6 (the reference's "schism" preset, config/schemes.toml): at
    512 x 512 the barotropic CFL is ~30 and the neutral theta = 0.5 scheme
    diverges after ~60 steps for this recipe, with or without wind, Coriolis,
    TKE, stretched levels or extra Picard passes; theta >= 0.6 is stable.
    """
    p = OceanParams(nx=nx, ny=ny, nz=nz, lx=lx, ly=ly, h0=depth, nu=1.0e-3, kappa=1.0e-3,
                    tau_x=0.1, scheme_name="theta", theta=0.6, n_picard=2,
                    solver_kind="multigrid", rtol=1.0e-12, max_iter=2000, dt=dt,
                    bc_x="closed", bc_y="closed", eos="teos10", pgf="keep",
                    advection="up3_tvd", tracers="TS", closure="tke", mxl="integral",
                    case_name="seamount_basin")
    p = p.replace(**over)
    rng = np.random.default_rng(seed)
    H = seamount_bathymetry(p, rng)
    mask = np.ones((ny, nx))
    h_max = float(np.max(H[mask > 0]))
    dzr = stretched_levels(nz, h_max) if stretched else None
    _, m3, zc = resting_layers(H, mask, dzr, nz, p.min_partial)
    T = 2.0 + 18.0 * np.exp(-zc / 800.0) + rng.normal(0.0, 0.01, size=zc.shape)
    S = 35.0 + 0.5 * np.exp(-zc / 500.0)
    _, y = centre_coords(p)
    taux = 0.1 * np.cos(2.0 * np.pi * y / p.ly) if wind_field else None
    tauy = np.zeros((ny, nx)) if wind_field else None
    zero3 = np.zeros((nz, ny, nx))
    return CaseSetup(p, H, mask, dzr, taux, tauy, T * m3, S * m3, zero3, zero3.copy(),
                     np.zeros((ny, nx)), seed=seed, name="seamount_basin")
