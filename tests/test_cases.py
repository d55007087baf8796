"""The seeded seamount-basin recipe behind the benchmark (cases.seamount_basin),
pinned on CPU to its stated description: depth 4000 m minus 8 Gaussian
seamounts (heights U(500, 2500) m, radii U(50, 200) km) clipped at 200 m; levels
growing geometrically from 10 to 250 m, scaled to the deepest column;
T = 2 + 18 exp(-d/800) + N(0, 0.01^2) and S = 35 + 0.5 exp(-d/500) on wet cells;
wind tau_x = 0.1 cos(2 pi y / Ly); theta = 0.6 with the multigrid at rtol 1e-12,
TKE, TVD3, polyTEOS10, closed walls, dt = 600 s."""

import numpy as np

from hydrostatic_ocean_core_benchmark_b200 import cases


def test_seamount_basin_recipe():
    s = cases.seamount_basin(nx=128, ny=128, nz=50, seed=11)
    p = s.params
    assert (p.scheme_name, p.theta, p.solver_kind, p.rtol, p.dt) == ("theta", 0.6, "multigrid", 1e-12, 600.0)
    assert (p.closure, p.advection, p.eos, p.tracers, p.bc_x, p.bc_y) == ("tke", "up3_tvd", "teos10", "TS",
                                                                          "closed", "closed")
    assert (p.lx, p.ly, p.h0, p.tau_x) == (2.0e6, 2.0e6, 4000.0, 0.1)
    H = s.H
    assert H.min() >= 200.0 and H.max() <= 4000.0 and H.min() < 3000.0  # seamounts are there
    assert (s.mask == 1.0).all()
    # levels: geometric from 10 to 250 m (ratio 25), scaled to the deepest column
    dz = s.dzr
    assert dz.shape == (50,) and np.all(np.diff(dz) > 0)
    assert np.isclose(dz[-1] / dz[0], 25.0, rtol=1e-12)
    assert np.isclose(np.sum(dz), H.max(), rtol=1e-12)
    ratios = dz[1:] / dz[:-1]
    assert np.allclose(ratios, ratios[0], rtol=1e-12)
    # tracer profiles on wet cells at the resting centre depth
    _, m3, zc = cases.resting_layers(H, s.mask, dz, 50, p.min_partial)
    wet = m3 > 0
    assert not s.T[~wet].any() and not s.S[~wet].any()
    assert np.allclose(s.S[wet], 35.0 + 0.5 * np.exp(-zc[wet] / 500.0), rtol=0, atol=1e-12)
    noise = s.T[wet] - (2.0 + 18.0 * np.exp(-zc[wet] / 800.0))
    assert abs(noise.mean()) < 1e-3 and 0.009 < noise.std() < 0.011
    # wind: a double gyre in tau_x, no tau_y
    _, y = cases.centre_coords(p)
    assert np.array_equal(s.taux_c, 0.1 * np.cos(2.0 * np.pi * y / p.ly)) and not s.tauy_c.any()
    # a resting start
    assert not s.eta.any() and not s.u.any() and not s.v.any()


def test_seamount_basin_is_seeded():
    a = cases.seamount_basin(nx=32, ny=32, nz=8, seed=3)
    b = cases.seamount_basin(nx=32, ny=32, nz=8, seed=3)
    c = cases.seamount_basin(nx=32, ny=32, nz=8, seed=4)
    for f in ("H", "T", "S", "dzr"):
        assert np.array_equal(getattr(a, f), getattr(b, f)), f
    assert not np.array_equal(a.H, c.H) and not np.array_equal(a.T, c.T)


def test_seamount_heights_and_radii_follow_their_draws():
    class Rng:
        """Stands in for the generator: fixed centres, the extreme heights and radii."""

        def __init__(self):
            self.vals = iter([1.0e6, 1.0e6, 2500.0, 2.0e5] + [0.0, 0.0, 500.0, 5.0e4] * 7)

        def uniform(self, lo, hi):
            v = next(self.vals)
            assert lo <= v <= hi
            return v

    s = cases.seamount_basin(nx=64, ny=64, nz=4, seed=1)
    H = cases.seamount_bathymetry(s.params, Rng())
    x, y = cases.centre_coords(s.params)
    r2 = (x - 1.0e6) ** 2 + (y - 1.0e6) ** 2
    corner = 7 * 500.0 * np.exp(-(x ** 2 + y ** 2) / 5.0e4 ** 2)
    want = np.maximum(4000.0 - 2500.0 * np.exp(-r2 / 2.0e5 ** 2) - corner, 200.0)
    assert np.allclose(H, want, rtol=0, atol=1e-9)
