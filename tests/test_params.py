"""Namelist contract: the reference's bundle namelists parse into the same parameters."""

from dataclasses import asdict

import pytest

from harness import fixture_names, load_fixture, params_from_meta
from hydrostatic_ocean_core_benchmark_b200.params import (OceanParams, read_namelist,
                                                          write_namelist)

GATES = [n for n in fixture_names() if n.startswith("gate_")]


@pytest.mark.parametrize("name", GATES)
def test_reference_namelist_parses_to_fixture_params(name, tmp_path):
    meta, _ = load_fixture(name)
    path = tmp_path / "run.nml"
    path.write_text(meta["nml_text"])
    got = read_namelist(path)
    want = params_from_meta(meta)
    for key in ("nx", "ny", "nz", "lx", "ly", "g", "f0", "h0", "n2", "nu", "kappa", "rho0", "tau_x",
                "tau_y", "bottom_drag", "scheme_name", "theta", "theta_cor", "theta_v", "n_picard",
                "solver_kind", "rtol", "max_iter", "dt", "bc_x", "bc_y", "face_rule", "min_partial",
                "eos", "pgf", "pgf_correction", "advection", "tracers", "alpha_t", "beta_s", "t0",
                "s0", "cp", "a_h", "k_h", "q_heat", "q_salt", "closure", "c_k", "c_eps", "pr_t",
                "z_0", "e_min", "l_min", "e_bb", "n2_min", "mxl"):
        assert getattr(got, key) == getattr(want, key), key


def test_namelist_round_trip(tmp_path):
    p = OceanParams(nx=17, ny=9, nz=5, dt=123.456, tau_x=0.1, eos="teos10", closure="tke",
                    pgf_correction=False, levels_file="x_levels.bin")
    q = read_namelist(write_namelist(tmp_path / "a.nml", p))
    assert asdict(p) == asdict(q)


def test_validate_refuses_unsupported():
    with pytest.raises(ValueError):
        OceanParams(dt=1.0, vcoord="sigma").validate()
    with pytest.raises(ValueError):
        OceanParams(dt=1.0, bc_x="open").validate()
    with pytest.raises(ValueError):
        OceanParams(dt=1.0, scheme_name="theta", theta=0.0).validate()


def test_params_from_reference_reads_every_attribute():
    """The reference's objects by attribute (model3d.py Physics3D, model3d_v05.py
    PhysicsV05 delegating to its ``base``, schemes.py SchemeParams, domain.py Domain
    with its CGrid): each parameter takes a distinctive value, so an attribute read
    under the wrong name (and silently defaulted) would show."""
    from types import SimpleNamespace

    from hydrostatic_ocean_core_benchmark_b200.params import params_from_reference

    base = SimpleNamespace(g=9.7, f=1.3e-4, H=4100.0, N2=2e-5, nu=3e-3, kappa=4e-4, rho0=1026.0, tau_x=0.11,
                           tau_y=-0.02, bottom_drag=1e-3, tracers="TS", alpha_T=2.1e-4, beta_S=7.5e-4, T0=11.0,
                           S0=34.5, cp=3991.0, A_h=50.0, K_h=20.0, q_heat=-5.0, q_salt=1e-6)

    class PhysicsV05:
        closure, c_k, c_eps, pr_t, z_0 = "tke", 0.11, 0.71, 1.1, 0.2
        e_min, l_min, e_bb, n2_min, mxl = 2e-6, 0.02, 3.8, 2e-8, "recursive"
        eos, pgf, pgf_correction = "seos", "keep", False

        def __init__(self, b):
            self.base = b

        def __getattr__(self, name):
            return getattr(self.base, name)

    scheme = SimpleNamespace(name="theta", theta=0.6, theta_cor=0.55, theta_v=0.45, n_picard=3, n_split=7,
                             barotropic_average="mean", solver="pcg_rbgs", rtol=1e-11, max_iter=1234,
                             advection="up3_tvd")
    grid = SimpleNamespace(nx=40, ny=36, nz=12, Lx=2.1e6, Ly=1.9e6)
    domain = SimpleNamespace(grid=grid, vcoord="zlevel", bc_x="closed", bc_y="periodic", face_rule="harmonic",
                             min_partial=0.15)
    p = params_from_reference(domain, PhysicsV05(base), scheme, 450.0)
    want = dict(nx=40, ny=36, nz=12, lx=2.1e6, ly=1.9e6, g=9.7, f0=1.3e-4, h0=4100.0, n2=2e-5, nu=3e-3,
                kappa=4e-4, rho0=1026.0, tau_x=0.11, tau_y=-0.02, bottom_drag=1e-3, tracers="TS", alpha_t=2.1e-4,
                beta_s=7.5e-4, t0=11.0, s0=34.5, cp=3991.0, a_h=50.0, k_h=20.0, q_heat=-5.0, q_salt=1e-6,
                closure="tke", c_k=0.11, c_eps=0.71, pr_t=1.1, z_0=0.2, e_min=2e-6, l_min=0.02, e_bb=3.8,
                n2_min=2e-8, mxl="recursive", eos="seos", pgf="keep", pgf_correction=False,
                scheme_name="theta", theta=0.6, theta_cor=0.55, theta_v=0.45, n_picard=3, n_split=7,
                barotropic_average="mean", solver_kind="pcg_rbgs", rtol=1e-11, max_iter=1234,
                advection="up3_tvd", dt=450.0, vcoord="zlevel", bc_x="closed", bc_y="periodic",
                face_rule="harmonic", min_partial=0.15)
    for k, v in want.items():
        assert getattr(p, k) == v, (k, getattr(p, k), v)
