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
