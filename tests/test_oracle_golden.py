"""The CPU oracle reproduces the unmodified reference bit for bit (up to signed zeros)."""

import numpy as np
import pytest

from harness import case_inputs, fixture_names, load_fixture, run_oracle
from oracle import ocean_oracle as orc

CASES = fixture_names()


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference_every_step(name):
    meta, arrays = load_fixture(name)
    st, s, hashes = run_oracle(meta, arrays)
    assert st.solve_log == meta["solve_log"]
    for step, (got, want) in enumerate(zip(hashes, meta["hashes"])):
        for f, h in want.items():
            assert got[f] == h, f"{name}: field {f} differs at step {step + 1}"
    counters = meta["counters"]
    assert st.solver_iterations == counters["solver_iterations"]
    assert st.solver_failures == counters["solver_failures"]
    assert st.solver_rebuilds == counters["solver_rebuilds"]
    assert st.tridiagonal_solves == counters["tridiagonal_solves"]
    assert st.barotropic_substeps == counters["barotropic_substeps"]


@pytest.mark.parametrize("name", [n for n in CASES if not n.startswith("gate_")])
def test_regenerated_initial_state_matches_reference(name):
    meta, arrays = load_fixture(name)
    p, H, mask, _, _, _, s = case_inputs(meta, arrays)
    from golden_io import fhash
    for f, h in meta["init_hashes"].items():
        val = H if f == "H" else getattr(s, f)
        assert fhash(val) == h, f"{name}: regenerated initial {f} differs from the reference"


def test_extensions_reduce_to_reference():
    """Uniform level table and a uniform stress field give the reference bit for bit."""
    meta, arrays = load_fixture("seamount_basin_ref_mg")
    p, H, mask, *_ = case_inputs(meta, arrays)
    h_max = float(np.max(H[mask > 0]))
    dzr = np.full(p.nz, h_max / p.nz)
    taux = np.full((p.ny, p.nx), p.tau_x)
    tauy = np.full((p.ny, p.nx), p.tau_y)
    st, s, hashes = run_oracle(meta, arrays, n_steps=3, dzr=dzr, taux=taux, tauy=tauy)
    for step in range(3):
        assert hashes[step] == meta["hashes"][step]
    assert st.solve_log == meta["solve_log"][:len(st.solve_log)]


def test_teos10_check_value():
    """Roquet et al. (2015) check value used by the reference (tools/verify_v05.py:96-110)."""
    rho = float(orc.rho_teos10(np.array(10.0), np.array(30.0), np.array(1000.0)))
    assert abs(rho - 1027.45140) < 1e-4


def test_field_error_state_scale_fallback():
    a = np.zeros(10)
    b = np.full(10, 1e-30)
    assert orc.field_error(a, b, 1.0) < 1e-20
    assert orc.field_error(b * 2, b, 0.0) > 0
