"""The sm_100a step against the reference: every golden case, every step.

Gate (the reference's, tools/compare_backends3d5.py:28-29, applied per step):
relative L2 < 1e-12 for every field and the per-solve Helmholtz iteration
counts identical. The stronger claim checked beside it: every field is
bit-identical to the reference (fingerprints of the fp64 bytes).
"""

import numpy as np
import pytest

from harness import case_inputs, fixture_names, load_fixture
from oracle import ocean_oracle as orc

pytestmark = pytest.mark.gpu

GATE_TOL = 1e-12
CASES = fixture_names()


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    import torch
    assert torch.cuda.is_available(), "gpu tests need a CUDA device"
    torch.cuda.set_device(0)


@pytest.mark.parametrize("name", CASES)
def test_bit_identical_to_reference_every_step(name):
    from gpu_util import gpu_case, gpu_hashes
    meta, arrays = load_fixture(name)
    p, st = gpu_case(meta, arrays)
    for step, want in enumerate(meta["hashes"]):
        st.step(1)
        got = gpu_hashes(p, st.get_state())
        bad = [f for f, h in want.items() if got[f] != h]
        assert not bad, f"{name}: fields {bad} differ from the reference at step {step + 1}"
    assert st.solve_log() == meta["solve_log"]
    stats = st.stats()
    c = meta["counters"]
    assert stats["solver_iterations"] == c["solver_iterations"]
    assert stats["solver_failures"] == c["solver_failures"]
    assert stats["solver_rebuilds"] == c["solver_rebuilds"]
    assert stats["tridiagonal_solves"] == c["tridiagonal_solves"]
    assert stats["barotropic_substeps"] == c["barotropic_substeps"]
    assert stats["n_split"] == c["n_split"]
    st.close()


@pytest.mark.parametrize("name", CASES)
def test_reference_gate_per_step(name):
    """rel L2 < 1e-12 per step against the oracle, identical iteration counts."""
    from gpu_util import gpu_case, state_errors
    meta, arrays = load_fixture(name)
    p, H, mask, dzr, taux, tauy, s = case_inputs(meta, arrays)
    ref = orc.OracleStepper(p, H, mask)
    p2, st = gpu_case(meta, arrays)
    for step in range(meta["n_steps"]):
        s = ref.step(s)
        st.step(1)
        errs = state_errors(p, st.get_state(), s)
        worst = max(errs.values())
        assert worst < GATE_TOL, f"{name} step {step + 1}: {errs}"
    assert st.solve_log() == ref.solve_log
    st.close()


@pytest.mark.parametrize("solver", ["multigrid", "pcg_jacobi"])
def test_stretched_levels_and_wind_field_match_oracle(solver):
    """The benchmark's extensions (stretched levels, stress field) against the oracle."""
    from hydrostatic_ocean_core_benchmark_b200 import cases
    from hydrostatic_ocean_core_benchmark_b200.stepper import OceanStepper
    s = cases.seamount_basin(nx=32, ny=48, nz=16, seed=11, solver_kind=solver)
    p = s.params
    geo = orc.Geometry(p, s.H, s.mask, s.dzr)
    b = orc.buoyancy(p.eos, s.T, s.S, geo.zc, p.g, p.rho0, p.alpha_t, p.beta_s, p.t0, p.s0) * geo.mask3
    ref = orc.OracleStepper(p, s.H, s.mask, dzr=s.dzr, taux_c=s.taux_c, tauy_c=s.tauy_c)
    st = OceanStepper(p, s.H, s.mask, dzr=s.dzr, taux_c=s.taux_c, tauy_c=s.tauy_c)
    st.set_state(eta=s.eta, u=s.u, v=s.v, T=s.T, S=s.S)   # b diagnosed on the GPU
    assert np.array_equal(st.get_state(fields=("b",))["b"], b)
    state = orc.OracleState(s.u, s.v, b, s.eta, s.T, s.S)
    for step in range(5):
        state = ref.step(state)
        st.step(1)
        got = st.get_state()
        for f in ("eta", "u", "v", "b", "T", "S", "e", "km", "kh"):
            want = {"km": ref.Km, "kh": ref.Kh}.get(f, None)
            want = getattr(state, f) if want is None else want
            assert np.array_equal(got[f], want), f"{solver} step {step + 1}: {f} differs"
    assert st.solve_log() == ref.solve_log
    st.close()


@pytest.mark.parametrize("rule", ["mean", "harmonic"])
def test_face_rules_and_horizontal_mixing_match_oracle(rule):
    """The partial-cell face rules other than min (domain.py:60-154), with
    horizontal viscosity and diffusion on, on a grid whose 40 columns leave a
    partial 32-column tile: bit-identical to the oracle every step."""
    from hydrostatic_ocean_core_benchmark_b200 import cases
    from hydrostatic_ocean_core_benchmark_b200.stepper import OceanStepper
    s = cases.seamount_basin(nx=40, ny=36, nz=12, seed=5, face_rule=rule, a_h=1.0e3, k_h=1.0e3)
    p = s.params
    geo = orc.Geometry(p, s.H, s.mask, s.dzr)
    b = orc.buoyancy(p.eos, s.T, s.S, geo.zc, p.g, p.rho0, p.alpha_t, p.beta_s, p.t0, p.s0) * geo.mask3
    ref = orc.OracleStepper(p, s.H, s.mask, dzr=s.dzr, taux_c=s.taux_c, tauy_c=s.tauy_c)
    st = OceanStepper(p, s.H, s.mask, dzr=s.dzr, taux_c=s.taux_c, tauy_c=s.tauy_c)
    st.set_state(eta=s.eta, u=s.u, v=s.v, b=b, T=s.T, S=s.S)
    state = orc.OracleState(s.u, s.v, b, s.eta, s.T, s.S)
    for step in range(4):
        state = ref.step(state)
        st.step(1)
        got = st.get_state()
        for f in ("eta", "u", "v", "b", "T", "S", "e", "km", "kh"):
            want = {"km": ref.Km, "kh": ref.Kh}.get(f, None)
            want = getattr(state, f) if want is None else want
            assert np.array_equal(got[f], want), f"{rule} step {step + 1}: {f} differs"
    assert st.solve_log() == ref.solve_log
    st.close()


def _recipe_run(s, n_steps, per_step_check):
    """Step the GPU and the oracle side by side from the same initial state."""
    from hydrostatic_ocean_core_benchmark_b200.stepper import OceanStepper
    p = s.params
    geo = orc.Geometry(p, s.H, s.mask, s.dzr)
    b = orc.buoyancy(p.eos, s.T, s.S, geo.zc, p.g, p.rho0, p.alpha_t, p.beta_s, p.t0, p.s0) * geo.mask3
    ref = orc.OracleStepper(p, s.H, s.mask, dzr=s.dzr, taux_c=s.taux_c, tauy_c=s.tauy_c)
    state = orc.OracleState(s.u, s.v, b, s.eta, s.T, s.S)
    st = OceanStepper(p, s.H, s.mask, dzr=s.dzr, taux_c=s.taux_c, tauy_c=s.tauy_c)
    st.set_state(eta=s.eta, u=s.u, v=s.v, b=b, T=s.T, S=s.S)
    for step in range(n_steps):
        state = ref.step(state)
        st.step(1)
        per_step_check(step + 1, st.get_state(), state, ref)
        # the solve log grows by the step's solves, each count equal to the oracle's
        assert st.solve_log() == ref.solve_log, f"step {step + 1}: solve logs differ"
    stats = st.stats()
    assert stats["solver_failures"] == 0 and not stats["diverged"]
    st.close()
    return ref


def _all_fields_equal(step, got, state, ref):
    for f in ("eta", "u", "v", "b", "T", "S", "e", "km", "kh"):
        want = {"km": ref.Km, "kh": ref.Kh}.get(f, None)
        want = getattr(state, f) if want is None else want
        assert np.array_equal(got[f], want), (
            f"step {step}: {f} differs from the oracle (max |diff| {np.max(np.abs(got[f] - want)):.3e})")


def test_benchmark_recipe_hundred_steps_against_oracle():
    """The benchmark's recipe (stretched levels, double-gyre wind field, TKE with
    integral mixing lengths, TVD3, polyTEOS10, theta = 0.6 + multigrid at rtol
    1e-12, dt = 600 s) at 128 x 128 x 50 for the benchmark's 100 steps: every
    field bit-identical to the oracle after every step, the reference gate's
    relative L2 below 1e-12 per step, and the per-solve iteration counts equal
    (reference model3d_v05.py:337-415; gate tools/compare_backends3d5.py:28-29)."""
    from hydrostatic_ocean_core_benchmark_b200 import cases
    from gpu_util import state_errors
    s = cases.seamount_basin(nx=128, ny=128, nz=50)

    def check(step, got, state, ref):
        errs = state_errors(s.params, got, state)
        assert max(errs.values()) < GATE_TOL, f"step {step}: {errs}"
        _all_fields_equal(step, got, state, ref)

    ref = _recipe_run(s, 100, check)
    assert len(ref.solve_log) == 200


def test_benchmark_size_first_steps_match_oracle():
    """512 x 512 x 50 seamount basin, three steps, bit-identical to the oracle.
    At this size the multigrid solve runs its level 0 in 128 x 16 tiles, keeps
    the level-0 coefficients in shared memory for the whole solve and forms the
    residual-norm leaf sums inside the last up phase: paths that only grids
    above about 150,000 columns take."""
    from hydrostatic_ocean_core_benchmark_b200 import cases
    _recipe_run(cases.seamount_basin(), 3, _all_fields_equal)


def test_full_size_properties_over_ten_steps():
    """At the benchmark size, ten steps: deterministic, finite, uniform T stays uniform."""
    from hydrostatic_ocean_core_benchmark_b200 import cases
    from hydrostatic_ocean_core_benchmark_b200.stepper import OceanStepper
    s = cases.seamount_basin()
    p = s.params
    runs = []
    for _ in range(2):
        st = OceanStepper(p, s.H, s.mask, dzr=s.dzr, taux_c=s.taux_c, tauy_c=s.tauy_c)
        st.set_state(eta=s.eta, u=s.u, v=s.v, T=s.T, S=s.S)
        st.step(10)
        runs.append(st.get_state())
        stats = st.stats()
        assert stats["solver_failures"] == 0 and not stats["diverged"]
        st.close()
    for f in runs[0]:
        assert np.array_equal(runs[0][f], runs[1][f]), f"{f} not reproducible run to run"
        assert np.all(np.isfinite(runs[0][f]))
    # constancy: a uniform tracer stays uniform where the ocean is wet
    st = OceanStepper(p, s.H, s.mask, dzr=s.dzr, taux_c=s.taux_c, tauy_c=s.tauy_c)
    T = np.where(s.T != 0, 7.0, 0.0)
    st.set_state(eta=s.eta, u=runs[0]["u"], v=runs[0]["v"], b=runs[0]["b"], T=T, S=s.S)
    st.step(3)
    Tn = st.get_state(fields=("T",))["T"]
    wet = T != 0
    assert np.max(np.abs(Tn[wet] - 7.0)) < 1e-10
    st.close()
