"""Failure reporting on the GPU, with every failure made on the host.

The reference binary stops a run and reports ``"diverged": true`` when the
surface elevation is NaN or above 1e6 at its every-tenth-step check
(libs/cuda/src/cfd_exp3d5_cuda.cu:1145-1154), and counts a Helmholtz solve that
hits ``max_iter`` as a solver failure (:410-411). Both are injected here through
the inputs (a NaN in the initial bundle, ``max_iter = 1``), so no kernel faults,
traps or hangs.
"""

import json
import subprocess
from pathlib import Path

import numpy as np
import pytest

from hydrostatic_ocean_core_benchmark_b200 import cases
from oracle import ocean_oracle as orc

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]
EXE = ROOT / "hydrostatic_ocean_core_benchmark_b200" / "bin" / "ocean3d5_b200"


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    import torch
    assert torch.cuda.is_available()
    torch.cuda.set_device(0)


def _bundle(tmp_path, p, s, eta=None):
    from hydrostatic_ocean_core_benchmark_b200.bundle import write_bundle
    geo = orc.Geometry(p, s.H, s.mask, s.dzr)
    b = orc.buoyancy(p.eos, s.T, s.S, geo.zc, p.g, p.rho0, p.alpha_t, p.beta_s, p.t0, p.s0) * geo.mask3
    st = orc.OracleState(s.u, s.v, b, s.eta if eta is None else eta, s.T, s.S)
    return write_bundle(str(tmp_path / "case"), p, s.H, s.mask, st, dzr=s.dzr, taux_c=s.taux_c,
                        tauy_c=s.tauy_c)


def test_nan_in_the_initial_bundle_is_reported_as_diverged(tmp_path):
    s = cases.seamount_basin(nx=16, ny=16, nz=6, seed=2, max_iter=20)
    p = s.params.replace(n_steps=20, n_warmup=0, n_repeat=1, out_prefix=str(tmp_path / "out"))
    eta = s.eta.copy()
    eta[5, 7] = np.nan
    r = subprocess.run([str(EXE), _bundle(tmp_path, p, s, eta)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    m = json.loads(Path(p.out_prefix + "_metrics.json").read_text())
    assert m["diverged"] is True
    assert "DIVERGED" in r.stdout


def test_nan_state_sets_the_handles_diverged_flag():
    from hydrostatic_ocean_core_benchmark_b200.stepper import OceanStepper
    s = cases.seamount_basin(nx=16, ny=16, nz=6, seed=2, max_iter=20)
    st = OceanStepper(s.params, s.H, s.mask, dzr=s.dzr, taux_c=s.taux_c, tauy_c=s.tauy_c)
    st.set_state(eta=s.eta, u=s.u, v=s.v, T=s.T, S=s.S)
    st.step(2)
    assert not st.stats()["diverged"]
    eta = s.eta.copy()
    eta[3, 3] = np.nan
    st.set_state(eta=eta, u=s.u, v=s.v, T=s.T, S=s.S)
    st.step(1)
    stats = st.stats()
    assert stats["diverged"] and stats["device_status"] == 0
    st.close()


@pytest.mark.parametrize("solver", ["multigrid", "pcg_jacobi"])
def test_max_iter_one_counts_solver_failures(tmp_path, solver):
    s = cases.seamount_basin(nx=32, ny=32, nz=8, seed=4, solver_kind=solver, max_iter=1)
    p = s.params.replace(n_steps=3, n_warmup=0, n_repeat=1, out_prefix=str(tmp_path / "out"))
    r = subprocess.run([str(EXE), _bundle(tmp_path, p, s)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    m = json.loads(Path(p.out_prefix + "_metrics.json").read_text())
    # two Picard passes, each one solve that stops unconverged after one iteration
    assert m["solver_failures"] == 6 and m["solver_iterations"] == 6
    # the same through the Python mirror, against the oracle's counts
    from hydrostatic_ocean_core_benchmark_b200.stepper import OceanStepper
    st = OceanStepper(s.params, s.H, s.mask, dzr=s.dzr, taux_c=s.taux_c, tauy_c=s.tauy_c)
    st.set_state(eta=s.eta, u=s.u, v=s.v, T=s.T, S=s.S)
    st.step(3)
    geo = orc.Geometry(s.params, s.H, s.mask, s.dzr)
    p0 = s.params
    b = orc.buoyancy(p0.eos, s.T, s.S, geo.zc, p0.g, p0.rho0, p0.alpha_t, p0.beta_s, p0.t0, p0.s0) * geo.mask3
    ref = orc.OracleStepper(p0, s.H, s.mask, dzr=s.dzr, taux_c=s.taux_c, tauy_c=s.tauy_c)
    state = orc.OracleState(s.u, s.v, b, s.eta, s.T, s.S)
    for _ in range(3):
        state = ref.step(state)
    stats = st.stats()
    assert stats["solver_failures"] == ref.solver_failures == 6
    assert st.solve_log() == ref.solve_log
    assert np.array_equal(st.get_state(fields=("eta",))["eta"], state.eta)
    st.close()


def test_a_barrier_wait_that_runs_out_returns_timeout_and_the_device_stays_usable():
    """The solve's grid barriers spin with a bound; a bound of 200 cycles runs
    out on the first barrier a CTA reaches before the others. Every CTA then
    leaves the solve, the handle reports OC_ERR_TIMEOUT, and a fresh handle on
    the same device steps normally."""
    from hydrostatic_ocean_core_benchmark_b200._lib import OceanError
    from hydrostatic_ocean_core_benchmark_b200.stepper import OceanStepper
    s = cases.seamount_basin(nx=128, ny=128, nz=6, seed=7)

    def fresh():
        st = OceanStepper(s.params, s.H, s.mask, dzr=s.dzr, taux_c=s.taux_c, tauy_c=s.tauy_c)
        st.set_state(eta=s.eta, u=s.u, v=s.v, T=s.T, S=s.S)
        return st

    st = fresh()
    st.set_wait_bound(200)
    st.step(1)
    with pytest.raises(OceanError, match="timed out"):
        st.stats()
    st.close()
    ok = fresh()
    ok.step(2)
    stats = ok.stats()
    assert stats["device_status"] == 0 and stats["solver_failures"] == 0 and not stats["diverged"]
    ok.close()
