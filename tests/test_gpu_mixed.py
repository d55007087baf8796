"""The mixed-precision step (precision = "mixed") against the fp64 oracle.

The mixed path keeps the 3D state and stencils in FP32 and the buoyancy, the
pressure gradient, the EOS, the surface elevation and the Helmholtz solve in
fp64 (the configured solver, to the same fp64 tolerance). It has no reference
counterpart, so its pins are the oracle (the fp64 path equals it bit for bit)
and the error bounds below, measured on the benchmark recipe: relative L2 of
every field against the oracle after a run.
"""

import numpy as np
import pytest

from hydrostatic_ocean_core_benchmark_b200 import cases
from oracle import ocean_oracle as orc

pytestmark = pytest.mark.gpu

# relative L2 against the oracle after 10 steps of the seamount-basin recipe at
# 48 x 40 x 12: about 4x the values measured on a B200 (eta 6.9e-5, u 9.6e-5,
# v 8.0e-5, b 2.5e-6, T 6.2e-7, S 8.0e-7, e 4.0e-8, K 4.0e-7)
TOL = {"eta": 3e-4, "u": 4e-4, "v": 4e-4, "b": 1e-5, "T": 3e-6, "S": 3e-6, "e": 1e-6, "km": 2e-6,
       "kh": 2e-6}


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    import torch
    assert torch.cuda.is_available()
    torch.cuda.set_device(0)


def _rel(a, b):
    den = float(np.sqrt(np.sum(b * b)))
    num = float(np.sqrt(np.sum((a - b) ** 2)))
    return num / den if den > 0 else num


def _mixed(s, steps, graph=False):
    from hydrostatic_ocean_core_benchmark_b200.stepper import OceanStepper
    st = OceanStepper(s.params, s.H, s.mask, dzr=s.dzr, taux_c=s.taux_c, tauy_c=s.tauy_c, precision="mixed")
    st.set_state(eta=s.eta, u=s.u, v=s.v, T=s.T, S=s.S)
    st.step(steps, graph=graph)
    out = st.get_state()
    log = st.solve_log()
    stats = st.stats()
    st.close()
    return out, log, stats


@pytest.mark.parametrize("solver", ["multigrid", "pcg_refined", "pcg_mg"])
def test_mixed_step_stays_within_its_bounds_of_the_oracle(solver):
    """With the configured multigrid (warm-started), the FP32-inner solve under
    FP64 refinement (pcg_refined), or MG-preconditioned CG (warm-started), all to
    the same FP64 stopping test."""
    s = cases.seamount_basin(nx=48, ny=40, nz=12, seed=3, solver_kind=solver)
    p = s.params
    steps = 10
    got, log, stats = _mixed(s, steps)
    p = p.replace(solver_kind="multigrid")  # the oracle runs the reference's solver
    geo = orc.Geometry(p, s.H, s.mask, s.dzr)
    b = orc.buoyancy(p.eos, s.T, s.S, geo.zc, p.g, p.rho0, p.alpha_t, p.beta_s, p.t0, p.s0) * geo.mask3
    ref = orc.OracleStepper(p, s.H, s.mask, dzr=s.dzr, taux_c=s.taux_c, tauy_c=s.tauy_c)
    state = orc.OracleState(s.u, s.v, b, s.eta, s.T, s.S)
    for _ in range(steps):
        state = ref.step(state)
    errs = {}
    for f in TOL:
        want = {"km": ref.Km, "kh": ref.Kh}.get(f, None)
        want = getattr(state, f) if want is None else want
        errs[f] = _rel(got[f], want)
    bad = {f: e for f, e in errs.items() if not e < TOL[f]}
    assert not bad, f"relative L2 above the bounds: {bad} (all: {errs})"
    assert stats["solver_failures"] == 0 and not stats["diverged"]
    assert len(log) == len(ref.solve_log)


@pytest.mark.parametrize("solver", ["multigrid", "pcg_refined", "pcg_mg"])
def test_mixed_graph_replay_equals_plain_steps(solver):
    s = cases.seamount_basin(nx=40, ny=36, nz=10, seed=5, solver_kind=solver)
    a, la, _ = _mixed(s, 6, graph=False)
    b, lb, _ = _mixed(s, 6, graph=True)
    for f in a:
        assert np.array_equal(a[f], b[f]), f
    assert la == lb


@pytest.mark.parametrize("over", [{"scheme_name": "split_explicit"}, {"tracers": "buoyancy"}])
def test_mixed_refuses_what_it_does_not_run(over):
    from hydrostatic_ocean_core_benchmark_b200._lib import OceanError
    from hydrostatic_ocean_core_benchmark_b200.stepper import OceanStepper
    s = cases.seamount_basin(nx=16, ny=16, nz=4, seed=1)
    with pytest.raises(OceanError, match="unsupported option"):
        OceanStepper(s.params.replace(**over), s.H, s.mask, dzr=s.dzr, precision="mixed")
