"""Batched-ensemble form on the GPU.

Members of uneven grid sizes advanced together by one recorded CUDA graph per
two steps (oc_ensemble_*) must equal the same members stepped alone, bit for
bit, with the same counters and solve logs; the tiling knob (levels per CTA of
the momentum and tracer kernels, set by hand or by the autotuner) must leave
every bit unchanged.
"""

import numpy as np
import pytest

from hydrostatic_ocean_core_benchmark_b200 import cases

pytestmark = pytest.mark.gpu
FIELDS = ("eta", "u", "v", "b", "T", "S", "e", "km", "kh")
# nx, ny, nz, seed: the solvers of the two larger grids need different amounts of
# shared memory, created largest first
MEMBERS = [(512, 512, 6, 3), (256, 256, 6, 4), (40, 36, 12, 5), (136, 200, 8, 6)]


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    import torch
    assert torch.cuda.is_available()
    torch.cuda.set_device(0)


def _member(nx, ny, nz, seed, precision="fp64"):
    from hydrostatic_ocean_core_benchmark_b200.stepper import OceanStepper
    s = cases.seamount_basin(nx=nx, ny=ny, nz=nz, seed=seed)
    st = OceanStepper(s.params, s.H, s.mask, dzr=s.dzr, taux_c=s.taux_c, tauy_c=s.tauy_c, precision=precision)
    st.set_state(eta=s.eta, u=s.u, v=s.v, T=s.T, S=s.S)
    return st


def _same(a, b, what):
    sa, sb = a.get_state(), b.get_state()
    for f in FIELDS:
        assert np.array_equal(sa[f], sb[f]), f"{what}: {f} differs"


def test_levels_per_cta_change_no_bit():
    a, b, c = (_member(40, 36, 12, 3) for _ in range(3))
    b.set_tiling(3, 5)
    mk, tk = c.autotune()
    assert 1 <= mk <= 12 and 1 <= tk <= 12
    for st in (a, b, c):
        st.step(4)
    _same(a, b, "levels per CTA 3 / 5")
    _same(a, c, f"autotuned levels per CTA {mk} / {tk}")
    with pytest.raises(Exception):
        a.set_tiling(0, 13)
    for st in (a, b, c):
        st.close()


def test_mixed_autotuned_tiling_changes_no_bit():
    """On a mixed-precision handle the autotuner times the FP32 kernels; its choice,
    like a tiling set by hand, leaves every bit of the FP32 step unchanged."""
    a, b, c = (_member(40, 36, 12, 7, precision="mixed") for _ in range(3))
    b.set_tiling(3, 5)
    mk, tk = c.autotune()
    assert 1 <= mk <= 12 and 1 <= tk <= 12
    for st in (a, b, c):
        st.step(4)
    _same(a, b, "mixed, levels per CTA 3 / 5")
    _same(a, c, f"mixed, autotuned levels per CTA {mk} / {tk}")
    for st in (a, b, c):
        st.close()


def test_ensemble_equals_members_stepped_alone():
    from hydrostatic_ocean_core_benchmark_b200.stepper import OceanEnsemble
    together = [_member(*m) for m in MEMBERS]
    alone = [_member(*m) for m in MEMBERS]
    for st in together:
        st.autotune()
    ens = OceanEnsemble(together)
    ens.step(5)   # two graph replays, then one step member after member
    ens.step(4)   # the buffers swapped: recorded again, then two replays
    for st in alone:
        st.step(9)
    keys = ("steps", "solver_iterations", "solver_failures", "solver_rebuilds", "tridiagonal_solves")
    for m, (a, b) in enumerate(zip(together, alone)):
        assert a.stats()["solver_failures"] == 0
        _same(a, b, f"member {m} {MEMBERS[m][:3]}")
        sa, sb = a.stats(), b.stats()
        assert all(sa[k] == sb[k] for k in keys), (m, {k: (sa[k], sb[k]) for k in keys})
        assert a.solve_log() == b.solve_log()
    # the two smaller members directly against the oracle, field by field
    for m in (1, 2):
        _equal_to_oracle(MEMBERS[m], together[m], 9)
    ens.close()
    for st in together + alone:
        st.close()


def test_mixed_precision_ensemble_equals_members_stepped_alone():
    """Members of the mixed-precision step in one ensemble (batched solves) give
    the bits of the same members stepped alone."""
    from hydrostatic_ocean_core_benchmark_b200.stepper import OceanEnsemble
    grids = [(96, 64, 8, 21), (136, 120, 6, 22), (48, 40, 10, 23)]
    together = [_member(*m, precision="mixed") for m in grids]
    alone = [_member(*m, precision="mixed") for m in grids]
    ens = OceanEnsemble(together)
    ens.step(6)
    for st in alone:
        st.step(6)
    for m, (a, b) in enumerate(zip(together, alone)):
        _same(a, b, f"mixed member {grids[m][:3]}")
        assert a.solve_log() == b.solve_log()
    ens.close()
    for st in together + alone:
        st.close()


def _equal_to_oracle(member, st, steps):
    from oracle import ocean_oracle as orc
    nx, ny, nz, seed = member
    s = cases.seamount_basin(nx=nx, ny=ny, nz=nz, seed=seed)
    p = s.params
    geo = orc.Geometry(p, s.H, s.mask, s.dzr)
    b = orc.buoyancy(p.eos, s.T, s.S, geo.zc, p.g, p.rho0, p.alpha_t, p.beta_s, p.t0, p.s0) * geo.mask3
    ref = orc.OracleStepper(p, s.H, s.mask, dzr=s.dzr, taux_c=s.taux_c, tauy_c=s.tauy_c)
    state = orc.OracleState(s.u, s.v, b, s.eta, s.T, s.S)
    for _ in range(steps):
        state = ref.step(state)
    got = st.get_state()
    for f in FIELDS:
        want = {"km": ref.Km, "kh": ref.Kh}.get(f, None)
        want = getattr(state, f) if want is None else want
        assert np.array_equal(got[f], want), f"member {member[:3]}: {f} differs from the oracle"
    assert st.solve_log() == ref.solve_log
