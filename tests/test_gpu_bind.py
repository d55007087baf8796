"""Caller-owned device tensors as the state (oc_bind_state): no copy in, and the
steps write into the two bound sets in turn, bit for bit as through the
handle's own buffers (which equal the oracle's, tests/test_gpu_parity.py)."""

import numpy as np
import pytest

from hydrostatic_ocean_core_benchmark_b200 import cases
from hydrostatic_ocean_core_benchmark_b200._lib import OceanError
from hydrostatic_ocean_core_benchmark_b200.stepper import OceanStepper

pytestmark = pytest.mark.gpu

FIELDS = ("eta", "u", "v", "b", "T", "S")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    import torch
    assert torch.cuda.is_available()
    torch.cuda.set_device(0)


def _stepper(s, **kw):
    return OceanStepper(s.params, s.H, s.mask, dzr=s.dzr, taux_c=s.taux_c, tauy_c=s.tauy_c, **kw)


def _copied_run(s, steps, graph):
    st = _stepper(s)
    st.set_state(eta=s.eta, u=s.u, v=s.v, T=s.T, S=s.S)
    st.step(steps, graph=graph)
    out = st.get_state()
    log = st.solve_log()
    st.close()
    return out, log


def _tensors(s):
    import torch
    b0 = _stepper(s)
    b0.set_state(eta=s.eta, u=s.u, v=s.v, T=s.T, S=s.S)
    b = b0.get_state(fields=("b",))["b"]  # b diagnosed from T and S by the step's EOS
    b0.close()
    src = {"eta": s.eta, "u": s.u, "v": s.v, "b": b, "T": s.T, "S": s.S}
    cur = {k: torch.tensor(np.ascontiguousarray(v), dtype=torch.float64, device="cuda") for k, v in src.items()}
    oth = {k: torch.full_like(v, float("nan")) for k, v in cur.items()}
    return cur, oth


@pytest.mark.parametrize("steps,graph", [(5, False), (6, True)])
def test_bound_tensors_step_like_the_copied_state(steps, graph):
    import torch
    s = cases.seamount_basin(nx=40, ny=36, nz=10, seed=11)
    want, want_log = _copied_run(s, steps, graph)
    st = _stepper(s)
    cur, oth = _tensors(s)
    ptrs = {k: v.data_ptr() for k, v in cur.items()}
    st.bind_state(cur, oth)
    st.step(steps, graph=graph)
    torch.cuda.synchronize()
    assert st.state_parity() == steps % 2
    live = st.bound_state()
    # the state lives in the caller's tensors: compare them, not a copy
    for f in FIELDS:
        assert np.array_equal(live[f].cpu().numpy(), want[f]), f
    got = st.get_state()
    for f in want:
        assert np.array_equal(got[f], want[f]), f
    assert st.solve_log() == want_log
    assert {k: v.data_ptr() for k, v in cur.items()} == ptrs
    st.close()


def test_bind_refuses_bad_buffers_and_unbinds():
    import torch
    s = cases.seamount_basin(nx=24, ny=20, nz=6, seed=2)
    st = _stepper(s)
    cur, oth = _tensors(s)
    alias = dict(oth, u=cur["u"])
    with pytest.raises(OceanError, match="overlap"):
        st.bind_state(cur, alias)
    with pytest.raises(ValueError):
        st.bind_state(cur, {k: v.cpu() for k, v in oth.items()})
    st.bind_state(cur, oth)
    st.step(2)
    st.bind_state(None)
    with pytest.raises(OceanError):
        st.step(1)  # unbound: no state until one is set again
    st.set_state(eta=s.eta, u=s.u, v=s.v, T=s.T, S=s.S)
    st.step(1)
    torch.cuda.synchronize()
    st.close()


def test_mixed_precision_handle_refuses_binding():
    s = cases.seamount_basin(nx=24, ny=20, nz=6, seed=2)
    st = _stepper(s, precision="mixed")
    cur, oth = _tensors(s)
    with pytest.raises(OceanError, match="FP32"):
        st.bind_state(cur, oth)
    st.close()
