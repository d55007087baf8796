"""The float64 torch restatement of the step (the adjoint's reference
gradient) against the oracle, on CPU: the restatement's forward must match the
oracle before its gradient is trusted."""

import numpy as np

from hydrostatic_ocean_core_benchmark_b200 import cases
from oracle import ocean_oracle as orc


def test_torch_restatement_forward_matches_the_oracle():
    import torch
    from torch_step import TorchStep
    s = cases.seamount_basin(nx=24, ny=20, nz=8, seed=3, closure="none")
    p = s.params
    ts = TorchStep(p, s.H, s.mask, s.dzr, device="cpu")
    geo = orc.Geometry(p, s.H, s.mask, s.dzr)
    b = orc.buoyancy(p.eos, s.T, s.S, geo.zc, p.g, p.rho0, p.alpha_t, p.beta_s, p.t0, p.s0) * geo.mask3
    ref = orc.OracleStepper(p, s.H, s.mask, dzr=s.dzr, taux_c=s.taux_c, tauy_c=s.tauy_c)
    st = orc.OracleState(s.u, s.v, b, s.eta, s.T, s.S)
    T = lambda a: torch.as_tensor(a, dtype=torch.float64)  # noqa: E731
    tst = {"u": T(s.u), "v": T(s.v), "b": T(b), "eta": T(s.eta), "T": T(s.T), "S": T(s.S)}
    assert float((tst["b"] - ts.buoyancy(tst["T"], tst["S"])).abs().max()) < 1e-13
    for _ in range(4):
        st = ref.step(st)
        tst = ts.step(tst, T(s.taux_c))
        for f in ("eta", "u", "v", "b", "T", "S"):
            want = getattr(st, f)
            err = np.linalg.norm(tst[f].numpy() - want) / np.linalg.norm(want)
            assert err < 1e-11, (f, err)
