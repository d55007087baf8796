"""The Python mirror of the reference's HelmholtzVar (solvers_var.HelmholtzVar).

CPU: the reference's argument errors. GPU: on the reference-written cases each
of the four FP64 methods returns the oracle's solution bit for bit with NumPy's
iteration count, also after update() with new face coefficients; pcg_refined
meets the FP64 stopping test; a zero right-hand side gives SolveReport(0, 0.0,
True) and x = 0, as in the reference.
"""

from types import SimpleNamespace

import numpy as np
import pytest

from hydrostatic_ocean_core_benchmark_b200.solvers_var import HelmholtzVar, SolveReport
from oracle import ocean_oracle as orc
from test_helmholtz_cases import SOLVERS, load_case


def _grid(meta):
    return SimpleNamespace(nx=meta["nx"], ny=meta["ny"], dx=meta["lx"] / meta["nx"], dy=meta["lx"] / meta["ny"])


def _oracle(meta, ku, kv, mask, kind, rtol):
    return orc.Helmholtz(meta["nx"], meta["ny"], meta["lx"], meta["lx"], meta["coef"], ku, kv, mask, kind, rtol,
                         meta["max_iter"])


def test_reference_argument_errors():
    meta, a = load_case(64)
    with pytest.raises(ValueError, match="unknown variable-coefficient solver"):
        HelmholtzVar(_grid(meta), meta["coef"], a["ku"], a["kv"], a["mask"], kind="sor")
    with pytest.raises(ValueError, match="V\\(2,2\\)"):
        HelmholtzVar(_grid(meta), meta["coef"], a["ku"], a["kv"], a["mask"], kind="multigrid", n_pre=3)
    assert SolveReport() == SolveReport(0, 0.0, True)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", SOLVERS)
def test_fp64_methods_equal_the_oracle_before_and_after_update(kind):
    meta, a = load_case(64)
    rtol = meta["rtol"]
    s = HelmholtzVar(_grid(meta), meta["coef"], a["ku"], a["kv"], a["mask"], kind=kind, rtol=rtol,
                     max_iter=meta["max_iter"])
    x, rep = s.solve(a["rhs"])
    xo, ito, oko = _oracle(meta, a["ku"], a["kv"], a["mask"], kind, rtol).solve(a["rhs"])
    assert rep.converged and oko and rep.iterations == ito == meta[f"numpy_iters_{kind}"]
    assert np.array_equal(x, xo)
    # new face coefficients, as a step-dependent viscosity gives them
    ku2, kv2 = 0.75 * a["ku"], 1.25 * a["kv"]
    s.update(ku2, kv2)
    x, rep = s.solve(a["rhs"])
    xo, ito, oko = _oracle(meta, ku2, kv2, a["mask"], kind, rtol).solve(a["rhs"])
    assert rep.converged == oko and rep.iterations == ito
    assert np.array_equal(x, xo)
    s.close()


@pytest.mark.gpu
def test_refined_kind_and_zero_right_hand_side():
    meta, a = load_case(96)
    s = HelmholtzVar(_grid(meta), meta["coef"], a["ku"], a["kv"], a["mask"], kind="pcg_refined", rtol=1e-12,
                     max_iter=meta["max_iter"])
    x, rep = s.solve(a["rhs"])
    op = orc.HelmOp(meta["nx"], meta["ny"], meta["lx"], meta["lx"], meta["coef"], a["ku"], a["kv"], a["mask"])
    b = a["rhs"] * a["mask"]
    assert rep.converged and rep.residual <= 1e-12
    assert np.linalg.norm(b - op.apply(x)) <= 1.01e-12 * np.linalg.norm(b)  # host sums in another order
    s.close()
    for kind in ("pcg_jacobi", "pcg_refined"):
        s = HelmholtzVar(_grid(meta), meta["coef"], a["ku"], a["kv"], a["mask"], kind=kind)
        x, rep = s.solve(np.zeros_like(a["rhs"]))
        assert rep == SolveReport(0, 0.0, True) and not x.any(), kind
        s.close()
