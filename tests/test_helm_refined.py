"""Mixed-precision Helmholtz solver (OC_SOLVER_PCG_REFINED): FP32 inner PCG,
FP64 refinement. No reference counterpart, so no bit parity: the pins are the
FP64 oracle's operator and solution on the reference-written cases.

CPU: the NumPy statement of the algorithm (refine_model.py) converges on both
cases to the FP64 stopping test and lands within 10 rtol (relative L2) of the
oracle's FP64 PCG solution.
GPU: the library's solve meets the same FP64 stopping test, recomputed here
with the oracle's operator; lands within 10 rtol of the oracle's solution; uses
the model's inner iteration count within 2; repeats bit for bit; and keeps the
solver's edge behaviour (zero right-hand side, iteration bound, the other
solvers refusing the refinement report).
"""

import ctypes as C
import json
import subprocess

import numpy as np
import pytest

from oracle import ocean_oracle as orc
from refine_model import refine
from test_helmholtz_cases import ROOT, SIZES, load_case

REFINED = 4  # OC_SOLVER_PCG_REFINED
RTOLS = (1e-10, 1e-13)


def _op(meta, a):
    return orc.HelmOp(meta["nx"], meta["ny"], meta["lx"], meta["lx"], meta["coef"], a["ku"], a["kv"], a["mask"])


def _fp64(meta, a, rtol):
    h = orc.Helmholtz(meta["nx"], meta["ny"], meta["lx"], meta["lx"], meta["coef"], a["ku"], a["kv"], a["mask"],
                      "pcg_jacobi", rtol, meta["max_iter"])
    return h.solve(a["rhs"])[0]


def _relres(op, rhs, x):
    b = rhs * op.mask
    return float(np.linalg.norm(b - op.apply(x)) / np.linalg.norm(b))


def _rel_l2(x, ref):
    return float(np.linalg.norm(x - ref) / np.linalg.norm(ref))


@pytest.mark.parametrize("nx", SIZES)
@pytest.mark.parametrize("rtol", RTOLS)
def test_model_meets_the_fp64_stopping_test(nx, rtol):
    meta, a = load_case(nx)
    op = _op(meta, a)
    x, inner, ok, outer, rel = refine(op, a["rhs"], rtol, meta["max_iter"])
    assert ok and 1 <= outer <= 8 and inner < 3 * meta["numpy_iters_pcg_jacobi"]
    assert rel <= rtol and _relres(op, a["rhs"], x) <= rtol
    assert _rel_l2(x, _fp64(meta, a, rtol)) <= 10 * rtol


def test_model_edges():
    meta, a = load_case(64)
    op = _op(meta, a)
    x, inner, ok, outer, rel = refine(op, np.zeros_like(a["rhs"]), 1e-10, 100)
    assert ok and inner == 0 and outer == 0 and not x.any()
    x, inner, ok, outer, rel = refine(op, a["rhs"], 1e-13, 5)
    assert not ok and inner == 5 and rel > 1e-13


# ---------------------------------------------------------------------- GPU
class Refined:
    def __init__(self, meta, a, rtol, max_iter=None, solver=REFINED):
        from hydrostatic_ocean_core_benchmark_b200 import _lib
        self.lib = _lib.load()
        cfg = _lib.OcHelmConfig(nx=meta["nx"], ny=meta["ny"], dx=meta["lx"] / meta["nx"],
                                dy=meta["lx"] / meta["ny"], coef=meta["coef"], solver=solver, rtol=rtol,
                                max_iter=max_iter or meta["max_iter"], device=0)
        self.arr = {k: np.ascontiguousarray(a[k], dtype=np.float64) for k in ("ku", "kv", "mask")}
        self.h = C.c_void_p()
        rc = self.lib.oc_helm_create(C.byref(cfg), self.arr["ku"].ctypes.data, self.arr["kv"].ctypes.data,
                                     self.arr["mask"].ctypes.data, C.byref(self.h))
        assert rc == 0

    def solve(self, rhs):
        rhs = np.ascontiguousarray(rhs, dtype=np.float64)
        x = np.full_like(rhs, np.nan)
        its, conv = C.c_int32(), C.c_int32()
        rc = self.lib.oc_helm_solve(self.h, rhs.ctypes.data, x.ctypes.data, 0, C.byref(its), C.byref(conv), None)
        assert rc == 0, self.lib.oc_helm_last_error(self.h)
        outer, rel = C.c_int32(), C.c_double()
        assert self.lib.oc_helm_refine_report(self.h, C.byref(outer), C.byref(rel)) == 0
        return x, its.value, bool(conv.value), outer.value, rel.value

    def close(self):
        self.lib.oc_helm_destroy(self.h)


@pytest.mark.gpu
@pytest.mark.parametrize("nx", SIZES)
@pytest.mark.parametrize("rtol", RTOLS)
def test_refined_solve_meets_fp64_test_and_model(nx, rtol):
    meta, a = load_case(nx)
    op = _op(meta, a)
    s = Refined(meta, a, rtol)
    x, inner, ok, outer, rel = s.solve(a["rhs"])
    again = s.solve(a["rhs"])
    s.close()
    xm, inner_m, ok_m, outer_m, _ = refine(op, a["rhs"], rtol, meta["max_iter"])
    assert ok and ok_m
    true_rel = _relres(op, a["rhs"], x)
    assert true_rel <= rtol and rel <= rtol
    assert abs(rel - true_rel) <= 1e-3 * rtol
    assert _rel_l2(x, _fp64(meta, a, rtol)) <= 10 * rtol
    assert abs(inner - inner_m) <= 2 and abs(outer - outer_m) <= 1, (inner, inner_m, outer, outer_m)
    assert np.array_equal(x, again[0]) and again[1:] == (inner, ok, outer, rel)


@pytest.mark.gpu
def test_refined_edges():
    meta, a = load_case(64)
    s = Refined(meta, a, 1e-13)
    x, inner, ok, outer, rel = s.solve(np.zeros_like(a["rhs"]))
    assert ok and inner == 0 and outer == 0 and rel == 0.0 and not x.any()
    s.close()
    s = Refined(meta, a, 1e-13, max_iter=5)
    x, inner, ok, outer, rel = s.solve(a["rhs"])
    assert not ok and inner == 5 and rel > 1e-13 and np.isfinite(x).all()
    s.close()
    # a tighter inner tolerance: fewer refinement steps, as in the model
    s = Refined(meta, a, 1e-13)
    assert s.lib.oc_helm_set_inner_rtol(s.h, 0.0) == 1 and s.lib.oc_helm_set_inner_rtol(s.h, 1e-5) == 0
    x, inner, ok, outer, rel = s.solve(a["rhs"])
    s.close()
    _, inner_m, _, outer_m, _ = refine(_op(meta, a), a["rhs"], 1e-13, meta["max_iter"], inner_rtol=1e-5)
    assert ok and rel <= 1e-13 and abs(inner - inner_m) <= 2 and abs(outer - outer_m) <= 1
    fp64 = Refined(meta, a, 1e-10, solver=0)
    outer_c, rel_c = C.c_int32(), C.c_double()
    assert fp64.lib.oc_helm_refine_report(fp64.h, C.byref(outer_c), C.byref(rel_c)) == 3
    assert fp64.lib.oc_helm_set_inner_rtol(fp64.h, 1e-4) == 3
    fp64.close()


@pytest.mark.gpu
def test_refined_bench_executable(tmp_path):
    meta, a = load_case(96)
    for name in ("ku", "kv", "mask", "rhs", "eta_ref"):
        np.ascontiguousarray(a[name], dtype=np.float64).tofile(tmp_path / f"{name}.bin")
    fd = lambda v: f"{float(v):.17e}".replace("e", "d")  # noqa: E731
    (tmp_path / "case.nml").write_text(
        "&helmholtz\n"
        f"  nx = {meta['nx']}\n  ny = {meta['ny']}\n  dx = {fd(meta['dx'])}\n  dy = {fd(meta['dy'])}\n"
        f"  coef = {fd(meta['coef'])}\n  rtol = {fd(meta['rtol'])}\n  max_iter = {meta['max_iter']}\n"
        f"  n_repeat = 3\n  n_warmup = 1\n  datadir = '{tmp_path}'\n/\n")
    exe = ROOT / "hydrostatic_ocean_core_benchmark_b200" / "bin" / "helmholtz_bench_b200"
    proc = subprocess.run([str(exe), str(tmp_path / "case.nml"), "pcg_refined"], capture_output=True, text=True,
                          timeout=300)
    assert proc.returncode == 0, proc.stderr
    m = json.loads((tmp_path / "metrics_b200_pcg_refined.json").read_text())
    assert m["precision"] == "fp32+fp64-refined" and m["converged"] is True
    assert m["residual"] <= meta["rtol"] * 1.0001
    assert m["l2_rel_vs_reference"] < 1e-8
