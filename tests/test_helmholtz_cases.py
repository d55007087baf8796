"""The standalone Helmholtz problem of the reference's bench (tools/write_helmholtz_case.py):
the oracle reproduces NumPy's HelmholtzVar on the reference-written cases (CPU), and
the B200 solver behind oc_helm_* and the helmholtz_bench_b200 executable reproduces
the oracle bit for bit with the same iteration counts (GPU)."""

import json
import subprocess
from pathlib import Path

import numpy as np
import pytest

from oracle import ocean_oracle as orc

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
SIZES = (64, 96)
SOLVERS = ("pcg_jacobi", "pcg_rbgs", "rbgs", "multigrid")


def load_case(nx):
    z = np.load(GOLDEN / "helmholtz" / f"case_{nx}.npz")
    meta = json.loads(str(z["meta"]))
    return meta, {k: z[k] for k in ("ku", "kv", "mask", "rhs", "eta_ref")}


def oracle_solver(meta, a, kind, rtol):
    nx, ny = meta["nx"], meta["ny"]
    return orc.Helmholtz(nx, ny, meta["lx"], meta["lx"], meta["coef"], a["ku"], a["kv"], a["mask"],
                         kind, rtol, meta["max_iter"])


@pytest.mark.parametrize("nx", SIZES)
def test_oracle_reproduces_reference_iterations_and_solution(nx):
    meta, a = load_case(nx)
    assert meta["nx"] * meta["dx"] == pytest.approx(meta["lx"], rel=1e-15)
    for kind in SOLVERS:
        x, its, ok = oracle_solver(meta, a, kind, meta["rtol"]).solve(a["rhs"])
        assert ok and its == meta[f"numpy_iters_{kind}"], kind
    # the reference's stored solution is its PCG-Jacobi solve at rtol 1e-13
    x, its, ok = oracle_solver(meta, a, "pcg_jacobi", 1e-13).solve(a["rhs"])
    assert its == meta["reference_iterations"]
    assert np.array_equal(x, a["eta_ref"])


def _lib_solve(meta, a, kind, rtol):
    import ctypes as C
    from hydrostatic_ocean_core_benchmark_b200 import _lib
    lib = _lib.load()
    cfg = _lib.OcHelmConfig(nx=meta["nx"], ny=meta["ny"], dx=meta["lx"] / meta["nx"], dy=meta["lx"] / meta["ny"],
                            coef=meta["coef"], solver=SOLVERS.index(kind), rtol=rtol,
                            max_iter=meta["max_iter"], device=0)
    arr = {k: np.ascontiguousarray(v, dtype=np.float64) for k, v in a.items()}
    h = C.c_void_p()
    assert lib.oc_helm_create(C.byref(cfg), arr["ku"].ctypes.data, arr["kv"].ctypes.data,
                              arr["mask"].ctypes.data, C.byref(h)) == 0
    x = np.zeros_like(arr["rhs"])
    its, conv = C.c_int32(), C.c_int32()
    for _ in range(2):  # a second solve on the same handle gives the same answer
        rc = lib.oc_helm_solve(h, arr["rhs"].ctypes.data, x.ctypes.data, 0, C.byref(its), C.byref(conv), None)
        assert rc == 0, lib.oc_helm_last_error(h)
    lib.oc_helm_destroy(h)
    return x, its.value, bool(conv.value)


@pytest.mark.gpu
@pytest.mark.parametrize("nx", SIZES)
@pytest.mark.parametrize("kind", SOLVERS)
def test_standalone_solver_matches_oracle_bitwise(nx, kind):
    meta, a = load_case(nx)
    x, its, ok = _lib_solve(meta, a, kind, meta["rtol"])
    xo, ito, oko = oracle_solver(meta, a, kind, meta["rtol"]).solve(a["rhs"])
    assert ok and its == ito == meta[f"numpy_iters_{kind}"]
    assert np.array_equal(x, xo)


@pytest.mark.gpu
def test_standalone_solver_reaches_the_reference_solution():
    meta, a = load_case(64)
    x, its, ok = _lib_solve(meta, a, "pcg_jacobi", 1e-13)
    assert ok and its == meta["reference_iterations"]
    assert np.array_equal(x, a["eta_ref"])


@pytest.mark.gpu
@pytest.mark.parametrize("kind", SOLVERS)
def test_helmholtz_bench_executable(tmp_path, kind):
    """The reference bench's protocol: case.nml + *.bin in, metrics JSON + one line out."""
    meta, a = load_case(96)
    for name in ("ku", "kv", "mask", "rhs", "eta_ref"):
        np.ascontiguousarray(a[name], dtype=np.float64).tofile(tmp_path / f"{name}.bin")
    fd = lambda v: f"{float(v):.17e}".replace("e", "d")  # noqa: E731 - the writer's Fortran literals
    (tmp_path / "case.nml").write_text(
        "&helmholtz\n"
        f"  nx = {meta['nx']}\n  ny = {meta['ny']}\n  dx = {fd(meta['dx'])}\n  dy = {fd(meta['dy'])}\n"
        f"  coef = {fd(meta['coef'])}\n  rtol = {fd(meta['rtol'])}\n  max_iter = {meta['max_iter']}\n"
        f"  n_repeat = 3\n  n_warmup = 1\n  datadir = '{tmp_path}'\n/\n")
    exe = ROOT / "hydrostatic_ocean_core_benchmark_b200" / "bin" / "helmholtz_bench_b200"
    proc = subprocess.run([str(exe), str(tmp_path / "case.nml"), kind], capture_output=True, text=True,
                          timeout=300)
    assert proc.returncode == 0, proc.stderr
    assert proc.stdout.startswith(f"solver={kind:>12s} iters=")
    m = json.loads((tmp_path / f"metrics_b200_{kind}.json").read_text())
    assert m["iterations"] == meta[f"numpy_iters_{kind}"] and m["converged"] is True
    assert m["residual"] <= meta["rtol"] * 1.0001
    assert 0.0 <= m["l2_rel_vs_reference"] < 1e-8
    assert m["wall_s"] > 0.0 and m["n_repeat"] == 3
