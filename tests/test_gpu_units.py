"""Unit pieces of the C ABI against the oracle: Thomas, Helmholtz, EOS, the binary protocol."""

import subprocess
from pathlib import Path

import numpy as np
import pytest

from harness import case_inputs, load_fixture
from oracle import ocean_oracle as orc

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    import torch
    assert torch.cuda.is_available()
    torch.cuda.set_device(0)


def test_thomas_matches_oracle_bitwise():
    from hydrostatic_ocean_core_benchmark_b200.stepper import thomas
    rng = np.random.default_rng(3)
    n, cols = 37, 5000
    sub = rng.uniform(-1, 0, (n, cols))
    sup = rng.uniform(-1, 0, (n, cols))
    diag = 2.5 + rng.uniform(0, 1, (n, cols))
    rhs = rng.standard_normal((n, cols))
    # dry-style identity rows
    sub[:, :100] = 0.0
    sup[:, :100] = 0.0
    diag[:, :100] = 1.0
    assert np.array_equal(thomas(sub, diag, sup, rhs), orc.thomas(sub, diag, sup, rhs))


@pytest.mark.parametrize("solver", ["pcg_jacobi", "pcg_rbgs", "rbgs", "multigrid"])
def test_helmholtz_iterations_and_solution_match(solver):
    from hydrostatic_ocean_core_benchmark_b200.stepper import OceanStepper
    meta, arrays = load_fixture("seamount_basin_ref_mg")
    p, H, mask, *_ = case_inputs(meta, arrays)
    p = p.replace(solver_kind=solver, max_iter=4000 if solver == "rbgs" else 2000)
    st = OceanStepper(p, H, mask)
    ku, kv = st.field("ku"), st.field("kv")
    ref_step = orc.OracleStepper(p, H, mask)
    assert np.array_equal(ku, ref_step.Ku) and np.array_equal(kv, ref_step.Kv)
    rng = np.random.default_rng(5)
    rhs = rng.standard_normal((p.ny, p.nx))
    x, its = st.helmholtz_solve(rhs)
    xr, itr, ok = ref_step.solver.solve(rhs)
    assert its == itr
    assert np.array_equal(x, xr)
    st.close()


@pytest.mark.parametrize("eos", ["linear", "seos", "teos10"])
def test_eos_bitwise(eos):
    from hydrostatic_ocean_core_benchmark_b200.params import OceanParams
    from hydrostatic_ocean_core_benchmark_b200.stepper import OceanStepper
    p = OceanParams(nx=8, ny=8, nz=4, dt=1.0, eos=eos, tracers="TS")
    st = OceanStepper(p, np.full((8, 8), 100.0), np.ones((8, 8)))
    rng = np.random.default_rng(9)
    T = rng.uniform(-2, 30, 100000)
    S = rng.uniform(0, 42, 100000)
    z = rng.uniform(0, 6000, 100000)
    got = st.buoyancy(T, S, z)
    want = orc.buoyancy(eos, T, S, z, p.g, p.rho0, p.alpha_t, p.beta_s, p.t0, p.s0)
    assert np.array_equal(got, want)
    if eos == "teos10":
        b = st.buoyancy(np.array([10.0]), np.array([30.0]), np.array([1000.0]))[0]
        rho = -b * p.rho0 / p.g + p.rho0
        assert abs(rho - 1027.45140) < 1e-4
    st.close()


def test_drop_in_binary_protocol(tmp_path):
    """The executable reads a reference bundle and writes the reference's outputs."""
    from hydrostatic_ocean_core_benchmark_b200 import bundle
    meta, arrays = load_fixture("gate_v06_seamount_tvd_tke_theta")
    p, H, mask, dzr, taux, tauy, s = case_inputs(meta, arrays)
    prefix = str(tmp_path / "run")
    nml = bundle.write_bundle(prefix, p.replace(n_steps=4, n_repeat=1, n_warmup=0, out_prefix=prefix),
                              H, mask, s)
    exe = ROOT / "hydrostatic_ocean_core_benchmark_b200" / "bin" / "ocean3d5_b200"
    proc = subprocess.run([str(exe), str(nml)], capture_output=True, text=True, timeout=300)
    assert proc.returncode == 0, proc.stderr
    got = bundle.read_state(prefix + "_state3d5.bin", p.nx, p.ny, p.nz, p.tracers == "TS")
    ref = orc.OracleStepper(p, H, mask).integrate(s, 4)
    for f in ("eta", "u", "v", "b", "T", "S"):
        assert np.array_equal(got[f], getattr(ref, f)), f
    import json
    metrics = json.loads(Path(prefix + "_metrics.json").read_text())
    for key in ("backend", "gpu", "nx", "ny", "nz", "cells", "n_steps", "scheme", "solver", "eos",
                "advection", "tracers", "theta", "dt", "solver_iterations", "solver_failures",
                "tridiagonal_solves", "solver_rebuilds", "n_split", "barotropic_substeps",
                "device_bytes", "bytes_per_cell", "diverged", "wall_s", "wall_mad_s", "n_repeat",
                "omp_num_threads"):
        assert key in metrics, key
    assert metrics["solver_iterations"] == sum(meta["solve_log"][:8])


def test_binary_refuses_open_boundaries(tmp_path):
    from hydrostatic_ocean_core_benchmark_b200.params import OceanParams, write_namelist
    p = OceanParams(nx=8, ny=8, nz=4, dt=1.0, n_steps=1, bc_x="open")
    nml = write_namelist(tmp_path / "x.nml", p)
    exe = ROOT / "hydrostatic_ocean_core_benchmark_b200" / "bin" / "ocean3d5_b200"
    proc = subprocess.run([str(exe), str(nml)], capture_output=True, text=True, timeout=60)
    assert proc.returncode != 0
    assert "FATAL" in proc.stderr


@pytest.mark.parametrize("nx,ny", [(66, 66), (50, 50), (96, 80), (256, 256), (40, 24), (512, 512),
                                   (640, 256), (512, 300)])
def test_multigrid_paths_match_oracle(nx, ny):
    """Every V-cycle layout: all levels on the grid (66: the coarsening stops at an odd
    33x33), partial tiles (50, 96x80), grid levels above CTA-0 levels (256), all in CTA 0
    (40x24); level 0 in 128x16 tiles whose rows are NumPy's leaves, so the up phase forms
    the residual sums (512), wide tiles with unaligned leaves (640x256), and wide partial
    tiles above a grid-wide coarsest level (512x300)."""
    from hydrostatic_ocean_core_benchmark_b200 import cases
    from hydrostatic_ocean_core_benchmark_b200.stepper import OceanStepper
    s = cases.seamount_basin(nx=nx, ny=ny, nz=8, seed=nx * 1000 + ny, solver_kind="multigrid")
    p = s.params
    st = OceanStepper(p, s.H, s.mask, dzr=s.dzr)
    ref = orc.OracleStepper(p, s.H, s.mask, dzr=s.dzr)
    assert np.array_equal(st.field("ku"), ref.Ku)
    rng = np.random.default_rng(nx + ny)
    for _ in range(2):
        rhs = rng.standard_normal((ny, nx))
        x, its = st.helmholtz_solve(rhs)
        xr, itr, ok = ref.solver.solve(rhs)
        assert its == itr
        assert np.array_equal(x, xr)
    st.close()


def test_async_state_round_trip_matches_synchronous():
    """oc_set_state_async / oc_step / oc_get_state_async on user streams (pinned host
    buffers, two handles alternating as in the end-to-end bench) give the bits of the
    synchronous set_state / step / get_state path."""
    import torch
    from hydrostatic_ocean_core_benchmark_b200 import cases
    from hydrostatic_ocean_core_benchmark_b200.stepper import OceanStepper
    s = cases.seamount_basin(nx=48, ny=40, nz=10, seed=7)
    p = s.params
    fields = ("eta", "u", "v", "b", "T", "S", "e")
    ref = OceanStepper(p, s.H, s.mask, dzr=s.dzr, taux_c=s.taux_c, tauy_c=s.tauy_c)
    ref.set_state(eta=s.eta, u=s.u, v=s.v, T=s.T, S=s.S)
    start = ref.get_state()
    cur = {k: start[k] for k in fields}
    for _ in range(3):
        ref.set_state(**cur)
        ref.step(1)
        cur = {k: v for k, v in ref.get_state().items() if k in fields}
    members = [OceanStepper(p, s.H, s.mask, dzr=s.dzr, taux_c=s.taux_c, tauy_c=s.tauy_c) for _ in range(2)]
    for m in members:
        m.set_state(eta=s.eta, u=s.u, v=s.v, T=s.T, S=s.S)
    bufs = [{k: torch.from_numpy(np.ascontiguousarray(start[k])).pin_memory() for k in fields}
            for _ in range(2)]
    s_in, s_cmp, s_out = (torch.cuda.Stream() for _ in range(3))
    ev_out = [None, None]
    for n in range(6):  # each member does three round trips, interleaved
        m = n % 2
        if ev_out[m] is not None:
            s_in.wait_event(ev_out[m])
        members[m].set_state_async(s_in, **bufs[m])
        e = torch.cuda.Event()
        e.record(s_in)
        s_cmp.wait_event(e)
        members[m].step(1, stream=s_cmp)
        e = torch.cuda.Event()
        e.record(s_cmp)
        s_out.wait_event(e)
        members[m].get_state_async(s_out, bufs[m])
        ev_out[m] = torch.cuda.Event()
        ev_out[m].record(s_out)
    torch.cuda.synchronize()
    for m in range(2):
        for k in fields:
            assert np.array_equal(bufs[m][k].numpy().reshape(cur[k].shape), cur[k]), (m, k)
        assert members[m].stats()["solver_failures"] == 0
    for st in [ref, *members]:
        st.close()


@pytest.mark.parametrize("case", ["seamount_basin_ref_mg", "gate_v06_seamount_tke_split",
                                  "gate_rough_TS_fb_upwind"])
def test_graph_steps_match_plain_steps(case):
    """oc_step_graph (two-step CUDA graphs per starting buffer, an odd last step run
    plainly) gives the bits, counters and solve log of oc_step."""
    from hydrostatic_ocean_core_benchmark_b200.stepper import OceanStepper
    meta, arrays = load_fixture(case)
    p, H, mask, dzr, tx, ty, s = case_inputs(meta, arrays)
    runs = []
    for graph in (False, True):
        st = OceanStepper(p, H, mask, dzr=dzr, taux_c=tx, tauy_c=ty)
        st.set_state(eta=s.eta, u=s.u, v=s.v, b=s.b, T=s.T, S=s.S)
        st.step(5, graph=graph)   # odd: 2 graph launches + 1 plain step
        st.step(4, graph=graph)   # starts from the other buffer: records its graph
        st.set_profiling(True)
        st.step(2, graph=graph)   # profiling falls back to plain launches
        st.set_profiling(False)
        st.step(3, graph=graph)
        stats = st.stats()
        runs.append((st.get_state(), stats, st.solve_log()))
        st.close()
    (a, sa, la), (b, sb, lb) = runs
    for k in a:
        assert np.array_equal(a[k], b[k]), k
    for k in ("steps", "solver_iterations", "solver_failures", "solver_rebuilds", "tridiagonal_solves",
              "barotropic_substeps", "solves"):
        assert sa[k] == sb[k], k
    assert la == lb


@pytest.mark.parametrize("n,solver", [(2048, "pcg_jacobi"), (2048, "multigrid"), (2000, "pcg_jacobi")])
def test_grids_above_one_ctas_fold_match_oracle(n, solver):
    """Above 16,384 NumPy leaves (about 2.1 M columns) the solver folds the
    pairwise tree in two levels (block subtrees, then the top over their roots).
    The sums are NumPy's all the same: iteration counts and solutions equal the
    oracle's bit for bit, on the grid of the reference's largest published runs
    (2000 x 2000, docs/32_hardware_ladder.md) and at 2048 x 2048."""
    from types import SimpleNamespace

    from hydrostatic_ocean_core_benchmark_b200.solvers_var import HelmholtzVar
    rng = np.random.default_rng(n)
    dx = 4.0e6 / n
    mask = np.ones((n, n))
    mask[n // 4:n // 3, n // 5:n // 2] = 0.0
    ku = (0.5 + 0.5 * rng.random((n, n))) * mask * np.roll(mask, -1, 1)
    kv = (0.5 + 0.5 * rng.random((n, n))) * mask * np.roll(mask, -1, 0)
    rhs = rng.standard_normal((n, n)) * mask
    coef = 0.5 * dx * dx
    grid = SimpleNamespace(nx=n, ny=n, dx=dx, dy=dx)
    solver_gpu = HelmholtzVar(grid, coef, ku, kv, mask, kind=solver, rtol=1e-10)
    x, rep = solver_gpu.solve(rhs)
    ref = orc.Helmholtz(n, n, 4.0e6, 4.0e6, coef, ku, kv, mask, solver, 1e-10, 2000)
    xr, itr, ok = ref.solve(rhs)
    assert ok and rep.converged
    assert rep.iterations == itr
    assert np.array_equal(x, xr)
    solver_gpu.close()
