"""The algorithmic-byte accounting behind bench.py's roofline fractions (CPU).

Every logical fp64 array access counts once: 44 accesses per cell and step with
the TKE closure, 29 without; 15 arrays per column per PCG-Jacobi iteration;
8 (32 sum_l n_l + 4 n_0) bytes per multigrid V(2,2) cycle, over the levels the
multigrid builds (halving while both sizes are even and at least 8 after the
halving). The mixed-precision solve's count is pass by pass (see
refined_bytes_per_cell); the seeded Helmholtz systems keep c K / dx^2 in
[0.25, 0.5], the reference cases' range.
"""

from types import SimpleNamespace

import numpy as np

import bench


def _p(**kw):
    base = dict(nx=512, ny=512, nz=50, closure="tke", solver_kind="multigrid")
    base.update(kw)
    return SimpleNamespace(**base)


def test_multigrid_levels_follow_the_coarsening_rule():
    assert bench.mg_level_cells(512, 512) == [512 * 512 // 4 ** k for k in range(7)]  # down to 8 x 8
    assert bench.mg_level_cells(40, 36) == [40 * 36, 20 * 18, 10 * 9]
    assert bench.mg_level_cells(24, 20) == [24 * 20, 12 * 10]
    assert bench.mg_level_cells(15, 16) == [15 * 16]


def test_helmholtz_iteration_bytes():
    assert bench.helm_bytes_per_iteration(_p(solver_kind="pcg_jacobi")) == 8 * 15 * 512 * 512
    levels = sum(bench.mg_level_cells(512, 512))
    assert bench.helm_bytes_per_iteration(_p()) == 8 * (32 * levels + 4 * 512 * 512)


def test_step_bytes_per_cell():
    n3 = 512 * 512 * 50
    assert bench.step_algorithmic_bytes(_p(), 0) == 8 * 44 * n3
    assert bench.step_algorithmic_bytes(_p(closure="none"), 0) == 8 * 29 * n3 == 232 * n3
    assert (bench.step_algorithmic_bytes(_p(), 22) - bench.step_algorithmic_bytes(_p(), 0)
            == 22 * bench.helm_bytes_per_iteration(_p()))
    # mixed precision: FP32 3D fields, b and the solver's arrays in fp64
    assert bench.step_algorithmic_bytes(_p(), 0, word=4) == (4 * 40 + 8 * 4) * n3
    assert bench.step_algorithmic_bytes(_p(closure="none"), 0, word=4) == (4 * 26 + 8 * 3) * n3
    assert (bench.step_algorithmic_bytes(_p(), 9, word=4) - bench.step_algorithmic_bytes(_p(), 0, word=4)
            == 9 * bench.helm_bytes_per_iteration(_p()))


def test_refined_solve_bytes():
    # start 40 B; 29 + 32 B per inner iteration, 4 B less in each inner solve's first; 76 B per step
    assert bench.refined_bytes_per_cell(0, 0) == 40
    assert bench.refined_bytes_per_cell(1, 1) == 40 + 25 + 32 + 76
    assert bench.refined_bytes_per_cell(28, 4) == 40 + 28 * 61 - 4 * 4 + 4 * 76


def test_seeded_helmholtz_systems():
    for n in (64, 128):
        dx, coef, ku, kv, mask, rhs = bench.helmholtz_system(n, 7)
        assert dx == 4.0e6 / n and 0.0 < mask.mean() < 1.0
        wet_u = ku[ku > 0] * coef / dx ** 2
        assert 0.25 <= wet_u.min() and wet_u.max() <= 0.5
        # closed faces on land and between land and water
        assert not (ku * (1 - mask)).any() and not (ku * (1 - np.roll(mask, -1, 1))).any()
        assert not (kv * (1 - mask)).any() and not (kv * (1 - np.roll(mask, -1, 0))).any()
        assert not (rhs * (1 - mask)).any()
        a = bench.helmholtz_system(n, 7)
        assert all(np.array_equal(x, y) for x, y in zip(a[2:], (ku, kv, mask, rhs)))


def test_profile_traffic_for_every_counted_kernel():
    """The committed ncu summary gives the DRAM bytes per launch of every kernel the
    accounting counts (and of the solve), which bench.py reads into its line."""
    for kernel in list(bench.ACCESSES_PER_CELL) + ["helm_solve"]:
        t = bench.dram_traffic_from_profiles(kernel)
        assert t is not None and t > 0, kernel
    assert bench.dram_traffic_from_profiles("no_such_kernel") is None
    # the column solves move about twice their algorithmic bytes, the streaming kernels about once
    n3 = 512 * 512 * 50

    def ratio(k):
        return bench.dram_traffic_from_profiles(k) / (8 * bench.ACCESSES_PER_CELL[k] * n3)

    assert 1.9 < ratio("momentum_solve") < 2.1 and 0.8 < ratio("backsub") < 1.1


def test_reference_arm_replicas_on_the_host_cores():
    """The reference arm's CPU oracle runs as independent single-threaded replicas in
    spawned processes; their aggregate rate counts every replica's cell-steps."""
    args = SimpleNamespace(cpu_nx=16, nz=6, seed=20261203, steps=1, warmup=1)
    assert 1 <= bench.oracle_replicas(args) <= max(1, bench.host_cpu()["usable"])
    rate, span, single = bench.cpu_oracle_rate_parallel(args, 1, 1, 2)
    assert span > 0 and single > 0
    assert rate == 2 * 16 * 16 * 6 / span
