"""The v0.5 driver's verify on the GPU: a case resolved from the TOML tree,
stepped by the GPU and by the oracle side by side through ``verify_run`` (the
reference gate of tools/compare_backends3d5.py:28-99: one step below 1e-12,
the run below 1e-9, solve logs equal). On a machine with the reference checkout
the CLI passes the reference's own NumPy stepper instead of the oracle."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("overrides,case", [
    (["physics3d_v06.closure=tke", "scheme.advection=up3_tvd"], "lock_exchange"),
    (["bathymetry.kind=rough", "scheme.name=fb", "physics3d_v06.closure=none"], "lock_exchange"),
    (["bathymetry.kind=flat", "physics3d_v04.tracers=buoyancy", "solver.kind=pcg_jacobi",
      "physics3d_v06.closure=none"], "seamount_rest"),
])
def test_verify_subcommand_passes_the_gate(overrides, case):
    import torch
    from hydrostatic_ocean_core_benchmark_b200 import toml_front as tf
    from hydrostatic_ocean_core_benchmark_b200.main import DEFAULT_CONFIG, verify_run
    from oracle import ocean_oracle as orc
    torch.cuda.set_device(0)
    config = tf.apply_overrides(tf.load_config(DEFAULT_CONFIG), overrides)
    run = tf.resolve_run(config, nx=24, nz=8, case=case, cfl=1.0, n_steps=5)
    p, s = run.params, run.state
    ref = orc.OracleStepper(p, run.H, run.mask)
    s0 = orc.OracleState(s.u, s.v, s.b, s.eta, s.T, s.S)
    report = verify_run(run, (ref, s0))
    assert report["pass"], report
    assert report["worst_step_error"] < 1e-12
    assert report.get("solve_log_equal", True)
