"""The C-ABI library loads and exports every entry point the public header declares."""

import re
from pathlib import Path

from hydrostatic_ocean_core_benchmark_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]


def header_functions():
    text = (ROOT / "include" / "ocean_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return set(re.findall(r"\b(oc_[a-z_]+)\s*\(", text))


def test_header_and_binding_agree():
    assert header_functions() == set(_lib.exported_symbols())


def test_library_exports_every_symbol():
    lib = _lib.load()
    for name in header_functions():
        assert hasattr(lib, name), name
    assert b"sm_100a" in lib.oc_version()


def test_config_struct_layout():
    import ctypes as C
    # 3 ints, 2+10 doubles, ... the struct must match the C layout byte for byte
    c = _lib.OcConfig()
    assert C.sizeof(c) % 8 == 0
    assert _lib.OcConfig.device.offset == C.sizeof(c) - 8


def test_library_refuses_invalid_config_without_a_gpu():
    import ctypes as C
    from hydrostatic_ocean_core_benchmark_b200.params import OceanParams
    lib = _lib.load()
    cfg = _lib.config_from_params(OceanParams(dt=1.0))
    cfg.nz = 0
    h = C.c_void_p()
    assert lib.oc_create(C.byref(cfg), C.byref(h)) == 1
    assert not h.value


def test_fp64_handles_refuse_the_refined_solver_without_a_gpu():
    """The FP32-inner refined solve serves the mixed-precision step only: an
    fp64 handle must reproduce the reference's solves."""
    import ctypes as C
    from hydrostatic_ocean_core_benchmark_b200.params import OceanParams
    lib = _lib.load()
    p = OceanParams(dt=1.0, scheme_name="theta", solver_kind="pcg_refined")
    h = C.c_void_p()
    assert lib.oc_create(C.byref(_lib.config_from_params(p, 0, "fp64")), C.byref(h)) == 1
    assert not h.value
    cfg = _lib.config_from_params(p, 0, "fp64")
    cfg.solver = 6
    assert lib.oc_create(C.byref(cfg), C.byref(h)) == 1


def test_entry_points_refuse_null_arguments_without_a_gpu():
    """Every entry point answers a null handle or a missing required pointer
    with OC_ERR_ARG before it touches a device; the error-string calls and
    oc_destroy accept null."""
    import ctypes as C
    lib = _lib.load()
    ARG = 1
    i32, i64, dbl = C.c_int32(), C.c_int64(), C.c_double()
    buf = (C.c_double * 8)()
    calls = {
        "oc_create": lambda: lib.oc_create(None, None),
        "oc_set_domain": lambda: lib.oc_set_domain(None, buf, buf, None),
        "oc_set_domain_slab": lambda: lib.oc_set_domain_slab(None, buf, buf, buf, buf, buf, 1.0, 1.0),
        "oc_set_forcing": lambda: lib.oc_set_forcing(None, buf, buf),
        "oc_set_state": lambda: lib.oc_set_state(None, None, 0),
        "oc_set_state_async": lambda: lib.oc_set_state_async(None, None, 0, None),
        "oc_reset_mixing": lambda: lib.oc_reset_mixing(None),
        "oc_bind_state": lambda: lib.oc_bind_state(None, None, None),
        "oc_set_wait_bound": lambda: lib.oc_set_wait_bound(None, 1000),
        "oc_state_parity": lambda: lib.oc_state_parity(None, None),
        "oc_get_state": lambda: lib.oc_get_state(None, None, 0),
        "oc_get_state_async": lambda: lib.oc_get_state_async(None, None, 0, None),
        "oc_step": lambda: lib.oc_step(None, 1, None),
        "oc_step_graph": lambda: lib.oc_step_graph(None, 1, None),
        "oc_get_stats": lambda: lib.oc_get_stats(None, None),
        "oc_set_profiling": lambda: lib.oc_set_profiling(None, 1),
        "oc_get_kernel_times": lambda: lib.oc_get_kernel_times(None, None, 0, C.byref(i32)),
        "oc_get_solve_log": lambda: lib.oc_get_solve_log(None, None, 0, C.byref(i32)),
        "oc_reset_stats": lambda: lib.oc_reset_stats(None),
        "oc_helmholtz_solve": lambda: lib.oc_helmholtz_solve(None, buf, buf, None, None),
        "oc_thomas": lambda: lib.oc_thomas(None, buf, buf, buf, buf, 4, 2, None),
        "oc_thomas_noalloc": lambda: lib.oc_thomas_noalloc(buf, buf, buf, buf, None, 4, 2, None),
        "oc_buoyancy": lambda: lib.oc_buoyancy(None, buf, buf, buf, buf, 8, None),
        "oc_helm_create": lambda: lib.oc_helm_create(None, buf, buf, buf, None),
        "oc_helm_solve": lambda: lib.oc_helm_solve(None, buf, buf, 0, None, None, None),
        "oc_helm_refine_report": lambda: lib.oc_helm_refine_report(None, C.byref(i32), C.byref(dbl)),
        "oc_helm_set_inner_rtol": lambda: lib.oc_helm_set_inner_rtol(None, 1e-3),
        "oc_helm_destroy": lambda: lib.oc_helm_destroy(None),
        "oc_density": lambda: lib.oc_density(0, 1.0, 0.0, 0.0, 0.0, 0.0, None, buf, buf, buf, 8, None),
        "oc_get_field": lambda: lib.oc_get_field(None, b"eta", buf, 8),
        "oc_halo_values_per_row": lambda: lib.oc_halo_values_per_row(None, C.byref(i64)),
        "oc_pack_rows": lambda: lib.oc_pack_rows(None, 0, 1, buf, None),
        "oc_unpack_rows": lambda: lib.oc_unpack_rows(None, 0, 1, buf, None),
        "oc_set_tiling": lambda: lib.oc_set_tiling(None, 1, 1),
        "oc_autotune": lambda: lib.oc_autotune(None, C.byref(i32), C.byref(i32)),
        "oc_ensemble_create": lambda: lib.oc_ensemble_create(None, 1, None),
        "oc_ensemble_step": lambda: lib.oc_ensemble_step(None, 1, None),
        "oc_ensemble_destroy": lambda: lib.oc_ensemble_destroy(None),
        "oc_adjoint_step": lambda: lib.oc_adjoint_step(None, buf, buf, buf, buf, buf, None, None),
        "oc_adjoint_eos": lambda: lib.oc_adjoint_eos(None, buf, buf, buf, buf, buf, None),
    }
    for name, call in calls.items():
        assert call() == ARG, name
    assert lib.oc_last_error(None) == b"null handle"
    assert lib.oc_helm_last_error(None) == b"null handle"
    assert lib.oc_ensemble_last_error(None) == b"null ensemble"
    lib.oc_destroy(None)
    # every header function is covered here, by the symbol tests or by the namelist protocol tests
    covered = set(calls) | {"oc_version", "oc_last_error", "oc_helm_last_error", "oc_ensemble_last_error",
                            "oc_destroy", "oc_run_namelist"}
    assert header_functions() <= covered, header_functions() - covered
