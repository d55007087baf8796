"""ctypes binding of ``lib/libocean_b200.so`` (the C ABI of ``include/ocean_b200.h``).

There is no fallback: if the library is missing or fails to load, every entry
point raises. Build it with ``python -m hydrostatic_ocean_core_benchmark_b200.build``.
"""

from __future__ import annotations

import ctypes as C
from pathlib import Path

from .params import OceanParams

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libocean_b200.so"

OC_OK = 0
ERRORS = {1: "invalid argument", 2: "CUDA error", 3: "unsupported option", 4: "call out of order",
          5: "device-side wait timed out", 6: "I/O error", 7: "request above a fixed buffer size"}

SCHEMES = {"fb": 0, "theta": 1, "split_explicit": 2}
SOLVERS = {"pcg_jacobi": 0, "pcg_rbgs": 1, "rbgs": 2, "multigrid": 3, "pcg_refined": 4, "pcg_mg": 5}
BCS = {"periodic": 0, "closed": 1}
FACE_RULES = {"min": 0, "mean": 1, "harmonic": 2}
EOS = {"linear": 0, "seos": 1, "teos10": 2}
PGF = {"remove": 0, "keep": 1}
ADVECTION = {"none": 0, "centered2": 1, "upwind1": 2, "up3": 3, "up3_tvd": 4}
TRACERS = {"buoyancy": 0, "TS": 1}
CLOSURES = {"none": 0, "tke": 1}
MXL = {"integral": 0, "recursive": 1}
BTAVG = {"none": 0, "mean": 1}


class OcConfig(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
        ("lx", C.c_double), ("ly", C.c_double),
        ("g", C.c_double), ("f0", C.c_double), ("h0", C.c_double), ("n2", C.c_double),
        ("nu", C.c_double), ("kappa", C.c_double), ("rho0", C.c_double), ("tau_x", C.c_double),
        ("tau_y", C.c_double), ("bottom_drag", C.c_double),
        ("scheme", C.c_int32),
        ("theta", C.c_double), ("theta_cor", C.c_double), ("theta_v", C.c_double),
        ("n_picard", C.c_int32), ("n_split", C.c_int32), ("barotropic_average", C.c_int32),
        ("solver", C.c_int32),
        ("rtol", C.c_double),
        ("max_iter", C.c_int32),
        ("dt", C.c_double),
        ("bc_x", C.c_int32), ("bc_y", C.c_int32), ("face_rule", C.c_int32),
        ("min_partial", C.c_double),
        ("eos", C.c_int32), ("pgf", C.c_int32), ("pgf_correction", C.c_int32),
        ("advection", C.c_int32), ("tracers", C.c_int32),
        ("alpha_t", C.c_double), ("beta_s", C.c_double), ("t0", C.c_double), ("s0", C.c_double),
        ("cp", C.c_double), ("a_h", C.c_double), ("k_h", C.c_double), ("q_heat", C.c_double),
        ("q_salt", C.c_double),
        ("closure", C.c_int32), ("mxl", C.c_int32),
        ("c_k", C.c_double), ("c_eps", C.c_double), ("pr_t", C.c_double), ("z_0", C.c_double),
        ("e_min", C.c_double), ("l_min", C.c_double), ("e_bb", C.c_double), ("n2_min", C.c_double),
        ("device", C.c_int32),
        ("precision", C.c_int32),
    ]


class OcStateView(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("eta", "u", "v", "b", "T", "S", "e", "km", "kh")]


class OcStats(C.Structure):
    _fields_ = [
        ("steps", C.c_int64), ("solver_iterations", C.c_int64), ("solver_failures", C.c_int64),
        ("solver_rebuilds", C.c_int64), ("tridiagonal_solves", C.c_int64),
        ("barotropic_substeps", C.c_int64), ("solves", C.c_int64),
        ("n_split", C.c_int32), ("n_levels", C.c_int32), ("diverged", C.c_int32),
        ("device_status", C.c_int32), ("device_bytes", C.c_int64), ("kernel_launches", C.c_int64),
    ]


class OcHelmConfig(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("dx", C.c_double), ("dy", C.c_double),
                ("coef", C.c_double), ("solver", C.c_int32), ("rtol", C.c_double),
                ("max_iter", C.c_int32), ("device", C.c_int32)]


class OcKernelTime(C.Structure):
    _fields_ = [("name", C.c_char * 32), ("launches", C.c_int64), ("total_ms", C.c_double)]


# every exported symbol of include/ocean_b200.h with its ctypes signature
_SIGNATURES = {
    "oc_version": (C.c_char_p, []),
    "oc_create": (C.c_int, [C.POINTER(OcConfig), C.POINTER(C.c_void_p)]),
    "oc_set_domain": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "oc_set_forcing": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "oc_set_state": (C.c_int, [C.c_void_p, C.POINTER(OcStateView), C.c_int32]),
    "oc_set_state_async": (C.c_int, [C.c_void_p, C.POINTER(OcStateView), C.c_int32, C.c_void_p]),
    "oc_reset_mixing": (C.c_int, [C.c_void_p]),
    "oc_set_wait_bound": (C.c_int, [C.c_void_p, C.c_int64]),
    "oc_bind_state": (C.c_int, [C.c_void_p, C.POINTER(OcStateView), C.POINTER(OcStateView)]),
    "oc_state_parity": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32)]),
    "oc_get_state": (C.c_int, [C.c_void_p, C.POINTER(OcStateView), C.c_int32]),
    "oc_get_state_async": (C.c_int, [C.c_void_p, C.POINTER(OcStateView), C.c_int32, C.c_void_p]),
    "oc_step": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p]),
    "oc_adjoint_step": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                  C.c_void_p, C.c_void_p]),
    "oc_adjoint_eos": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                 C.c_void_p]),
    "oc_step_graph": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p]),
    "oc_get_stats": (C.c_int, [C.c_void_p, C.POINTER(OcStats)]),
    "oc_set_profiling": (C.c_int, [C.c_void_p, C.c_int32]),
    "oc_get_kernel_times": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.POINTER(C.c_int32)]),
    "oc_get_solve_log": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.POINTER(C.c_int32)]),
    "oc_reset_stats": (C.c_int, [C.c_void_p]),
    "oc_helmholtz_solve": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_int32),
                                     C.c_void_p]),
    "oc_thomas": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                            C.c_int32, C.c_int32, C.c_void_p]),
    "oc_thomas_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.c_int32, C.c_int32, C.c_void_p]),
    "oc_buoyancy": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                              C.c_int64, C.c_void_p]),
    "oc_helm_create": (C.c_int, [C.POINTER(OcHelmConfig), C.c_void_p, C.c_void_p, C.c_void_p,
                                 C.POINTER(C.c_void_p)]),
    "oc_helm_solve": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.POINTER(C.c_int32),
                                C.POINTER(C.c_int32), C.c_void_p]),
    "oc_helm_last_error": (C.c_char_p, [C.c_void_p]),
    "oc_helm_destroy": (C.c_int, [C.c_void_p]),
    "oc_helm_refine_report": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_double)]),
    "oc_helm_set_inner_rtol": (C.c_int, [C.c_void_p, C.c_double]),
    "oc_density": (C.c_int, [C.c_int32, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                             C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p]),
    "oc_get_field": (C.c_int, [C.c_void_p, C.c_char_p, C.c_void_p, C.c_int64]),
    "oc_set_domain_slab": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_double, C.c_double]),
    "oc_halo_values_per_row": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    "oc_set_tiling": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32]),
    "oc_ensemble_create": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p]),
    "oc_ensemble_step": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p]),
    "oc_ensemble_last_error": (C.c_char_p, [C.c_void_p]),
    "oc_ensemble_destroy": (C.c_int, [C.c_void_p]),
    "oc_autotune": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "oc_pack_rows": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p]),
    "oc_unpack_rows": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p]),
    "oc_run_namelist": (C.c_int, [C.c_char_p]),
    "oc_last_error": (C.c_char_p, [C.c_void_p]),
    "oc_destroy": (None, [C.c_void_p]),
}

_lib = None


def load() -> C.CDLL:
    """Load the library once; raise if it is missing (no CPU fallback exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: build it with "
                           "`python -m hydrostatic_ocean_core_benchmark_b200.build`")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def exported_symbols() -> list[str]:
    return list(_SIGNATURES)


PRECISIONS = {"fp64": 0, "mixed": 1}


def config_from_params(p: OceanParams, device: int = 0, precision: str = "fp64") -> OcConfig:
    p.validate()
    if precision not in PRECISIONS:
        raise ValueError(f"precision must be one of {sorted(PRECISIONS)}")
    c = OcConfig()
    for name in ("nx", "ny", "nz", "n_picard", "n_split", "max_iter"):
        setattr(c, name, int(getattr(p, name)))
    for name in ("lx", "ly", "g", "f0", "h0", "n2", "nu", "kappa", "rho0", "tau_x", "tau_y",
                 "bottom_drag", "theta", "theta_cor", "theta_v", "rtol", "dt", "min_partial",
                 "alpha_t", "beta_s", "t0", "s0", "cp", "a_h", "k_h", "q_heat", "q_salt", "c_k",
                 "c_eps", "pr_t", "z_0", "e_min", "l_min", "e_bb", "n2_min"):
        setattr(c, name, float(getattr(p, name)))
    c.scheme = SCHEMES[p.scheme_name]
    c.solver = SOLVERS.get(p.solver_kind, 0) if p.scheme_name != "theta" else SOLVERS[p.solver_kind]
    c.bc_x, c.bc_y = BCS[p.bc_x], BCS[p.bc_y]
    c.face_rule = FACE_RULES[p.face_rule]
    c.eos = EOS[p.eos]
    c.pgf = PGF[p.pgf]
    c.pgf_correction = 1 if p.pgf_correction else 0
    c.advection = ADVECTION[p.advection]
    c.tracers = TRACERS[p.tracers]
    c.closure = CLOSURES[p.closure]
    c.mxl = MXL[p.mxl]
    c.barotropic_average = BTAVG[p.barotropic_average]
    c.device = int(device)
    c.precision = PRECISIONS[precision]
    return c


class OceanError(RuntimeError):
    pass


def check(rc: int, handle=None, what: str = "") -> None:
    if rc != OC_OK:
        msg = ""
        if handle is not None:
            raw = load().oc_last_error(handle)
            msg = raw.decode() if raw else ""
        raise OceanError(f"{what}: {ERRORS.get(rc, rc)}" + (f" ({msg})" if msg else ""))
