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
