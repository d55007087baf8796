"""The bundle files of the backend protocol, on CPU: what write_bundle writes,
the namelist reader, read_domain / read_state and the multi-device front end's
reader give back exactly (reference layout, tools/toml2nml.py:143-273 and
tools/compare_backends3d5.py:32-43)."""

import numpy as np
import pytest

from hydrostatic_ocean_core_benchmark_b200 import cases
from hydrostatic_ocean_core_benchmark_b200.bundle import read_domain, read_state, write_bundle
from hydrostatic_ocean_core_benchmark_b200.params import read_namelist
from hydrostatic_ocean_core_benchmark_b200.slab import _read_bundle


class _State:
    def __init__(self, **kw):
        self.__dict__.update(kw)


@pytest.mark.parametrize("tracers", ["TS", "buoyancy"])
def test_bundle_round_trip(tmp_path, tracers):
    s = cases.seamount_basin(nx=12, ny=10, nz=5, seed=4)
    p = s.params.replace(tracers=tracers, out_prefix=str(tmp_path / "out"))
    rng = np.random.default_rng(1)
    b = rng.standard_normal((5, 10, 12))
    st = _State(eta=s.eta, u=s.u, v=s.v, b=b, T=s.T, S=s.S)
    nml = write_bundle(str(tmp_path / "case"), p, s.H, s.mask, st, dzr=s.dzr, taux_c=s.taux_c, tauy_c=s.tauy_c)
    q = read_namelist(nml)
    for k in ("nx", "ny", "nz", "dt", "theta", "solver_kind", "scheme_name", "eos", "tracers", "closure"):
        assert getattr(q, k) == getattr(p, k), k
    H, mask = read_domain(q.domain_file, q.nx, q.ny)
    assert np.array_equal(H, s.H) and np.array_equal(mask, s.mask)
    init = read_state(q.init_file, q.nx, q.ny, q.nz, tracers == "TS")
    want = {"eta": s.eta, "u": s.u, "v": s.v, "b": b}
    if tracers == "TS":
        want.update(T=s.T, S=s.S)
    assert set(init) == set(want)
    for k, a in want.items():
        assert np.array_equal(init[k], a), k
    H2, mask2, state2, dzr2, taux2, tauy2 = _read_bundle(q)
    assert np.array_equal(H2, s.H) and np.array_equal(mask2, s.mask)
    assert all(np.array_equal(state2[k], a) for k, a in want.items())
    assert np.array_equal(dzr2, s.dzr) and np.array_equal(taux2, s.taux_c) and np.array_equal(tauy2, s.tauy_c)


def test_short_files_are_refused(tmp_path):
    (tmp_path / "short.bin").write_bytes(np.zeros(7).tobytes())
    with pytest.raises(ValueError, match="expected"):
        read_state(tmp_path / "short.bin", 4, 3, 2, True)
    with pytest.raises(ValueError, match="expected"):
        read_domain(tmp_path / "short.bin", 4, 3)
    with pytest.raises(ValueError, match="needs b"):
        write_bundle(str(tmp_path / "x"), cases.seamount_basin(nx=8, ny=8, nz=3, seed=1).params,
                     np.ones((8, 8)), np.ones((8, 8)), _State(eta=0, u=0, v=0, b=None))
