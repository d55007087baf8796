"""The binary protocol's refusals, on CPU: ``ocean3d5_b200 <prefix>.nml`` checks
the namelist and the bundle files before it touches a GPU, and refuses what the
step cannot run with ``FATAL: ...`` on stderr and exit code 1, the reference
binary's convention (libs/cuda/src/cfd_exp3d5_cuda.cu:111-114,1117-1127 and
libs/cuda/src/config.hpp:78,153-163)."""

import subprocess
from pathlib import Path

import numpy as np
import pytest

from hydrostatic_ocean_core_benchmark_b200 import cases
from hydrostatic_ocean_core_benchmark_b200.bundle import write_bundle
from oracle import ocean_oracle as orc

ROOT = Path(__file__).resolve().parents[1]
EXE = ROOT / "hydrostatic_ocean_core_benchmark_b200" / "bin" / "ocean3d5_b200"


@pytest.fixture(scope="module")
def bundle(tmp_path_factory):
    d = tmp_path_factory.mktemp("bundle")
    s = cases.seamount_basin(nx=16, ny=16, nz=6, seed=1)
    p = s.params.replace(n_steps=2, n_warmup=0, n_repeat=1, out_prefix=str(d / "out"))
    geo = orc.Geometry(p, s.H, s.mask, s.dzr)
    b = orc.buoyancy(p.eos, s.T, s.S, geo.zc, p.g, p.rho0, p.alpha_t, p.beta_s, p.t0, p.s0) * geo.mask3
    nml = write_bundle(str(d / "case"), p, s.H, s.mask, orc.OracleState(s.u, s.v, b, s.eta, s.T, s.S),
                       dzr=s.dzr, taux_c=s.taux_c, tauy_c=s.tauy_c)
    return Path(nml)


def _run(*args):
    if not EXE.exists():
        pytest.fail(f"{EXE} is missing: build the package first")
    return subprocess.run([str(EXE), *map(str, args)], capture_output=True, text=True, timeout=60)


def _mutated(bundle: Path, tmp_path: Path, key: str, value: str) -> Path:
    lines = bundle.read_text().splitlines()
    hits = [i for i, ln in enumerate(lines) if ln.strip().startswith(f"{key} =")]
    assert len(hits) == 1, key
    lines[hits[0]] = f"  {key} = {value}"
    out = tmp_path / "case.nml"
    out.write_text("\n".join(lines) + "\n")
    return out


def test_usage_and_missing_namelist(tmp_path):
    r = _run()
    assert r.returncode == 1 and "usage: ocean3d5_b200 <namelist>" in r.stderr
    r = _run(tmp_path / "absent.nml")
    assert r.returncode == 1 and "FATAL: cannot open namelist" in r.stderr


@pytest.mark.parametrize("key,value,message", [
    ("scheme_name", "'leapfrog'", "unknown scheme leapfrog"),
    ("solver_kind", "'sor'", "unknown variable-coefficient solver sor"),
    ("theta", "0.0d+00", "theta must lie in (0,1]"),
    ("n_picard", "0", "dt, n_steps and n_picard must come from the driver"),
    ("vcoord", "'sigma'", "vcoord=zlevel only"),
    ("bc_x", "'open'", "periodic|closed boundaries only"),
    ("face_rule", "'max'", "face_rule must be min|mean|harmonic"),
    ("eos", "'unesco'", "eos must be linear|seos|teos10"),
    ("advection", "'weno5'", "unknown advection weno5"),
    ("tracers", "'passive'", "tracers must be buoyancy|TS"),
    ("closure", "'kpp'", "closure must be none|tke"),
    ("mxl", "'blackadar'", "mxl must be integral|recursive"),
    ("barotropic_average", "'cosine'", "barotropic_average must be none|mean"),
])
def test_unsupported_options_are_refused(bundle, tmp_path, key, value, message):
    r = _run(_mutated(bundle, tmp_path, key, value))
    assert r.returncode == 1, r.stdout + r.stderr
    assert f"FATAL: {message}" in r.stderr


def test_missing_and_short_bundle_files(bundle, tmp_path):
    r = _run(_mutated(bundle, tmp_path, "domain_file", f"'{tmp_path / 'absent.bin'}'"))
    assert r.returncode == 1 and "FATAL: cannot read" in r.stderr
    short = tmp_path / "short_init.bin"
    short.write_bytes(np.zeros(10).tobytes())
    r = _run(_mutated(bundle, tmp_path, "init_file", f"'{short}'"))
    assert r.returncode == 1 and "is shorter than the state it must hold" in r.stderr
    short_lv = tmp_path / "short_levels.bin"
    short_lv.write_bytes(np.ones(2).tobytes())
    r = _run(_mutated(bundle, tmp_path, "levels_file", f"'{short_lv}'"))
    assert r.returncode == 1 and "is shorter than nz doubles" in r.stderr


@pytest.mark.parametrize("line,message", [
    # a doubled quote inside a quoted value stands for one quote
    ("  scheme_name = 'leap''frog'", "unknown scheme leap'frog"),
    # names are case-insensitive and a comment may follow the value
    ("  SCHEME_NAME = \"leapfrog\"   ! not a scheme", "unknown scheme leapfrog"),
    # several items on one line, separated by commas; a D exponent
    ("  theta = 0.0D0, n_picard = 2", "theta must lie in (0,1]"),
    ("  theta = 1.5d+00", "theta must lie in (0,1]"),
])
def test_namelist_format_variants(bundle, tmp_path, line, message):
    """The namelist reader follows the Fortran namelist format the bundle
    writer emits (reference tools/toml2nml.py:27-34,188-268), including forms
    the writer does not use but a hand-edited file may: doubled quotes, upper
    case names, trailing comments and comma-separated items."""
    key = line.split("=")[0].strip().lower()
    lines = bundle.read_text().splitlines()
    hits = [i for i, ln in enumerate(lines) if ln.strip().lower().startswith(f"{key} =")]
    assert len(hits) == 1, key
    lines[hits[0]] = line
    nml = tmp_path / "case.nml"
    nml.write_text("\n".join(lines) + "\n")
    r = _run(nml)
    assert r.returncode == 1, r.stdout + r.stderr
    assert f"FATAL: {message}" in r.stderr


def test_group_end_forms(bundle, tmp_path):
    """`&end` closes a group as `/` does; items outside any group are ignored."""
    text = bundle.read_text().replace("\n/\n", "\n&end\n")
    text = "scheme_name = 'leapfrog'\n" + text
    nml = tmp_path / "case.nml"
    nml.write_text(text.replace("scheme_name = 'theta'", "scheme_name = 'split'"))
    r = _run(nml)
    assert r.returncode == 1 and "FATAL: unknown scheme split" in r.stderr, r.stderr
