"""The TOML front end against the reference's own bundle writer, on CPU.

``tests/golden/make_v05_bundles.py`` ran the reference's ``write_v05_bundle``
(tools/toml2nml.py:143-273) on this package's default TOML tree under several
override sets (bathymetry kinds, cases, schemes, EOS, face rules, an island,
a band-limited rough field). Resolving the same tree and overrides here must
give the same namelist values and byte-identical domain and initial-state
files."""

import hashlib
import json
from pathlib import Path

import pytest

from hydrostatic_ocean_core_benchmark_b200 import toml_front as tf
from hydrostatic_ocean_core_benchmark_b200.bundle import write_bundle
from hydrostatic_ocean_core_benchmark_b200.params import parse_namelist_text

ROOT = Path(__file__).resolve().parents[1]
CONFIG = ROOT / "hydrostatic_ocean_core_benchmark_b200" / "config"
CASES = json.loads((ROOT / "tests" / "golden" / "v05_bundles.json").read_text())
# keys the reference writes that this front end does not carry, or that name files
NOT_COMPARED = {"omp_min_points", "tridiag_kernel", "pcg_sync", "pcg_check_every", "out_prefix", "domain_file",
                "init_file", "n_repeat", "n_warmup"}


def _sha(path):
    return hashlib.sha256(Path(path).read_bytes()).hexdigest()


def _value(raw):
    try:
        return float(raw.replace("d", "e").replace("D", "e"))
    except ValueError:
        return raw


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_front_end_writes_the_reference_bundle(case, tmp_path):
    config = tf.apply_overrides(tf.load_config(CONFIG), case["overrides"])
    run = tf.resolve_run(config, nx=case["nx"], nz=case["nz"], case=case["case"], cfl=case["cfl"],
                         n_steps=case["steps"])
    prefix = str(tmp_path / "b")
    nml = write_bundle(prefix, run.params.replace(n_repeat=1, n_warmup=0), run.H, run.mask, run.state)
    ours = parse_namelist_text(Path(nml).read_text())
    want = case["namelist"]
    compared = 0
    for key, raw in want.items():
        if key in NOT_COMPARED or key not in ours:
            continue
        assert _value(ours[key]) == _value(raw), (key, ours[key], raw)
        compared += 1
    assert compared >= 50
    assert _sha(prefix + "_domain.bin") == case["domain_sha256"]
    assert _sha(prefix + "_init.bin") == case["init_sha256"]


def test_overrides_parse_as_the_reference_driver():
    assert tf.parse_override("12") == 12 and isinstance(tf.parse_override("12"), int)
    assert tf.parse_override("1e-3") == 1e-3
    assert tf.parse_override("TRUE") is True and tf.parse_override("false") is False
    assert tf.parse_override("up3_tvd") == "up3_tvd"
    c = tf.apply_overrides(tf.load_config(CONFIG), ["grid.nx=40", "new.table.key=x"])
    assert c.get("grid.nx") == 40 and c.get("new.table.key") == "x"
    with pytest.raises(SystemExit):
        tf.apply_overrides(c, ["no_equals_sign"])


def test_refused_cases_name_themselves():
    c = tf.load_config(CONFIG)
    with pytest.raises(ValueError, match="zstar_constancy"):
        tf.resolve_run(c.with_overrides({"case.zstar_constancy.eta0": 0.1}), nx=8, nz=2, case="zstar_constancy")


def test_main_bundle_subcommand_writes_the_reference_bundle(tmp_path, capsys):
    from hydrostatic_ocean_core_benchmark_b200 import main
    case = CASES[0]
    prefix = str(tmp_path / "cli")
    args = ["bundle", "--config", str(CONFIG), "--case", case["case"], "--nx", str(case["nx"]), "--nz",
            str(case["nz"]), "--cfl", str(case["cfl"]), "--steps", str(case["steps"]), "--prefix", prefix]
    for o in case["overrides"]:
        args += ["--set", o]
    assert main.main(args) == 0
    assert "v0.5 bundle" in capsys.readouterr().out
    assert _sha(prefix + "_domain.bin") == case["domain_sha256"]
    assert _sha(prefix + "_init.bin") == case["init_sha256"]


def test_verify_gate_metric():
    """field_error: relative L2, or over the state scale for a near-zero field
    (reference tools/compare_backends3d.py:52-67)."""
    import numpy as np
    from hydrostatic_ocean_core_benchmark_b200.main import field_error
    a = np.array([1.0, 2.0, 3.0])
    assert field_error(a, a, 1.0) == 0.0
    assert abs(field_error(a * (1 + 1e-13), a, 1.0) - 1e-13) < 1e-15
    z = np.zeros(3)
    assert field_error(z + 1e-20, z, 10.0) == pytest.approx(np.sqrt(3) * 1e-20 / 10.0)


def _reference_dir():
    import os
    d = Path(os.environ.get("OCEAN_REFERENCE", str(ROOT.parent / "reference")))
    return d if (d / "libs" / "core" / "model3d_v05.py").exists() else None


@pytest.mark.skipif(_reference_dir() is None, reason="needs the reference checkout")
def test_verify_builds_the_reference_stepper_of_the_run():
    """verify's reference side: the reference's own NumPy stepper built for a
    TOML-resolved run takes the oracle's step, bit for bit."""
    import numpy as np
    from hydrostatic_ocean_core_benchmark_b200.main import reference_stepper_factory
    from oracle import ocean_oracle as orc
    config = tf.apply_overrides(tf.load_config(CONFIG), ["physics3d_v06.closure=tke"])
    run = tf.resolve_run(config, nx=16, nz=6, case="lock_exchange", cfl=1.0, n_steps=2)
    stepper, s0 = reference_stepper_factory(_reference_dir(), config, run)
    p, s = run.params, run.state
    ref = orc.OracleStepper(p, run.H, run.mask)
    o = orc.OracleState(s.u, s.v, s.b, s.eta, s.T, s.S)
    for _ in range(2):
        s0 = stepper.step(s0)
        o = ref.step(o)
    for f in ("eta", "u", "v", "b", "T", "S"):
        assert np.array_equal(getattr(s0, f), getattr(o, f)), f


LADDER = json.loads((Path(__file__).resolve().parent / "golden" / "ladder_case.json").read_text())


@pytest.mark.parametrize("case", LADDER, ids=[c["name"] for c in LADDER])
def test_ladder_case_matches_the_reference_tree(case, tmp_path):
    """The reference's hardware-ladder case (lock_exchange, theta 0.5, 50 steps),
    bundled by the reference's tool on the reference's own tree, is what this
    package's tree gives under the same flags plus `extra`."""
    config = tf.apply_overrides(tf.load_config(CONFIG), case["overrides"] + case["extra"])
    run = tf.resolve_run(config, nx=case["nx"], nz=case["nz"], case=case["case"], cfl=case["cfl"],
                         n_steps=case["steps"])
    prefix = str(tmp_path / "b")
    nml = write_bundle(prefix, run.params.replace(n_repeat=1, n_warmup=0), run.H, run.mask, run.state)
    ours = parse_namelist_text(Path(nml).read_text())
    compared = 0
    for key, raw in case["namelist"].items():
        if key in NOT_COMPARED or key not in ours:
            continue
        assert _value(ours[key]) == _value(raw), (key, ours[key], raw)
        compared += 1
    assert compared >= 50
    assert _sha(prefix + "_domain.bin") == case["domain_sha256"]
    assert _sha(prefix + "_init.bin") == case["init_sha256"]
