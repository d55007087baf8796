"""The y-slab fb driver on the GPU against the single-device step.

The reference's gate for its multi-device driver (docs/03 section 12): the owned
rows of every slab equal the single-device run, maximum absolute difference 0.
Here the slabs are processes sharing the one GPU of the test box and exchange
their halos through gloo (host memory); their kernels never wait on one another.
"""

import os
import socket
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from hydrostatic_ocean_core_benchmark_b200 import cases

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]
FIELDS = ("eta", "u", "v", "b", "T", "S", "e", "km", "kh")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    import torch
    assert torch.cuda.is_available()
    torch.cuda.set_device(0)


def _case(bc_y="closed"):
    # fb at dt = 100 s keeps the gravity-wave CFL below 1 on this 50 km grid
    return cases.seamount_basin(nx=40, ny=40, nz=12, seed=7, scheme_name="fb", dt=100.0, bc_y=bc_y)


def _single(s, steps):
    from hydrostatic_ocean_core_benchmark_b200.stepper import OceanStepper
    st = OceanStepper(s.params, s.H, s.mask, dzr=s.dzr, taux_c=s.taux_c, tauy_c=s.tauy_c)
    st.set_state(eta=s.eta, u=s.u, v=s.v, T=s.T, S=s.S)
    st.step(steps)
    out = st.get_state()
    st.close()
    return out


def test_pack_and_unpack_rows():
    import torch
    from hydrostatic_ocean_core_benchmark_b200.stepper import OceanStepper
    s = _case()
    st = OceanStepper(s.params, s.H, s.mask, dzr=s.dzr, taux_c=s.taux_c, tauy_c=s.tauy_c)
    st.set_state(eta=s.eta, u=s.u, v=s.v, T=s.T, S=s.S)
    st.step(2)
    full = st.get_state()
    j0, nr = 7, 5
    n = st.halo_values_per_row()
    assert n == s.params.nx * (1 + 5 * s.params.nz + 3 * (s.params.nz + 1))
    buf = torch.empty(n * nr, dtype=torch.float64, device="cuda")
    st.pack_rows(j0, nr, buf)
    torch.cuda.synchronize()
    want = np.concatenate([full[f][..., j0:j0 + nr, :].reshape(-1) for f in FIELDS])
    assert np.array_equal(buf.cpu().numpy(), want)
    # rows written back elsewhere appear there, field by field
    st.unpack_rows(20, nr, buf)
    after = st.get_state()
    for f in FIELDS:
        assert np.array_equal(after[f][..., 20:20 + nr, :], full[f][..., j0:j0 + nr, :]), f
        assert np.array_equal(after[f][..., :20, :], full[f][..., :20, :]), f
    st.close()


@pytest.mark.parametrize("bc_y", ["closed", "periodic"])
def test_one_slab_with_itself_equals_the_single_device_step(bc_y):
    from hydrostatic_ocean_core_benchmark_b200.slab import FbSlabRun
    s = _case(bc_y)
    steps = 6
    run = FbSlabRun(s.params, s.H, s.mask, s.dzr, s.taux_c, s.tauy_c, rank=0, nranks=1)
    run.set_state(eta=s.eta, u=s.u, v=s.v, T=s.T, S=s.S)
    run.step(steps)
    got = run.gather_state()
    run.close()
    want = _single(s, steps)
    for f in FIELDS:
        assert np.array_equal(got[f], want[f]), f"{f} differs ({bc_y})"


def _rank_main(rank, world, port, steps, out_dir):
    import torch
    import torch.distributed as dist
    from hydrostatic_ocean_core_benchmark_b200.slab import FbSlabRun
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        s = _case()
        run = FbSlabRun(s.params, s.H, s.mask, s.dzr, s.taux_c, s.tauy_c)
        run.set_state(eta=s.eta, u=s.u, v=s.v, T=s.T, S=s.S)
        run.step(steps)
        got = run.gather_state()
        if rank == 0:
            np.savez(os.path.join(out_dir, "slabs.npz"), **got)
        run.close()
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


@pytest.mark.parametrize("world", [2])
def test_slabs_on_ranks_equal_the_single_device_step(tmp_path, world):
    import torch.multiprocessing as mp
    steps = 6
    mp.spawn(_rank_main, args=(world, _free_port(), steps, str(tmp_path)), nprocs=world, join=True)
    got = dict(np.load(tmp_path / "slabs.npz"))
    want = _single(_case(), steps)
    for f in FIELDS:
        assert np.array_equal(got[f], want[f]), f"{f} differs with {world} ranks"
    # and directly against the oracle's whole-domain fb run
    _equal_to_oracle(_case(), got, steps, f"{world} slabs")


def _equal_to_oracle(s, got, steps, what):
    from oracle import ocean_oracle as orc
    p = s.params
    geo = orc.Geometry(p, s.H, s.mask, s.dzr)
    b = orc.buoyancy(p.eos, s.T, s.S, geo.zc, p.g, p.rho0, p.alpha_t, p.beta_s, p.t0, p.s0) * geo.mask3
    ref = orc.OracleStepper(p, s.H, s.mask, dzr=s.dzr, taux_c=s.taux_c, tauy_c=s.tauy_c)
    state = orc.OracleState(s.u, s.v, b, s.eta, s.T, s.S)
    for _ in range(steps):
        state = ref.step(state)
    for f in FIELDS:
        want = {"km": ref.Km, "kh": ref.Kh}.get(f, None)
        want = getattr(state, f) if want is None else want
        assert np.array_equal(got[f], want), f"{what}: {f} differs from the oracle"


@pytest.mark.parametrize("bc_y", ["closed", "periodic"])
def test_one_slab_with_itself_equals_the_oracle(bc_y):
    """The gathered slab run against the oracle's whole-domain fb step, bit for bit."""
    from hydrostatic_ocean_core_benchmark_b200.slab import FbSlabRun
    s = _case(bc_y)
    steps = 6
    run = FbSlabRun(s.params, s.H, s.mask, s.dzr, s.taux_c, s.tauy_c, rank=0, nranks=1)
    run.set_state(eta=s.eta, u=s.u, v=s.v, T=s.T, S=s.S)
    run.step(steps)
    got = run.gather_state()
    run.close()
    _equal_to_oracle(s, got, steps, f"one slab ({bc_y})")


def test_namelist_front_end_matches_the_single_device_binary(tmp_path):
    """The multi-device protocol under torchrun (2 ranks) against ocean3d5_b200 on the
    same bundle: the state files are byte-identical."""
    from hydrostatic_ocean_core_benchmark_b200.bundle import write_bundle
    from oracle import ocean_oracle as orc
    s = _case()
    p = s.params
    geo = orc.Geometry(p, s.H, s.mask, s.dzr)
    bb = orc.buoyancy(p.eos, s.T, s.S, geo.zc, p.g, p.rho0, p.alpha_t, p.beta_s, p.t0, p.s0) * geo.mask3
    b = orc.OracleState(s.u, s.v, bb, s.eta, s.T, s.S)
    outs = {}
    for name in ("one", "slabs"):
        p = s.params.replace(n_steps=6, n_warmup=0, n_repeat=1, out_prefix=str(tmp_path / f"out_{name}"))
        nml = write_bundle(str(tmp_path / f"case_{name}"), p, s.H, s.mask, b, dzr=s.dzr, taux_c=s.taux_c,
                           tauy_c=s.tauy_c)
        outs[name] = (nml, p.out_prefix)
    exe = ROOT / "hydrostatic_ocean_core_benchmark_b200" / "bin" / "ocean3d5_b200"
    r = subprocess.run([str(exe), str(outs["one"][0])], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    env = dict(os.environ, PYTHONPATH=str(ROOT))
    r = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
                        "--master-addr=127.0.0.1", f"--master-port={_free_port()}", "-m",
                        "hydrostatic_ocean_core_benchmark_b200.slab", str(outs["slabs"][0]), "--halo", "16"],
                       capture_output=True, text=True, timeout=900, cwd=ROOT, env=env)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-3000:]
    one = Path(outs["one"][1] + "_state3d5.bin").read_bytes()
    slabs = Path(outs["slabs"][1] + "_state3d5.bin").read_bytes()
    assert one == slabs
    import json
    m = json.loads(Path(outs["slabs"][1] + "_metrics.json").read_text())
    assert m["n_devices"] == 2 and m["halo"] == 16 and m["scheme"] == "fb" and not m["diverged"]
