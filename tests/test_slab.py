"""Host logic of the y-slab fb driver (hydrostatic_ocean_core_benchmark_b200/slab.py), on CPU.

The rows each rank owns and stores, the whole domain's face masks against the
oracle's, and the halo exchange itself: two gloo ranks run the driver over a
stand-in stepper whose step is a nonlinear stencil reaching two rows, and their
owned rows must equal a single-domain run of the same stencil bit for bit.
"""

import os
import socket

import numpy as np
import pytest

from hydrostatic_ocean_core_benchmark_b200 import cases
from hydrostatic_ocean_core_benchmark_b200.params import OceanParams
from hydrostatic_ocean_core_benchmark_b200.slab import FbSlabRun, SlabLayout, face_masks
from oracle import ocean_oracle as orc


@pytest.mark.parametrize("ny,n,halo", [(64, 4, 16), (50, 3, 16), (33, 2, 16), (16, 1, 16), (20, 3, 5)])
def test_layout_owns_every_row_once(ny, n, halo):
    lay = SlabLayout(ny, n, halo)
    owned = np.concatenate([np.arange(*(lambda j0, m: (j0, j0 + m))(*lay.owned(r))) for r in range(n)])
    assert np.array_equal(owned, np.arange(ny))
    for r in range(n):
        j0, m = lay.owned(r)
        rows = lay.rows(r)
        assert len(rows) == m + 2 * halo == lay.ny_ext(r)
        assert np.array_equal(rows[halo:halo + m], np.arange(j0, j0 + m))
        assert np.array_equal(rows, (np.arange(j0 - halo, j0 + m + halo)) % ny)


def test_layout_refuses_ranks_thinner_than_the_halo():
    with pytest.raises(ValueError, match="halo"):
        SlabLayout(30, 2, 16)
    with pytest.raises(ValueError):
        SlabLayout(30, 0, 4)


@pytest.mark.parametrize("bc", [("closed", "closed"), ("periodic", "periodic"), ("periodic", "closed")])
def test_face_masks_equal_the_oracle(bc):
    s = cases.seamount_basin(nx=24, ny=20, nz=6, seed=3, bc_x=bc[0], bc_y=bc[1])
    mask = s.mask.copy()
    mask[5:8, 10:14] = 0.0   # an island
    mask[:, 0] = 0.0         # a coast
    g = orc.Geometry(s.params, s.H, mask, s.dzr)
    mu, mv = face_masks(mask, *bc)
    assert np.array_equal(mu, g.mask_u) and np.array_equal(mv, g.mask_v)


def test_slab_refuses_schemes_other_than_fb():
    p = OceanParams(nx=8, ny=40, nz=4, scheme_name="theta")
    with pytest.raises(ValueError, match="fb only"):
        FbSlabRun(p, np.ones((40, 8)), np.ones((40, 8)), rank=0, nranks=1)


# ---------------------------------------------------------------------- stand-in stepper
class StencilStepper:
    """A stepper with the OceanStepper interface the driver uses: fields eta
    [ny, nx] and u, v [nz, ny, nx], a step that reaches two rows each way and
    stops at closed v faces, rows packed field after field, level after level."""

    def __init__(self, params, H, mask, dzr=None, taux_c=None, tauy_c=None, device=0, slab=None):
        self.p = params
        self.mv = np.asarray(slab[1]) if slab is not None else face_masks(mask, params.bc_x, params.bc_y)[1]
        self.H = np.asarray(H)
        self.levels = [1, params.nz, params.nz]

    def halo_values_per_row(self):
        return sum(self.levels) * self.p.nx

    def set_state(self, eta, u, v, **_):
        self.s = {"eta": np.array(eta, dtype=np.float64), "u": np.array(u, dtype=np.float64),
                  "v": np.array(v, dtype=np.float64)}

    def get_state(self):
        return {k: a.copy() for k, a in self.s.items()}

    def step(self, n=1, stream=None):
        for _ in range(n):
            eta, u, v = self.s["eta"], self.s["u"], self.s["v"]
            mv = self.mv
            # flux through v faces, zero at closed faces, reaching j-1 .. j+1
            flux = mv * (np.roll(u, -1, axis=-2) - u) * (0.5 + 0.25 * v)
            un = u + 0.1 * (flux - np.roll(flux, 1, axis=-2)) + 0.01 * np.sin(self.H / 1000.0)
            vn = v * 0.99 + 0.02 * np.roll(u, 2, axis=-2) * mv + 0.001 * eta
            etan = eta - 0.05 * (vn[0] - np.roll(vn[0], 1, axis=-2) * np.roll(mv, 1, axis=-2))
            self.s = {"eta": etan, "u": un, "v": vn}

    def _rows(self, j0, nrows):
        return [self.s["eta"][None, j0:j0 + nrows], self.s["u"][:, j0:j0 + nrows],
                self.s["v"][:, j0:j0 + nrows]]

    def pack_rows(self, j0, nrows, buf, stream=None):
        flat = np.concatenate([a.reshape(-1) for a in self._rows(j0, nrows)])
        buf[:flat.size] = __import__("torch").from_numpy(flat)

    def unpack_rows(self, j0, nrows, buf, stream=None):
        data = buf.numpy()
        off = 0
        for name, lev in (("eta", 1), ("u", self.p.nz), ("v", self.p.nz)):
            n = lev * nrows * self.p.nx
            blk = data[off:off + n].reshape(lev, nrows, self.p.nx)
            if name == "eta":
                self.s[name][j0:j0 + nrows] = blk[0]
            else:
                self.s[name][:, j0:j0 + nrows] = blk
            off += n

    def stats(self):
        return {"device_bytes": 0}

    def close(self):
        pass


def _inputs(bc_y):
    p = OceanParams(nx=12, ny=24, nz=3, scheme_name="fb", bc_x="closed", bc_y=bc_y, lx=1.0e5, ly=2.0e5)
    rng = np.random.default_rng(5)
    H = 1000.0 + 500.0 * rng.random((24, 12))
    mask = np.ones((24, 12))
    mask[10:13, 4:7] = 0.0
    st = {"eta": rng.standard_normal((24, 12)), "u": rng.standard_normal((3, 24, 12)),
          "v": rng.standard_normal((3, 24, 12))}
    return p, H, mask, st


def _global_run(bc_y, steps):
    p, H, mask, st = _inputs(bc_y)
    ref = StencilStepper(p, H, mask)
    ref.set_state(**st)
    ref.step(steps)
    return ref.get_state()


def _rank_main(rank, world, port, bc_y, steps, out_dir):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        p, H, mask, st = _inputs(bc_y)
        run = FbSlabRun(p, H, mask, halo=4, stepper_factory=StencilStepper, torch_device="cpu")
        run.set_state(**st)
        run.step(steps)
        got = run.gather_state()
        if rank == 0:
            np.savez(os.path.join(out_dir, "slabs.npz"), **got)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("bc_y", ["closed", "periodic"])
@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_reproduce_the_single_domain_run(tmp_path, bc_y, world):
    import torch.multiprocessing as mp
    steps = 6
    mp.spawn(_rank_main, args=(world, _free_port(), bc_y, steps, str(tmp_path)), nprocs=world, join=True)
    got = dict(np.load(tmp_path / "slabs.npz"))
    want = _global_run(bc_y, steps)
    for k in want:
        assert np.array_equal(got[k], want[k]), f"{k} differs with {world} ranks, bc_y={bc_y}"


def test_one_rank_exchanges_with_itself():
    p, H, mask, st = _inputs("closed")
    run = FbSlabRun(p, H, mask, halo=4, rank=0, nranks=1, stepper_factory=StencilStepper, torch_device="cpu")
    run.set_state(**st)
    run.step(5)
    got = run.gather_state()
    want = _global_run("closed", 5)
    for k in want:
        assert np.array_equal(got[k], want[k]), k


def _bundle(tmp_path, scheme, ny):
    from hydrostatic_ocean_core_benchmark_b200.params import write_namelist
    p = OceanParams(nx=8, ny=ny, nz=4, scheme_name=scheme, out_prefix=str(tmp_path / "out"))
    return write_namelist(str(tmp_path / "case.nml"), p)


@pytest.mark.parametrize("scheme,ny,halo,what", [("theta", 40, 16, "fb only"), ("fb", 12, 16, "halo")])
def test_front_end_refuses_before_any_device_work(tmp_path, scheme, ny, halo, what):
    """The multi-device front end refuses other schemes and ranks thinner than the
    halo with FATAL and exit code 2, as the reference's binary does."""
    import subprocess
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    nml = _bundle(tmp_path, scheme, ny)
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK")}
    r = subprocess.run([sys.executable, "-m", "hydrostatic_ocean_core_benchmark_b200.slab", str(nml),
                        "--halo", str(halo)], capture_output=True, text=True, cwd=root, timeout=300,
                       env={**env, "PYTHONPATH": str(root)})
    assert r.returncode == 2, r.stdout + r.stderr
    assert "FATAL" in r.stderr and what in r.stderr


def _front_end(tmp_path, nml, *flags, env_extra=None):
    import subprocess
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK")}
    env.update(PYTHONPATH=str(root), **(env_extra or {}))
    return subprocess.run([sys.executable, "-m", "hydrostatic_ocean_core_benchmark_b200.slab", str(nml), *flags],
                          capture_output=True, text=True, cwd=root, timeout=300, env=env)


@pytest.mark.parametrize("flags,env_extra,what", [
    (("--ndev", "0"), None, "--ndev must be >= 1"),
    (("--devices", "0,x"), None, "comma-separated list"),
    (("--devices", "1,1"), None, "distinct non-negative"),
    (("--ndev", "3", "--devices", "0,1"), None, "disagree"),
    (("--ndev", "3"), {"WORLD_SIZE": "2"}, "the launcher started 2 ranks"),
    (("--devices", "5"), None, "device 5 does not exist"),
])
def test_front_end_command_line_refusals(tmp_path, flags, env_extra, what):
    """--ndev and --devices as the reference binary takes them, refused before any
    rendezvous or device work (a CPU box has no device 5)."""
    r = _front_end(tmp_path, _bundle(tmp_path, "fb", 40), *flags, env_extra=env_extra)
    assert r.returncode == 2, r.stdout + r.stderr
    assert "FATAL" in r.stderr and what in r.stderr


def test_front_end_starts_its_own_ranks(tmp_path):
    """Without a launcher, --ndev 2 starts two ranks that meet over gloo on
    127.0.0.1; here both refuse the theta scheme, and the exit code comes back."""
    r = _front_end(tmp_path, _bundle(tmp_path, "theta", 40), "--ndev", "2")
    assert r.returncode == 2, r.stdout + r.stderr
    assert r.stderr.count("FATAL") >= 1 and "fb only" in r.stderr
