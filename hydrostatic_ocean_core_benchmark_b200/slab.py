"""Multi-GPU run of the fb scheme on y-slabs with deep halos.

The reference's multi-device driver (libs/cuda/src/cfd_exp3d5_cuda_multi.cu,
design in docs/03 section 12) cuts the domain into y-slabs, one per device.
Each device stores its owned rows plus ``halo`` rows on either side (global
rows wrap periodically) and runs the unchanged single-device step on that
extended slab; after every step the halo rows of the state are refreshed from
the neighbours' owned rows. The static arrays are those of the whole domain,
cut by rows, and the whole domain's spacing is kept. While ``halo`` is at
least the stencil reach of one step, every owned row is bit-identical to the
single-device run. Only the forward-backward (fb) scheme decomposes this way:
theta needs a global elliptic solve, split_explicit a halo per substep.

Here each rank is one process on one GPU (``torch.distributed``): its slab is
an ``OceanStepper`` built with ``oc_set_domain_slab``, and a halo refresh packs
the first and last ``halo`` owned rows of every exchanged field into one
device buffer each (``oc_pack_rows``), swaps them with the two neighbours in
one batch of point-to-point transfers (NCCL between GPUs; gloo stages them
through host memory) and unpacks the received rows into the halos
(``oc_unpack_rows``, which also recomputes w for the new velocities).

    python -m torch.distributed.run --nproc-per-node N -m \\
        hydrostatic_ocean_core_benchmark_b200.slab <prefix>.nml [--halo H] [--devices 0,1,..]
    python -m hydrostatic_ocean_core_benchmark_b200.slab <prefix>.nml --ndev N [--halo H] [--devices ..]

(the second form starts the N ranks itself, as the reference binary's
``--ndev``; ``--devices`` maps rank r to the r-th listed device) reads the reference's bundle, runs ``n_warmup`` + ``n_repeat`` repeats of
``n_steps`` and writes ``<out_prefix>_state3d5.bin`` and
``<out_prefix>_metrics.json`` as the reference's multi-device binary does.
"""

from __future__ import annotations

import argparse
import json
import os
import socket
import sys
import statistics
import time
from pathlib import Path

import numpy as np

from .params import OceanParams, read_namelist

DEFAULT_HALO = 16  # the reference's default depth (cfd_exp3d5_cuda_multi.cu:59)


class SlabLayout:
    """Owned and stored rows of each rank (cfd_exp3d5_cuda_multi.cu:100-104):
    rank g owns rows [ny g / n, ny (g + 1) / n) and stores ``halo`` more rows on
    each side, wrapped periodically."""

    def __init__(self, ny: int, nranks: int, halo: int = DEFAULT_HALO):
        if nranks < 1:
            raise ValueError("nranks must be >= 1")
        if halo < 1:
            raise ValueError("halo must be >= 1")
        if ny // nranks < halo:
            raise ValueError(f"ny/nranks = {ny // nranks} < halo = {halo}: every rank must own at "
                             "least as many rows as the halo is deep")
        self.ny, self.nranks, self.halo = ny, nranks, halo

    def owned(self, rank: int) -> tuple[int, int]:
        """(first global row owned, rows owned)."""
        j0 = (self.ny * rank) // self.nranks
        j1 = (self.ny * (rank + 1)) // self.nranks
        return j0, j1 - j0

    def ny_ext(self, rank: int) -> int:
        return self.owned(rank)[1] + 2 * self.halo

    def rows(self, rank: int) -> np.ndarray:
        """Global row of each stored row of the rank's slab."""
        j0, _ = self.owned(rank)
        return (j0 - self.halo + np.arange(self.ny_ext(rank))) % self.ny


def face_masks(mask, bc_x: str, bc_y: str) -> tuple[np.ndarray, np.ndarray]:
    """The whole domain's 2D face masks as oc_set_domain forms them
    (domain.py:60-97): the product of the two cells' masks, closed at the last
    column / row when that boundary is closed."""
    m = np.asarray(mask, dtype=np.float64)
    mask_u = m * np.roll(m, -1, axis=1)
    mask_v = m * np.roll(m, -1, axis=0)
    if bc_x != "periodic":
        mask_u[:, -1] = 0.0
    if bc_y != "periodic":
        mask_v[-1, :] = 0.0
    return mask_u, mask_v


def uniform_levels(H, mask, nz: int) -> np.ndarray:
    """The whole domain's uniform level table max(H over wet cells) / nz."""
    hmax = float(np.max(np.asarray(H)[np.asarray(mask) > 0]))
    return np.full(nz, hmax / nz)


def _dist():
    import torch.distributed as dist
    return dist if dist.is_available() and dist.is_initialized() else None


class FbSlabRun:
    """This rank's slab of a y-slab run of the fb scheme.

    Every rank constructs it with the whole domain's inputs; ``rank`` and
    ``nranks`` default to the torch.distributed process group (one rank when
    there is none). ``set_state`` takes the whole domain's state, ``step`` runs
    steps with a halo refresh after each, ``gather_state`` returns the whole
    domain's state on rank 0 (None elsewhere)."""

    def __init__(self, params: OceanParams, H, mask, dzr=None, taux_c=None, tauy_c=None, *,
                 halo: int = DEFAULT_HALO, rank: int | None = None, nranks: int | None = None,
                 device: int = 0, stepper_factory=None, torch_device=None):
        """``stepper_factory(params, H, mask, dzr, taux_c, tauy_c, device, slab)`` builds
        the slab's stepper (default ``OceanStepper``); ``torch_device`` holds the halo
        buffers (default the CUDA device)."""
        import torch
        from .stepper import OceanStepper
        if params.scheme_name != "fb":
            raise ValueError(f"the slab run supports scheme fb only (got {params.scheme_name}): theta "
                             "needs a global elliptic solve and split_explicit a halo per substep")
        dist = _dist()
        self.dist = dist
        self.rank = rank if rank is not None else (dist.get_rank() if dist else 0)
        self.nranks = nranks if nranks is not None else (dist.get_world_size() if dist else 1)
        self.layout = SlabLayout(params.ny, self.nranks, halo)
        self.halo = halo
        self.p = params
        self.j0, self.ny_loc = self.layout.owned(self.rank)
        self.rows = self.layout.rows(self.rank)
        H = np.asarray(H, dtype=np.float64)
        mask = np.asarray(mask, dtype=np.float64)
        dzr = uniform_levels(H, mask, params.nz) if dzr is None else np.asarray(dzr, dtype=np.float64)
        mask_u, mask_v = face_masks(mask, params.bc_x, params.bc_y)
        r = self.rows
        cut = lambda a: None if a is None else np.ascontiguousarray(np.asarray(a, np.float64)[r, :])  # noqa: E731
        self.device = device
        make = stepper_factory or (lambda *a, **k: OceanStepper(*a, **k))
        self.stepper = make(params.replace(ny=len(r)), cut(H), cut(mask), dzr=dzr, taux_c=cut(taux_c),
                            tauy_c=cut(tauy_c), device=device,
                            slab=(cut(mask_u), cut(mask_v), params.lx / params.nx, params.ly / params.ny))
        n = self.stepper.halo_values_per_row() * halo
        self.tdev = torch.device("cuda", device) if torch_device is None else torch.device(torch_device)
        self.send_lo, self.send_hi, self.recv_lo, self.recv_hi = (
            torch.empty(n, dtype=torch.float64, device=self.tdev) for _ in range(4))
        self.exchanges = 0

    # ------------------------------------------------------------------ state
    def _cut(self, a):
        if a is None:
            return None
        a = np.asarray(a, dtype=np.float64)
        return np.ascontiguousarray(a[..., self.rows, :])

    def set_state(self, eta, u, v, b=None, T=None, S=None, e=None, km=None, kh=None):
        """The whole domain's state; this rank keeps its stored rows."""
        self.stepper.set_state(eta=self._cut(eta), u=self._cut(u), v=self._cut(v), b=self._cut(b),
                               T=self._cut(T), S=self._cut(S), e=self._cut(e), km=self._cut(km),
                               kh=self._cut(kh))

    def reset_mixing(self):
        """The configuration's constant viscosity and diffusivity again (oc_reset_mixing)."""
        self.stepper.reset_mixing()

    def owned_state(self) -> dict:
        """This rank's owned rows of every state field (host arrays)."""
        full = self.stepper.get_state()
        h, n = self.halo, self.ny_loc
        return {k: np.ascontiguousarray(a[..., h:h + n, :]) for k, a in full.items()}

    def gather_state(self) -> dict | None:
        """The whole domain's state on rank 0 (None on the other ranks)."""
        mine = (self.j0, self.owned_state())
        if self.dist is None or self.nranks == 1:
            parts = [mine]
        else:
            parts = [None] * self.nranks if self.rank == 0 else None
            self.dist.gather_object(mine, parts, dst=0)
        if self.rank != 0:
            return None
        out = {}
        for j0, st in parts:
            for k, a in st.items():
                if k not in out:
                    shape = a.shape[:-2] + (self.p.ny, self.p.nx)
                    out[k] = np.empty(shape)
                out[k][..., j0:j0 + a.shape[-2], :] = a
        return out

    # ------------------------------------------------------------------ steps
    def exchange(self):
        """Refresh both halos from the neighbours' owned rows
        (cfd_exp3d5_cuda_multi.cu:133-172): the low halo takes the previous
        rank's last owned rows, the high halo the next rank's first ones."""
        st = self.stepper
        h, n = self.halo, self.ny_loc
        stream = self._stream()
        st.pack_rows(h, h, self.send_lo, stream)      # my first owned rows -> previous rank
        st.pack_rows(n, h, self.send_hi, stream)      # my last owned rows -> next rank
        if self.nranks == 1:
            self.recv_lo.copy_(self.send_hi)
            self.recv_hi.copy_(self.send_lo)
        else:
            self._swap()
        st.unpack_rows(0, h, self.recv_lo, stream)
        st.unpack_rows(h + n, h, self.recv_hi, stream)
        self.exchanges += 1

    def _swap(self):
        """One batch of point-to-point transfers with both neighbours. Sends go
        to the previous rank then the next, receives come from the next rank
        then the previous: with two ranks both neighbours are the same rank and
        the transfers pair up in this order."""
        import torch
        dist = self.dist
        prev, nxt = (self.rank - 1) % self.nranks, (self.rank + 1) % self.nranks
        if dist.get_backend() == "nccl" or self.tdev.type == "cpu":
            bufs = (self.send_lo, self.send_hi, self.recv_hi, self.recv_lo)
        else:  # gloo moves host tensors
            torch.cuda.current_stream(self.device).synchronize()
            bufs = (self.send_lo.cpu(), self.send_hi.cpu(), torch.empty_like(self.recv_hi, device="cpu"),
                    torch.empty_like(self.recv_lo, device="cpu"))
        ops = [dist.P2POp(dist.isend, bufs[0], prev), dist.P2POp(dist.isend, bufs[1], nxt),
               dist.P2POp(dist.irecv, bufs[2], nxt), dist.P2POp(dist.irecv, bufs[3], prev)]
        for w in dist.batch_isend_irecv(ops):
            w.wait()
        if bufs[2] is not self.recv_hi:
            self.recv_hi.copy_(bufs[2])
            self.recv_lo.copy_(bufs[3])

    def _stream(self):
        import torch
        return torch.cuda.current_stream(self.device) if self.tdev.type == "cuda" else None

    def step(self, n_steps: int = 1):
        stream = self._stream()
        for _ in range(n_steps):
            self.stepper.step(1, stream)
            self.exchange()

    def stats(self) -> dict:
        return self.stepper.stats()

    def close(self):
        self.stepper.close()


# ---------------------------------------------------------------------- front end
def _read_bundle(p: OceanParams):
    """The whole domain's inputs named by the namelist: H, mask, the initial state
    (the init file has the state file's layout), levels and forcing if given."""
    from .bundle import read_domain, read_state
    nx, ny, nz = p.nx, p.ny, p.nz
    n2 = nx * ny
    H, mask = read_domain(p.domain_file, nx, ny)
    state = read_state(p.init_file, nx, ny, nz, p.tracers == "TS")
    dzr = None
    if getattr(p, "levels_file", ""):
        dzr = np.fromfile(p.levels_file, dtype=np.float64)
    taux = tauy = None
    if getattr(p, "forcing_file", ""):
        f = np.fromfile(p.forcing_file, dtype=np.float64)
        taux, tauy = f[:n2].reshape(ny, nx), f[n2:2 * n2].reshape(ny, nx)
    return H, mask, state, dzr, taux, tauy


def run_namelist(nml: str, halo: int = DEFAULT_HALO, devices: list[int] | None = None) -> int:
    """The multi-device binary's protocol (cfd_exp3d5_cuda_multi.cu:58-265) for the
    rank this process is; rank 0 writes the state and metrics files. ``devices``:
    the device of each rank (default: the launcher's local rank)."""
    p = read_namelist(nml)
    dist = _dist()
    rank = dist.get_rank() if dist else 0
    nranks = dist.get_world_size() if dist else 1
    # what the run refuses, before any device work (cfd_exp3d5_cuda_multi.cu:73-76)
    if p.scheme_name != "fb":
        raise ValueError(f"the multi-device run supports scheme fb only (got {p.scheme_name})")
    SlabLayout(p.ny, nranks, halo)
    if devices is not None and len(devices) != nranks:
        raise ValueError(f"--devices lists {len(devices)} devices for {nranks} ranks")
    import torch
    if devices is not None:
        device = devices[rank]
        if not 0 <= device < torch.cuda.device_count():
            raise ValueError(f"device {device} does not exist ({torch.cuda.device_count()} visible)")
    else:
        device = int(os.environ.get("LOCAL_RANK", 0)) if torch.cuda.device_count() > 1 else 0
    torch.cuda.set_device(device)
    H, mask, state, dzr, taux, tauy = _read_bundle(p)
    run = FbSlabRun(p, H, mask, dzr, taux, tauy, halo=halo, device=device)
    samples, diverged = [], False

    def one_repeat():
        nonlocal diverged
        run.reset_mixing()
        run.set_state(**state)
        for s in range(p.n_steps):
            run.step(1)
            if s % 10 == 9:
                eta = run.owned_state()["eta"]
                bad = not (np.max(np.abs(eta)) < 1.0e6)
                flag = torch.tensor([1.0 if bad else 0.0])
                if dist:
                    dist.all_reduce(flag, op=dist.ReduceOp.MAX)
                if flag.item() > 0:
                    diverged = True
                    return

    for _ in range(p.n_warmup):
        one_repeat()
        if diverged:
            break
    for _ in range(p.n_repeat if not diverged else 0):
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        one_repeat()
        torch.cuda.synchronize()
        dt = torch.tensor([time.perf_counter() - t0])
        if dist:
            dist.all_reduce(dt, op=dist.ReduceOp.MAX)   # the slowest rank's time
        samples.append(float(dt.item()))
        if diverged:
            break
    out = run.gather_state()
    if rank == 0:
        ts = p.tracers == "TS"
        with open(f"{p.out_prefix}_state3d5.bin", "wb") as fh:
            for k in ["eta", "u", "v", "b"] + (["T", "S"] if ts else []):
                fh.write(np.ascontiguousarray(out[k], dtype=np.float64).tobytes())
        med = statistics.median(samples) if samples else float("nan")
        mad = statistics.median([abs(x - med) for x in samples]) if samples else float("nan")
        metrics = {"backend": "cuda_b200_slabs", "gpu": torch.cuda.get_device_name(device),
                   "n_devices": nranks, "halo": halo, "nx": p.nx, "ny": p.ny, "nz": p.nz,
                   "cells": p.nx * p.ny * p.nz, "n_steps": p.n_steps, "scheme": p.scheme_name,
                   "solver": p.solver_kind, "eos": p.eos, "advection": p.advection, "tracers": p.tracers,
                   "closure": p.closure, "dt": p.dt,
                   "device_bytes": int(run.stats()["device_bytes"]) * nranks,
                   "diverged": diverged, "wall_s": med, "wall_mad_s": mad, "n_repeat": len(samples),
                   "omp_num_threads": 0}
        Path(f"{p.out_prefix}_metrics.json").write_text(json.dumps(metrics, indent=2) + "\n")
    run.close()
    return 3 if diverged else 0


def parse_devices(text: str) -> list[int]:
    """``--devices 0,1,..`` (cfd_exp3d5_cuda_multi.cu:67): distinct non-negative ids."""
    try:
        ids = [int(t) for t in text.split(",")]
    except ValueError:
        raise ValueError(f"--devices takes a comma-separated list of device ids (got {text!r})") from None
    if min(ids) < 0 or len(set(ids)) != len(ids):
        raise ValueError(f"--devices must list distinct non-negative ids (got {text!r})")
    return ids


def _free_port() -> int:
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def _spawned_rank(rank: int, world: int, port: int, argv: list[str]) -> None:
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), LOCAL_WORLD_SIZE=str(world),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    rc = main(argv)
    if rc:
        sys.exit(rc)


def _spawn(ndev: int, argv: list[str]) -> int:
    """Start the ranks of one run on this node, as the reference binary does for --ndev."""
    import torch.multiprocessing as mp
    try:
        mp.spawn(_spawned_rank, args=(ndev, _free_port(), argv), nprocs=ndev, join=True)
    except mp.ProcessExitedException as e:
        return e.exit_code if e.exit_code and e.exit_code > 0 else 1
    except mp.ProcessRaisedException:
        return 1
    return 0


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description="y-slab multi-GPU run of the fb scheme (one rank per GPU)")
    ap.add_argument("namelist")
    ap.add_argument("--halo", type=int, default=DEFAULT_HALO)
    ap.add_argument("--ndev", type=int, default=None,
                    help="number of ranks; without a launcher, this process starts them")
    ap.add_argument("--devices", default=None, help="device of each rank, e.g. 0,1,2,3")
    args = ap.parse_args(argv)
    argv = list(sys.argv[1:] if argv is None else argv)
    # the command line's refusals, before any rendezvous or device work
    try:
        devices = parse_devices(args.devices) if args.devices is not None else None
        ndev = args.ndev if args.ndev is not None else (len(devices) if devices else None)
        if ndev is not None and ndev < 1:
            raise ValueError(f"--ndev must be >= 1 (got {ndev})")
        if devices is not None and ndev != len(devices):
            raise ValueError(f"--ndev {ndev} and --devices {args.devices} disagree")
        launched = "WORLD_SIZE" in os.environ
        if launched and ndev is not None and ndev != int(os.environ["WORLD_SIZE"]):
            raise ValueError(f"--ndev {ndev}, but the launcher started {os.environ['WORLD_SIZE']} ranks")
    except ValueError as e:
        print(f"FATAL: {e}", file=sys.stderr, flush=True)
        return 2
    if not launched and ndev is not None and ndev > 1:
        return _spawn(ndev, argv)
    import torch
    import torch.distributed as dist
    if "WORLD_SIZE" in os.environ and not dist.is_initialized():
        import datetime
        backend = "nccl" if torch.cuda.device_count() >= int(os.environ["WORLD_SIZE"]) else "gloo"
        # a rank that dies ends the others' next exchange with an error, not a hang
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    try:
        rc = run_namelist(args.namelist, args.halo, devices)
    except ValueError as e:
        print(f"FATAL: {e}", file=sys.stderr, flush=True)
        rc = 2
    if dist.is_initialized():
        dist.destroy_process_group()
    return rc


if __name__ == "__main__":
    raise SystemExit(main())
