"""Host-side mirror of the reference's stepper interface, over the C ABI.

``OceanStepper`` is the device-level API: one handle, state kept in HBM,
``step(n)`` enqueues n steps on a CUDA stream. Arrays crossing the boundary
are NumPy arrays (host, copied with cudaMemcpy) or contiguous fp64 CUDA
tensors (device pointers, copied device to device).

``Stepper3DV05`` reproduces the reference class of the same name
(``libs/core/model3d_v05.py:78-545``): constructed from ``(domain, physics,
params, dt)`` -- the reference's own objects or this package's mirrors, by
attribute -- with ``step(state)`` / ``integrate(state, n)`` returning a new
state and the counters ``solver_iterations``, ``solver_failures``,
``solver_rebuilds``, ``tridiagonal_solves``, ``barotropic_substeps``.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from .params import OceanParams, params_from_reference

FIELDS3 = ("u", "v", "b", "T", "S")
FIELDSI = ("e", "km", "kh")


def _is_tensor(a) -> bool:
    return type(a).__module__.startswith("torch")


class OceanStepper:
    """One model instance on one GPU."""

    def __init__(self, params: OceanParams, H, mask, dzr=None, taux_c=None, tauy_c=None,
                 device: int = 0, slab=None, precision: str = "fp64"):
        """``slab``: for one y-slab of a larger domain (fb scheme, multi-GPU), the
        tuple (mask_u, mask_v, dx, dy) of the larger domain -- its face masks at
        this handle's rows and its spacing (oc_set_domain_slab); dzr is then
        required and is the larger domain's level table.

        ``precision``: "fp64" (bit-identical to the reference) or "mixed" (the 3D
        state and stencils in FP32; b, the pressure gradient, the EOS, eta and the
        Helmholtz solve in fp64). States go in and come out as float64 either way."""
        self.lib = _lib.load()
        self.p = params
        self.precision = precision
        cfg = _lib.config_from_params(params, device, precision)
        h = C.c_void_p()
        _lib.check(self.lib.oc_create(C.byref(cfg), C.byref(h)), None, "oc_create")
        self.h = h
        self.shape2 = (params.ny, params.nx)
        self.shape3 = (params.nz, params.ny, params.nx)
        self.shapei = (params.nz + 1, params.ny, params.nx)
        Hh = np.ascontiguousarray(H, dtype=np.float64).reshape(self.shape2)
        mh = np.ascontiguousarray(mask, dtype=np.float64).reshape(self.shape2)
        dz = None if dzr is None else np.ascontiguousarray(dzr, dtype=np.float64).reshape(params.nz)
        self._keep = [Hh, mh, dz]
        if slab is None:
            self._call("oc_set_domain", self.lib.oc_set_domain, self.h, Hh.ctypes.data, mh.ctypes.data,
                       None if dz is None else dz.ctypes.data)
        else:
            mu, mv, dx, dy = slab
            mu = np.ascontiguousarray(mu, dtype=np.float64).reshape(self.shape2)
            mv = np.ascontiguousarray(mv, dtype=np.float64).reshape(self.shape2)
            self._keep += [mu, mv]
            self._call("oc_set_domain_slab", self.lib.oc_set_domain_slab, self.h, Hh.ctypes.data,
                       mh.ctypes.data, None if dz is None else dz.ctypes.data, mu.ctypes.data, mv.ctypes.data,
                       float(dx), float(dy))
        if taux_c is not None or tauy_c is not None:
            self.set_forcing(taux_c, tauy_c)

    # ------------------------------------------------------------------ plumbing
    def _call(self, what, fn, *args):
        _lib.check(fn(*args), self.h, what)

    def close(self):
        if getattr(self, "h", None):
            self.lib.oc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass

    def _view(self, arrays: dict, shapes: dict, writable: bool):
        """(OcStateView, on_device, keep-alive list) for numpy arrays or CUDA tensors."""
        view = _lib.OcStateView()
        keep = []
        on_device = None
        for name, a in arrays.items():
            if a is None:
                continue
            if _is_tensor(a):
                import torch
                if a.dtype != torch.float64 or not a.is_contiguous():
                    raise ValueError(f"{name}: tensors must be contiguous float64")
                if a.numel() != int(np.prod(shapes[name])):
                    raise ValueError(f"{name}: expected {shapes[name]} elements")
                dev = 1 if a.is_cuda else 0
                ptr = a.data_ptr()
            else:
                if writable:
                    if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and
                            a.flags.c_contiguous and a.flags.writeable):
                        raise ValueError(f"{name}: output arrays must be writable C-contiguous float64")
                    arr = a
                else:
                    arr = np.ascontiguousarray(a, dtype=np.float64)
                if arr.size != int(np.prod(shapes[name])):
                    raise ValueError(f"{name}: expected shape {shapes[name]}, got {arr.shape}")
                keep.append(arr)
                dev = 0
                ptr = arr.ctypes.data
            if on_device is None:
                on_device = dev
            elif on_device != dev:
                raise ValueError("mix of host and device arrays in one call")
            setattr(view, name, ptr)
        return view, (on_device or 0), keep

    def _shapes(self):
        s = {"eta": self.shape2}
        s.update({k: self.shape3 for k in FIELDS3})
        s.update({k: self.shapei for k in FIELDSI})
        return s

    # ------------------------------------------------------------------ API
    def set_forcing(self, taux_c=None, tauy_c=None):
        tx = None if taux_c is None else np.ascontiguousarray(taux_c, np.float64).reshape(self.shape2)
        ty = None if tauy_c is None else np.ascontiguousarray(tauy_c, np.float64).reshape(self.shape2)
        self._keep_forcing = [tx, ty]
        self._call("oc_set_forcing", self.lib.oc_set_forcing, self.h,
                   None if tx is None else tx.ctypes.data, None if ty is None else ty.ctypes.data)

    def set_state(self, eta, u, v, b=None, T=None, S=None, e=None, km=None, kh=None):
        view, dev, keep = self._view(dict(eta=eta, u=u, v=v, b=b, T=T, S=S, e=e, km=km, kh=kh),
                                     self._shapes(), writable=False)
        self._call("oc_set_state", self.lib.oc_set_state, self.h, C.byref(view), dev)

    def set_state_async(self, stream, eta, u, v, b=None, T=None, S=None, e=None, km=None, kh=None):
        """Enqueue the state copies on `stream` without waiting (oc_set_state_async).
        Inputs must be contiguous float64 tensors (pinned host or CUDA) or C-contiguous
        float64 arrays that stay alive and unchanged until the stream passes the copies."""
        arrays = dict(eta=eta, u=u, v=v, b=b, T=T, S=S, e=e, km=km, kh=kh)
        for name, a in arrays.items():
            if a is not None and not _is_tensor(a) and not (
                    isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous):
                raise ValueError(f"{name}: asynchronous inputs must be contiguous float64")
        view, dev, keep = self._view(arrays, self._shapes(), writable=False)
        sp = getattr(stream, "cuda_stream", stream)
        self._call("oc_set_state_async", self.lib.oc_set_state_async, self.h, C.byref(view), dev, sp)

    def bind_state(self, current: dict | None, other: dict | None = None):
        """Make caller-owned CUDA tensors the state, without a copy (oc_bind_state).

        ``current`` holds the state to start from (eta, u, v, b and, with TS
        tracers, T and S; optionally e, km, kh, used in place); ``other`` names
        tensors of the same fields (without e, km, kh) that the step writes
        into. The state alternates between the two sets, one step each:
        ``state_parity()`` says which holds it. The stepper keeps both sets
        alive until the next bind_state; ``bind_state(None)`` returns to the
        handle's own buffers (set the state again after it)."""
        if current is None:
            if other is not None:
                raise ValueError("give both sets, or neither")
            self._call("oc_bind_state", self.lib.oc_bind_state, self.h, None, None)
            self._bound = None
            return
        if other is None:
            raise ValueError("bind_state needs the second set the step writes into")
        for name, a in list(current.items()) + list(other.items()):
            if a is not None and not (_is_tensor(a) and a.is_cuda):
                raise ValueError(f"{name}: bound buffers must be CUDA tensors")
        if any(other.get(k) is not None for k in FIELDSI):
            raise ValueError("e, km and kh are bound once, in the current set")
        va, _, _ = self._view(current, self._shapes(), writable=True)
        vb, _, _ = self._view(other, self._shapes(), writable=True)
        self._call("oc_bind_state", self.lib.oc_bind_state, self.h, C.byref(va), C.byref(vb))
        self._bound = (dict(current), dict(other))

    def state_parity(self) -> int:
        """0 when the bound ``current`` set holds the state, 1 when ``other`` does."""
        w = C.c_int32()
        self._call("oc_state_parity", self.lib.oc_state_parity, self.h, C.byref(w))
        return int(w.value)

    def bound_state(self) -> dict:
        """The bound tensors that hold the current state (no copy; read after the
        stream has passed the steps)."""
        if not getattr(self, "_bound", None):
            raise RuntimeError("no state is bound")
        cur, oth = self._bound
        src = oth if self.state_parity() else cur
        out = {k: v for k, v in src.items() if v is not None and k not in FIELDSI}
        out.update({k: v for k, v in cur.items() if v is not None and k in FIELDSI})
        return out

    def get_state_async(self, stream, out: dict):
        """Enqueue the copies of the current state into ``out`` on `stream` without
        waiting (oc_get_state_async); ``out`` is complete once the stream passes them."""
        view, dev, keep = self._view(out, self._shapes(), writable=True)
        sp = getattr(stream, "cuda_stream", stream)
        self._call("oc_get_state_async", self.lib.oc_get_state_async, self.h, C.byref(view), dev, sp)

    # ------------------------------------------------------------------ tiling
    def set_tiling(self, mom_levels: int, tracer_levels: int):
        """Levels one CTA marches in the momentum / tracer kernels (oc_set_tiling)."""
        self._call("oc_set_tiling", self.lib.oc_set_tiling, self.h, int(mom_levels), int(tracer_levels))

    def autotune(self) -> tuple[int, int]:
        """Time the candidates on the current state and keep the fastest (oc_autotune)."""
        mk, tk = C.c_int32(), C.c_int32()
        self._call("oc_autotune", self.lib.oc_autotune, self.h, C.byref(mk), C.byref(tk))
        return int(mk.value), int(tk.value)

    # ------------------------------------------------------------------ slab halos
    def halo_values_per_row(self) -> int:
        """Doubles one row of all exchanged fields takes (oc_halo_values_per_row)."""
        n = C.c_int64()
        self._call("oc_halo_values_per_row", self.lib.oc_halo_values_per_row, self.h, C.byref(n))
        return int(n.value)

    def _rows_buffer(self, buf, nrows: int):
        import torch
        if not (_is_tensor(buf) and buf.is_cuda and buf.dtype == torch.float64 and buf.is_contiguous()):
            raise ValueError("row buffers must be contiguous float64 CUDA tensors")
        if buf.numel() < self.halo_values_per_row() * nrows:
            raise ValueError("row buffer too small")
        return buf.data_ptr()

    def pack_rows(self, j0: int, nrows: int, buf, stream=None):
        """Rows [j0, j0 + nrows) of every exchanged field into ``buf`` (oc_pack_rows)."""
        ptr = self._rows_buffer(buf, nrows)
        sp = getattr(stream, "cuda_stream", stream)
        self._call("oc_pack_rows", self.lib.oc_pack_rows, self.h, int(j0), int(nrows), ptr, sp)

    def unpack_rows(self, j0: int, nrows: int, buf, stream=None):
        """``buf`` into rows [j0, j0 + nrows) of every exchanged field (oc_unpack_rows)."""
        ptr = self._rows_buffer(buf, nrows)
        sp = getattr(stream, "cuda_stream", stream)
        self._call("oc_unpack_rows", self.lib.oc_unpack_rows, self.h, int(j0), int(nrows), ptr, sp)

    def set_wait_bound(self, cycles: int):
        """Bound of the solve's device-side waits in SM clock cycles (oc_set_wait_bound)."""
        self._call("oc_set_wait_bound", self.lib.oc_set_wait_bound, self.h, int(cycles))

    def reset_mixing(self):
        self._call("oc_reset_mixing", self.lib.oc_reset_mixing, self.h)

    def get_state(self, out: dict | None = None, fields=("eta", "u", "v", "b", "T", "S", "e",
                                                        "km", "kh")) -> dict:
        """Copy the state into ``out`` (arrays or tensors) or into new NumPy arrays."""
        shapes = self._shapes()
        if out is None:
            ts = self.p.tracers == "TS"
            out = {f: np.empty(shapes[f]) for f in fields if ts or f not in ("T", "S")}
        view, dev, keep = self._view(out, shapes, writable=True)
        self._call("oc_get_state", self.lib.oc_get_state, self.h, C.byref(view), dev)
        return out

    def step(self, n_steps: int = 1, stream=None, graph: bool = False):
        """Enqueue n_steps on `stream` (torch.cuda.Stream, raw cudaStream_t int, or None);
        graph=True replays recorded two-step CUDA graphs (oc_step_graph)."""
        sp = None
        if stream is not None:
            sp = getattr(stream, "cuda_stream", stream)
        if graph:
            self._call("oc_step_graph", self.lib.oc_step_graph, self.h, int(n_steps), sp)
        else:
            self._call("oc_step", self.lib.oc_step, self.h, int(n_steps), sp)

    def stats(self) -> dict:
        st = _lib.OcStats()
        self._call("oc_get_stats", self.lib.oc_get_stats, self.h, C.byref(st))
        return {name: getattr(st, name) for name, _ in st._fields_}

    def set_profiling(self, enable: bool = True):
        self._call("oc_set_profiling", self.lib.oc_set_profiling, self.h, 1 if enable else 0)

    def kernel_times(self) -> dict:
        """{kernel class: (launches, total device ms)} since the last call; synchronises."""
        buf = (_lib.OcKernelTime * 64)()
        n = C.c_int32()
        self._call("oc_get_kernel_times", self.lib.oc_get_kernel_times, self.h, buf, 64, C.byref(n))
        return {buf[i].name.decode(): (int(buf[i].launches), float(buf[i].total_ms))
                for i in range(min(n.value, 64))}

    def solve_log(self) -> list[int]:
        n = C.c_int32()
        self._call("oc_get_solve_log", self.lib.oc_get_solve_log, self.h, None, 0, C.byref(n))
        buf = np.zeros(max(1, n.value), dtype=np.int32)
        self._call("oc_get_solve_log", self.lib.oc_get_solve_log, self.h, buf.ctypes.data,
                   int(buf.size), C.byref(n))
        return [int(x) for x in buf[:n.value]]

    def reset_stats(self):
        self._call("oc_reset_stats", self.lib.oc_reset_stats, self.h)

    def field(self, name: str) -> np.ndarray:
        shapes = {"dz3": self.shape3, "mask3": self.shape3, "mask3u": self.shape3,
                  "mask3v": self.shape3, "dz3u": self.shape3, "dz3v": self.shape3,
                  "zc": self.shape3, "q": self.shape3, "ku": self.shape2, "kv": self.shape2,
                  "mask_u": self.shape2, "mask_v": self.shape2}
        out = np.empty(shapes[name])
        self._call("oc_get_field", self.lib.oc_get_field, self.h, name.encode(),
                   out.ctypes.data, int(out.size))
        return out

    def helmholtz_solve(self, rhs) -> tuple:
        """x = A^-1 rhs with the current face coefficients; (x, iterations)."""
        import torch
        r = torch.as_tensor(np.ascontiguousarray(rhs, np.float64).reshape(self.shape2),
                            device=f"cuda:{torch.cuda.current_device()}")
        x = torch.empty_like(r)
        its = C.c_int32()
        self._call("oc_helmholtz_solve", self.lib.oc_helmholtz_solve, self.h, r.data_ptr(),
                   x.data_ptr(), C.byref(its), None)
        return x.cpu().numpy(), int(its.value)

    def buoyancy(self, T, S, z):
        """b = -g rho'(T, S, z) / rho0 with the configured EOS, computed on the GPU."""
        import torch
        dev = f"cuda:{torch.cuda.current_device()}"
        t = torch.as_tensor(np.ascontiguousarray(T, np.float64), device=dev)
        s = torch.as_tensor(np.ascontiguousarray(S, np.float64), device=dev)
        zz = torch.as_tensor(np.ascontiguousarray(z, np.float64), device=dev)
        b = torch.empty_like(t)
        self._call("oc_buoyancy", self.lib.oc_buoyancy, self.h, t.data_ptr(), s.data_ptr(),
                   zz.data_ptr(), b.data_ptr(), int(t.numel()), None)
        return b.cpu().numpy()

    def integrate(self, state: dict, n_steps: int) -> dict:
        """Upload a host state, advance n_steps, return the host state."""
        self.set_state(**{k: state.get(k) for k in ("eta", "u", "v", "b", "T", "S", "e")})
        self.step(n_steps)
        return self.get_state()


def thomas(sub, diag, sup, rhs):
    """Batched tridiagonal solve on the GPU (reference vertical.py:17-44)."""
    import torch
    lib = _lib.load()
    dev = f"cuda:{torch.cuda.current_device()}"
    arrs = [torch.as_tensor(np.ascontiguousarray(a, np.float64), device=dev)
            for a in (sub, diag, sup, rhs)]
    n = arrs[0].shape[0]
    ncols = arrs[0].numel() // n
    x = torch.empty_like(arrs[3])
    rc = lib.oc_thomas(*(a.data_ptr() for a in arrs), x.data_ptr(), int(n), int(ncols), None)
    _lib.check(rc, None, "oc_thomas")
    return x.cpu().numpy()


# ---------------------------------------------------------------------------
# reference-shaped interface


class OceanEnsemble:
    """Members (``OceanStepper`` objects of any grid size, on one GPU, states set)
    advanced together by one recorded CUDA graph per two steps (oc_ensemble_*):
    every member on its own branch, the Helmholtz solves one after another.
    Each member's results equal those of the member stepped alone."""

    def __init__(self, members):
        self.lib = _lib.load()
        self.members = list(members)
        arr = (C.c_void_p * len(self.members))(*[m.h.value for m in self.members])
        e = C.c_void_p()
        rc = self.lib.oc_ensemble_create(arr, len(self.members), C.byref(e))
        if rc:
            raise _lib.OceanError(f"oc_ensemble_create failed ({rc})")
        self.e = e

    def step(self, n_steps: int = 1, stream=None):
        sp = getattr(stream, "cuda_stream", stream)
        rc = self.lib.oc_ensemble_step(self.e, int(n_steps), sp)
        if rc:
            msg = self.lib.oc_ensemble_last_error(self.e)
            raise _lib.OceanError(f"oc_ensemble_step failed ({rc}): {msg.decode() if msg else ''}")

    def close(self):
        if getattr(self, "e", None):
            self.lib.oc_ensemble_destroy(self.e)
            self.e = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass


@dataclass(frozen=True)
class State3D:
    """Prognostic state, field for field the reference's State3D (model3d.py:34-47)."""

    u: np.ndarray
    v: np.ndarray
    b: np.ndarray
    eta: np.ndarray
    t: float = 0.0
    T: np.ndarray | None = None
    S: np.ndarray | None = None
    e: np.ndarray | None = None


class Stepper3DV05:
    """Drop-in for the reference ``Stepper3DV05`` running on the B200 path.

    ``domain`` may carry ``dzr_levels`` (stretched level table) and
    ``physics`` may carry ``taux_field``/``tauy_field`` (surface stress at
    cell centres); without them the reference's uniform levels and scalar
    stress apply.
    """

    def __init__(self, domain, physics, params, dt, device: int = 0):
        self.p: OceanParams = params_from_reference(domain, physics, params, dt)
        self.p.validate()
        self.dt = float(dt)
        self.domain, self.physics, self.params = domain, physics, params
        self._dev = OceanStepper(self.p, domain.H, domain.mask,
                                 dzr=getattr(domain, "dzr_levels", None),
                                 taux_c=getattr(physics, "taux_field", None),
                                 tauy_c=getattr(physics, "tauy_field", None), device=device)
        self._last = None
        self.solver_iterations = 0
        self.solver_failures = 0
        self.solver_rebuilds = 0
        self.tridiagonal_solves = 1
        self.barotropic_substeps = 0
        self.n_split = self._dev.stats()["n_split"]

    def _sync_counters(self, st: dict):
        self.solver_iterations = int(st["solver_iterations"])
        self.solver_failures = int(st["solver_failures"])
        self.solver_rebuilds = int(st["solver_rebuilds"])
        self.tridiagonal_solves = int(st["tridiagonal_solves"])
        self.barotropic_substeps = int(st["barotropic_substeps"])

    def _upload(self, s):
        if self._last is not None and s is self._last:
            return
        ts = self.p.tracers == "TS"
        self._dev.set_state(eta=s.eta, u=s.u, v=s.v, b=s.b, T=s.T if ts else None,
                            S=s.S if ts else None, e=getattr(s, "e", None))

    def _download(self, s, n) -> State3D:
        out = self._dev.get_state()
        e = out.get("e") if self.p.closure == "tke" else getattr(s, "e", None)
        new = State3D(u=out["u"], v=out["v"], b=out["b"], eta=out["eta"],
                      t=float(getattr(s, "t", 0.0)) + n * self.dt, T=out.get("T"), S=out.get("S"),
                      e=e)
        self._sync_counters(self._dev.stats())
        self._last = new
        return new

    @property
    def nu(self) -> np.ndarray:
        """Current interface viscosity (the reference stepper's ``self.nu``)."""
        return self._dev.get_state(fields=("km",))["km"]

    @property
    def kappa(self) -> np.ndarray:
        return self._dev.get_state(fields=("kh",))["kh"]

    def step(self, s) -> State3D:
        self._upload(s)
        self._dev.step(1)
        return self._download(s, 1)

    def integrate(self, s, n_steps: int) -> State3D:
        self._upload(s)
        self._dev.step(int(n_steps))
        return self._download(s, n_steps)

    def solve_log(self) -> list[int]:
        return self._dev.solve_log()
