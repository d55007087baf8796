"""Host-side mirror of the reference's variable-coefficient Helmholtz solver.

``HelmholtzVar`` reproduces the reference class of the same name
(``libs/core/solvers_var.py:72-197``): constructed from a grid (any object with
``nx``, ``ny``, ``dx``, ``dy``, such as the reference's ``CGrid``), the coefficient
``coef = g theta^2 dt^2``, the depth-integrated face coefficients ``Ku``, ``Kv``
and an optional wet mask, with ``update(Ku, Kv)`` and ``solve(rhs)`` returning
``(x, SolveReport)``. The solve runs on the GPU through the standalone entry
points ``oc_helm_*`` (the step's own persistent solver, so iteration counts and
solutions are NumPy's bit for bit); there is no CPU path.

Differences from the reference class:
- ``kind`` also accepts ``"pcg_refined"``: FP32 inner PCG inside FP64 iterative
  refinement (no reference counterpart, no bit parity; same FP64 stopping test);
- the multigrid is V(2,2) coarsened down to 8 cells, the reference defaults;
  other ``n_pre``, ``n_post`` or ``min_size`` values are refused;
- ``SolveReport.residual`` is the relative residual for ``pcg_refined`` and for a
  zero right-hand side, and NaN otherwise: the FP64 solvers' C ABI does not
  report it (no caller in the reference reads it).
"""

from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from . import _lib

KINDS = {"pcg_jacobi": 0, "pcg_rbgs": 1, "rbgs": 2, "multigrid": 3, "pcg_refined": 4, "pcg_mg": 5}


@dataclass
class SolveReport:
    """Per-solve diagnostics (reference ``libs/core/solvers.py:25-30``)."""

    iterations: int = 0
    residual: float = 0.0
    converged: bool = True


class HelmholtzVar:
    """A = I - coef D[K G[.]] on one GPU; see the module docstring."""

    def __init__(self, grid, coef: float, Ku, Kv, mask=None, kind: str = "pcg_jacobi",
                 rtol: float = 1e-12, max_iter: int = 2000, n_pre: int = 2, n_post: int = 2,
                 min_size: int = 8, device: int = 0) -> None:
        if kind not in KINDS:
            raise ValueError(f"unknown variable-coefficient solver '{kind}' "
                             "(expected pcg_jacobi|pcg_rbgs|rbgs|multigrid|pcg_refined|pcg_mg)")
        if (n_pre, n_post, min_size) != (2, 2, 8):
            raise ValueError("the B200 multigrid is V(2,2) coarsened down to 8 cells "
                             "(n_pre=2, n_post=2, min_size=8)")
        self.kind, self.rtol, self.max_iter = kind, float(rtol), int(max_iter)
        self.grid, self.coef, self.device = grid, float(coef), int(device)
        self.nx, self.ny = int(grid.nx), int(grid.ny)
        self.dx, self.dy = float(grid.dx), float(grid.dy)
        shape = (self.ny, self.nx)
        self.mask = (np.ones(shape) if mask is None
                     else np.ascontiguousarray(mask, dtype=np.float64).reshape(shape))
        self.lib = _lib.load()
        self.h = None
        self.update(Ku, Kv)

    def update(self, Ku, Kv) -> None:
        """New face coefficients: the solver is built again (its multigrid levels
        included), as the reference rebuilds its operator."""
        shape = (self.ny, self.nx)
        ku = np.ascontiguousarray(Ku, dtype=np.float64).reshape(shape)
        kv = np.ascontiguousarray(Kv, dtype=np.float64).reshape(shape)
        cfg = _lib.OcHelmConfig(nx=self.nx, ny=self.ny, dx=self.dx, dy=self.dy, coef=self.coef,
                                solver=KINDS[self.kind], rtol=self.rtol, max_iter=self.max_iter,
                                device=self.device)
        h = C.c_void_p()
        rc = self.lib.oc_helm_create(C.byref(cfg), ku.ctypes.data, kv.ctypes.data, self.mask.ctypes.data,
                                     C.byref(h))
        if rc != _lib.OC_OK:
            raise _lib.OceanError(f"oc_helm_create: {_lib.ERRORS.get(rc, rc)}")
        self.close()
        self.h = h

    def _check(self, rc: int, what: str) -> None:
        if rc != _lib.OC_OK:
            msg = self.lib.oc_helm_last_error(self.h)
            raise _lib.OceanError(f"{what}: {_lib.ERRORS.get(rc, rc)}" + (f" ({msg.decode()})" if msg else ""))

    def solve(self, rhs) -> tuple[np.ndarray, SolveReport]:
        r = np.ascontiguousarray(rhs, dtype=np.float64).reshape(self.ny, self.nx)
        x = np.empty_like(r)
        its, conv = C.c_int32(), C.c_int32()
        self._check(self.lib.oc_helm_solve(self.h, r.ctypes.data, x.ctypes.data, 0, C.byref(its), C.byref(conv),
                                           None), "oc_helm_solve")
        residual = math.nan
        if self.kind == "pcg_refined":
            steps, rel = C.c_int32(), C.c_double()
            self._check(self.lib.oc_helm_refine_report(self.h, C.byref(steps), C.byref(rel)),
                        "oc_helm_refine_report")
            residual = rel.value
        elif its.value == 0 and conv.value:
            residual = 0.0  # a zero right-hand side, solved by x = 0
        return x, SolveReport(its.value, residual, bool(conv.value))

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.oc_helm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass
