"""NumPy statement of the mixed-precision Helmholtz solve (test infrastructure).

The solver behind ``OC_SOLVER_PCG_REFINED`` (csrc/helm_refined.cu) has no
reference counterpart: this model states its algorithm with the same FP32
arithmetic, so the tests can check the library's iteration counts against it,
and its answer against the FP64 oracle (``oracle.ocean_oracle.HelmOp``, the
reference's operator, libs/core/solvers_var.py:22-60).

  x = 0, r = b = rhs * mask                         FP64
  while |r|_2 > rtol |b|_2:
      PCG-Jacobi on A d = r from d = 0 in FP32,     FP32 operator and vectors,
          until |r - A d|_2 <= inner_rtol |r|_2     dot products summed in FP64
      x += d;  r = b - A x                          FP64

The FP32 operator is diag p - (ax_e p_e + ax_w p_w + ay_n p_n + ay_s p_s) with
ax = c Ku / dx^2, ay = c Kv / dy^2 and diag = 1 + ax + ax_w + ay + ay_s, the
identity on dry cells; each FP32 expression is evaluated in the kernel's order.
"""

from __future__ import annotations

import numpy as np

F = np.float32


def _e(a):
    return np.roll(a, -1, axis=-1)


def _w(a):
    return np.roll(a, 1, axis=-1)


def _n(a):
    return np.roll(a, -1, axis=-2)


def _s(a):
    return np.roll(a, 1, axis=-2)


def refine(op, rhs, rtol, max_iter, inner_rtol=1e-3, max_outer=64):
    """Solve ``op`` x = rhs; returns (x, inner iterations, converged,
    refinement steps, FP64 relative residual)."""
    ax, ay = (op.cx * op.Ku).astype(F), (op.cy * op.Kv).astype(F)
    d64 = 1.0 + op.cx * (op.Ku + _w(op.Ku)) + op.cy * (op.Kv + _s(op.Kv))
    wet = op.mask > 0
    diag = d64.astype(F)
    dinv = np.where(wet, 1.0 / np.where(wet, d64, 1.0), 1.0).astype(F)

    def a32(p):
        off = ax * _e(p) + _w(ax) * _w(p) + ay * _n(p) + _s(ay) * _s(p)
        return np.where(wet, diag * p - off, p).astype(F)

    def dot(a, b):
        return float(np.sum(a.astype(np.float64) * b.astype(np.float64)))

    b = rhs * op.mask
    norm_b = float(np.sqrt(np.sum(b * b)))
    x = np.zeros_like(b)
    if norm_b == 0.0:
        return x, 0, True, 0, 0.0
    tol = rtol * norm_b
    r, res, inner, outer = b.copy(), norm_b, 0, 0
    while True:
        if res <= tol:
            return x, inner, True, outer, res / norm_b
        if inner >= max_iter or outer >= max_outer:
            return x, inner, False, outer, res / norm_b
        outer += 1
        rr = r.astype(F)
        z = (dinv * rr).astype(F)
        p, d = z.copy(), np.zeros_like(rr)
        rz, itol = dot(rr, z), inner_rtol * res
        while True:
            ap = a32(p)
            pap = dot(p, ap)
            if not pap > 0.0:
                break
            alpha = F(rz / pap)
            d = (d + alpha * p).astype(F)
            rr = (rr - alpha * ap).astype(F)
            z = (dinv * rr).astype(F)
            inner += 1
            if np.sqrt(dot(rr, rr)) <= itol or inner >= max_iter:
                break
            rz_new = dot(rr, z)
            p = (z + F(rz_new / rz) * p).astype(F)
            rz = rz_new
        x = x + d.astype(np.float64)
        r = b - op.apply(x)
        res = float(np.sqrt(np.sum(r * r)))
