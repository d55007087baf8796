"""Gradients of a run of the fp64 step through its hand-written adjoint.

``OceanRollout`` advances a model state n steps on the GPU keeping a
checkpoint every ``every`` steps; its ``backward`` recomputes each segment's
states from the segment's checkpoint and walks the segment backwards with
``oc_adjoint_step`` (the transpose of the step's Jacobian, csrc/adjoint.cu).
``rollout_apply`` wraps the pair in a ``torch.autograd.Function`` whose inputs
are the initial temperature and the surface x-stress field at cell centres,
so any torch objective of the final state differentiates with respect to them.

Covered: the theta scheme with TS tracers, the closure off (constant
viscosity and diffusivity) and pgf keep; other configurations are refused by
the C ABI. No reference counterpart: the reference has no adjoint.
"""

from __future__ import annotations

import ctypes as C
import time

import numpy as np

from . import _lib
from .stepper import OceanStepper

STATE = ("eta", "u", "v", "b", "T", "S")


class OceanRollout:
    """n fp64 steps from a state on the GPU, with checkpoints every `every` steps."""

    def __init__(self, params, H, mask, dzr=None, n_steps: int = 20, every: int = 5, device: int = 0):
        self.p = params
        self.n, self.every = int(n_steps), max(1, int(every))
        self.st = OceanStepper(params, H, mask, dzr=dzr, device=device)
        self.lib = self.st.lib
        self.device = device
        self.timing = {}

    def close(self):
        self.st.close()

    def _new(self, like: dict) -> dict:
        import torch
        return {k: torch.empty_like(v) for k, v in like.items()}

    def _shapes(self):
        st = self.st
        return {"eta": st.shape2, "u": st.shape3, "v": st.shape3, "b": st.shape3, "T": st.shape3, "S": st.shape3}

    def _zeros(self) -> dict:
        import torch
        dev = f"cuda:{self.device}"
        return {k: torch.zeros(s, dtype=torch.float64, device=dev) for k, s in self._shapes().items()}

    def _set_forcing(self, taux):
        t = taux.detach().cpu().numpy()
        self.st.set_forcing(t, np.zeros_like(t))

    def _stream(self):
        import torch
        return torch.cuda.current_stream(self.device)

    def _fetch(self) -> dict:
        """The current state into new tensors, enqueued on the current stream."""
        out = {k: v for k, v in zip(STATE, self._empty())}
        self.st.get_state_async(self._stream(), out)
        return out

    def _empty(self):
        import torch
        dev = f"cuda:{self.device}"
        return [torch.empty(s, dtype=torch.float64, device=dev) for s in self._shapes().values()]

    def _segment(self, state: dict, n: int) -> list:
        """The n states after `state` (which carries its b), one per step."""
        st = self.st
        st.set_state(eta=state["eta"], u=state["u"], v=state["v"], b=state["b"], T=state["T"], S=state["S"])
        out = []
        for _ in range(n):
            st.step(1, stream=self._stream())
            out.append(self._fetch())
        return out

    def forward(self, state0: dict, taux) -> dict:
        """state0: eta, u, v, T, S (device tensors; b is diagnosed from T and S).
        The steps run back to back; the state is fetched at the checkpoints only."""
        import torch
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        self._set_forcing(taux)
        st = self.st
        st.set_state(eta=state0["eta"], u=state0["u"], v=state0["v"], T=state0["T"], S=state0["S"])
        cur = self._zeros()
        st.get_state(out=cur, fields=STATE)
        self.checkpoints = {0: cur}
        done = 0
        while done < self.n:
            m = min(self.every, self.n - done)
            st.step(m, stream=self._stream())
            done += m
            cur = self._fetch()
            if done < self.n:
                self.checkpoints[done] = cur
        torch.cuda.synchronize()
        self.timing["forward_s"] = time.perf_counter() - t0
        return cur

    def _adjoint_step(self, x0: dict, x1: dict, x1_b: dict, taux_b):
        x0_b = self._zeros()
        views = []
        for d in (x0, x1, x1_b, x0_b):
            v, _, keep = self.st._view(d, self._shapes(), writable=False)
            views.append((v, keep))
        _lib.check(self.lib.oc_adjoint_step(self.st.h, C.byref(views[0][0]), C.byref(views[1][0]),
                                            C.byref(views[2][0]), C.byref(views[3][0]), taux_b.data_ptr(), None,
                                            None), self.st.h, "oc_adjoint_step")
        return x0_b

    def backward(self, final_b: dict, taux):
        """Cotangents of the initial state (eta, u, v, T, S; the initial b's
        cotangent already folded into T and S through the EOS) and of the
        x-stress field, given the cotangents of the final state."""
        import torch
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        self._set_forcing(taux)
        taux_b = torch.zeros(self.st.shape2, dtype=torch.float64, device=f"cuda:{self.device}")
        cot = {k: final_b[k].contiguous() if k in final_b and final_b[k] is not None else None for k in STATE}
        zeros = self._zeros()
        cot = {k: (v if v is not None else zeros[k]) for k, v in cot.items()}
        starts = sorted(self.checkpoints)
        for si in range(len(starts) - 1, -1, -1):
            s0 = starts[si]
            s1 = starts[si + 1] if si + 1 < len(starts) else self.n
            states = [self.checkpoints[s0]] + self._segment(self.checkpoints[s0], s1 - s0)
            for t in range(s1 - s0 - 1, -1, -1):
                cot = self._adjoint_step(states[t], states[t + 1], cot, taux_b)
            del states
        # the initial b was diagnosed from T and S by the EOS
        x0 = self.checkpoints[0]
        _lib.check(self.lib.oc_adjoint_eos(self.st.h, x0["T"].data_ptr(), x0["S"].data_ptr(), cot["b"].data_ptr(),
                                           cot["T"].data_ptr(), cot["S"].data_ptr(), None), self.st.h,
                   "oc_adjoint_eos")
        torch.cuda.synchronize()
        self.timing["backward_s"] = time.perf_counter() - t0
        return cot, taux_b


def rollout_apply(rollout: OceanRollout, T0, taux, fixed: dict):
    """Final state (eta, u, v, b, T, S) of `rollout` from the initial state
    `fixed` (eta, u, v, S) with temperature T0, under the x-stress field taux,
    differentiable with respect to T0 and taux."""
    import torch

    class _Rollout(torch.autograd.Function):
        @staticmethod
        def forward(ctx, T0_, taux_):
            state0 = {"eta": fixed["eta"], "u": fixed["u"], "v": fixed["v"], "T": T0_.detach().contiguous(),
                      "S": fixed["S"]}
            out = rollout.forward(state0, taux_.detach())
            ctx.save_for_backward(taux_)
            return tuple(out[k] for k in STATE)

        @staticmethod
        def backward(ctx, *grads):
            (taux_,) = ctx.saved_tensors
            fb = {k: g for k, g in zip(STATE, grads)}
            cot, taux_b = rollout.backward(fb, taux_.detach())
            return cot["T"], taux_b

    return dict(zip(STATE, _Rollout.apply(T0, taux)))
