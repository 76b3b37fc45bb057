"""Differentiable rollouts: repeated (semi-Lagrangian advection -> projection)
with a hand-written adjoint and checkpointed recomputation.

    r = Rollout(mat, steps=16, checkpoint_every=4, dt_over_dx=c, box=...)
    loss = r.forward(u0, v0, w0)        # CUDA tensors, float64 or float32
    gu, gv, gw = r.backward()           # dL/d(u0, v0, w0)

Every step runs libxfp kernels only: ``xfp_advect_*`` then ``xfp_project_*``
forward; ``xfp_project_backward_*`` (g - D^T A^{-1} G^T g, a second MIC(0)-PCG
solve with the same matrix) then ``xfp_advect_backward_*`` in reverse.  The
forward pass keeps the state every ``checkpoint_every`` steps; the reverse
pass recomputes one segment at a time, so memory is steps/checkpoint_every +
checkpoint_every states instead of steps.  The loss is the sum of squared face
velocities inside a box of the unit cube (``xfp_box_loss_*``).

xFluid is not differentiable; this is an extension beside the drop-in.
"""
from __future__ import annotations

import ctypes as C

from . import _lib
from ._lib import Context, XfpStats


class Rollout:
    def __init__(self, mat, steps: int = 16, checkpoint_every: int = 4, dt_over_dx: float = 1.0,
                 box=((0.6, 0.9), (0.6, 0.9), (0.6, 0.9)), precision: str = "f64", tol: float = 1e-10,
                 max_iter: int = 5000, device: int = 0, weights=(None, None, None)):
        if steps < 1 or checkpoint_every < 1:
            raise ValueError("steps and checkpoint_every must be >= 1")
        o = _lib.default_options()
        o.precision = _lib.PREC[precision]
        o.tol, o.max_iter, o.device, o.device_pointers = tol, max_iter, device, 1
        # torch produces and consumes every tensor this class passes.  The
        # library runs on torch's current stream when that is a created stream;
        # torch's default stream has the handle NULL, which gives the context a
        # stream of its own that is not ordered after torch's work, so every
        # library call below first waits for torch's stream (_wait_torch).  Each
        # call returns only after its own kernels are done.
        o.stream = _lib.torch_stream(device)
        self.device = device
        self._ctx = Context(o)
        self.mat = mat
        self.nk, self.nj, self.ni = mat.shape
        self.steps, self.every, self.c = steps, checkpoint_every, float(dt_over_dx)
        self.box = (C.c_double * 6)(*[float(x) for pair in box for x in pair])
        self.weights = weights
        self._ck: dict = {}
        self._final = None
        self.iterations = {"forward": 0, "backward": 0}
        # |G^T g|_inf of every adjoint projection (the right-hand side of its
        # MIC(0)-PCG solve), in the order the reverse pass runs them: zero when
        # the loss's sensitivity has not reached a face next to fluid
        self.adjoint_rhs_inf: list[float] = []

    def close(self) -> None:
        self._ctx.close()

    # ---- one step, forward and adjoint ----
    def _fn(self, name, t):
        return getattr(self._ctx.lib, name + ("_f64" if str(t.dtype) == "torch.float64" else "_f32"))

    @staticmethod
    def _P(x):
        return None if x is None else C.c_void_p(x.data_ptr())

    def _wait_torch(self):
        _lib.sync_torch(self.device)

    def step(self, u, v, w):
        """advect then project; returns new tensors."""
        P = self._P
        ou, ov, ow = (a.clone() for a in (u, v, w))
        # the clones (torch) must land before the advection overwrites them
        self._wait_torch()
        self._ctx.check(self._fn("xfp_advect", u)(self._ctx.ptr, self.ni, self.nj, self.nk, P(u), P(v), P(w),
                                                  P(ou), P(ov), P(ow), self.c))
        st = XfpStats()
        rc = self._fn("xfp_project", u)(self._ctx.ptr, self.ni, self.nj, self.nk, P(self.mat), P(ou), P(ov), P(ow),
                                        *map(P, self.weights), None, C.byref(st))
        if self._ctx.check(rc) != _lib.XFP_OK:
            raise _lib.XfpError(rc, "projection did not converge")
        self.iterations["forward"] += st.iterations
        return ou, ov, ow

    def step_adjoint(self, state, g):
        """(J_advect^T P^T) g for the step taken from `state`."""
        P = self._P
        u, v, w = state
        pu, pv, pw = (torch_empty_like(a) for a in g)
        self._wait_torch()
        st = XfpStats()
        rc = self._fn("xfp_project_backward", u)(self._ctx.ptr, self.ni, self.nj, self.nk, P(self.mat),
                                                 *map(P, self.weights), P(g[0]), P(g[1]), P(g[2]), P(pu), P(pv),
                                                 P(pw), C.byref(st))
        if self._ctx.check(rc) != _lib.XFP_OK:
            raise _lib.XfpError(rc, "adjoint projection did not converge")
        self.iterations["backward"] += st.iterations
        self.adjoint_rhs_inf.append(float(st.b_inf))
        du, dv, dw = (torch_empty_like(a) for a in g)
        self._ctx.check(self._fn("xfp_advect_backward", u)(self._ctx.ptr, self.ni, self.nj, self.nk, P(u), P(v),
                                                           P(w), P(pu), P(pv), P(pw), P(du), P(dv), P(dw), self.c))
        return du, dv, dw

    def loss(self, u, v, w, grad: bool = False):
        P = self._P
        out = C.c_double(0.0)
        g = tuple(torch_empty_like(a) for a in (u, v, w)) if grad else (None, None, None)
        self._wait_torch()
        self._ctx.check(self._fn("xfp_box_loss", u)(self._ctx.ptr, self.ni, self.nj, self.nk, P(u), P(v), P(w),
                                                    self.box, C.byref(out), *map(P, g)))
        return (out.value, g) if grad else out.value

    # ---- rollout ----
    def forward(self, u0, v0, w0) -> float:
        self._ck = {}
        u, v, w = u0, v0, w0
        for n in range(self.steps):
            if n % self.every == 0:
                self._ck[n] = (u.clone(), v.clone(), w.clone())
            u, v, w = self.step(u, v, w)
        self._final = (u, v, w)
        return self.loss(u, v, w)

    def backward(self):
        if self._final is None:
            raise RuntimeError("forward() first")
        _, g = self.loss(*self._final, grad=True)
        self.adjoint_rhs_inf = []
        for s0 in sorted(self._ck, reverse=True):
            states = []
            u, v, w = self._ck[s0]
            for _ in range(s0, min(s0 + self.every, self.steps)):
                states.append((u, v, w))
                u, v, w = self.step(u, v, w)
            for st in reversed(states):
                g = self.step_adjoint(st, g)
        return g


def torch_empty_like(a):
    import torch
    return torch.empty_like(a)
