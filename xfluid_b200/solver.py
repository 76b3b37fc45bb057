"""Python mirror of xFluid's pressure-solver interface, backed by libxfp.

``VariationalPressureSolver`` keeps the reference class's nine methods
(xFluid/xFluid/variationalpressure/variational_pressuresolver.h:33-44) with the
same meaning: the setters store sizes and borrowed arrays, ``solve(pressure)``
assembles the variational system, runs MIC(0)-PCG and fills ``pressure`` for
every cell, and ``applyPressure(pressure)`` updates the borrowed velocity arrays
in place.  As in the reference, ``setDensity``, ``setDt``, ``setDx`` and
``setDisField`` are stored but do not change the result (the reference's
pressure scale factor is fixed at 1.0, variational_pressuresolver.cpp:122).

Arrays are numpy arrays (host memory; the library copies) or CUDA torch tensors
(device memory; used in place), shaped like xFluid's Array3d with k slowest:
material (nk,nj,ni) uint8, u (nk,nj,ni+1), v (nk,nj+1,ni), w (nk+1,nj,ni),
pressure (nk,nj,ni).  float64 arrays use the *_f64 entry points, float32 the
*_f32 ones.

Differences from the reference, by design: ``solve`` returns False on
non-convergence but still writes the last iterate (the reference leaves the
grid unsized, variational_pressuresolver.cpp:80-86), and the PCG tolerance and
iteration cap are settable (``set_solver_parameters``, pcg_solver.h:234).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import Context, XfpStats


def _is_torch(a) -> bool:
    return type(a).__module__.startswith("torch")


def _ptr(a):
    if a is None:
        return None
    if _is_torch(a):
        if not a.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return C.c_void_p(a.data_ptr())
    if not (a.flags["C_CONTIGUOUS"] and a.flags["ALIGNED"]):
        raise ValueError("array must be C-contiguous")
    return C.c_void_p(a.ctypes.data)


def _dtype_name(a) -> str:
    if _is_torch(a):
        import torch
        return {torch.float64: "f64", torch.float32: "f32"}[a.dtype]
    return {np.dtype(np.float64): "f64", np.dtype(np.float32): "f32"}[a.dtype]


def _on_device(a) -> bool:
    return _is_torch(a) and a.is_cuda


class VariationalPressureSolver:
    """Drop-in for xFluid's VariationalPressureSolver on a B200."""

    _MATRIX = "variational"

    def __init__(self, precision: str = "f64", device: int = 0, tol: float = 1e-5, max_iter: int = 100,
                 omega: float = 0.97, min_diag_ratio: float = 0.25, check_every: int = 8,
                 timeout_ms: float = 2000.0, tile_k: int = 0):
        o = _lib.default_options()
        o.tol, o.max_iter, o.omega, o.min_diag_ratio = tol, max_iter, omega, min_diag_ratio
        o.precision = _lib.PREC[precision]
        o.device, o.check_every, o.timeout_ms, o.tile_k = device, check_every, timeout_ms, tile_k
        o.matrix = _lib.MATRIX[self._MATRIX]
        self._ctx = Context(o)
        self._size = (0, 0, 0)
        self._u = self._v = self._w = None
        self._mat = None
        self._weights = (None, None, None)
        self._density = self._dt = self._dx = None
        self._disfield = None
        self.stats: dict = {}

    # ---- the reference's setters (variational_pressuresolver.cpp:11-48) ----
    def setSize(self, sizei: int, sizej: int, sizek: int) -> None:
        self._size = (int(sizei), int(sizej), int(sizek))

    def setVelocityField(self, u, v, w) -> None:
        self._u, self._v, self._w = u, v, w

    def setMaterial(self, material) -> None:
        self._mat = material

    def setDisField(self, disfield) -> None:
        self._disfield = disfield

    def setDensity(self, density: float) -> None:
        self._density = density

    def setDt(self, dt: float) -> None:
        self._dt = dt

    def setDx(self, dx: float) -> None:
        self._dx = dx

    # ---- extensions ----
    def set_solver_parameters(self, tol: float, max_iter: int, omega: float = 0.97,
                              min_diag_ratio: float = 0.25) -> None:
        """PCGSolver::set_solver_parameters (pcg_solver.h:234-241)."""
        o = self._ctx.opts
        o.tol, o.max_iter, o.omega, o.min_diag_ratio = tol, max_iter, omega, min_diag_ratio
        self._ctx.set_options(o)

    def set_precision(self, precision: str) -> None:
        o = self._ctx.opts
        o.precision = _lib.PREC[precision]
        self._ctx.set_options(o)

    def setFaceWeights(self, wu, wv, ww) -> None:
        """Open fractions per face in [0,1] (None for the reference's matrix)."""
        self._weights = (wu, wv, ww)

    # ---- the solve / apply pair (variational_pressuresolver.cpp:50-220) ----
    def _prep(self, arrays):
        dev = {_on_device(a) for a in arrays if a is not None}
        if len(dev) != 1:
            raise ValueError("arrays must all be host numpy arrays or all CUDA tensors")
        o = self._ctx.opts
        want = 1 if dev.pop() else 0
        if o.device_pointers != want:
            o.device_pointers = want
            self._ctx.set_options(o)
        if want:
            # the context's stream is not ordered after torch's: finish the
            # torch work that produced the tensors (each call returns only
            # after its own stream is done)
            _lib.sync_torch(o.device)

    def solve(self, pressure) -> bool:
        """Fills pressure (nk,nj,ni) for every cell; True when converged."""
        ni, nj, nk = self._size
        wu, wv, ww = self._weights
        arrs = [self._mat, self._u, self._v, self._w, wu, wv, ww, pressure]
        self._prep(arrs)
        st = XfpStats()
        fn = self._ctx.lib.xfp_solve_f64 if _dtype_name(pressure) == "f64" else self._ctx.lib.xfp_solve_f32
        rc = self._ctx.check(fn(self._ctx.ptr, ni, nj, nk, *map(_ptr, arrs), C.byref(st)))
        self.stats = st.as_dict()
        return rc == _lib.XFP_OK

    # ---- the simulator steps either side of the projection (FluidSimulator.cpp) ----
    def applyForces(self, force, dt: float) -> None:
        """FluidSimulator::_applyForces (:429-499) on the borrowed velocities:
        force (the summed constant force, 3 values) * dt on every face that
        borders fluid."""
        ni, nj, nk = self._size
        arrs = [self._mat, self._u, self._v, self._w]
        self._prep(arrs)
        f3 = (C.c_double * 3)(*[float(x) for x in force])
        fn = self._ctx.lib.xfp_apply_forces_f64 if _dtype_name(self._u) == "f64" else self._ctx.lib.xfp_apply_forces_f32
        self._ctx.check(fn(self._ctx.ptr, ni, nj, nk, *map(_ptr, arrs), f3, float(dt)))

    def extrapolateVelocity(self, layers: int) -> None:
        """FluidSimulator::_expolateVelocity (:511-650) on the borrowed
        velocities; the reference uses layers = int(CFL number + 5)."""
        ni, nj, nk = self._size
        arrs = [self._mat, self._u, self._v, self._w]
        self._prep(arrs)
        fn = self._ctx.lib.xfp_extrapolate_f64 if _dtype_name(self._u) == "f64" else self._ctx.lib.xfp_extrapolate_f32
        self._ctx.check(fn(self._ctx.ptr, ni, nj, nk, *map(_ptr, arrs), int(layers)))

    def calculateDivergence(self, div) -> None:
        """VariationalPressureSolver::_calculate_divergience (variational_
        pressuresolver.cpp:526-597) of the borrowed velocities into `div`
        (ni*nj*nk, the velocities' dtype): per fluid cell the unit-weight sum
        over faces whose neighbour is not solid, 0 elsewhere."""
        ni, nj, nk = self._size
        arrs = [self._mat, self._u, self._v, self._w, div]
        self._prep(arrs)
        fn = self._ctx.lib.xfp_divergence_f64 if _dtype_name(self._u) == "f64" else self._ctx.lib.xfp_divergence_f32
        self._ctx.check(fn(self._ctx.ptr, ni, nj, nk, *map(_ptr, arrs)))

    def projectStep(self, pressure, force, dt: float, layers: int) -> bool:
        """applyForces, solve, applyPressure and extrapolateVelocity in one
        call, the force fused into the assembly and apply kernels; True when
        the solve converged."""
        ni, nj, nk = self._size
        wu, wv, ww = self._weights
        arrs = [self._mat, self._u, self._v, self._w, wu, wv, ww, pressure]
        self._prep(arrs)
        st = XfpStats()
        f3 = (C.c_double * 3)(*[float(x) for x in force])
        fn = (self._ctx.lib.xfp_project_step_f64 if _dtype_name(self._u) == "f64"
              else self._ctx.lib.xfp_project_step_f32)
        rc = self._ctx.check(fn(self._ctx.ptr, ni, nj, nk, *map(_ptr, arrs), f3, float(dt), int(layers),
                                C.byref(st)))
        self.stats = st.as_dict()
        return rc == _lib.XFP_OK

    def applyPressure(self, pressure) -> bool:
        """u,v,w -= grad p on every face that touches fluid."""
        ni, nj, nk = self._size
        wu, wv, ww = self._weights
        arrs = [self._mat, wu, wv, ww, pressure, self._u, self._v, self._w]
        self._prep(arrs)
        fn = (self._ctx.lib.xfp_apply_pressure_f64 if _dtype_name(pressure) == "f64"
              else self._ctx.lib.xfp_apply_pressure_f32)
        self._ctx.check(fn(self._ctx.ptr, ni, nj, nk, *map(_ptr, arrs)))
        return True

    def project(self, pressure=None) -> bool:
        """solve + applyPressure in one call (FluidSimulator::_solvePressure)."""
        ni, nj, nk = self._size
        wu, wv, ww = self._weights
        arrs = [self._mat, self._u, self._v, self._w, wu, wv, ww, pressure]
        self._prep(arrs)
        st = XfpStats()
        fn = self._ctx.lib.xfp_project_f64 if _dtype_name(self._u) == "f64" else self._ctx.lib.xfp_project_f32
        rc = self._ctx.check(fn(self._ctx.ptr, ni, nj, nk, *map(_ptr, arrs), C.byref(st)))
        self.stats = st.as_dict()
        return rc == _lib.XFP_OK

    def backward(self, gu, gv, gw, du=None, dv=None, dw=None):
        """Adjoint of project(): given dL/du_out returns dL/du_in."""
        ni, nj, nk = self._size
        wu, wv, ww = self._weights
        if du is None:
            du, dv, dw = (g.clone() if _is_torch(g) else g.copy() for g in (gu, gv, gw))
        arrs = [self._mat, wu, wv, ww, gu, gv, gw, du, dv, dw]
        self._prep(arrs)
        st = XfpStats()
        fn = (self._ctx.lib.xfp_project_backward_f64 if _dtype_name(gu) == "f64"
              else self._ctx.lib.xfp_project_backward_f32)
        self._ctx.check(fn(self._ctx.ptr, ni, nj, nk, *map(_ptr, arrs), C.byref(st)))
        self.stats = st.as_dict()
        return du, dv, dw

    def close(self) -> None:
        self._ctx.close()


def project_scene(sc, precision: str = "f64", tol: float = 1e-6, max_iter: int = 200,
                  solver: VariationalPressureSolver | None = None, fractional: bool = True, **kw):
    """Project a scenes.Scene (numpy arrays) on the GPU.  Returns
    (ok, pressure, u, v, w, stats) with new arrays; the scene is not modified."""
    s = solver or VariationalPressureSolver(precision=precision, **kw)
    if solver is not None:
        s.set_precision(precision)
    s.set_solver_parameters(tol, max_iter)
    u, v, w = sc.u.copy(), sc.v.copy(), sc.w.copy()
    p = np.zeros((sc.nk, sc.nj, sc.ni), dtype=u.dtype)
    s.setSize(sc.ni, sc.nj, sc.nk)
    s.setMaterial(np.ascontiguousarray(sc.mat, dtype=np.uint8))
    s.setVelocityField(u, v, w)
    if fractional and sc.wu is not None:
        s.setFaceWeights(*(np.ascontiguousarray(a, dtype=u.dtype) for a in (sc.wu, sc.wv, sc.ww)))
    else:
        s.setFaceWeights(None, None, None)
    ok = s.project(p)
    return ok, p, u, v, w, dict(s.stats)


class NormalPressureSolver(VariationalPressureSolver):
    """Drop-in for xFluid's NormalPressureSolver (pressuresolver.h:9-25), the
    classic Poisson matrix on the same MIC(0)-PCG: for every fluid cell the
    diagonal is the number of in-range non-solid neighbours and -1 couples it
    to each fluid neighbour (pressuresolver.cpp:220-347); applyPressure
    updates faces touching fluid with solid faces reflecting and air faces at
    zero pressure (:109-212).  The same nine methods with the same meanings;
    the reference class has no face weights, so setFaceWeights is refused."""

    _MATRIX = "normal"

    def setFaceWeights(self, wu, wv, ww) -> None:
        raise ValueError("the normal pressure matrix has no face weights")
