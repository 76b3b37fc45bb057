"""The particle steps around the projection, on the device: a mirror of
xFluid's FluidSimulator particle methods over the C ABI (include/xfp.h).

    s = ParticleSteps(dx=1/64)
    s.advectParticles(parts, mat, (u, v, w), (us, vs, ws), dt, ratio=0.95)   # _advectParticles a-b
    s.updateVelocityByParticles(parts, (u, v, w))                            # _updateVelocityByParticles
    s.updateMaterial(parts, mat)                                             # _updateMaterial
    phi = s.updateField(parts, mat, subdiv=2, radius=r, threshold=0.4)       # updateFeild + updateSurfaceInfo

Particles are an (n, 6) float64 array (or CUDA tensor) laid out as xFluid's
struct Particle {Vec3d p; Vec3d v;}; grids are the simulator's Array3d
layout ((nk, nj, ni+1) for u and so on).  Arrays are updated in place.  numpy
arrays go through host staging; CUDA tensors are used in place.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import Context


def _is_cuda(a) -> bool:
    return getattr(a, "is_cuda", False)


def _ptr(a):
    if a is None:
        return None
    if _is_cuda(a):
        return C.c_void_p(a.data_ptr())
    if not (isinstance(a, np.ndarray) and a.flags.c_contiguous):
        raise ValueError("arrays must be C-contiguous numpy arrays or CUDA tensors")
    return C.c_void_p(a.ctypes.data)


def _check(a, dtype, shape, name):
    sh = tuple(a.shape)
    if sh != tuple(shape):
        raise ValueError(f"{name}: shape {sh}, expected {tuple(shape)}")
    dt = str(a.dtype).replace("torch.", "")
    if dt != dtype:
        raise ValueError(f"{name}: dtype {dt}, expected {dtype}")


class ParticleSteps:
    def __init__(self, dx: float, device: int = 0):
        self.dx = float(dx)
        self.device = device
        self._ctx: dict[bool, Context] = {}

    def close(self) -> None:
        for c in self._ctx.values():
            c.close()
        self._ctx = {}

    def _context(self, arrays) -> Context:
        dev = [_is_cuda(a) for a in arrays if a is not None]
        if any(dev) and not all(dev):
            raise ValueError("pass either all numpy arrays or all CUDA tensors")
        on_dev = bool(dev) and dev[0]
        if on_dev:
            # the kernels read and write len(a) contiguous elements from data_ptr()
            # on the context's device: a strided view (x[:, :6] of an (n, 8)
            # tensor) would have memory outside the view overwritten, and a
            # tensor on another GPU would be dereferenced from this one
            for a in arrays:
                if a is None:
                    continue
                if not a.is_contiguous():
                    raise ValueError("CUDA tensors must be contiguous")
                if a.device.index != self.device:
                    raise ValueError(f"CUDA tensor on {a.device}, expected cuda:{self.device}")
        if on_dev:
            _lib.sync_torch(self.device)
        if on_dev not in self._ctx:
            o = _lib.default_options()
            o.device, o.device_pointers = self.device, int(on_dev)
            self._ctx[on_dev] = Context(o)
        return self._ctx[on_dev]

    @staticmethod
    def _dims(mat):
        nk, nj, ni = (int(x) for x in mat.shape)
        return ni, nj, nk

    def _faces(self, dims, uvw, name):
        ni, nj, nk = dims
        for a, sh, nm in zip(uvw, ((nk, nj, ni + 1), (nk, nj + 1, ni), (nk + 1, nj, ni)), "uvw"):
            _check(a, "float64", sh, f"{name}{nm}")

    def advectParticles(self, parts, mat, uvw, saved, dt: float, ratio: float = 0.95) -> None:
        """FluidSimulator::_advectParticles steps a-b (FluidSimulator.cpp:652-723):
        FLIP/PIC velocity update from `uvw` and the pre-force `saved` faces,
        RK4 advection over dt, solid collisions.  The last n mod 6 particles
        stay unchanged, as in the reference."""
        dims = self._dims(mat)
        _check(parts, "float64", (parts.shape[0], 6), "particles")
        _check(mat, "uint8", mat.shape, "material")
        self._faces(dims, uvw, "")
        self._faces(dims, saved, "saved ")
        ctx = self._context([parts, mat, *uvw, *saved])
        ctx.check(ctx.lib.xfp_advect_particles_f64(ctx.ptr, *dims, self.dx, _ptr(mat), *map(_ptr, uvw),
                                                   *map(_ptr, saved), float(ratio), float(dt),
                                                   int(parts.shape[0]), _ptr(parts)))

    def maxVelocity(self, parts) -> float:
        """FluidSimulator::_maxVelocity (FluidSimulator.cpp:387-400): the
        largest particle speed, rounded as the reference rounds it."""
        _check(parts, "float64", (parts.shape[0], 6), "particles")
        ctx = self._context([parts])
        out = C.c_double(0.0)
        ctx.check(ctx.lib.xfp_max_speed_f64(ctx.ptr, int(parts.shape[0]), _ptr(parts), C.byref(out)))
        return out.value

    def updateVelocityByParticles(self, parts, uvw) -> None:
        """FluidSimulator::_updateVelocityByParticles (:909-1085) into uvw."""
        nk, nj, ni1 = (int(x) for x in uvw[0].shape)
        dims = (ni1 - 1, nj, nk)
        _check(parts, "float64", (parts.shape[0], 6), "particles")
        self._faces(dims, uvw, "")
        ctx = self._context([parts, *uvw])
        ctx.check(ctx.lib.xfp_particles_to_grid_f64(ctx.ptr, *dims, self.dx, int(parts.shape[0]), _ptr(parts),
                                                    *map(_ptr, uvw)))

    def updateMaterial(self, parts, mat) -> None:
        """FluidSimulator::_updateMaterial (:402-427) on `mat` in place."""
        _check(parts, "float64", (parts.shape[0], 6), "particles")
        _check(mat, "uint8", mat.shape, "material")
        ctx = self._context([parts, mat])
        ctx.check(ctx.lib.xfp_update_material(ctx.ptr, *self._dims(mat), self.dx, int(parts.shape[0]), _ptr(parts),
                                              _ptr(mat)))

    def updateField(self, parts, mat, subdiv: int = 2, radius: float | None = None, threshold: float = 0.4,
                    classify: bool = True, phi=None):
        """DirectedDistanceField::updateFeild (directeddistancefield.cpp:122-165)
        and, with classify=True, updateSurfaceInfo's material classification
        (:167-215) on `mat` in place.  radius defaults to FluidSimulator's:
        3x the particle radius (3 dx^3/8 / (4 pi))^(1/3) (FluidSimulator.cpp:
        380-385, 210).  Returns phi ((nk*s+1, nj*s+1, ni*s+1) float64)."""
        ni, nj, nk = self._dims(mat)
        s = int(subdiv)
        if radius is None:
            radius = 3.0 * (3 * (self.dx ** 3 / 8.0) / (4 * 3.141592653)) ** (1.0 / 3.0)
        shape = (nk * s + 1, nj * s + 1, ni * s + 1)
        if phi is None:
            if _is_cuda(parts):
                import torch
                phi = torch.zeros(shape, dtype=torch.float64, device=parts.device)
            else:
                phi = np.zeros(shape)
        _check(phi, "float64", shape, "phi")
        _check(parts, "float64", (parts.shape[0], 6), "particles")
        _check(mat, "uint8", mat.shape, "material")
        ctx = self._context([parts, mat, phi])
        ctx.check(ctx.lib.xfp_distance_field_f64(ctx.ptr, ni, nj, nk, self.dx, s, float(radius), float(threshold),
                                                 int(parts.shape[0]), _ptr(parts), _ptr(phi),
                                                 _ptr(mat) if classify else None))
        return phi
