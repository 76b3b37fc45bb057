"""xFluid's whole time step on the device: FluidSimulator::timeStep
(FluidSimulator.cpp:265-335) through the library's entry points, with the
state (particles, face velocities, material) resident in device memory.

    sim = Simulation(mat, particles, dx=1/64, cfl=5.0, tol=1e-6, max_iter=200)
    dt = sim.step_dt(max_dt=1/30)     # frameStep's rule from _maxVelocity (:228-241)
    ok = sim.time_step(dt)            # one step, as timeStep runs it

A step runs, in the reference's order:
  1. the distance field and its classification (updateFeild,
     updateSurfaceInfo, :274-275) -- optional: _updateMaterial overwrites the
     classification, so it changes nothing downstream; the reference computes
     it for the mesh output -- then _updateMaterial (:276);
  2. _saveVelocity (:285): the faces before the force;
  3. _applyForces, _solvePressure and _expolateVelocity (:309-322) fused in
     one call (xfp_project_step_f64: the force enters the assembly and apply
     kernels; int(CFL + 5) extrapolation layers, :513);
  4. _advectParticles (:327): the FLIP/PIC update from the saved faces, RK4
     advection with solid collisions, then the particle-to-grid transfer
     (_updateVelocityByParticles) into the faces.
The mesh output (:291-305) and fluid sources are not part of it.

Particles are an (n, 6) float64 CUDA tensor in xFluid's Particle layout
(p then v); faces and material use the Array3d layouts ((nk, nj, ni+1) for u
and so on).  Everything is FP64, as the reference; the projection can run in
the mixed form (FP64 faces, FP32 inner PCG with FP64 refinement).
"""
from __future__ import annotations

import math

from .particles import ParticleSteps
from .solver import VariationalPressureSolver


class Simulation:
    def __init__(self, mat, particles, dx: float, force=(0.0, -9.8, 0.0), cfl: float = 1.0, max_step: float = 0.5,
                 ratio_flip: float = 0.95, tol: float = 1e-5, max_iter: int = 100, subdiv: int = 2,
                 radius: float | None = None, threshold: float = 0.4, field: bool = True, precision: str = "f64",
                 device: int = 0, uvw=None):
        import torch
        if not (getattr(mat, "is_cuda", False) and getattr(particles, "is_cuda", False)):
            raise ValueError("material and particles must be CUDA tensors")
        self.mat, self.particles = mat, particles
        nk, nj, ni = (int(x) for x in mat.shape)
        self.dims = (ni, nj, nk)
        self.dx = float(dx)
        self.force = tuple(float(f) for f in force)
        self.cfl, self.max_step, self.ratio = float(cfl), float(max_step), float(ratio_flip)
        self.subdiv, self.threshold, self.field = int(subdiv), float(threshold), bool(field)
        # FluidSimulator's particle radius (:380-385) times 3, as init passes it (:210)
        self.radius = (3.0 * (3 * (self.dx ** 3 / 8.0) / (4 * 3.141592653)) ** (1.0 / 3.0)
                       if radius is None else float(radius))
        dev = mat.device
        shapes = ((nk, nj, ni + 1), (nk, nj + 1, ni), (nk + 1, nj, ni))
        if uvw is None:
            uvw = tuple(torch.zeros(s, dtype=torch.float64, device=dev) for s in shapes)
        self.u, self.v, self.w = uvw
        self.pressure = torch.zeros((nk, nj, ni), dtype=torch.float64, device=dev)
        self.phi = None
        self.steps = ParticleSteps(self.dx, device=device)
        self.solver = VariationalPressureSolver(precision, device=device, tol=tol, max_iter=max_iter)
        self.solver.setSize(ni, nj, nk)
        self.solver.setVelocityField(self.u, self.v, self.w)
        self.solver.setMaterial(self.mat)
        self.solver.setDx(self.dx)
        self.stats: dict = {}
        # with keep_intermediates: the faces the last step's advection used
        # (saved: before the force; uvw: after projection and extrapolation)
        self.keep_intermediates = False
        self.last: dict = {}

    def close(self) -> None:
        self.steps.close()
        self.solver.close()

    def set_state(self, particles=None, uvw=None, mat=None) -> None:
        """Copies a state in (in place, so the solver keeps its borrowed arrays)."""
        if particles is not None:
            if tuple(particles.shape) != tuple(self.particles.shape):
                self.particles = particles.clone()
            else:
                self.particles.copy_(particles)
        if uvw is not None:
            for dst, src in zip((self.u, self.v, self.w), uvw):
                dst.copy_(src)
        if mat is not None:
            self.mat.copy_(mat)

    def max_velocity(self) -> float:
        return self.steps.maxVelocity(self.particles)

    def step_dt(self, max_dt: float = math.inf) -> float:
        """frameStep's substep (:228-241): CFL * dx / max speed, at most the
        maximum step time (and max_dt)."""
        maxv = self.max_velocity()
        dt = self.max_step if maxv == 0.0 else self.cfl * self.dx / maxv
        dt = dt if dt < self.max_step else self.max_step
        return dt if dt < max_dt else max_dt

    def time_step(self, dt: float) -> bool:
        """One timeStep (:265-335) without the mesh output; True when the
        pressure solve converged."""
        P, m = self.particles, self.mat
        if self.field:
            self.phi = self.steps.updateField(P, m, subdiv=self.subdiv, radius=self.radius,
                                              threshold=self.threshold, classify=True, phi=self.phi)
        self.steps.updateMaterial(P, m)
        saved = (self.u.clone(), self.v.clone(), self.w.clone())
        ok = self.solver.projectStep(self.pressure, self.force, dt, int(self.cfl + 5))
        self.stats = dict(self.solver.stats)
        if self.keep_intermediates:
            self.last = {"saved": saved, "uvw": (self.u.clone(), self.v.clone(), self.w.clone()),
                         "mat": self.mat.clone(), "particles_in": P.clone()}
        self.steps.advectParticles(P, m, (self.u, self.v, self.w), saved, dt, ratio=self.ratio)
        self.steps.updateVelocityByParticles(P, (self.u, self.v, self.w))
        return ok

    def frame_step(self, frame_dt: float) -> int:
        """frameStep (:224-262): substeps until frame_dt is covered; returns
        the number of substeps."""
        left, n = float(frame_dt), 0
        while left > 0.0:
            dt = self.step_dt()
            if left <= dt:
                dt, left = left, 0.0
            else:
                left -= dt
            self.time_step(dt)
            n += 1
        return n
