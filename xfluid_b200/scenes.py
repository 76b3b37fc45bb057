"""Seeded synthetic scenes for the pressure projection.

Every array uses xFluid's grid layout (``Array3d``, xFluid/xFluid/array3d.h:143-146):
flat index ``k*ni*nj + j*ni + i``, i.e. numpy shape ``(nk, nj, ni)`` in C order.
MAC faces follow xFluid/xFluid/FluidSimulator.h:177-181: ``u`` is (ni+1, nj, nk),
``v`` is (ni, nj+1, nk), ``w`` is (ni, nj, nk+1); ``u(i,j,k)`` sits on the face
between cells i-1 and i.  Materials use ``enum class Material : char`` values
(xFluid/xFluid/material.h:4-8): air 0, fluid 1, solid 2.

A scene may carry per-face open fractions ``wu, wv, ww`` (same shapes as the
velocities, values in [0, 1]).  They scale every face's contribution to the
Poisson system and are ``None`` in reference mode, where the matrix is exactly
xFluid's (all faces fully open).

Workloads:
  dam_break      -- 64^3 dam break: fluid x<0.4, y<0.5, solid border.
  pool_drop      -- 128^3 pool (depth 0.3) plus a falling fluid sphere and a
                    static solid sphere that gives fractional face weights.
  blob_scene     -- 256^3 standalone projection: fluid = sum of 32 Gaussian
                    blobs thresholded at 0.5, a random box obstacle covering 10%
                    of the volume, U[-1,1] face velocities.
  batch_scenes   -- uneven blob scenes with nx,ny,nz ~ U[32,160].
All inputs are synthetic and seeded; none is read from a dataset.
"""
from __future__ import annotations

import dataclasses
import numpy as np

AIR, FLUID, SOLID = 0, 1, 2


@dataclasses.dataclass
class Scene:
    ni: int
    nj: int
    nk: int
    mat: np.ndarray            # uint8 (nk, nj, ni)
    u: np.ndarray              # (nk, nj, ni+1)
    v: np.ndarray              # (nk, nj+1, ni)
    w: np.ndarray              # (nk+1, nj, ni)
    wu: np.ndarray | None = None
    wv: np.ndarray | None = None
    ww: np.ndarray | None = None
    name: str = ""

    @property
    def ncells(self) -> int:
        return self.ni * self.nj * self.nk

    def astype(self, dtype) -> "Scene":
        cv = lambda a: None if a is None else np.ascontiguousarray(a, dtype=dtype)
        return dataclasses.replace(self, u=cv(self.u), v=cv(self.v), w=cv(self.w),
                                   wu=cv(self.wu), wv=cv(self.wv), ww=cv(self.ww))

    def copy(self) -> "Scene":
        cp = lambda a: None if a is None else a.copy()
        return dataclasses.replace(self, mat=self.mat.copy(), u=cp(self.u), v=cp(self.v),
                                   w=cp(self.w), wu=cp(self.wu), wv=cp(self.wv), ww=cp(self.ww))

    def reference_mode(self) -> "Scene":
        return dataclasses.replace(self, wu=None, wv=None, ww=None)


def _centres(n: int) -> np.ndarray:
    return (np.arange(n, dtype=np.float64) + 0.5) / n


def solid_border(mat: np.ndarray) -> None:
    """Outermost cell layer becomes solid (FluidSimulator::setSolidBoundary,
    xFluid/xFluid/FluidSimulator.cpp:64-96)."""
    mat[0, :, :] = SOLID
    mat[-1, :, :] = SOLID
    mat[:, 0, :] = SOLID
    mat[:, -1, :] = SOLID
    mat[:, :, 0] = SOLID
    mat[:, :, -1] = SOLID


def face_shapes(ni: int, nj: int, nk: int):
    return (nk, nj, ni + 1), (nk, nj + 1, ni), (nk + 1, nj, ni)


def fluid_adjacent_faces(mat: np.ndarray):
    """Masks of faces bordering at least one fluid cell (the faces
    FluidSimulator::_applyForces touches, FluidSimulator.cpp:429-499)."""
    fl = mat == FLUID
    nk, nj, ni = mat.shape
    su, sv, sw = face_shapes(ni, nj, nk)
    mu = np.zeros(su, bool); mu[:, :, :-1] |= fl; mu[:, :, 1:] |= fl
    mv = np.zeros(sv, bool); mv[:, :-1, :] |= fl; mv[:, 1:, :] |= fl
    mw = np.zeros(sw, bool); mw[:-1, :, :] |= fl; mw[1:, :, :] |= fl
    return mu, mv, mw


def random_faces(rng, ni, nj, nk, lo=-1.0, hi=1.0, dtype=np.float32):
    su, sv, sw = face_shapes(ni, nj, nk)
    return (rng.uniform(lo, hi, su).astype(dtype), rng.uniform(lo, hi, sv).astype(dtype),
            rng.uniform(lo, hi, sw).astype(dtype))


def dam_break(n: int = 64, seed: int = 1, dt: float = 1.0 / 30.0, noise: float = 0.0,
              dims: tuple[int, int, int] | None = None, dtype=np.float64) -> Scene:
    """Dam break: fluid where the cell centre has x<0.4 and y<0.5, solid border.
    Velocities are the first step's gravity impulse (-9.8*dt on v faces that
    border fluid, as _applyForces does) plus optional seeded U[-noise, noise]."""
    ni, nj, nk = dims if dims is not None else (n, n, n)
    mat = np.zeros((nk, nj, ni), np.uint8)
    x, y = _centres(ni), _centres(nj)
    box = (x[None, None, :] < 0.4) & (y[None, :, None] < 0.5)
    mat[np.broadcast_to(box, mat.shape)] = FLUID
    solid_border(mat)
    rng = np.random.default_rng(seed)
    su, sv, sw = face_shapes(ni, nj, nk)
    u = np.zeros(su); v = np.zeros(sv); w = np.zeros(sw)
    _, mv, _ = fluid_adjacent_faces(mat)
    v[mv] += -9.8 * dt
    if noise > 0:
        nu, nv, nw = random_faces(rng, ni, nj, nk, -noise, noise, np.float64)
        u += nu; v += nv; w += nw
    return Scene(ni, nj, nk, mat, u.astype(dtype), v.astype(dtype), w.astype(dtype),
                 name=f"dam_break_{ni}x{nj}x{nk}")


def _gaussian_sum(ni, nj, nk, rng, nblobs, sig_lo, sig_hi):
    x, y, z = _centres(ni), _centres(nj), _centres(nk)
    phi = np.zeros((nk, nj, ni), np.float64)
    cen = rng.uniform(0.0, 1.0, (nblobs, 3))
    sig = rng.uniform(sig_lo, sig_hi, nblobs)
    for c, s in zip(cen, sig):
        inv = 1.0 / (2.0 * s * s)
        gx = np.exp(-(x - c[0]) ** 2 * inv)
        gy = np.exp(-(y - c[1]) ** 2 * inv)
        gz = np.exp(-(z - c[2]) ** 2 * inv)
        phi += gz[:, None, None] * (gy[:, None] * gx[None, :])[None, :, :]
    return phi


def _overlap_1d(a0, a1, lo, hi):
    """Length of [a0,a1] inside [lo,hi], elementwise, divided by (a1-a0)."""
    return np.clip(np.minimum(a1, hi) - np.maximum(a0, lo), 0.0, None) / (a1 - a0)


def _box_face_fractions(ni, nj, nk, lo, hi):
    """Open fraction of every MAC face against an axis-aligned solid box
    [lo,hi] (world units, grid spacing 1/n per axis)."""
    def axis(n):
        e = np.arange(n + 1, dtype=np.float64) / n       # face positions
        c0 = np.arange(n, dtype=np.float64) / n           # cell extents
        c1 = c0 + 1.0 / n
        return e, c0, c1
    ex, x0, x1 = axis(ni)
    ey, y0, y1 = axis(nj)
    ez, z0, z1 = axis(nk)
    inx = ((ex > lo[0]) & (ex < hi[0])).astype(np.float64)
    iny = ((ey > lo[1]) & (ey < hi[1])).astype(np.float64)
    inz = ((ez > lo[2]) & (ez < hi[2])).astype(np.float64)
    ox, oy, oz = _overlap_1d(x0, x1, lo[0], hi[0]), _overlap_1d(y0, y1, lo[1], hi[1]), _overlap_1d(z0, z1, lo[2], hi[2])
    wu = 1.0 - oz[:, None, None] * oy[None, :, None] * inx[None, None, :]
    wv = 1.0 - oz[:, None, None] * iny[None, :, None] * ox[None, None, :]
    ww = 1.0 - inz[:, None, None] * oy[None, :, None] * ox[None, None, :]
    return wu, wv, ww


def blob_scene(n: int = 256, seed: int = 3, nblobs: int = 32, obstacle_frac: float = 0.10,
               dims: tuple[int, int, int] | None = None, fractional: bool = True,
               dtype=np.float32) -> Scene:
    """Standalone projection scene: fluid = {sum of nblobs Gaussians (sigma ~
    U[0.03,0.12], centres ~ U[0,1]^3) > 0.5}, a random axis-aligned box obstacle
    covering ``obstacle_frac`` of the volume (cells whose centre is inside are
    solid; faces it cuts get fractional open weights), solid border, face
    velocities U[-1,1]."""
    ni, nj, nk = dims if dims is not None else (n, n, n)
    rng = np.random.default_rng(seed)
    phi = _gaussian_sum(ni, nj, nk, rng, nblobs, 0.03, 0.12)
    mat = np.where(phi > 0.5, FLUID, AIR).astype(np.uint8)
    # box obstacle: sides with product obstacle_frac, random placement
    sx, sy = rng.uniform(0.35, 0.65, 2)
    sz = min(0.95, obstacle_frac / (sx * sy))
    side = np.array([sx, sy, sz])
    lo = rng.uniform(0.0, 1.0 - side)
    hi = lo + side
    x, y, z = _centres(ni), _centres(nj), _centres(nk)
    inside = ((z[:, None, None] > lo[2]) & (z[:, None, None] < hi[2]) &
              (y[None, :, None] > lo[1]) & (y[None, :, None] < hi[1]) &
              (x[None, None, :] > lo[0]) & (x[None, None, :] < hi[0]))
    mat[inside] = SOLID
    solid_border(mat)
    u, v, w = random_faces(rng, ni, nj, nk, -1.0, 1.0, np.float32)
    wu = wv = ww = None
    if fractional:
        wu, wv, ww = (a.astype(np.float32) for a in _box_face_fractions(ni, nj, nk, lo, hi))
    sc = Scene(ni, nj, nk, mat, u, v, w, wu, wv, ww, name=f"blob_{ni}x{nj}x{nk}_s{seed}")
    return sc.astype(dtype)


def _sphere_face_fractions(ni, nj, nk, centre, radius, sub=4):
    """Open fraction of every MAC face against a solid sphere, by sub x sub
    point sampling of each face."""
    off = (np.arange(sub) + 0.5) / sub

    def frac(shape, fixed_axis):
        # fixed_axis: 0 -> x faces (u), 1 -> y faces (v), 2 -> z faces (w)
        nkf, njf, nif = shape
        kk = np.arange(nkf, dtype=np.float64)
        jj = np.arange(njf, dtype=np.float64)
        ii = np.arange(nif, dtype=np.float64)
        acc = np.zeros(shape)
        for a in off:
            for b in off:
                if fixed_axis == 0:
                    X = ii[None, None, :] / ni; Y = (jj[None, :, None] + a) / nj; Z = (kk[:, None, None] + b) / nk
                elif fixed_axis == 1:
                    X = (ii[None, None, :] + a) / ni; Y = jj[None, :, None] / nj; Z = (kk[:, None, None] + b) / nk
                else:
                    X = (ii[None, None, :] + a) / ni; Y = (jj[None, :, None] + b) / nj; Z = kk[:, None, None] / nk
                d2 = (X - centre[0]) ** 2 + (Y - centre[1]) ** 2 + (Z - centre[2]) ** 2
                acc += (d2 < radius * radius)
        return 1.0 - acc / (sub * sub)
    su, sv, sw = face_shapes(ni, nj, nk)
    return frac(su, 0), frac(sv, 1), frac(sw, 2)


def pool_drop(n: int = 128, seed: int = 2, dt: float = 1.0 / 30.0, noise: float = 0.5,
              dims: tuple[int, int, int] | None = None, dtype=np.float32) -> Scene:
    """Drop into a pool: fluid pool y<0.3 plus a fluid sphere (r=0.15, centre
    (0.5,0.7,0.5)); a static solid sphere (r=0.1, centre (0.3,0.2,0.5)) whose
    cells are solid and whose cut faces get fractional open weights.  Velocities:
    gravity impulse on fluid faces plus seeded U[-noise, noise]."""
    ni, nj, nk = dims if dims is not None else (n, n, n)
    x, y, z = _centres(ni), _centres(nj), _centres(nk)
    X, Y, Z = x[None, None, :], y[None, :, None], z[:, None, None]
    mat = np.zeros((nk, nj, ni), np.uint8)
    fluid = (Y < 0.3) | ((X - 0.5) ** 2 + (Y - 0.7) ** 2 + (Z - 0.5) ** 2 < 0.15 ** 2)
    mat[np.broadcast_to(fluid, mat.shape)] = FLUID
    solid = (X - 0.3) ** 2 + (Y - 0.2) ** 2 + (Z - 0.5) ** 2 < 0.1 ** 2
    mat[np.broadcast_to(solid, mat.shape)] = SOLID
    solid_border(mat)
    rng = np.random.default_rng(seed)
    u, v, w = random_faces(rng, ni, nj, nk, -noise, noise, np.float64)
    _, mv, _ = fluid_adjacent_faces(mat)
    v[mv] += -9.8 * dt
    wu, wv, ww = _sphere_face_fractions(ni, nj, nk, (0.3, 0.2, 0.5), 0.1)
    sc = Scene(ni, nj, nk, mat, u, v, w, wu, wv, ww, name=f"pool_{ni}x{nj}x{nk}")
    return sc.astype(dtype)


def batch_scenes(count: int = 64, seed: int = 4, lo: int = 32, hi: int = 160,
                 dtype=np.float32) -> list[Scene]:
    """Uneven batch: each scene's nx, ny, nz ~ U[lo, hi] (inclusive), blob
    masks and U[-1,1] velocities as in blob_scene, each with its own seed."""
    rng = np.random.default_rng(seed)
    dims = rng.integers(lo, hi + 1, size=(count, 3))
    return [blob_scene(dims=(int(d[0]), int(d[1]), int(d[2])), seed=seed * 1000 + s, dtype=dtype)
            for s, d in enumerate(dims)]


def active_mask(mat: np.ndarray) -> np.ndarray:
    """Unknown rows of xFluid's system: fluid cells plus solid cells with a
    fluid neighbour (variational_pressuresolver.cpp:309-321)."""
    fl = mat == FLUID
    adj = np.zeros_like(fl)
    adj[1:] |= fl[:-1]; adj[:-1] |= fl[1:]
    adj[:, 1:] |= fl[:, :-1]; adj[:, :-1] |= fl[:, 1:]
    adj[:, :, 1:] |= fl[:, :, :-1]; adj[:, :, :-1] |= fl[:, :, 1:]
    return fl | ((mat == SOLID) & adj)


# xFluid's eight seeding points per fluid cell (FluidSimulator::_addParticle,
# FluidSimulator.cpp:347-370): cell centre +- dx/4 on each axis, in this order
_SEED_OFFSETS = np.array([(-1, -1, -1), (1, -1, -1), (1, -1, 1), (-1, -1, 1),
                          (-1, 1, -1), (1, 1, -1), (1, 1, 1), (-1, 1, 1)], np.float64)


def seed_particles(mat: np.ndarray, dx: float, seed: int = 0, jitter: float = 0.01, vel_scale: float = 1.0,
                   vel=None) -> np.ndarray:
    """Particles in every fluid cell of `mat` as xFluid seeds them: eight per
    cell at the centre +- dx/4 with a U[-jitter, jitter] offset (the reference's
    scale 0.01, FluidSimulator.cpp:364-369).  Velocities are U[-vel_scale,
    vel_scale] (the reference starts at rest; random velocities exercise the
    transfers), or `vel` (n, 3) when given.  Returns (n, 6) FP64 rows laid out
    as struct Particle {Vec3d p; Vec3d v;} (particle.h:5-15)."""
    rng = np.random.default_rng(seed)
    k, j, i = np.nonzero(mat == 1)
    c = (np.stack([i, j, k], 1).astype(np.float64) + 0.5) * dx
    p = (c[:, None, :] + 0.25 * dx * _SEED_OFFSETS[None]).reshape(-1, 3)
    p = p + rng.uniform(-jitter, jitter, p.shape)
    v = rng.uniform(-vel_scale, vel_scale, p.shape) if vel is None else np.asarray(vel, np.float64)
    return np.ascontiguousarray(np.concatenate([p, v], 1))
