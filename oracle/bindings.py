"""ctypes bindings for the oracle libraries -- TEST INFRASTRUCTURE ONLY.

Arrays follow xFluid's layout (numpy shape (nk, nj, ni), faces
(nk,nj,ni+1) / (nk,nj+1,ni) / (nk+1,nj,ni)); all values are float64.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SRC = HERE / "xfp_oracle.c"
ORACLE_SRCS = [ORACLE_SRC, HERE / "xfp_particles_oracle.c"]
ORACLE_LIB = HERE / "_build" / "libxfp_oracle.so"
REF_LIB = HERE / "_ref" / "libxfref.so"
SIM_LIB = HERE / "_ref" / "libxfsim.so"
DROPIN_LIB = HERE / "_ref" / "libxfsim_dropin.so"

_dp = C.POINTER(C.c_double)
_u8 = C.POINTER(C.c_uint8)


def _parts(a) -> np.ndarray:
    """Particles as xFluid's struct Particle {Vec3d p; Vec3d v;}: (n, 6) FP64."""
    return np.ascontiguousarray(np.asarray(a, np.float64).reshape(-1, 6))


def build_oracle(force: bool = False) -> Path:
    """Compile the C restatement (gcc, -O2, no FP contraction)."""
    if ORACLE_LIB.exists() and not force and \
            ORACLE_LIB.stat().st_mtime >= max(f.stat().st_mtime for f in ORACLE_SRCS):
        return ORACLE_LIB
    ORACLE_LIB.parent.mkdir(parents=True, exist_ok=True)
    tmp = ORACLE_LIB.with_suffix(".so.tmp")
    subprocess.check_call(["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-ffp-contract=off",
                           "-fno-fast-math", *map(str, ORACLE_SRCS), "-lm", "-o", str(tmp)])
    os.replace(tmp, ORACLE_LIB)
    return ORACLE_LIB


def build_reference(ref_root: str | None = None) -> Path | None:
    """Compile xFluid's own solver into oracle/_ref when its sources exist."""
    env = dict(os.environ)
    if ref_root:
        env["XFLUID_REF"] = ref_root
    # XFLUID_REF, else a checkout named `reference` beside this repository
    root = Path(env.get("XFLUID_REF", str(HERE.parent.parent / "reference")))
    if not (root / "xFluid" / "xFluid" / "variationalpressure").is_dir():
        return None
    subprocess.check_call(["bash", str(HERE / "build_ref.sh")], env=env,
                          stdout=subprocess.DEVNULL)
    subprocess.check_call(["bash", str(HERE / "build_sim.sh")], env=env,
                          stdout=subprocess.DEVNULL)
    return REF_LIB


def sim_available() -> bool:
    return SIM_LIB.exists()


def dropin_available() -> bool:
    return DROPIN_LIB.exists()


def seed_rand(seed: int) -> None:
    """srand() of the process's C library: xFluid's FluidSimulator::init
    jitters its particles with rand() (xfluidutil.cpp:67-70), so two simulators
    seeded alike start from the same particles."""
    C.CDLL(None).srand(C.c_uint(seed))


def oracle_available() -> bool:
    return ORACLE_LIB.exists()


def reference_available() -> bool:
    return REF_LIB.exists()


def _p(a):
    if a is None:
        return None
    return a.ctypes.data_as(_dp if a.dtype == np.float64 else _u8)


def _f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


class _Lib:
    def __init__(self, path: Path):
        if not path.exists():
            raise FileNotFoundError(f"oracle library missing: {path}")
        self.lib = C.CDLL(str(path))


class Oracle(_Lib):
    """The FP64 C restatement (oracle/xfp_oracle.c)."""

    def __init__(self):
        super().__init__(ORACLE_LIB if ORACLE_LIB.exists() else build_oracle())
        L = self.lib
        L.xo_assemble.argtypes = [C.c_int] * 3 + [_u8] + [_dp] * 11
        L.xo_spmv.argtypes = [C.c_int] * 3 + [_dp] * 6
        L.xo_factor.argtypes = [C.c_int] * 3 + [_dp] * 4 + [C.c_double] * 2 + [_dp] * 4
        L.xo_precond.argtypes = [C.c_int] * 3 + [_dp] * 6
        L.xo_forward.argtypes = [C.c_int] * 3 + [_dp] * 6
        L.xo_backward.argtypes = [C.c_int] * 3 + [_dp] * 6
        L.xo_pcg.argtypes = ([C.c_int] * 3 + [_dp] * 5 + [C.c_double, C.c_int, C.c_double, C.c_double,
                             _dp, C.POINTER(C.c_int), _dp])
        L.xo_pcg.restype = C.c_int
        L.xo_apply.argtypes = [C.c_int] * 3 + [_u8] + [_dp] * 7
        L.xo_apply_T.argtypes = [C.c_int] * 3 + [_u8] + [_dp] * 7
        L.xo_rhs_T.argtypes = [C.c_int] * 3 + [_u8] + [_dp] * 7
        L.xo_divergence_ref.argtypes = [C.c_int] * 3 + [_u8] + [_dp] * 4
        L.xo_project.argtypes = ([C.c_int] * 3 + [_u8] + [_dp] * 6 + [C.c_double, C.c_int, _dp,
                                 C.POINTER(C.c_int), _dp])
        L.xo_project.restype = C.c_int
        L.xo_assemble_normal.argtypes = [C.c_int] * 3 + [_u8] + [_dp] * 8
        L.xo_apply_normal.argtypes = [C.c_int] * 3 + [_u8] + [_dp] * 4
        L.xo_project_normal.argtypes = ([C.c_int] * 3 + [_u8] + [_dp] * 3 + [C.c_double, C.c_int, _dp,
                                        C.POINTER(C.c_int), _dp])
        L.xo_project_normal.restype = C.c_int
        L.xo_apply_forces.argtypes = [C.c_int] * 3 + [_u8] + [_dp] * 3 + [C.c_double] * 4
        L.xo_advect_particles.argtypes = ([C.c_int] * 3 + [C.c_double, _u8] + [_dp] * 6 +
                                          [C.c_double, C.c_double, C.c_longlong, _dp, C.POINTER(C.c_int)])
        L.xo_p2g.argtypes = [C.c_int] * 3 + [C.c_double, C.c_longlong] + [_dp] * 4
        L.xo_update_material.argtypes = [C.c_int] * 3 + [C.c_double, C.c_longlong, _dp, _u8]
        L.xo_distance_field.argtypes = ([C.c_int] * 3 + [C.c_double, C.c_int, C.c_double, C.c_double,
                                        C.c_longlong, _dp, _dp, _u8])
        L.xo_extrapolate.argtypes = [C.c_int] * 3 + [_u8] + [_dp] * 3 + [C.c_int]

    @staticmethod
    def _dims(sc):
        return sc.ni, sc.nj, sc.nk

    def assemble(self, sc):
        n = (sc.nk, sc.nj, sc.ni)
        out = [np.zeros(n) for _ in range(5)]
        u, v, w, wu, wv, ww = map(_f64, (sc.u, sc.v, sc.w, sc.wu, sc.wv, sc.ww))
        self.lib.xo_assemble(*self._dims(sc), _p(np.ascontiguousarray(sc.mat)), _p(u), _p(v), _p(w),
                             _p(wu), _p(wv), _p(ww), *[_p(a) for a in out])
        return dict(zip(("diag", "ax", "ay", "az", "b"), out))

    def spmv(self, sc, A, s):
        z = np.zeros_like(A["diag"])
        self.lib.xo_spmv(*self._dims(sc), _p(A["diag"]), _p(A["ax"]), _p(A["ay"]), _p(A["az"]),
                         _p(_f64(s)), _p(z))
        return z

    def factor(self, sc, A, omega=0.97, ratio=0.25):
        out = [np.zeros_like(A["diag"]) for _ in range(4)]
        self.lib.xo_factor(*self._dims(sc), _p(A["diag"]), _p(A["ax"]), _p(A["ay"]), _p(A["az"]),
                           omega, ratio, *[_p(a) for a in out])
        return dict(zip(("inv", "lx", "ly", "lz"), out))

    def precond(self, sc, F, r):
        z = np.zeros_like(F["inv"])
        self.lib.xo_precond(*self._dims(sc), _p(F["inv"]), _p(F["lx"]), _p(F["ly"]), _p(F["lz"]),
                            _p(_f64(r)), _p(z))
        return z

    def forward(self, sc, F, r):
        y = np.zeros_like(F["inv"])
        self.lib.xo_forward(*self._dims(sc), _p(F["inv"]), _p(F["lx"]), _p(F["ly"]), _p(F["lz"]),
                            _p(_f64(r)), _p(y))
        return y

    def backward(self, sc, F, y):
        z = np.zeros_like(F["inv"])
        self.lib.xo_backward(*self._dims(sc), _p(F["inv"]), _p(F["lx"]), _p(F["ly"]), _p(F["lz"]),
                             _p(_f64(y)), _p(z))
        return z

    def pcg(self, sc, A, tol=1e-6, maxit=200, omega=0.97, ratio=0.25):
        x = np.zeros_like(A["diag"])
        it = C.c_int(0)
        res = C.c_double(0)
        ok = self.lib.xo_pcg(*self._dims(sc), _p(A["diag"]), _p(A["ax"]), _p(A["ay"]), _p(A["az"]),
                             _p(A["b"]), tol, maxit, omega, ratio, _p(x), C.byref(it), C.byref(res))
        return dict(ok=bool(ok), p=x, iters=it.value, resid=res.value)

    def apply(self, sc, p):
        u, v, w = (np.array(a, dtype=np.float64) for a in (sc.u, sc.v, sc.w))
        wu, wv, ww = map(_f64, (sc.wu, sc.wv, sc.ww))
        self.lib.xo_apply(*self._dims(sc), _p(np.ascontiguousarray(sc.mat)), _p(wu), _p(wv), _p(ww),
                          _p(_f64(p)), _p(u), _p(v), _p(w))
        return u, v, w

    def apply_T(self, sc, gu, gv, gw):
        q = np.zeros((sc.nk, sc.nj, sc.ni))
        wu, wv, ww = map(_f64, (sc.wu, sc.wv, sc.ww))
        self.lib.xo_apply_T(*self._dims(sc), _p(np.ascontiguousarray(sc.mat)), _p(wu), _p(wv), _p(ww),
                            _p(_f64(gu)), _p(_f64(gv)), _p(_f64(gw)), _p(q))
        return q

    def rhs_T(self, sc, lam):
        gu = np.zeros(sc.u.shape); gv = np.zeros(sc.v.shape); gw = np.zeros(sc.w.shape)
        wu, wv, ww = map(_f64, (sc.wu, sc.wv, sc.ww))
        self.lib.xo_rhs_T(*self._dims(sc), _p(np.ascontiguousarray(sc.mat)), _p(wu), _p(wv), _p(ww),
                          _p(_f64(lam)), _p(gu), _p(gv), _p(gw))
        return gu, gv, gw

    def divergence_ref(self, sc, u, v, w):
        d = np.zeros((sc.nk, sc.nj, sc.ni))
        self.lib.xo_divergence_ref(*self._dims(sc), _p(np.ascontiguousarray(sc.mat)), _p(_f64(u)),
                                   _p(_f64(v)), _p(_f64(w)), _p(d))
        return d

    def project(self, sc, tol=1e-6, maxit=200):
        """Full projection (assemble, PCG, apply).  Returns dict with p, u, v, w."""
        u, v, w = (np.array(a, dtype=np.float64) for a in (sc.u, sc.v, sc.w))
        wu, wv, ww = map(_f64, (sc.wu, sc.wv, sc.ww))
        p = np.zeros((sc.nk, sc.nj, sc.ni))
        it = C.c_int(0)
        res = C.c_double(0)
        ok = self.lib.xo_project(*self._dims(sc), _p(np.ascontiguousarray(sc.mat)), _p(u), _p(v), _p(w),
                                 _p(wu), _p(wv), _p(ww), tol, maxit, _p(p), C.byref(it), C.byref(res))
        return dict(ok=bool(ok), p=p, u=u, v=v, w=w, iters=it.value, resid=res.value)

    # ---- the simulator steps either side of the projection ----
    def apply_forces(self, sc, force, dt, uvw=None):
        u, v, w = (np.array(a, dtype=np.float64) for a in (uvw or (sc.u, sc.v, sc.w)))
        self.lib.xo_apply_forces(*self._dims(sc), _p(np.ascontiguousarray(sc.mat)), _p(u), _p(v), _p(w),
                                 *map(float, force), float(dt))
        return u, v, w

    def extrapolate(self, sc, layers, uvw=None):
        u, v, w = (np.array(a, dtype=np.float64) for a in (uvw or (sc.u, sc.v, sc.w)))
        self.lib.xo_extrapolate(*self._dims(sc), _p(np.ascontiguousarray(sc.mat)), _p(u), _p(v), _p(w), int(layers))
        return u, v, w

    # ---- particle steps (oracle/xfp_particles_oracle.c) ----
    def advect_particles(self, sc, saved, parts, ratio, dt, dx, status=False):
        """_advectParticles steps a, b on the faces of sc (current) and `saved`;
        with status=True also the per-particle outcome (xo_advect_particles)."""
        out = _parts(parts).copy()
        g = [_f64(a) for a in (sc.u, sc.v, sc.w, *saved)]
        st = np.zeros(len(out), np.int32)
        self.lib.xo_advect_particles(*self._dims(sc), float(dx), _p(np.ascontiguousarray(sc.mat, np.uint8)),
                                     *map(_p, g), float(ratio), float(dt), len(out), _p(out),
                                     st.ctypes.data_as(C.POINTER(C.c_int)))
        return (out, st) if status else out

    def p2g(self, dims, dx, parts):
        ni, nj, nk = dims
        P = _parts(parts)
        u, v, w = np.zeros((nk, nj, ni + 1)), np.zeros((nk, nj + 1, ni)), np.zeros((nk + 1, nj, ni))
        self.lib.xo_p2g(ni, nj, nk, float(dx), len(P), _p(P), _p(u), _p(v), _p(w))
        return u, v, w

    def update_material(self, mat, dx, parts):
        nk, nj, ni = mat.shape
        P = _parts(parts)
        m = np.array(mat, np.uint8)
        self.lib.xo_update_material(ni, nj, nk, float(dx), len(P), _p(P), _p(m))
        return m

    def distance_field(self, mat, dx, subdiv, radius, threshold, parts):
        nk, nj, ni = mat.shape
        P = _parts(parts)
        s = int(subdiv)
        phi = np.zeros((nk * s + 1, nj * s + 1, ni * s + 1))
        m = np.array(mat, np.uint8)
        self.lib.xo_distance_field(ni, nj, nk, float(dx), s, float(radius), float(threshold), len(P), _p(P),
                                   _p(phi), _p(m))
        return phi, m

    # ---- NormalPressureSolver (classic Poisson matrix) ----
    def assemble_normal(self, sc):
        n = (sc.nk, sc.nj, sc.ni)
        out = [np.zeros(n) for _ in range(5)]
        u, v, w = map(_f64, (sc.u, sc.v, sc.w))
        self.lib.xo_assemble_normal(*self._dims(sc), _p(np.ascontiguousarray(sc.mat)), _p(u), _p(v), _p(w),
                                    *[_p(a) for a in out])
        return dict(zip(("diag", "ax", "ay", "az", "b"), out))

    def apply_normal(self, sc, p):
        u, v, w = (np.array(a, dtype=np.float64) for a in (sc.u, sc.v, sc.w))
        self.lib.xo_apply_normal(*self._dims(sc), _p(np.ascontiguousarray(sc.mat)), _p(_f64(p)), _p(u), _p(v),
                                 _p(w))
        return u, v, w

    def project_normal(self, sc, tol=1e-6, maxit=200):
        u, v, w = (np.array(a, dtype=np.float64) for a in (sc.u, sc.v, sc.w))
        p = np.zeros((sc.nk, sc.nj, sc.ni))
        it = C.c_int(0)
        res = C.c_double(0)
        ok = self.lib.xo_project_normal(*self._dims(sc), _p(np.ascontiguousarray(sc.mat)), _p(u), _p(v), _p(w),
                                        tol, maxit, _p(p), C.byref(it), C.byref(res))
        return dict(ok=bool(ok), p=p, u=u, v=v, w=w, iters=it.value, resid=res.value)

    def weighted_divergence(self, sc, u, v, w):
        """Per-cell m-weighted divergence that the projection drives to zero:
        the right-hand side b assembled from the given face velocities."""
        s2 = sc.copy()
        s2.u, s2.v, s2.w = u, v, w
        return self.assemble(s2)["b"]


class Reference(_Lib):
    """xFluid's own solver, built from the reference sources (oracle/_ref)."""

    def __init__(self):
        super().__init__(REF_LIB)
        L = self.lib
        L.xfref_solve.argtypes = ([C.c_int] * 3 + [_u8] + [_dp] * 3 + [C.c_double, C.c_int, _dp,
                                  C.POINTER(C.c_int), _dp])
        L.xfref_solve.restype = C.c_int
        L.xfref_project.argtypes = [C.c_int] * 3 + [_u8] + [_dp] * 3 + [C.c_double, C.c_int, _dp]
        L.xfref_project.restype = C.c_int
        L.xfref_apply.argtypes = [C.c_int] * 3 + [_u8] + [_dp] * 4
        L.xfref_set_threads.argtypes = [C.c_int]
        L.xfref_set_threads.restype = C.c_int
        L.xfref_time_apply.argtypes = [C.c_int] * 3 + [_u8] + [_dp] * 4 + [C.c_int, C.c_int]
        L.xfref_time_apply.restype = C.c_double
        L.xfref_assemble.argtypes = [C.c_int] * 3 + [_u8] + [_dp] * 8
        L.xfref_assemble.restype = C.c_int
        L.xfref_factor.argtypes = [C.c_int] * 3 + [_u8] + [_dp] * 7
        L.xfref_precond.argtypes = [C.c_int] * 3 + [_u8] + [_dp] * 5
        L.xfref_divergence.argtypes = [C.c_int] * 3 + [_u8] + [_dp] * 4

    def _normal_argtypes(self):
        L = self.lib
        L.xfref_normal_assemble.argtypes = [C.c_int] * 3 + [_u8] + [_dp] * 8
        L.xfref_normal_assemble.restype = C.c_int
        L.xfref_normal_solve.argtypes = ([C.c_int] * 3 + [_u8] + [_dp] * 3 + [C.c_double, C.c_int, _dp,
                                         C.POINTER(C.c_int), _dp])
        L.xfref_normal_solve.restype = C.c_int
        L.xfref_normal_apply.argtypes = [C.c_int] * 3 + [_u8] + [_dp] * 4

    def normal_assemble(self, sc):
        self._normal_argtypes()
        n = (sc.nk, sc.nj, sc.ni)
        out = [np.zeros(n) for _ in range(5)]
        self.lib.xfref_normal_assemble(*self._in(sc), *[_p(a) for a in out])
        return dict(zip(("diag", "ax", "ay", "az", "b"), out))

    def normal_solve(self, sc, tol=1e-6, maxit=200):
        self._normal_argtypes()
        p = np.zeros((sc.nk, sc.nj, sc.ni))
        it = C.c_int(0)
        res = C.c_double(0)
        ok = self.lib.xfref_normal_solve(*self._in(sc), tol, maxit, _p(p), C.byref(it), C.byref(res))
        return dict(ok=bool(ok), p=p, iters=it.value, resid=res.value)

    def normal_apply(self, sc, p):
        self._normal_argtypes()
        u, v, w = (np.array(a, dtype=np.float64) for a in (sc.u, sc.v, sc.w))
        self.lib.xfref_normal_apply(sc.ni, sc.nj, sc.nk, _p(np.ascontiguousarray(sc.mat)), _p(_f64(p)),
                                    _p(u), _p(v), _p(w))
        return u, v, w

    def _in(self, sc):
        return (sc.ni, sc.nj, sc.nk, _p(np.ascontiguousarray(sc.mat)), _p(_f64(sc.u)),
                _p(_f64(sc.v)), _p(_f64(sc.w)))

    def solve(self, sc, tol=1e-6, maxit=200):
        p = np.zeros((sc.nk, sc.nj, sc.ni))
        it = C.c_int(0)
        res = C.c_double(0)
        ok = self.lib.xfref_solve(*self._in(sc), tol, maxit, _p(p), C.byref(it), C.byref(res))
        return dict(ok=bool(ok), p=p, iters=it.value, resid=res.value)

    def project(self, sc, tol=1e-6, maxit=200):
        u, v, w = (np.array(a, dtype=np.float64) for a in (sc.u, sc.v, sc.w))
        p = np.zeros((sc.nk, sc.nj, sc.ni))
        ok = self.lib.xfref_project(sc.ni, sc.nj, sc.nk, _p(np.ascontiguousarray(sc.mat)), _p(u),
                                    _p(v), _p(w), tol, maxit, _p(p))
        return dict(ok=bool(ok), p=p, u=u, v=v, w=w)

    def set_threads(self, n: int) -> int:
        """OpenMP threads for the reference's parallel loops; returns the
        previous count (1 for a build without OpenMP)."""
        return int(self.lib.xfref_set_threads(int(n)))

    def time_apply(self, sc, p, threads: int, reps: int = 3) -> float:
        """Mean seconds of the reference's applyPressure on `threads` threads."""
        u, v, w = (np.array(a, dtype=np.float64) for a in (sc.u, sc.v, sc.w))
        return float(self.lib.xfref_time_apply(sc.ni, sc.nj, sc.nk, _p(np.ascontiguousarray(sc.mat, np.uint8)),
                                               _p(_f64(p)), _p(u), _p(v), _p(w), int(threads), int(reps)))

    def apply(self, sc, p):
        u, v, w = (np.array(a, dtype=np.float64) for a in (sc.u, sc.v, sc.w))
        self.lib.xfref_apply(sc.ni, sc.nj, sc.nk, _p(np.ascontiguousarray(sc.mat)), _p(_f64(p)),
                             _p(u), _p(v), _p(w))
        return u, v, w

    def assemble(self, sc):
        n = (sc.nk, sc.nj, sc.ni)
        out = [np.zeros(n) for _ in range(5)]
        maxrow = self.lib.xfref_assemble(*self._in(sc), *[_p(a) for a in out])
        d = dict(zip(("diag", "ax", "ay", "az", "b"), out))
        d["maxrow"] = maxrow
        return d

    def factor(self, sc):
        n = (sc.nk, sc.nj, sc.ni)
        out = [np.zeros(n) for _ in range(4)]
        self.lib.xfref_factor(*self._in(sc), *[_p(a) for a in out])
        return dict(zip(("inv", "lx", "ly", "lz"), out))

    def precond(self, sc, r):
        z = np.zeros((sc.nk, sc.nj, sc.ni))
        self.lib.xfref_precond(*self._in(sc), _p(_f64(r)), _p(z))
        return z

    def divergence(self, sc, u, v, w):
        d = np.zeros((sc.nk, sc.nj, sc.ni))
        self.lib.xfref_divergence(sc.ni, sc.nj, sc.nk, _p(np.ascontiguousarray(sc.mat)), _p(_f64(u)),
                                  _p(_f64(v)), _p(_f64(w)), _p(d))
        return d


class RefSim(_Lib):
    """xFluid's own FluidSimulator on the dam-break scene (oracle/_ref/libxfsim.so,
    oracle/sim_harness.cpp), stepped up to and through the projection."""

    def __init__(self, n=64, cfl=5.0, gravity=-9.8, tol=1e-6, maxit=200, boxes=None, spheres=()):
        """boxes: fluid boxes ((x0,y0,z0),(x1,y1,z1)) (default: the dam break);
        spheres: fluid spheres ((cx,cy,cz), r); unit-cube coordinates."""
        super().__init__(SIM_LIB)
        L = self.lib
        L.xfsim_create.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, C.c_int]
        L.xfsim_create.restype = C.c_void_p
        L.xfsim_add_box.argtypes = [C.c_void_p] + [C.c_double] * 6
        L.xfsim_add_sphere.argtypes = [C.c_void_p] + [C.c_double] * 4
        L.xfsim_init.argtypes = [C.c_void_p]
        L.xfsim_destroy.argtypes = [C.c_void_p]
        L.xfsim_begin_step.argtypes = [C.c_void_p, C.c_double, _u8, _dp, _dp, _dp]
        L.xfsim_begin_step.restype = C.c_double
        L.xfsim_project.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp, C.POINTER(C.c_int)]
        L.xfsim_project.restype = C.c_int
        L.xfsim_end_step.argtypes = [C.c_void_p]
        L.xfsim_fluid_cells.argtypes = [C.c_void_p]
        L.xfsim_fluid_cells.restype = C.c_int
        L.xfsim_particle_count.argtypes = [C.c_void_p]
        L.xfsim_particle_count.restype = C.c_longlong
        L.xfsim_particles.argtypes = [C.c_void_p, _dp]
        L.xfsim_fields.argtypes = [C.c_void_p, _u8, _dp, _dp, _dp]
        self.n = n
        self.h = L.xfsim_create(n, cfl, gravity, tol, maxit)
        for lo, hi in (boxes if boxes is not None else [((0.0, 0.0, 0.0), (0.4, 0.5, 1.0))]):
            L.xfsim_add_box(self.h, *lo, *hi)
        for c, r in spheres:
            L.xfsim_add_sphere(self.h, *c, r)
        L.xfsim_init(self.h)

    def close(self):
        if self.h:
            self.lib.xfsim_destroy(self.h)
            self.h = None

    def _shapes(self):
        n = self.n
        return (n, n, n), (n, n, n + 1), (n, n + 1, n), (n + 1, n, n)

    def begin_step(self, max_dt=1.0 / 30.0):
        """Runs the step up to the projection; returns (dt, mat, u, v, w)."""
        sm, su, sv, sw = self._shapes()
        mat = np.zeros(sm, np.uint8)
        u, v, w = np.zeros(su), np.zeros(sv), np.zeros(sw)
        dt = self.lib.xfsim_begin_step(self.h, max_dt, _p(mat), _p(u), _p(v), _p(w))
        return dt, mat, u, v, w

    def project(self, iterations=True):
        """The reference's own projection: (ok, pressure, u, v, w, iterations);
        iterations (a rerun of the same PCG) is -1 when not asked for."""
        sm, su, sv, sw = self._shapes()
        p = np.zeros(sm)
        u, v, w = np.zeros(su), np.zeros(sv), np.zeros(sw)
        it = C.c_int(-1)
        ok = self.lib.xfsim_project(self.h, _p(p), _p(u), _p(v), _p(w), C.byref(it) if iterations else None)
        return bool(ok), p, u, v, w, it.value

    def end_step(self):
        self.lib.xfsim_end_step(self.h)

    def fluid_cells(self):
        return self.lib.xfsim_fluid_cells(self.h)

    def particles(self):
        P = np.zeros((self.lib.xfsim_particle_count(self.h), 6))
        self.lib.xfsim_particles(self.h, _p(P))
        return P

    def fields(self):
        """The current (material, u, v, w), without stepping."""
        sm, su, sv, sw = self._shapes()
        mat = np.zeros(sm, np.uint8)
        u, v, w = np.zeros(su), np.zeros(sv), np.zeros(sw)
        self.lib.xfsim_fields(self.h, _p(mat), _p(u), _p(v), _p(w))
        return mat, u, v, w


class RefSimDropIn(_Lib):
    """xFluid's own FluidSimulator built with this project's solver class as
    its pressure-solver member (oracle/_ref/libxfsim_dropin.so,
    oracle/sim_dropin_harness.cpp): the dam break, stepped as RefSim steps the
    stock build, with the simulator's own _solvePressure calling the library."""

    def __init__(self, n=64, cfl=5.0, gravity=-9.8, tol=1e-6, maxit=200):
        super().__init__(DROPIN_LIB)
        L = self.lib
        L.xfsd_solver_type.restype = C.c_char_p
        L.xfsd_create_dam.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, C.c_int]
        L.xfsd_create_dam.restype = C.c_void_p
        L.xfsd_destroy.argtypes = [C.c_void_p]
        L.xfsd_begin_step.argtypes = [C.c_void_p, C.c_double, _u8, _dp, _dp, _dp]
        L.xfsd_begin_step.restype = C.c_double
        L.xfsd_project.argtypes = [C.c_void_p, _dp, _dp, _dp, C.POINTER(C.c_int)]
        L.xfsd_project.restype = C.c_int
        L.xfsd_end_step.argtypes = [C.c_void_p]
        L.xfsd_particle_count.argtypes = [C.c_void_p]
        L.xfsd_particle_count.restype = C.c_longlong
        L.xfsd_particles.argtypes = [C.c_void_p, _dp]
        self.n = n
        self.solver_type = L.xfsd_solver_type().decode()
        self.h = L.xfsd_create_dam(n, cfl, gravity, tol, maxit)

    def close(self):
        if self.h:
            self.lib.xfsd_destroy(self.h)
            self.h = None

    def begin_step(self, max_dt=1.0 / 30.0):
        n = self.n
        mat = np.zeros((n, n, n), np.uint8)
        u, v, w = np.zeros((n, n, n + 1)), np.zeros((n, n + 1, n)), np.zeros((n + 1, n, n))
        dt = self.lib.xfsd_begin_step(self.h, max_dt, _p(mat), _p(u), _p(v), _p(w))
        return dt, mat, u, v, w

    def project(self):
        """The simulator's _solvePressure through the library: (status, u, v, w, iterations)."""
        n = self.n
        u, v, w = np.zeros((n, n, n + 1)), np.zeros((n, n + 1, n)), np.zeros((n + 1, n, n))
        it = C.c_int(-1)
        rc = self.lib.xfsd_project(self.h, _p(u), _p(v), _p(w), C.byref(it))
        return rc, u, v, w, it.value

    def end_step(self):
        self.lib.xfsd_end_step(self.h)

    def particles(self):
        P = np.zeros((self.lib.xfsd_particle_count(self.h), 6))
        self.lib.xfsd_particles(self.h, _p(P))
        return P


class RefSteps(_Lib):
    """xFluid's own FluidSimulator::_applyForces and _expolateVelocity on given
    arrays (oracle/sim_harness.cpp, built from the reference sources)."""

    def __init__(self):
        super().__init__(SIM_LIB)
        L = self.lib
        L.xfsim_apply_forces.argtypes = [C.c_int] * 3 + [_u8] + [_dp] * 3 + [C.c_double] * 4
        L.xfsim_extrapolate.argtypes = [C.c_int] * 3 + [_u8] + [_dp] * 3 + [C.c_int]
        L.xfsim_advect_particles.argtypes = ([C.c_int] * 3 + [C.c_double, _u8] + [_dp] * 6 +
                                             [C.c_double, C.c_double, C.c_longlong, _dp] + [_dp] * 3)
        L.xfsim_p2g.argtypes = [C.c_int] * 3 + [C.c_double, C.c_longlong] + [_dp] * 4
        L.xfsim_material.argtypes = ([C.c_int] * 3 + [C.c_double, C.c_int, C.c_double, C.c_double,
                                     C.c_longlong, _dp, _u8, _dp, _u8, _u8])

    def apply_forces(self, sc, force, dt, uvw=None):
        u, v, w = (np.array(a, dtype=np.float64) for a in (uvw or (sc.u, sc.v, sc.w)))
        self.lib.xfsim_apply_forces(sc.ni, sc.nj, sc.nk, _p(np.ascontiguousarray(sc.mat)), _p(u), _p(v), _p(w),
                                    *map(float, force), float(dt))
        return u, v, w

    def extrapolate(self, sc, layers, uvw=None):
        u, v, w = (np.array(a, dtype=np.float64) for a in (uvw or (sc.u, sc.v, sc.w)))
        self.lib.xfsim_extrapolate(sc.ni, sc.nj, sc.nk, _p(np.ascontiguousarray(sc.mat)), _p(u), _p(v), _p(w),
                                   int(layers))
        return u, v, w

    def advect_particles(self, sc, saved, parts, ratio, dt, dx, grids=False):
        """The reference's _advectParticles(dt) (steps a, b, then its own P2G);
        returns the particles, and with grids=True also the faces after P2G."""
        out = _parts(parts).copy()
        g = [_f64(a) for a in (sc.u, sc.v, sc.w, *saved)]
        u, v, w = (np.zeros_like(a) for a in g[:3])
        self.lib.xfsim_advect_particles(sc.ni, sc.nj, sc.nk, float(dx), _p(np.ascontiguousarray(sc.mat, np.uint8)),
                                        *map(_p, g), float(ratio), float(dt), len(out), _p(out), _p(u), _p(v), _p(w))
        return (out, (u, v, w)) if grids else out

    def p2g(self, dims, dx, parts):
        ni, nj, nk = dims
        P = _parts(parts)
        u, v, w = np.zeros((nk, nj, ni + 1)), np.zeros((nk, nj + 1, ni)), np.zeros((nk + 1, nj, ni))
        self.lib.xfsim_p2g(ni, nj, nk, float(dx), len(P), _p(P), _p(u), _p(v), _p(w))
        return u, v, w

    def material(self, mat, dx, subdiv, radius, threshold, parts):
        """updateFeild + updateSurfaceInfo, then _updateMaterial: (phi, material
        after updateSurfaceInfo, material after _updateMaterial)."""
        nk, nj, ni = mat.shape
        P = _parts(parts)
        s = int(subdiv)
        phi = np.zeros((nk * s + 1, nj * s + 1, ni * s + 1))
        m0 = np.ascontiguousarray(mat, np.uint8)
        ms, mf = np.zeros_like(m0), np.zeros_like(m0)
        self.lib.xfsim_material(ni, nj, nk, float(dx), s, float(radius), float(threshold), len(P), _p(P), _p(m0),
                                _p(phi), _p(ms), _p(mf))
        return phi, ms, mf
