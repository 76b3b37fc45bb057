"""Helpers for the GPU tests: direct calls through the C ABI (libxfp.so)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from xfluid_b200 import _lib


def ptr(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


def f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


def make_ctx(precision="f64", **kw):
    o = _lib.default_options()
    o.precision = _lib.PREC[precision]
    for k, v in kw.items():
        setattr(o, k, v)
    return _lib.Context(o)


def debug_stages(ctx, sc, r=None, fractional=False):
    """Dense internal stages (assembly, factor, M^-1 r, A r) from the GPU."""
    shp = (sc.nk, sc.nj, sc.ni)
    names = ("diag", "ax", "ay", "az", "b", "inv", "lx", "ly", "lz", "y", "z", "q")
    out = {k: np.zeros(shp) for k in names}
    w = (sc.wu, sc.wv, sc.ww) if fractional else (None, None, None)
    args = [ptr(np.ascontiguousarray(sc.mat, np.uint8)), *(ptr(f64(a)) for a in (sc.u, sc.v, sc.w)),
            *(ptr(f64(a)) for a in w), ptr(f64(r))]
    keep = [f64(a) for a in (sc.u, sc.v, sc.w, *w, r)]  # noqa: F841 (keep buffers alive)
    rc = ctx.lib.xfp_debug_stages(ctx.ptr, sc.ni, sc.nj, sc.nk, *args, *(ptr(out[k]) for k in names))
    ctx.check(rc)
    return out


def project(ctx, sc, dtype=np.float64, fractional=True, with_pressure=True):
    """xfp_project_{f64,f32} with host pointers; returns (rc, p, u, v, w, stats)."""
    u, v, w = (np.array(a, dtype=dtype) for a in (sc.u, sc.v, sc.w))
    wts = (sc.wu, sc.wv, sc.ww) if (fractional and sc.wu is not None) else (None, None, None)
    wts = [None if a is None else np.ascontiguousarray(a, dtype=dtype) for a in wts]
    p = np.zeros((sc.nk, sc.nj, sc.ni), dtype=dtype) if with_pressure else None
    st = _lib.XfpStats()
    fn = ctx.lib.xfp_project_f64 if dtype == np.float64 else ctx.lib.xfp_project_f32
    rc = fn(ctx.ptr, sc.ni, sc.nj, sc.nk, ptr(np.ascontiguousarray(sc.mat, np.uint8)), ptr(u), ptr(v), ptr(w),
            *(ptr(a) for a in wts), ptr(p), C.byref(st))
    ctx.check(rc)
    return rc, p, u, v, w, st.as_dict()


def solve(ctx, sc, dtype=np.float64, fractional=True):
    u, v, w = (np.ascontiguousarray(a, dtype=dtype) for a in (sc.u, sc.v, sc.w))
    wts = (sc.wu, sc.wv, sc.ww) if (fractional and sc.wu is not None) else (None, None, None)
    wts = [None if a is None else np.ascontiguousarray(a, dtype=dtype) for a in wts]
    p = np.zeros((sc.nk, sc.nj, sc.ni), dtype=dtype)
    st = _lib.XfpStats()
    fn = ctx.lib.xfp_solve_f64 if dtype == np.float64 else ctx.lib.xfp_solve_f32
    rc = fn(ctx.ptr, sc.ni, sc.nj, sc.nk, ptr(np.ascontiguousarray(sc.mat, np.uint8)), ptr(u), ptr(v), ptr(w),
            *(ptr(a) for a in wts), ptr(p), C.byref(st))
    ctx.check(rc)
    return rc, p, st.as_dict()


def set_tol(ctx, tol, maxit, **kw):
    o = ctx.opts
    o.tol, o.max_iter = tol, maxit
    for k, v in kw.items():
        setattr(o, k, v)
    ctx.set_options(o)


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    d = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (d if d > 0 else 1.0))


def bits_equal(a, b):
    """Bit-identical FP64 arrays, except that -0.0 and +0.0 compare equal (the
    reference keeps the sign of zero in rows without an unknown; the GPU
    output grid holds +0.0 there)."""
    a = np.ascontiguousarray(a, dtype=np.float64) + 0.0
    b = np.ascontiguousarray(b, dtype=np.float64) + 0.0
    return a.shape == b.shape and np.array_equal(a.view(np.uint64), b.view(np.uint64))
