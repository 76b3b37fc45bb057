"""The simulator steps either side of the projection: xFluid's
FluidSimulator::_applyForces (the constant body force) before it and
_expolateVelocity (layered velocity extrapolation) after it
(FluidSimulator.cpp:429-499, 511-650), and the fused call that does both around
one projection (xfp_project_step_*).

The oracle's C restatement is pinned bitwise to golden vectors produced by the
reference's own simulator code (tests/golden/make_golden.py, the steps_*.npz
fixtures) and, where that build is present, to it on further seeded scenes.
The CUDA path is checked through the C ABI: the separate steps bitwise in
FP64, the fused step against the reference's forces -> projection ->
extrapolation to 1e-12 and bitwise against the same three GPU calls made one
after another, and FP32 to 1e-5 against the FP64 oracle."""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

import oracle
from xfluid_b200 import scenes

GOLDEN = Path(__file__).parent / "golden" / "steps_dam20x14x18.npz"


def _scene(z):
    ni, nj, nk = (int(x) for x in z["dims"])
    return scenes.Scene(ni, nj, nk, z["mat"], z["u"], z["v"], z["w"])


def _rel(a, b):
    d = np.linalg.norm(b)
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / (d if d > 0 else 1.0))


def test_oracle_steps_match_reference_golden_vectors():
    z = np.load(GOLDEN)
    sc = _scene(z)
    O = oracle.Oracle()
    f = O.apply_forces(sc, z["force"], float(z["dt"]))
    for a, k in zip(f, ("u_forced", "v_forced", "w_forced")):
        assert np.array_equal(a, z[k]), k
    e = O.extrapolate(sc, int(z["layers"]))
    for a, k in zip(e, ("u_extrap", "v_extrap", "w_extrap")):
        assert np.array_equal(a, z[k]), k
    s2 = sc.copy()
    s2.u, s2.v, s2.w = f
    pr = O.project(s2, float(z["tol"]), int(z["maxit"]))
    assert np.array_equal(pr["p"], z["p_step"])
    st = O.extrapolate(sc, int(z["layers"]), uvw=(pr["u"], pr["v"], pr["w"]))
    for a, k in zip(st, ("u_step", "v_step", "w_step")):
        assert np.array_equal(a, z[k]), k


@pytest.mark.skipif(not oracle.sim_available(), reason="reference simulator build absent (oracle/_ref)")
@pytest.mark.parametrize("seed,dims,layers", [(4, (17, 21, 15), 3), (5, (26, 11, 19), 10)])
def test_oracle_steps_match_reference_build(seed, dims, layers):
    sc = scenes.dam_break(dims=dims, seed=seed, noise=0.4)
    O, R = oracle.Oracle(), oracle.RefSteps()
    for force in ((0.0, -9.8, 0.0), (1.5, 0.0, -2.0), (0.0, 5e-9, 0.0)):
        for x, y in zip(O.apply_forces(sc, force, 0.02), R.apply_forces(sc, force, 0.02)):
            assert np.array_equal(x, y), force
    for x, y in zip(O.extrapolate(sc, layers), R.extrapolate(sc, layers)):
        assert np.array_equal(x, y)


def _ctx(prec, **kw):
    from gpu_util import make_ctx
    return make_ctx(prec, **kw)


def _arrays(sc, dtype):
    mat = np.ascontiguousarray(sc.mat, np.uint8)
    return mat, [np.array(a, dtype) for a in (sc.u, sc.v, sc.w)]


@pytest.mark.gpu
def test_gpu_forces_and_extrapolation_are_bit_identical_in_fp64():
    from gpu_util import ptr
    z = np.load(GOLDEN)
    sc = _scene(z)
    ctx = _ctx("f64")
    try:
        mat, uvw = _arrays(sc, np.float64)
        f3 = (C.c_double * 3)(*z["force"])
        ctx.check(ctx.lib.xfp_apply_forces_f64(ctx.ptr, sc.ni, sc.nj, sc.nk, ptr(mat), *map(ptr, uvw), f3,
                                               float(z["dt"])))
        for a, k in zip(uvw, ("u_forced", "v_forced", "w_forced")):
            assert np.array_equal(a, z[k]), k
        mat, uvw = _arrays(sc, np.float64)
        ctx.check(ctx.lib.xfp_extrapolate_f64(ctx.ptr, sc.ni, sc.nj, sc.nk, ptr(mat), *map(ptr, uvw),
                                              int(z["layers"])))
        for a, k in zip(uvw, ("u_extrap", "v_extrap", "w_extrap")):
            assert np.array_equal(a, z[k]), k
    finally:
        ctx.close()


@pytest.mark.gpu
def test_gpu_fused_step_matches_reference_sequence_and_separate_calls():
    from gpu_util import ptr
    from xfluid_b200 import _lib
    z = np.load(GOLDEN)
    sc = _scene(z)
    f3 = (C.c_double * 3)(*z["force"])
    dt, layers = float(z["dt"]), int(z["layers"])
    ctx = _ctx("f64", tol=float(z["tol"]), max_iter=int(z["maxit"]))
    try:
        mat, uvw = _arrays(sc, np.float64)
        p = np.zeros((sc.nk, sc.nj, sc.ni))
        st = _lib.XfpStats()
        ctx.check(ctx.lib.xfp_project_step_f64(ctx.ptr, sc.ni, sc.nj, sc.nk, ptr(mat), *map(ptr, uvw), None, None,
                                               None, ptr(p), f3, dt, layers, C.byref(st)))
        assert _rel(p, z["p_step"]) <= 1e-12
        for a, k in zip(uvw, ("u_step", "v_step", "w_step")):
            assert _rel(a, z[k]) <= 1e-12, (k, _rel(a, z[k]))
        # the same three steps as separate calls give the same bits
        mat, sep = _arrays(sc, np.float64)
        p2 = np.zeros_like(p)
        ctx.check(ctx.lib.xfp_apply_forces_f64(ctx.ptr, sc.ni, sc.nj, sc.nk, ptr(mat), *map(ptr, sep), f3, dt))
        ctx.check(ctx.lib.xfp_project_f64(ctx.ptr, sc.ni, sc.nj, sc.nk, ptr(mat), *map(ptr, sep), None, None, None,
                                          ptr(p2), C.byref(st)))
        ctx.check(ctx.lib.xfp_extrapolate_f64(ctx.ptr, sc.ni, sc.nj, sc.nk, ptr(mat), *map(ptr, sep), layers))
        assert np.array_equal(p, p2)
        for a, b in zip(uvw, sep):
            assert np.array_equal(a, b)
        assert ctx.lib.xfp_extrapolate_f64(ctx.ptr, sc.ni, sc.nj, sc.nk, ptr(mat), *map(ptr, sep), -1) \
            == _lib.XFP_ERR_ARGS
    finally:
        ctx.close()


@pytest.mark.gpu
def test_gpu_fp32_step_and_python_methods_vs_fp64_oracle():
    from xfluid_b200.solver import VariationalPressureSolver
    sc = scenes.dam_break(dims=(30, 26, 22), seed=7, noise=0.3)
    force, dt, layers = (0.0, -9.8, 0.5), 0.02, 8
    O = oracle.Oracle()
    f = O.apply_forces(sc, force, dt)
    s2 = sc.copy()
    s2.u, s2.v, s2.w = f
    pr = O.project(s2, 1e-7, 1000)
    ref = O.extrapolate(sc, layers, uvw=(pr["u"], pr["v"], pr["w"]))
    s = VariationalPressureSolver(precision="f32", tol=1e-7, max_iter=1000)
    try:
        u, v, w = (np.array(a, np.float32) for a in (sc.u, sc.v, sc.w))
        s.setSize(sc.ni, sc.nj, sc.nk)
        s.setMaterial(np.ascontiguousarray(sc.mat, np.uint8))
        s.setVelocityField(u, v, w)
        p = np.zeros((sc.nk, sc.nj, sc.ni), np.float32)
        assert s.projectStep(p, force, dt, layers)
    finally:
        s._ctx.close()
    assert _rel(p, pr["p"]) <= 1e-5, _rel(p, pr["p"])
    got = np.concatenate([a.ravel() for a in (u, v, w)])
    want = np.concatenate([a.ravel() for a in ref])
    assert _rel(got, want) <= 1e-5, _rel(got, want)
    # the separate Python methods (FP64) reproduce the oracle's forces and extrapolation
    s = VariationalPressureSolver(precision="f64")
    try:
        u, v, w = (np.array(a, np.float64) for a in (sc.u, sc.v, sc.w))
        s.setSize(sc.ni, sc.nj, sc.nk)
        s.setMaterial(np.ascontiguousarray(sc.mat, np.uint8))
        s.setVelocityField(u, v, w)
        s.applyForces(force, dt)
        for a, b in zip((u, v, w), f):
            assert np.array_equal(a, b)
        s.extrapolateVelocity(layers)
        for a, b in zip((u, v, w), O.extrapolate(sc, layers, uvw=f)):
            assert np.array_equal(a, b)
    finally:
        s._ctx.close()
