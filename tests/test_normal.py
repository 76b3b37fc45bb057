"""xFluid's NormalPressureSolver (pressuresolver.cpp: the classic Poisson matrix
and its applyPressure) as the library's second matrix mode, XFP_MATRIX_NORMAL.

The oracle's C restatement is pinned bitwise to golden vectors that the
reference's own NormalPressureSolver produced (tests/golden/make_golden.py) and,
where the reference build is present, to that build on further seeded scenes.
The CUDA path is then checked through the C ABI against those vectors: FP64 to
1e-12 relative with the reference's iteration count, mixed precision and FP32
to 1e-4 against the FP64 oracle, and the normal mode's argument rules."""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

import oracle
from xfluid_b200 import scenes

GOLDEN = Path(__file__).parent / "golden"
CASES = ["normal_dam16.npz", "normal_blob24x20x22.npz"]


def _scene(z):
    ni, nj, nk = (int(x) for x in z["dims"])
    return scenes.Scene(ni, nj, nk, z["mat"], z["u"], z["v"], z["w"])


def _rel(a, b):
    d = np.linalg.norm(b)
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / (d if d > 0 else 1.0))


@pytest.mark.parametrize("name", CASES)
def test_oracle_normal_matches_reference_golden_vectors(name):
    z = np.load(GOLDEN / name)
    sc = _scene(z)
    O = oracle.Oracle()
    A = O.assemble_normal(sc)
    for k in ("diag", "ax", "ay", "az", "b"):
        assert np.array_equal(A[k], z[k]), k
    r = O.project_normal(sc, tol=float(z["tol"]), maxit=int(z["maxit"]))
    assert r["ok"] and r["iters"] == int(z["iters"])
    assert np.array_equal(r["p"], z["p"])
    for a, k in zip((r["u"], r["v"], r["w"]), ("u_out", "v_out", "w_out")):
        assert np.array_equal(a, z[k]), k


@pytest.mark.skipif(not oracle.reference_available(), reason="reference build absent (oracle/_ref)")
@pytest.mark.parametrize("seed,dims", [(3, (19, 23, 17)), (4, (31, 12, 25))])
def test_oracle_normal_matches_reference_build(seed, dims):
    sc = scenes.blob_scene(dims=dims, seed=seed, fractional=False, dtype=np.float64)
    O, R = oracle.Oracle(), oracle.Reference()
    a, r = O.assemble_normal(sc), R.normal_assemble(sc)
    for k in ("diag", "ax", "ay", "az", "b"):
        assert np.array_equal(a[k], r[k]), k
    ro, po = R.normal_solve(sc, tol=1e-8, maxit=500), O.project_normal(sc, tol=1e-8, maxit=500)
    assert ro["ok"] and po["ok"] and ro["iters"] == po["iters"]
    assert np.array_equal(ro["p"], po["p"])
    p = np.random.default_rng(seed).standard_normal(sc.mat.shape)
    for x, y in zip(O.apply_normal(sc, p), R.normal_apply(sc, p)):
        assert np.array_equal(x, y)


def _ctx(prec, **kw):
    from gpu_util import make_ctx
    from xfluid_b200 import _lib
    return make_ctx(prec, matrix=_lib.MATRIX["normal"], **kw)


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_gpu_normal_fp64_matches_reference_vectors(name):
    from gpu_util import project
    z = np.load(GOLDEN / name)
    sc = _scene(z)
    ctx = _ctx("f64", tol=float(z["tol"]), max_iter=int(z["maxit"]))
    try:
        rc, p, u, v, w, st = project(ctx, sc, dtype=np.float64, fractional=False)
    finally:
        ctx.close()
    assert rc == 0
    assert abs(st["iterations"] - int(z["iters"])) <= 1, (st["iterations"], int(z["iters"]))
    assert _rel(p, z["p"]) <= 1e-12, _rel(p, z["p"])
    for a, k in zip((u, v, w), ("u_out", "v_out", "w_out")):
        assert _rel(a, z[k]) <= 1e-12, (k, _rel(a, z[k]))


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["mixed", "f32"])
def test_gpu_normal_reduced_precision_vs_fp64_oracle(prec):
    from gpu_util import project
    sc = scenes.blob_scene(dims=(48, 40, 44), seed=11, fractional=False, dtype=np.float32)
    ref = oracle.Oracle().project_normal(sc, tol=1e-6, maxit=2000)
    ctx = _ctx(prec, tol=1e-6, max_iter=2000)
    try:
        rc, p, u, v, w, st = project(ctx, sc, dtype=np.float32, fractional=False)
    finally:
        ctx.close()
    assert rc == 0 and ref["ok"]
    assert _rel(p, ref["p"]) <= 1e-4, _rel(p, ref["p"])
    assert max(_rel(a, ref[k]) for a, k in zip((u, v, w), "uvw")) <= 1e-4


@pytest.mark.gpu
def test_gpu_normal_mode_argument_rules():
    """Face weights are refused (the reference class has none); the batch and
    backward entry points report XFP_ERR_UNSUPPORTED for the normal matrix."""
    from gpu_util import ptr
    from xfluid_b200 import _lib
    sc = scenes.blob_scene(dims=(12, 10, 9), seed=2, fractional=False, dtype=np.float64)
    ni, nj, nk = sc.ni, sc.nj, sc.nk
    mat = np.ascontiguousarray(sc.mat, np.uint8)
    u, v, w = (np.array(a, np.float64) for a in (sc.u, sc.v, sc.w))
    ones = [np.ones_like(a) for a in (u, v, w)]
    p = np.zeros((nk, nj, ni))
    ctx = _ctx("f64")
    try:
        st = _lib.XfpStats()
        rc = ctx.lib.xfp_project_f64(ctx.ptr, ni, nj, nk, ptr(mat), ptr(u), ptr(v), ptr(w), *map(ptr, ones),
                                     ptr(p), C.byref(st))
        assert rc == _lib.XFP_ERR_ARGS and "face weights" in ctx.last_error()
        rc = ctx.lib.xfp_apply_pressure_f64(ctx.ptr, ni, nj, nk, ptr(mat), *map(ptr, ones), ptr(p), ptr(u),
                                            ptr(v), ptr(w))
        assert rc == _lib.XFP_ERR_ARGS
        g = [np.zeros_like(a) for a in (u, v, w)]
        d = [np.zeros_like(a) for a in (u, v, w)]
        rc = ctx.lib.xfp_project_backward_f64(ctx.ptr, ni, nj, nk, ptr(mat), None, None, None, *map(ptr, g),
                                              *map(ptr, d), C.byref(st))
        assert rc == _lib.XFP_ERR_UNSUPPORTED
        scn = _lib.XfpScene(ni, nj, nk, mat.ctypes.data, u.ctypes.data, v.ctypes.data, w.ctypes.data,
                            None, None, None, p.ctypes.data)
        arr = (_lib.XfpScene * 1)(scn)
        sts = (_lib.XfpStats * 1)()
        rc = ctx.lib.xfp_project_batch_f64(ctx.ptr, 1, arr, sts)
        assert rc == _lib.XFP_ERR_UNSUPPORTED
        # the context still projects afterwards
        rc = ctx.lib.xfp_project_f64(ctx.ptr, ni, nj, nk, ptr(mat), ptr(u), ptr(v), ptr(w), None, None, None,
                                     ptr(p), C.byref(st))
        assert rc == 0
    finally:
        ctx.close()


@pytest.mark.gpu
def test_python_normal_solver_mirrors_the_reference_class():
    """NormalPressureSolver's nine methods drive the normal mode: solve then
    applyPressure on numpy arrays match the FP64 oracle's projection."""
    from xfluid_b200.solver import NormalPressureSolver
    sc = scenes.dam_break(dims=(20, 16, 14), seed=3, noise=0.3)
    ref = oracle.Oracle().project_normal(sc, tol=1e-9, maxit=500)
    s = NormalPressureSolver(precision="f64", tol=1e-9, max_iter=500)
    try:
        u, v, w = (np.array(a, np.float64) for a in (sc.u, sc.v, sc.w))
        s.setSize(sc.ni, sc.nj, sc.nk)
        s.setMaterial(np.ascontiguousarray(sc.mat, np.uint8))
        s.setVelocityField(u, v, w)
        s.setDensity(1.0)
        s.setDt(0.01)
        s.setDx(1.0 / sc.ni)
        s.setDisField(None)
        p = np.zeros((sc.nk, sc.nj, sc.ni))
        assert s.solve(p)
        assert s.applyPressure(p)
        with pytest.raises(ValueError):
            s.setFaceWeights(u, v, w)
    finally:
        s._ctx.close()
    assert _rel(p, ref["p"]) <= 1e-9
    # all faces together: at a solid face the reference forms u - ((p1 + u) - p1),
    # a rounding residue of p's size that differs with p's last bits, so a
    # component that is nearly zero everywhere is not compared on its own
    got = np.concatenate([a.ravel() for a in (u, v, w)])
    want = np.concatenate([ref[k].ravel() for k in "uvw"])
    assert _rel(got, want) <= 1e-9, _rel(got, want)
