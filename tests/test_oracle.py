"""The CPU oracle (oracle/xfp_oracle.c) pinned against xFluid's own solver.

Bit-exact checks use the golden vectors in tests/golden/, produced by running
the reference code (tests/golden/make_golden.py).  Fractional face weights have
no reference counterpart; they are checked through properties the variational
system must have and against scipy.
"""
import numpy as np
import pytest

from golden_io import CASES, bits_equal, load
from xfluid_b200 import scenes


@pytest.mark.parametrize("name", CASES)
def test_assembly_matches_reference_bitwise(oracle_lib, name):
    sc, g = load(name)
    A = oracle_lib.assemble(sc)
    assert int(g["maxrow"]) <= 7
    for k in ("diag", "ax", "ay", "az", "b"):
        assert bits_equal(A[k], g[k]), k


@pytest.mark.parametrize("name", CASES)
def test_mic0_factor_matches_reference_bitwise(oracle_lib, name):
    sc, g = load(name)
    F = oracle_lib.factor(sc, oracle_lib.assemble(sc))
    for k in ("inv", "lx", "ly", "lz"):
        assert bits_equal(F[k], g[k]), k


@pytest.mark.parametrize("name", CASES)
def test_preconditioner_matches_reference_bitwise(oracle_lib, name):
    sc, g = load(name)
    F = oracle_lib.factor(sc, oracle_lib.assemble(sc))
    assert bits_equal(oracle_lib.precond(sc, F, g["r"]), g["z"])


@pytest.mark.parametrize("name", CASES)
def test_pcg_matches_reference_bitwise(oracle_lib, name):
    sc, g = load(name)
    sol = oracle_lib.pcg(sc, oracle_lib.assemble(sc), float(g["tol"]), int(g["maxit"]))
    assert sol["ok"]
    assert sol["iters"] == int(g["iters"])
    assert sol["resid"] == float(g["resid"])
    assert bits_equal(sol["p"], g["p"])


@pytest.mark.parametrize("name", CASES)
def test_apply_and_divergence_match_reference_bitwise(oracle_lib, name):
    sc, g = load(name)
    u, v, w = oracle_lib.apply(sc, g["p"])
    assert bits_equal(u, g["u_out"]) and bits_equal(v, g["v_out"]) and bits_equal(w, g["w_out"])
    assert bits_equal(oracle_lib.divergence_ref(sc, u, v, w), g["div"])


@pytest.mark.parametrize("name", CASES)
def test_project_zeroes_weighted_divergence(oracle_lib, name):
    sc, g = load(name)
    out = oracle_lib.project(sc, tol=1e-12, maxit=2000)
    assert out["ok"]
    d = oracle_lib.weighted_divergence(sc, out["u"], out["v"], out["w"])
    bnorm = np.abs(oracle_lib.assemble(sc)["b"]).max()
    assert np.abs(d).max() <= 1e-9 * bnorm


def _dense(sc, A):
    import scipy.sparse as sp
    n = sc.ncells
    ni, nn = sc.ni, sc.ni * sc.nj
    rows, cols, vals = [], [], []
    for off, key in ((1, "ax"), (ni, "ay"), (nn, "az")):
        a = A[key].ravel()
        idx = np.nonzero(a)[0]
        rows += [idx, idx - off]; cols += [idx - off, idx]; vals += [a[idx], a[idx]]
    d = A["diag"].ravel()
    idx = np.nonzero(d)[0]
    rows.append(idx); cols.append(idx); vals.append(d[idx])
    return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))


@pytest.mark.parametrize("fractional", [False, True])
def test_matrix_properties(oracle_lib, fractional):
    """Symmetric M-matrix with non-negative row sums; solid rows sum to zero
    (each solid unknown only couples to fluid with matching weights)."""
    sc = scenes.pool_drop(dims=(18, 20, 16), dtype=np.float64)
    if not fractional:
        sc = sc.reference_mode()
    A = oracle_lib.assemble(sc)
    M = _dense(sc, A)
    assert abs(M - M.T).max() == 0
    off = M - __import__("scipy.sparse", fromlist=["diags"]).diags(M.diagonal())
    assert off.max() <= 0
    rs = np.asarray(M.sum(axis=1)).ravel()
    assert rs.min() >= -1e-12
    solid = (sc.mat.ravel() == scenes.SOLID) & (A["diag"].ravel() != 0)
    assert np.abs(rs[solid]).max() <= 1e-12
    if fractional:
        assert np.any((sc.wu > 0) & (sc.wu < 1))


@pytest.mark.parametrize("fractional", [False, True])
def test_pcg_agrees_with_scipy_direct_solve(oracle_lib, fractional):
    import scipy.sparse.linalg as spla
    sc = scenes.blob_scene(dims=(20, 18, 16), seed=11, fractional=fractional, dtype=np.float64)
    A = oracle_lib.assemble(sc)
    M = _dense(sc, A)
    act = A["diag"].ravel() != 0
    Ma = M[act][:, act]
    x_ref = spla.spsolve(Ma.tocsc(), A["b"].ravel()[act])
    sol = oracle_lib.pcg(sc, A, 1e-13, 5000)
    assert sol["ok"]
    x = sol["p"].ravel()[act]
    assert np.linalg.norm(x - x_ref) <= 1e-9 * np.linalg.norm(x_ref)


def test_adjoint_matches_finite_differences(oracle_lib):
    """Projection P(u) = u - G A^{-1} D u; its adjoint is g - D^T A^{-1} G^T g.
    Checked along random directions by FP64 central differences."""
    sc = scenes.pool_drop(dims=(12, 14, 10), dtype=np.float64)
    A = oracle_lib.assemble(sc)
    rng = np.random.default_rng(3)
    gu, gv, gw = (rng.standard_normal(a.shape) for a in (sc.u, sc.v, sc.w))
    # backward
    q = oracle_lib.apply_T(sc, gu, gv, gw)
    lam = oracle_lib.pcg(sc, dict(A, b=q), 1e-14, 5000)["p"]
    du, dv, dw = oracle_lib.rhs_T(sc, lam)
    bu, bv, bw = gu - du, gv - dv, gw - dw

    def loss(s):
        out = oracle_lib.project(s, tol=1e-14, maxit=5000)
        return float((out["u"] * gu).sum() + (out["v"] * gv).sum() + (out["w"] * gw).sum())

    for _ in range(4):
        eu, ev, ew = (rng.standard_normal(a.shape) for a in (sc.u, sc.v, sc.w))
        eps = 1e-3
        sp_, sm_ = sc.copy(), sc.copy()
        sp_.u = sc.u + eps * eu; sp_.v = sc.v + eps * ev; sp_.w = sc.w + eps * ew
        sm_.u = sc.u - eps * eu; sm_.v = sc.v - eps * ev; sm_.w = sc.w - eps * ew
        fd = (loss(sp_) - loss(sm_)) / (2 * eps)
        an = float((bu * eu).sum() + (bv * ev).sum() + (bw * ew).sum())
        assert abs(fd - an) <= 1e-7 * max(1.0, abs(an))


def test_reference_apply_does_not_depend_on_its_thread_count():
    """oracle/_ref is built with OpenMP, as xFluid's project is: applyPressure's
    loop over i (variational_pressuresolver.cpp:134) runs in parallel.  Its
    iterations write disjoint faces, so one thread and all host threads give the
    same bits (the golden vectors do not depend on the build's thread count)."""
    import os

    import oracle
    if not oracle.reference_available():
        pytest.skip("reference build absent (oracle/_ref)")
    R = oracle.Reference()
    sc = scenes.dam_break(dims=(40, 34, 30), seed=4, noise=0.5)
    p = np.random.default_rng(4).standard_normal((sc.nk, sc.nj, sc.ni))
    before = R.set_threads(1)
    try:
        one = R.apply(sc, p)
        R.set_threads(max(2, os.cpu_count() or 2))
        many = R.apply(sc, p)
    finally:
        R.set_threads(before)
    for a, b in zip(one, many):
        assert np.array_equal(a, b)
    assert R.time_apply(sc, p, 1, 1) > 0.0


def test_full_size_fixture_matches_the_seeded_scene():
    """The 256^3 fixture (xFluid's own solver on the benchmark scene) was made
    on the scene scenes.blob_scene(256, seed=3) generates here, and its sample
    indices are unknown rows of that scene."""
    import hashlib
    from golden_io import GOLDEN
    g = dict(np.load(GOLDEN / "full_blob256.npz"))
    sc = scenes.blob_scene(int(g["n"]), seed=int(g["seed"]), dtype=np.float32)
    h = hashlib.sha256()
    for a in (sc.mat, sc.u, sc.v, sc.w):
        h.update(np.ascontiguousarray(a).tobytes())
    assert h.hexdigest() == str(g["digest"])
    fl = sc.mat == scenes.FLUID
    nb = np.zeros_like(fl)
    nb[1:] |= fl[:-1]; nb[:-1] |= fl[1:]
    nb[:, 1:] |= fl[:, :-1]; nb[:, :-1] |= fl[:, 1:]
    nb[:, :, 1:] |= fl[:, :, :-1]; nb[:, :, :-1] |= fl[:, :, 1:]
    rows = fl | ((sc.mat == scenes.SOLID) & nb)
    assert int(rows.sum()) == int(g["rows"])
    assert rows.ravel()[g["idx_p"]].all()
    assert int(g["iters"]) < int(g["iters_exact"]) and g["p_minus_pe_l2"] < 1e-4 * g["pe_l2"]
