"""The oracle against xFluid's own build on a seeded sweep of small random
scenes: random fluid/air/solid masks inside the solid border ring the
reference's assembly relies on (its neighbour lookup has no bounds check,
variational_pressuresolver.cpp:292), thin and ragged dimensions down to 3
cells, velocities of several scales.  Every stage of both matrix modes must be
bit-identical: assembly, MIC(0) factor, preconditioner, PCG (iterations,
residual, pressure), applyPressure and the divergence diagnostic,
NormalPressureSolver's assembly, solve and apply, and the simulator's forces and
velocity extrapolation.  Needs oracle/_ref."""
import numpy as np
import pytest

import oracle
from golden_io import bits_equal
from xfluid_b200 import scenes

pytestmark = pytest.mark.skipif(not oracle.reference_available(), reason="reference build absent (oracle/_ref)")

SEEDS = list(range(12))


def _random_scene(seed):
    rng = np.random.default_rng(1000 + seed)
    ni, nj, nk = (int(x) for x in rng.integers(3, 19, 3))
    p_fluid, p_solid = rng.uniform(0.3, 0.8), rng.uniform(0.0, 0.25)
    r = rng.uniform(size=(nk, nj, ni))
    mat = np.where(r < p_fluid, scenes.FLUID, np.where(r < p_fluid + p_solid, scenes.SOLID, scenes.AIR))
    mat = mat.astype(np.uint8)
    scenes.solid_border(mat)
    scale = 10.0 ** rng.uniform(-3, 2)
    u, v, w = (rng.standard_normal(sh) * scale for sh in scenes.face_shapes(ni, nj, nk))
    return scenes.Scene(ni, nj, nk, mat, u, v, w, name=f"sweep{seed}")


@pytest.fixture(scope="module")
def libs():
    return oracle.Oracle(), oracle.Reference()


@pytest.mark.parametrize("seed", SEEDS)
def test_variational_stages_match_reference_bitwise(libs, seed):
    O, R = libs
    sc = _random_scene(seed)
    A, Ar = O.assemble(sc), R.assemble(sc)
    for k in ("diag", "ax", "ay", "az", "b"):
        assert bits_equal(A[k], Ar[k]), k
    F, Fr = O.factor(sc, A), R.factor(sc)
    for k in ("inv", "lx", "ly", "lz"):
        assert bits_equal(F[k], Fr[k]), k
    rv = np.random.default_rng(seed).standard_normal(A["diag"].shape) * (A["diag"] != 0)
    assert bits_equal(O.precond(sc, F, rv), R.precond(sc, rv))
    so, sr = O.pcg(sc, A, 1e-8, 400), R.solve(sc, 1e-8, 400)
    assert so["ok"] == sr["ok"]
    if sr["ok"]:
        assert so["iters"] == sr["iters"] and so["resid"] == sr["resid"]
        assert bits_equal(so["p"], sr["p"])
    p = sr["p"]
    uo, ur = O.apply(sc, p), R.apply(sc, p)
    for a, b in zip(uo, ur):
        assert bits_equal(a, b)
    assert bits_equal(O.divergence_ref(sc, *uo), R.divergence(sc, *ur))


@pytest.mark.parametrize("seed", SEEDS[::2])
def test_normal_solver_matches_reference_bitwise(libs, seed):
    O, R = libs
    sc = _random_scene(seed)
    a, r = O.assemble_normal(sc), R.normal_assemble(sc)
    for k in ("diag", "ax", "ay", "az", "b"):
        assert np.array_equal(a[k], r[k]), k
    po, pr = O.project_normal(sc, tol=1e-8, maxit=400), R.normal_solve(sc, tol=1e-8, maxit=400)
    assert po["ok"] == pr["ok"]
    if pr["ok"]:
        assert po["iters"] == pr["iters"] and np.array_equal(po["p"], pr["p"])
    p = np.random.default_rng(seed).standard_normal(sc.mat.shape)
    for x, y in zip(O.apply_normal(sc, p), R.normal_apply(sc, p)):
        assert np.array_equal(x, y)


@pytest.mark.skipif(not oracle.sim_available(), reason="reference simulator build absent (oracle/_ref)")
@pytest.mark.parametrize("seed", SEEDS[:6])
def test_simulator_steps_match_reference_bitwise(libs, seed):
    """_applyForces with random forces (a component below the reference's
    1e-10 cut-off included) and _expolateVelocity with random layer counts on
    the same random scenes, against the reference's own simulator code."""
    O, _ = libs
    S = oracle.RefSteps()
    sc = _random_scene(seed)
    rng = np.random.default_rng(2000 + seed)
    force = rng.standard_normal(3) * 10.0
    force[rng.integers(0, 3)] = 3e-11 / 0.02   # |force*dt| = 3e-11: below the cut-off
    for x, y in zip(O.apply_forces(sc, force, 0.02), S.apply_forces(sc, force, 0.02)):
        assert np.array_equal(x, y)
    layers = int(rng.integers(0, 9))
    for x, y in zip(O.extrapolate(sc, layers), S.extrapolate(sc, layers)):
        assert np.array_equal(x, y)
