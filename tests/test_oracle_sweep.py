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


@pytest.mark.skipif(not oracle.sim_available(), reason="reference simulator build absent (oracle/_ref)")
@pytest.mark.parametrize("seed", SEEDS[:8])
def test_particle_steps_match_reference_on_random_masks(libs, seed):
    """The particle steps on the random masks, whose solids sit inside the
    domain too: collisions walk through interior solid voxels and hit their
    boxes from every side.  Particles are seeded in the fluid cells as xFluid
    seeds them, plus some anywhere in the box (solid cells included), with
    velocities fast enough to cross cells.  Bit-identical where the reference
    reads inside its arrays (the oracle's status 2 marks the rest)."""
    O, _ = libs
    S = oracle.RefSteps()
    sc = _random_scene(seed)
    rng = np.random.default_rng(3000 + seed)
    dx = 1.0 / max(sc.ni, sc.nj, sc.nk)
    P = scenes.seed_particles(sc.mat, dx, seed=seed, jitter=0.3 * dx, vel_scale=4.0)
    extra = np.concatenate([rng.uniform(0, 1, (200, 3)) * np.array([sc.ni, sc.nj, sc.nk]) * dx,
                            rng.uniform(-4, 4, (200, 3))], 1)
    P = np.concatenate([P, extra])[: len(P) + 200 - (seed % 5)]
    uvw = [np.clip(a, -50.0, 50.0) for a in (sc.u, sc.v, sc.w)]
    sc = scenes.Scene(sc.ni, sc.nj, sc.nk, sc.mat, *uvw)
    saved = [a + 0.1 * rng.standard_normal(a.shape) for a in uvw]
    for dt in (0.01, 0.08):
        po, st = O.advect_particles(sc, saved, P, 0.95, dt, dx, status=True)
        pr = S.advect_particles(sc, saved, P, 0.95, dt, dx)
        keep = st != 2
        assert np.array_equal(po[keep], pr[keep])
    dims = (sc.ni, sc.nj, sc.nk)
    for a, b in zip(O.p2g(dims, dx, P), S.p2g(dims, dx, P)):
        assert np.array_equal(a, b)
    radius = 3.0 * (3 * (dx ** 3 / 8.0) / (4 * 3.141592653)) ** (1.0 / 3.0)
    phi_o, m_o = O.distance_field(sc.mat, dx, 2, radius, 0.4, P)
    phi_r, m_s, m_f = S.material(sc.mat, dx, 2, radius, 0.4, P)
    assert np.array_equal(phi_o, phi_r) and np.array_equal(m_o, m_s)
    assert np.array_equal(O.update_material(m_s, dx, P), m_f)
