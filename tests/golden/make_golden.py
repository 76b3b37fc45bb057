"""Generate the golden vectors in tests/golden/ from xFluid's own solver.

The reference ships no tests, fixtures or known-answer vectors, so the golden
vectors are produced by running the reference code itself: oracle/build_ref.sh
compiles xFluid's VariationalPressureSolver / PCGSolver from the reference
sources into oracle/_ref/libxfref.so and this script drives it on small seeded
scenes (reference mode: all faces fully open).  Run from the repository root:

    python tests/golden/make_golden.py

Each ``<case>.npz`` holds the scene inputs and the reference's outputs:
assembly (diag, ax, ay, az, b), MIC(0) factor (inv, lx, ly, lz), the
preconditioner applied to a seeded residual (r -> z), the PCG pressure at
tol 1e-6 (iterations, residual), the velocities after applyPressure, and the
reference's divergence diagnostic after the projection.

``normal_<case>.npz`` holds the same scene inputs run through xFluid's
NormalPressureSolver (pressuresolver.cpp, the classic Poisson matrix): its
assembly (diag, ax, ay, az, b), its PCG pressure at tol 1e-6 (iterations,
residual) and the velocities after its applyPressure.  ``--normal-only``
writes just those (and the step fixtures); ``--steps-only`` writes only the
``steps_<case>.npz`` fixtures (see step_fixtures); ``--particles-only`` writes
only the ``particles_<case>.npz`` fixtures (see particle_fixtures).

``full_blob256.npz`` (``--full-only``; about two minutes on one core) pins the
reference on the full-size 256^3 blob scene (see full_size_fixture).
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import Reference, build_reference  # noqa: E402
from xfluid_b200 import scenes  # noqa: E402

OUT = Path(__file__).resolve().parent
TOL, MAXIT = 1e-6, 500


def cases():
    return {
        "dam16": scenes.dam_break(16, seed=1, noise=0.3),
        "dam20x14x18": scenes.dam_break(dims=(20, 14, 18), seed=2, noise=0.5),
        "blob24x20x22": scenes.blob_scene(dims=(24, 20, 22), seed=5, fractional=False, dtype=np.float64),
        "pool20x22x18": scenes.pool_drop(dims=(20, 22, 18), seed=2, dtype=np.float64).reference_mode(),
    }


NORMAL_CASES = ("dam16", "blob24x20x22")
STEP_CASES = ("dam20x14x18",)
FORCE, DT, LAYERS = (0.3, -9.8, 0.0), 0.01, 6


def step_fixtures(R):
    """``steps_<case>.npz``: FluidSimulator::_applyForces (force FORCE, dt DT)
    and _expolateVelocity (LAYERS layers) on the scene's faces, and the whole
    sequence forces -> projection (tol 1e-6) -> extrapolation, all run by the
    reference's own code (oracle/sim_harness.cpp, oracle/ref_harness.cpp)."""
    from oracle import RefSteps  # noqa: E402
    S = RefSteps()
    for name, sc in cases().items():
        if name not in STEP_CASES:
            continue
        f = S.apply_forces(sc, FORCE, DT)
        e = S.extrapolate(sc, LAYERS)
        s2 = sc.copy()
        s2.u, s2.v, s2.w = f
        pr = R.project(s2, TOL, MAXIT)
        assert pr["ok"], name
        st = S.extrapolate(sc, LAYERS, uvw=(pr["u"], pr["v"], pr["w"]))
        np.savez_compressed(
            OUT / f"steps_{name}.npz",
            dims=np.array([sc.ni, sc.nj, sc.nk]), mat=sc.mat, u=sc.u, v=sc.v, w=sc.w,
            force=np.array(FORCE), dt=DT, layers=LAYERS, tol=TOL, maxit=MAXIT,
            u_forced=f[0], v_forced=f[1], w_forced=f[2], u_extrap=e[0], v_extrap=e[1], w_extrap=e[2],
            p_step=pr["p"], u_step=st[0], v_step=st[1], w_step=st[2])
        print(f"steps_{name}: forces, {LAYERS}-layer extrapolation, full step")


PARTICLE_CASES = {"dam17x13x11": dict(dims=(17, 13, 11), seed=2, dt=0.2, vel=2.0),
                  "dam19x15x13": dict(dims=(19, 15, 13), seed=3, dt=0.05, vel=4.0)}
RATIO_FLIP, SUBDIV, THRESHOLD = 0.95, 2, 0.4


def particle_fixtures():
    """``particles_<case>.npz``: the particle steps around the projection, run
    by the reference's own code (oracle/sim_harness.cpp) on xFluid-seeded
    particles (scenes.seed_particles, jitter dx/5 so particles cross faces)
    with random velocities, and one particle dropped so n is not a multiple of
    six:
      - _advectParticles(dt) (FluidSimulator.cpp:652-728) with ratio 0.95 on
        the scene's faces and a perturbed saved copy: particles_out, and the
        faces after its own particle-to-grid transfer (u_p2g_adv, ...);
      - _updateVelocityByParticles on the input particles (u_p2g, ...);
      - updateFeild + updateSurfaceInfo (subdivision 2, radius 3 x the
        simulator's particle radius, threshold 0.4, FluidSimulator.cpp:207-213):
        phi, mat_surface; then _updateMaterial: mat_final.
    `ub` marks the particles whose collision point lies in a cell outside the
    grid: the reference reads the material out of bounds there (:714), so those
    particles are not compared (the oracle's status 2)."""
    from oracle import Oracle, RefSteps  # noqa: E402
    S, O = RefSteps(), Oracle()
    for name, cfg in PARTICLE_CASES.items():
        ni, nj, nk = cfg["dims"]
        sc = scenes.dam_break(dims=cfg["dims"], seed=cfg["seed"], noise=0.4)
        dx = 1.0 / ni
        P = scenes.seed_particles(sc.mat, dx, seed=cfg["seed"], jitter=0.2 * dx, vel_scale=cfg["vel"])[:-1]
        rng = np.random.default_rng(cfg["seed"])
        saved = [a + 0.1 * rng.standard_normal(a.shape) for a in (sc.u, sc.v, sc.w)]
        out, g = S.advect_particles(sc, saved, P, RATIO_FLIP, cfg["dt"], dx, grids=True)
        _, st = O.advect_particles(sc, saved, P, RATIO_FLIP, cfg["dt"], dx, status=True)
        p2g = S.p2g((ni, nj, nk), dx, P)
        radius = 3.0 * (3 * (dx * dx * dx / 8.0) / (4 * 3.141592653)) ** (1.0 / 3.0)
        phi, ms, mf = S.material(sc.mat, dx, SUBDIV, radius, THRESHOLD, P)
        np.savez_compressed(
            OUT / f"particles_{name}.npz",
            dims=np.array([ni, nj, nk]), dx=dx, mat=sc.mat, u=sc.u, v=sc.v, w=sc.w,
            us=saved[0], vs=saved[1], ws=saved[2], ratio=RATIO_FLIP, dt=cfg["dt"], parts_in=P,
            parts_out=out, ub=(st == 2), u_p2g_adv=g[0], v_p2g_adv=g[1], w_p2g_adv=g[2],
            u_p2g=p2g[0], v_p2g=p2g[1], w_p2g=p2g[2], subdiv=SUBDIV, radius=radius, threshold=THRESHOLD,
            phi=phi, mat_surface=ms, mat_final=mf)
        print(f"particles_{name}: {len(P)} particles, status counts {np.bincount(st, minlength=5).tolist()}")


def scene_digest(sc) -> str:
    """sha256 over the scene's material bytes and its FP32 face velocities, as
    generated: the full-size test checks it before comparing results."""
    import hashlib
    h = hashlib.sha256()
    for a in (sc.mat, sc.u, sc.v, sc.w):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


FULL_N, FULL_SEED, FULL_MAXIT = 256, 3, 20000


def full_size_fixture(R):
    """``full_blob256.npz``: xFluid's own solver on the 256^3 blob scene
    (scenes.blob_scene(256, seed=3), reference mode: the same mask, obstacle
    and FP32 faces without fractional weights), single-threaded:
      - solve to tol 1e-6 (iterations, residual) and to tol 1e-12 (the exact
        solution the convergence error is measured against);
      - the full-field L2 norms of both pressures and of their difference;
      - a fixed sample of the pressures (every 97th unknown row, flat indices
        stored) and of the velocities after applyPressure (every 389th face
        that borders fluid);
      - the reference's own divergence diagnostic's L-inf after the projection.
    The whole fields (16.7M cells) are too large to commit; the sample pins the
    live reference run the GPU test makes beside it."""
    sc32 = scenes.blob_scene(FULL_N, seed=FULL_SEED, dtype=np.float32)
    sc = sc32.astype(np.float64).reference_mode()
    before = R.set_threads(1)
    try:
        sol = R.solve(sc, TOL, FULL_MAXIT)
        ex = R.solve(sc, 1e-12, FULL_MAXIT)
        assert sol["ok"] and ex["ok"]
        u2, v2, w2 = R.apply(sc, sol["p"])
        div = R.divergence(sc, u2, v2, w2)
    finally:
        R.set_threads(before)
    fl = sc.mat == scenes.FLUID
    nb = np.zeros_like(fl)
    nb[1:] |= fl[:-1]; nb[:-1] |= fl[1:]
    nb[:, 1:] |= fl[:, :-1]; nb[:, :-1] |= fl[:, 1:]
    nb[:, :, 1:] |= fl[:, :, :-1]; nb[:, :, :-1] |= fl[:, :, 1:]
    rows = np.flatnonzero(fl | ((sc.mat == scenes.SOLID) & nb))
    prow = rows[::97].astype(np.int64)
    mu, mv, mw = scenes.fluid_adjacent_faces(sc.mat)
    fu, fv, fw = (np.flatnonzero(m)[::389].astype(np.int64) for m in (mu, mv, mw))
    p, pe = sol["p"].ravel(), ex["p"].ravel()
    np.savez_compressed(
        OUT / "full_blob256.npz", n=FULL_N, seed=FULL_SEED, digest=scene_digest(sc32), tol=TOL,
        maxit=FULL_MAXIT, rows=len(rows), iters=sol["iters"], resid=sol["resid"], iters_exact=ex["iters"],
        p_l2=np.linalg.norm(p), pe_l2=np.linalg.norm(pe), p_minus_pe_l2=np.linalg.norm(p - pe),
        idx_p=prow, p=p[prow], pe=pe[prow], idx_u=fu, idx_v=fv, idx_w=fw,
        u_out=u2.ravel()[fu], v_out=v2.ravel()[fv], w_out=w2.ravel()[fw],
        div_inf=np.abs(div).max())
    print(f"full_blob256: {len(rows)} rows, {sol['iters']} iterations (exact: {ex['iters']}), "
          f"reference vs exact rel L2 {np.linalg.norm(p - pe) / np.linalg.norm(pe):.3e}")


def normal_fixtures(R):
    for name, sc in cases().items():
        if name not in NORMAL_CASES:
            continue
        A = R.normal_assemble(sc)
        sol = R.normal_solve(sc, TOL, MAXIT)
        assert sol["ok"], name
        u2, v2, w2 = R.normal_apply(sc, sol["p"])
        np.savez_compressed(
            OUT / f"normal_{name}.npz",
            dims=np.array([sc.ni, sc.nj, sc.nk]), mat=sc.mat, u=sc.u, v=sc.v, w=sc.w,
            diag=A["diag"], ax=A["ax"], ay=A["ay"], az=A["az"], b=A["b"],
            p=sol["p"], iters=sol["iters"], resid=sol["resid"], tol=TOL, maxit=MAXIT,
            u_out=u2, v_out=v2, w_out=w2)
        print(f"normal_{name}: {int((A['diag'] != 0).sum())} rows, {sol['iters']} iterations")


def main():
    if build_reference() is None:
        raise SystemExit("reference sources not found; cannot regenerate golden vectors")
    R = Reference()
    if "--full-only" in sys.argv:
        full_size_fixture(R)
        return
    if "--particles-only" in sys.argv:
        particle_fixtures()
        return
    if "--steps-only" not in sys.argv:
        normal_fixtures(R)
    step_fixtures(R)
    if "--normal-only" in sys.argv or "--steps-only" in sys.argv:
        return
    for name, sc in cases().items():
        A = R.assemble(sc)
        F = R.factor(sc)
        rng = np.random.default_rng(7)
        r = rng.standard_normal(A["diag"].shape) * (A["diag"] != 0)
        z = R.precond(sc, r)
        sol = R.solve(sc, TOL, MAXIT)
        assert sol["ok"], name
        u2, v2, w2 = R.apply(sc, sol["p"])
        div = R.divergence(sc, u2, v2, w2)
        np.savez_compressed(
            OUT / f"{name}.npz",
            dims=np.array([sc.ni, sc.nj, sc.nk]), mat=sc.mat, u=sc.u, v=sc.v, w=sc.w,
            diag=A["diag"], ax=A["ax"], ay=A["ay"], az=A["az"], b=A["b"], maxrow=A["maxrow"],
            inv=F["inv"], lx=F["lx"], ly=F["ly"], lz=F["lz"], r=r, z=z,
            p=sol["p"], iters=sol["iters"], resid=sol["resid"], tol=TOL, maxit=MAXIT,
            u_out=u2, v_out=v2, w_out=w2, div=div)
        print(f"{name}: {int((A['diag'] != 0).sum())} rows, {sol['iters']} iterations")


if __name__ == "__main__":
    main()
