"""Differentiable rollouts (advect -> project, repeated): the advection kernels
and the checkpointed adjoint, checked by FP64 central differences and against
the oracle's FP64 CPU adjoint (oracle/advect.py)."""
import numpy as np
import pytest

from xfluid_b200 import scenes
from oracle import advect as adv

BOX = ((0.6, 0.9), (0.6, 0.9), (0.6, 0.9))


def _rand_state(rng, ni, nj, nk, lo=-0.5, hi=0.5):
    return (rng.uniform(lo, hi, (nk, nj, ni + 1)), rng.uniform(lo, hi, (nk, nj + 1, ni)),
            rng.uniform(lo, hi, (nk + 1, nj, ni)))


def _dot(a, b):
    return float(sum((x * y).sum() for x, y in zip(a, b)))


# ------------------------------------------------------------------ oracle (CPU)
def test_oracle_advect_adjoint_matches_central_differences():
    rng = np.random.default_rng(5)
    ni, nj, nk, c = 7, 5, 6, 0.9
    st = _rand_state(rng, ni, nj, nk)
    g = _rand_state(rng, ni, nj, nk, -1, 1)
    jt = adv.advect_adjoint(*st, *g, c)
    for _ in range(6):
        e = _rand_state(rng, ni, nj, nk, -1, 1)
        eps = 1e-6
        fp = adv.advect(*(s + eps * d for s, d in zip(st, e)), c)
        fm = adv.advect(*(s - eps * d for s, d in zip(st, e)), c)
        fd = (_dot(fp, g) - _dot(fm, g)) / (2 * eps)
        an = _dot(jt, e)
        assert abs(fd - an) <= 1e-6 * max(1.0, abs(an)), (fd, an)


def test_oracle_rollout_gradient_matches_central_differences():
    import oracle
    O = oracle.Oracle()
    sc = scenes.dam_break(10, seed=1)
    rng = np.random.default_rng(8)
    u0 = _rand_state(rng, sc.ni, sc.nj, sc.nk)
    c, steps = 10 / 30, 4
    loss, g = adv.rollout_grad(O, sc.mat, *u0, steps, c, BOX, 1e-13, checkpoint_every=2)
    assert loss > 0
    for _ in range(4):
        e = _rand_state(rng, sc.ni, sc.nj, sc.nk, -1, 1)
        eps = 1e-4
        lp = adv.rollout_loss(O, sc.mat, *(a + eps * d for a, d in zip(u0, e)), steps, c, BOX, 1e-13)
        lm = adv.rollout_loss(O, sc.mat, *(a - eps * d for a, d in zip(u0, e)), steps, c, BOX, 1e-13)
        fd = (lp - lm) / (2 * eps)
        an = _dot(g, e)
        assert abs(fd - an) <= 1e-5 * max(abs(an), 1e-3), (fd, an)


# ------------------------------------------------------------------ GPU
def _t(a, dtype=None):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda() if dtype is None else \
        torch.from_numpy(np.ascontiguousarray(a, dtype)).cuda()


@pytest.mark.gpu
def test_gpu_advection_and_adjoint_match_oracle():
    from xfluid_b200.rollout import Rollout
    rng = np.random.default_rng(2)
    ni, nj, nk, c = 20, 16, 18, 1.3
    st = _rand_state(rng, ni, nj, nk)
    g = _rand_state(rng, ni, nj, nk, -1, 1)
    mat = np.zeros((nk, nj, ni), np.uint8)
    r = Rollout(_t(mat), steps=1, dt_over_dx=c)
    try:
        P = r._P
        out = [_t(np.zeros_like(a)) for a in st]
        ts = [_t(a) for a in st]
        r._ctx.check(r._ctx.lib.xfp_advect_f64(r._ctx.ptr, ni, nj, nk, *map(P, ts), *map(P, out), c))
        ref = adv.advect(*st, c)
        for a, b in zip(out, ref):
            assert np.allclose(a.cpu().numpy(), b, rtol=0, atol=1e-13)
        tg = [_t(a) for a in g]
        d = [_t(np.zeros_like(a)) for a in st]
        r._ctx.check(r._ctx.lib.xfp_advect_backward_f64(r._ctx.ptr, ni, nj, nk, *map(P, ts), *map(P, tg), *map(P, d), c))
        ref = adv.advect_adjoint(*st, *g, c)
        for a, b in zip(d, ref):
            assert np.allclose(a.cpu().numpy(), b, rtol=1e-12, atol=1e-12)
        loss, grads = r.loss(*ts, grad=True)
        rl, rg = adv.box_loss(*st, BOX)
        assert abs(loss - rl) <= 1e-12 * rl
        for a, b in zip(grads, rg):
            assert np.array_equal(a.cpu().numpy(), b)
    finally:
        r.close()


@pytest.mark.gpu
def test_gpu_rollout_gradient_vs_central_differences_and_cpu_adjoint():
    """The differentiable-rollout configuration at 24^3: 16 advect+project steps
    from u0 ~ U[-0.5,0.5] over a dam-break mask, checkpoints every 4 steps,
    loss = sum of squared velocity in [0.6,0.9]^3.  The GPU gradient must match
    the oracle's FP64 CPU adjoint, and FP64 central differences along 32 random
    directions to 1e-4 relative.  The step size is 1e-6: trilinear sampling is
    piecewise linear in the departure point, so a perturbation of 1e-3 moves
    some departure points across cell faces within 16 steps and the central
    difference then straddles a kink (it misses by about 1e-2 even for one
    step); as eps shrinks the differences converge to the adjoint (1e-5 gives
    ~1e-5, 1e-6 gives ~1e-8)."""
    import oracle
    from xfluid_b200.rollout import Rollout
    sc = scenes.dam_break(24, seed=1)
    rng = np.random.default_rng(13)
    u0 = _rand_state(rng, sc.ni, sc.nj, sc.nk)
    c = 24 / 30
    r = Rollout(_t(sc.mat), steps=16, checkpoint_every=4, dt_over_dx=c, box=BOX, precision="f64", tol=1e-13)
    try:
        t0 = [_t(a) for a in u0]
        loss = r.forward(*t0)
        g = [a.cpu().numpy() for a in r.backward()]
        assert loss > 0 and all(np.isfinite(a).all() for a in g)
        errs = []
        for _ in range(32):
            e = _rand_state(rng, sc.ni, sc.nj, sc.nk, -1, 1)
            eps = 1e-6
            lp = r.forward(*(_t(a + eps * d) for a, d in zip(u0, e)))
            lm = r.forward(*(_t(a - eps * d) for a, d in zip(u0, e)))
            fd = (lp - lm) / (2 * eps)
            an = _dot(g, e)
            # relative to the derivative, or to the gradient's scale along e
            # when the derivative itself is nearly zero
            scale = 1e-6 * np.sqrt(_dot(g, g) * _dot(e, e))
            errs.append(abs(fd - an) / max(abs(an), scale))
        assert np.median(errs) <= 1e-6 and max(errs) <= 1e-4, sorted(errs)[-5:]
    finally:
        r.close()
    O = oracle.Oracle()
    lref, gref = adv.rollout_grad(O, sc.mat, *u0, 16, c, BOX, 1e-13, checkpoint_every=4)
    assert abs(loss - lref) <= 1e-9 * lref
    num = np.sqrt(sum(((a - b) ** 2).sum() for a, b in zip(g, gref)))
    den = np.sqrt(sum((b ** 2).sum() for b in gref))
    assert num / den <= 1e-12, num / den


@pytest.mark.gpu
def test_gpu_rollout_f32_tracks_f64():
    from xfluid_b200.rollout import Rollout
    sc = scenes.dam_break(24, seed=1)
    rng = np.random.default_rng(4)
    u0 = _rand_state(rng, sc.ni, sc.nj, sc.nk)
    out = {}
    for prec, dt in (("f64", np.float64), ("mixed", np.float32)):
        r = Rollout(_t(sc.mat), steps=8, checkpoint_every=4, dt_over_dx=1.0, box=BOX, precision=prec,
                    tol=1e-10 if prec == "f64" else 1e-6)
        try:
            loss = r.forward(*(_t(a, dt) for a in u0))
            out[prec] = (loss, [a.double().cpu().numpy() for a in r.backward()])
        finally:
            r.close()
    (l64, g64), (l32, g32) = out["f64"], out["mixed"]
    assert abs(l32 - l64) <= 1e-4 * l64
    num = np.sqrt(sum(((a - b) ** 2).sum() for a, b in zip(g32, g64)))
    den = np.sqrt(sum((b ** 2).sum() for b in g64))
    assert num / den <= 1e-3, num / den


DAM_BOX = ((0.1, 0.35), (0.1, 0.45), (0.2, 0.8))   # inside the dam-break fluid (x < 0.4, y < 0.5)


@pytest.mark.gpu
def test_gpu_rollout_gradient_through_the_adjoint_solve():
    """The rollout of the configuration above with the loss box inside the
    dam-break fluid instead of [0.6,0.9]^3: the loss's sensitivity then sits
    on faces next to fluid from the last step on, so every adjoint projection
    has a nonzero right-hand side G^T g and its MIC(0)-PCG solve does work
    (with the configured box in air that right-hand side stays zero for the
    first steps of the reverse pass).  The gradient must match the oracle's
    FP64 CPU adjoint and FP64 central differences along 32 random directions
    to 1e-4 relative.  The step is 1e-7: trilinear sampling is piecewise
    linear (above), and with the box in the fluid the departure points of the
    faces that matter sit where the flow moves, so at 1e-6 one direction in 32
    straddled a kink (1.2e-4 off, unchanged at tighter solver tolerances);
    FP64 rounding of the loss stays below 1e-8 relative at 1e-7."""
    import oracle
    from xfluid_b200.rollout import Rollout
    sc = scenes.dam_break(24, seed=1)
    rng = np.random.default_rng(17)
    u0 = _rand_state(rng, sc.ni, sc.nj, sc.nk)
    c = 24 / 30
    r = Rollout(_t(sc.mat), steps=16, checkpoint_every=4, dt_over_dx=c, box=DAM_BOX, precision="f64", tol=1e-13)
    try:
        t0 = [_t(a) for a in u0]
        loss = r.forward(*t0)
        r.iterations = {"forward": 0, "backward": 0}
        g = [a.cpu().numpy() for a in r.backward()]
        assert loss > 0 and all(np.isfinite(a).all() for a in g)
        assert len(r.adjoint_rhs_inf) == 16 and min(r.adjoint_rhs_inf) > 0, r.adjoint_rhs_inf
        assert r.iterations["backward"] >= 16, r.iterations
        errs = []
        for _ in range(32):
            e = _rand_state(rng, sc.ni, sc.nj, sc.nk, -1, 1)
            eps = 1e-7
            lp = r.forward(*(_t(a + eps * d) for a, d in zip(u0, e)))
            lm = r.forward(*(_t(a - eps * d) for a, d in zip(u0, e)))
            fd = (lp - lm) / (2 * eps)
            an = _dot(g, e)
            scale = 1e-6 * np.sqrt(_dot(g, g) * _dot(e, e))
            errs.append(abs(fd - an) / max(abs(an), scale))
        assert np.median(errs) <= 1e-6 and max(errs) <= 1e-4, sorted(errs)[-5:]
    finally:
        r.close()
    O = oracle.Oracle()
    lref, gref = adv.rollout_grad(O, sc.mat, *u0, 16, c, DAM_BOX, 1e-13, checkpoint_every=4)
    assert abs(loss - lref) <= 1e-9 * lref
    num = np.sqrt(sum(((a - b) ** 2).sum() for a, b in zip(g, gref)))
    den = np.sqrt(sum((b ** 2).sum() for b in gref))
    assert num / den <= 1e-12, num / den


def test_oracle_rollout_adjoint_rhs_zero_in_air_nonzero_in_the_dam():
    """CPU check of what the two GPU rollout tests rely on: the first adjoint
    projection of the reverse pass solves A lam = G^T g for the box loss's
    gradient g.  With the configured box [0.6,0.9]^3 (in air, away from the
    dam-break fluid) G^T g is exactly zero, so that solve has nothing to do;
    with the box inside the fluid it is not."""
    import oracle
    O = oracle.Oracle()
    sc = scenes.dam_break(12, seed=1)
    rng = np.random.default_rng(3)
    u = _rand_state(rng, sc.ni, sc.nj, sc.nk)
    c, steps = 12 / 30, 4
    for _ in range(steps):
        u = adv.project(O, sc.mat, *adv.advect(*u, c), 1e-13)
    q = {}
    for name, box in (("air", BOX), ("dam", DAM_BOX)):
        _, g = adv.box_loss(*u, box)
        q[name] = np.abs(O.apply_T(adv._scene(sc.mat, *g), *g)).max()
    assert q["air"] == 0.0 and q["dam"] > 0.0, q
