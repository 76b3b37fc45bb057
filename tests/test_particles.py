"""The particle steps around the projection (FLIP/PIC): xFluid's
FluidSimulator::_advectParticles steps a-b (FluidSimulator.cpp:652-723),
_updateVelocityByParticles (:909-1085), _updateMaterial (:402-427) and
DirectedDistanceField::updateFeild + updateSurfaceInfo's material
(directeddistancefield.cpp:122-215).

The oracle's C restatement (oracle/xfp_particles_oracle.c) is pinned bitwise to
golden vectors the reference's own simulator code produced
(tests/golden/make_golden.py, particles_*.npz) and, where that build is present,
to it on further seeded scenes.  Particles whose collision point lies in a cell
outside the grid are left out of those comparisons: the reference reads the
material out of bounds there (the oracle's status 2).

The CUDA path is checked through the C ABI: advection and the material update
bitwise against the oracle on every particle; the two transfers (particle ->
faces, particle -> distance field), which sum the same contributions in another
order, to 1e-12 of the field's scale; the field's fluid/air classification
exactly, away from cells whose value is within rounding of the threshold."""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

import oracle
from xfluid_b200 import scenes

GOLDEN = Path(__file__).parent / "golden"
CASES = ["particles_dam17x13x11.npz", "particles_dam19x15x13.npz"]
TRANSFER_TOL = 1e-12


def _scene(z):
    ni, nj, nk = (int(x) for x in z["dims"])
    return scenes.Scene(ni, nj, nk, z["mat"], z["u"], z["v"], z["w"])


def _saved(z):
    return z["us"], z["vs"], z["ws"]


def _maxrel(a, b):
    s = max(float(np.abs(b).max()), 1e-300)
    return float(np.abs(np.asarray(a) - b).max()) / s


def _case(seed, dims, jitter=0.2, vel=3.0):
    sc = scenes.dam_break(dims=dims, seed=seed, noise=0.4)
    dx = 1.0 / dims[0]
    P = scenes.seed_particles(sc.mat, dx, seed=seed, jitter=jitter * dx, vel_scale=vel)[:-1]
    rng = np.random.default_rng(seed)
    saved = [a + 0.1 * rng.standard_normal(a.shape) for a in (sc.u, sc.v, sc.w)]
    return sc, dx, P, saved


# ------------------------------------------------------------------ CPU: the oracle
@pytest.mark.parametrize("name", CASES)
def test_oracle_particles_match_reference_golden_vectors(name):
    z = np.load(GOLDEN / name)
    sc, dx, P = _scene(z), float(z["dx"]), z["parts_in"]
    O = oracle.Oracle()
    out, st = O.advect_particles(sc, _saved(z), P, float(z["ratio"]), float(z["dt"]), dx, status=True)
    keep = ~z["ub"]
    assert np.array_equal(st == 2, z["ub"])
    assert np.array_equal(out[keep], z["parts_out"][keep])
    assert (st == 1).sum() > 0 and (st == 3).sum() > 0 and (st == 4).sum() == len(P) % 6  # collisions exercised
    dims = (sc.ni, sc.nj, sc.nk)
    for a, k in zip(O.p2g(dims, dx, P), ("u_p2g", "v_p2g", "w_p2g")):
        assert np.array_equal(a, z[k]), k
    if not z["ub"].any():   # the reference's own transfer after its advection
        for a, k in zip(O.p2g(dims, dx, out), ("u_p2g_adv", "v_p2g_adv", "w_p2g_adv")):
            assert np.array_equal(a, z[k]), k
    phi, ms = O.distance_field(z["mat"], dx, int(z["subdiv"]), float(z["radius"]), float(z["threshold"]), P)
    assert np.array_equal(phi, z["phi"])
    assert np.array_equal(ms, z["mat_surface"])
    assert np.array_equal(O.update_material(ms, dx, P), z["mat_final"])


@pytest.mark.skipif(not oracle.sim_available(), reason="reference simulator build absent (oracle/_ref)")
@pytest.mark.parametrize("seed,dims,dt", [(4, (16, 12, 14), 0.1), (6, (13, 17, 11), 0.4)])
def test_oracle_particles_match_reference_build(seed, dims, dt):
    sc, dx, P, saved = _case(seed, dims)
    O, R = oracle.Oracle(), oracle.RefSteps()
    po, st = O.advect_particles(sc, saved, P, 0.9, dt, dx, status=True)
    pr = R.advect_particles(sc, saved, P, 0.9, dt, dx)
    keep = st != 2
    assert np.array_equal(po[keep], pr[keep])
    for a, b in zip(O.p2g((sc.ni, sc.nj, sc.nk), dx, P), R.p2g((sc.ni, sc.nj, sc.nk), dx, P)):
        assert np.array_equal(a, b)
    for s, rad in ((2, 0.93 * dx), (3, 1.4 * dx)):
        phi_o, m_o = O.distance_field(sc.mat, dx, s, rad, 0.4, P)
        phi_r, m_s, m_f = R.material(sc.mat, dx, s, rad, 0.4, P)
        assert np.array_equal(phi_o, phi_r) and np.array_equal(m_o, m_s)
        assert np.array_equal(O.update_material(m_s, dx, P), m_f)


@pytest.mark.skipif(not oracle.sim_available(), reason="reference simulator build absent (oracle/_ref)")
def test_oracle_particles_match_reference_on_lattice_and_edge_positions():
    """Particles exactly on cell faces and centres (the half-cell lattice), just
    below zero (where C's truncation and floor differ: pos2Index gives 0 and
    the particle counts as inside), and just inside the far wall, with fast
    velocities so many collide: the oracle equals the reference everywhere the
    reference reads inside its arrays."""
    sc = scenes.dam_break(dims=(14, 12, 10), seed=5, noise=0.6)
    ni, nj, nk = sc.ni, sc.nj, sc.nk
    dx = 1.0 / ni
    rng = np.random.default_rng(5)
    n = 3000
    lat = np.stack([rng.integers(0, 2 * m, n) for m in (ni, nj, nk)], 1) * (0.5 * dx)
    lat[:300, 0] = -rng.uniform(0, 0.9, 300) * dx
    lat[300:600, 1] = -rng.uniform(0, 0.9, 300) * dx
    lat[600:900, 2] = (nk - rng.uniform(0.001, 0.5, 300)) * dx
    P = np.concatenate([lat, rng.uniform(-3, 3, (n, 3))], 1)
    saved = [a + 0.1 * rng.standard_normal(a.shape) for a in (sc.u, sc.v, sc.w)]
    O, R = oracle.Oracle(), oracle.RefSteps()
    for dt in (0.005, 0.3):
        po, st = O.advect_particles(sc, saved, P, 0.9, dt, dx, status=True)
        pr = R.advect_particles(sc, saved, P, 0.9, dt, dx)
        keep = st != 2
        assert (st == 1).sum() > 0 and keep.sum() > 0.95 * n
        assert np.array_equal(po[keep], pr[keep])
    for a, b in zip(O.p2g((ni, nj, nk), dx, P), R.p2g((ni, nj, nk), dx, P)):
        assert np.array_equal(a, b)
    for s, rad in ((2, 0.93 * dx), (1, 1.0 * dx), (3, 0.5 * dx)):
        phi_o, m_o = O.distance_field(sc.mat, dx, s, rad, 0.4, P)
        phi_r, m_s, m_f = R.material(sc.mat, dx, s, rad, 0.4, P)
        assert np.array_equal(phi_o, phi_r) and np.array_equal(m_o, m_s)
        assert np.array_equal(O.update_material(m_s, dx, P), m_f)


def _trunc_div(x, dx):
    """C's (int)(x / dx): truncation toward zero."""
    return np.trunc(x / dx).astype(np.int64)


@pytest.mark.parametrize("spec", ["faces0", "faces1", "faces2", "field2", "field3", "field1"])
def test_gather_bin_windows_cover_every_box(spec):
    """The binning of xfp_particles.cu restated in integers: a particle's key is
    the bin of its box's low corner, clamped to [0, nb-1]; an output at index t
    scans bins [b(t) - span, b(t)] per axis, b(t) = min(t/s, nb-1), span = the
    widest box.  Every output inside a particle's box must scan the particle's
    bin (that is what makes the gather see exactly the reference's
    contributions).  Checked on random, lattice and out-of-domain positions."""
    ni, nj, nk, dx = 13, 9, 11, 0.07
    rng = np.random.default_rng(8)
    n = 20000
    lo_b, hi_b = np.array([-2.0, -2.0, -2.0]), np.array([ni + 2.0, nj + 2.0, nk + 2.0])
    pos = rng.uniform(lo_b, hi_b, (n, 3)) * dx
    pos[: n // 4] = rng.integers(-4, 2 * max(ni, nj, nk) + 4, (n // 4, 3)) * (0.5 * dx)   # lattice
    if spec.startswith("faces"):
        a = int(spec[-1])
        s, r = 1, 1.5 * dx
        sh = np.zeros(3)
        sh[a] = 0.5 * dx
        ext = np.array([ni, nj, nk]) + (np.arange(3) == a)
    else:
        s, r = int(spec[-1]), 0.93 * dx * (1 + (spec == "field1"))
        sh = np.zeros(3)
        ext = np.array([ni, nj, nk]) * s + 1
    p = pos + sh
    g0 = _trunc_div((-r) + p, dx)
    g1 = _trunc_div(p + r, dx)
    lo, hi = (g0, g1) if s == 1 else (g0 * s, (g1 + 1) * s)
    nb = (ext + s - 1) // s
    hits = np.all((hi >= 0) & (lo <= ext - 1), axis=1)
    assert hits.sum() > n // 2 and (~hits).sum() > 0
    bc = np.minimum(np.maximum(lo, 0) // s, nb - 1)
    span = (np.minimum(hi, ext - 1) // s - bc)[hits].max(axis=0)
    assert (span >= 0).all()
    lo_t, hi_t = np.maximum(lo, 0)[hits], np.minimum(hi, ext - 1)[hits]
    b = lambda t: np.minimum(t // s, nb - 1)   # noqa: E731
    # b is monotone: the window condition at both ends of the covered range
    assert (bc[hits] <= b(lo_t)).all()
    assert (bc[hits] >= b(hi_t) - span).all()


def test_seed_particles_follow_the_reference_layout():
    mat = np.zeros((3, 3, 3), np.uint8)
    mat[1, 2, 0] = 1
    P = scenes.seed_particles(mat, 0.5, jitter=0.0, vel_scale=0.0)
    c = np.array([0.25, 1.25, 0.75])
    assert P.shape == (8, 6) and not P[:, 3:].any()
    assert np.allclose(P[:, :3] - c, 0.125 * np.array(
        [(-1, -1, -1), (1, -1, -1), (1, -1, 1), (-1, -1, 1), (-1, 1, -1), (1, 1, -1), (1, 1, 1), (-1, 1, 1)]))


def test_python_particle_steps_check_arguments_before_the_library():
    """Shapes and dtypes are checked on the host, before any library call."""
    from xfluid_b200.particles import ParticleSteps
    s = ParticleSteps(0.1)
    mat = np.zeros((4, 5, 6), np.uint8)
    P = np.zeros((10, 6))
    faces = [np.zeros(sh) for sh in scenes.face_shapes(6, 5, 4)]
    with pytest.raises(ValueError):
        s.updateMaterial(np.zeros((10, 5)), mat)
    with pytest.raises(ValueError):
        s.updateMaterial(P.astype(np.float32), mat)
    with pytest.raises(ValueError):
        s.updateMaterial(P, mat.astype(np.int32))
    with pytest.raises(ValueError):
        s.advectParticles(P, mat, faces, [np.zeros((4, 5, 8))] * 3, 0.1)
    with pytest.raises(ValueError):
        s.advectParticles(P, mat, faces[::-1], faces, 0.1)
    with pytest.raises(ValueError):
        s.updateVelocityByParticles(P, [faces[0], faces[0], faces[2]])
    with pytest.raises(ValueError):
        s.updateField(P, mat, subdiv=2, phi=np.zeros((9, 11, 12)))
    assert s._ctx == {}


class _FakeCudaTensor:
    """Stands in for a CUDA tensor on a CPU-only host: shape, dtype, layout and
    device are all the argument checks look at."""

    def __init__(self, shape, dtype, contiguous=True, index=0):
        self.shape, self.dtype, self._contig = tuple(shape), dtype, contiguous
        self.is_cuda = True
        self.device = type("Dev", (), {"index": index, "__str__": lambda d: f"cuda:{d.index}"})()

    def is_contiguous(self):
        return self._contig


def test_python_particle_steps_reject_strided_and_foreign_device_tensors():
    """A strided view such as x[:, :6] of an (n, 8) tensor has the right shape
    and dtype, but the kernels would read and write 6n contiguous doubles from
    its data pointer; a tensor on another GPU would be dereferenced from the
    context's device.  Both are refused before any library call."""
    from xfluid_b200.particles import ParticleSteps
    s = ParticleSteps(0.1, device=0)
    mat = _FakeCudaTensor((4, 5, 6), "torch.uint8")
    sliced = _FakeCudaTensor((10, 6), "torch.float64", contiguous=False)
    with pytest.raises(ValueError, match="contiguous"):
        s.updateMaterial(sliced, mat)
    other = _FakeCudaTensor((10, 6), "torch.float64", index=1)
    with pytest.raises(ValueError, match="cuda:1"):
        s.updateMaterial(other, mat)
    with pytest.raises(ValueError, match="contiguous"):
        s.updateMaterial(_FakeCudaTensor((10, 6), "torch.float64"),
                         _FakeCudaTensor((4, 5, 6), "torch.uint8", contiguous=False))
    assert s._ctx == {}


# ------------------------------------------------------------------ GPU: the C ABI
def _ctx(**kw):
    from gpu_util import make_ctx
    return make_ctx("f64", **kw)


def _p(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


def _gpu_advect(ctx, sc, saved, P, ratio, dt, dx):
    out = np.array(P)
    g = [np.ascontiguousarray(a, np.float64) for a in (sc.u, sc.v, sc.w, *saved)]
    ctx.check(ctx.lib.xfp_advect_particles_f64(ctx.ptr, sc.ni, sc.nj, sc.nk, dx,
                                               _p(np.ascontiguousarray(sc.mat, np.uint8)), *map(_p, g), ratio, dt,
                                               len(out), _p(out)))
    return out


def _gpu_p2g(ctx, dims, dx, P):
    ni, nj, nk = dims
    u, v, w = np.full((nk, nj, ni + 1), 7.0), np.full((nk, nj + 1, ni), 7.0), np.full((nk + 1, nj, ni), 7.0)
    ctx.check(ctx.lib.xfp_particles_to_grid_f64(ctx.ptr, ni, nj, nk, dx, len(P), _p(np.ascontiguousarray(P)),
                                                _p(u), _p(v), _p(w)))
    return u, v, w


def _gpu_field(ctx, mat, dx, s, rad, thr, P):
    nk, nj, ni = mat.shape
    phi = np.zeros((nk * s + 1, nj * s + 1, ni * s + 1))
    m = np.array(mat, np.uint8)
    ctx.check(ctx.lib.xfp_distance_field_f64(ctx.ptr, ni, nj, nk, dx, s, rad, thr, len(P),
                                             _p(np.ascontiguousarray(P)), _p(phi), _p(m)))
    return phi, m


def _classification_equal(m_gpu, m_ref, phi_ref, s, thr):
    """Equal material, except at cells whose vertices hold a value within
    rounding of the threshold (phi's summation order can move such a value
    across it); every other difference fails."""
    diff = m_gpu != m_ref
    if not diff.any():
        return True
    nk, nj, ni = m_ref.shape
    near = 0
    for k, j, i in zip(*np.nonzero(diff)):
        blk = phi_ref[k * s:k * s + s + 1, j * s:j * s + s + 1, i * s:i * s + s + 1]
        near += bool((np.abs(blk - thr) <= 1e-12 * max(1.0, abs(thr))).any())
    return near == int(diff.sum())


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_gpu_particle_steps_match_reference_vectors(name):
    z = np.load(GOLDEN / name)
    sc, dx, P = _scene(z), float(z["dx"]), z["parts_in"]
    ctx = _ctx()
    try:
        out = _gpu_advect(ctx, sc, _saved(z), P, float(z["ratio"]), float(z["dt"]), dx)
        keep = ~z["ub"]
        assert np.array_equal(out[keep], z["parts_out"][keep])
        dims = (sc.ni, sc.nj, sc.nk)
        for a, k in zip(_gpu_p2g(ctx, dims, dx, P), ("u_p2g", "v_p2g", "w_p2g")):
            assert _maxrel(a, z[k]) <= TRANSFER_TOL, (k, _maxrel(a, z[k]))
        s, rad, thr = int(z["subdiv"]), float(z["radius"]), float(z["threshold"])
        phi, ms = _gpu_field(ctx, z["mat"], dx, s, rad, thr, P)
        assert _maxrel(phi, z["phi"]) <= TRANSFER_TOL
        assert _classification_equal(ms, z["mat_surface"], z["phi"], s, thr)
        m = np.array(z["mat_surface"])
        ctx.check(ctx.lib.xfp_update_material(ctx.ptr, *dims, dx, len(P), _p(np.ascontiguousarray(P)), _p(m)))
        assert np.array_equal(m, z["mat_final"])
    finally:
        ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("seed,dims,dt,jitter", [(7, (40, 36, 44), 0.05, 0.2), (8, (33, 29, 31), 0.3, 0.45)])
def test_gpu_particle_steps_vs_oracle_every_particle(seed, dims, dt, jitter):
    """Every particle, the collision outcomes included (status 2 too: both
    sides keep those particles in place), bitwise; transfers to 1e-12."""
    sc, dx, P, saved = _case(seed, dims, jitter=jitter, vel=4.0)
    O = oracle.Oracle()
    ref, st = O.advect_particles(sc, saved, P, 0.95, dt, dx, status=True)
    assert (st == 1).sum() > 0 and (st == 3).sum() > 0
    ctx = _ctx()
    try:
        out = _gpu_advect(ctx, sc, saved, P, 0.95, dt, dx)
        assert np.array_equal(out, ref)
        g = _gpu_p2g(ctx, (sc.ni, sc.nj, sc.nk), dx, out)
        for a, b in zip(g, O.p2g((sc.ni, sc.nj, sc.nk), dx, out)):
            assert _maxrel(a, b) <= TRANSFER_TOL
        for s, rad in ((2, 0.93 * dx), (3, 2.2 * dx), (1, 1.5 * dx)):
            phi, m = _gpu_field(ctx, sc.mat, dx, s, rad, 0.4, out)
            phi_o, m_o = O.distance_field(sc.mat, dx, s, rad, 0.4, out)
            assert _maxrel(phi, phi_o) <= TRANSFER_TOL, (s, _maxrel(phi, phi_o))
            assert _classification_equal(m, m_o, phi_o, s, 0.4)
        m = np.array(sc.mat)
        ctx.check(ctx.lib.xfp_update_material(ctx.ptr, sc.ni, sc.nj, sc.nk, dx, len(out), _p(out), _p(m)))
        assert np.array_equal(m, O.update_material(sc.mat, dx, out))
    finally:
        ctx.close()


@pytest.mark.gpu
def test_gpu_particles_outside_the_grid_and_edge_cases():
    """Particles outside the domain (they bin at the edge and cover no face, or
    the faces their boxes reach), on the far walls exactly, no particles, and
    the argument rules."""
    from xfluid_b200 import _lib
    ni, nj, nk, dx = 12, 10, 9, 0.1
    rng = np.random.default_rng(3)
    P = np.zeros((600, 6))
    P[:, :3] = rng.uniform(-0.35, 1.35, (600, 3)) * np.array([ni, nj, nk]) * dx
    P[:, 3:] = rng.standard_normal((600, 3))
    P[:6, 0] = ni * dx   # on the far x wall (the reference reads face ni+1 there)
    P[6:12, 1] = nj * dx
    O = oracle.Oracle()
    mat = np.zeros((nk, nj, ni), np.uint8)
    scenes.solid_border(mat)
    mat[2:6, 3:7, 4:8] = 1
    sc = scenes.Scene(ni, nj, nk, mat, *[rng.standard_normal(s) for s in scenes.face_shapes(ni, nj, nk)])
    saved = [rng.standard_normal(a.shape) for a in (sc.u, sc.v, sc.w)]
    ctx = _ctx()
    try:
        assert np.array_equal(_gpu_advect(ctx, sc, saved, P, 0.95, 0.02, dx),
                              O.advect_particles(sc, saved, P, 0.95, 0.02, dx))
        for a, b in zip(_gpu_p2g(ctx, (ni, nj, nk), dx, P), O.p2g((ni, nj, nk), dx, P)):
            assert _maxrel(a, b) <= TRANSFER_TOL
        for a in _gpu_p2g(ctx, (ni, nj, nk), dx, P[:0]):
            assert not a.any()   # no particles: every face 0
        phi, m = _gpu_field(ctx, mat, dx, 2, 0.093, 0.4, P)
        phi_o, m_o = O.distance_field(mat, dx, 2, 0.093, 0.4, P)
        assert _maxrel(phi, phi_o) <= TRANSFER_TOL and _classification_equal(m, m_o, phi_o, 2, 0.4)
        # argument rules
        assert ctx.lib.xfp_particles_to_grid_f64(ctx.ptr, ni, nj, nk, dx, 5, None, _p(sc.u), _p(sc.v),
                                                 _p(sc.w)) == _lib.XFP_ERR_ARGS
        assert ctx.lib.xfp_particles_to_grid_f64(ctx.ptr, ni, nj, nk, 0.0, len(P), _p(P), _p(sc.u), _p(sc.v),
                                                 _p(sc.w)) == _lib.XFP_ERR_ARGS
        assert ctx.lib.xfp_distance_field_f64(ctx.ptr, ni, nj, nk, dx, 0, 0.1, 0.4, len(P), _p(P), _p(phi),
                                              None) == _lib.XFP_ERR_ARGS
        assert ctx.lib.xfp_distance_field_f64(ctx.ptr, ni, nj, nk, dx, 2, 0.1, 0.4, len(P), _p(P), None,
                                              None) == _lib.XFP_ERR_ARGS
    finally:
        ctx.close()


@pytest.mark.gpu
def test_python_particle_steps_on_cuda_tensors_match_host_arrays():
    """ParticleSteps (the Python mirror) on CUDA tensors in place gives the
    same bits as on numpy arrays."""
    import torch
    from xfluid_b200.particles import ParticleSteps
    sc, dx, P, saved = _case(9, (30, 26, 22), jitter=0.3, vel=3.0)
    uvw = [np.array(a, np.float64) for a in (sc.u, sc.v, sc.w)]
    host = ParticleSteps(dx)
    try:
        Ph = np.array(P)
        mat_h = np.array(sc.mat, np.uint8)
        host.advectParticles(Ph, mat_h, uvw, saved, 0.1)
        gh = [np.zeros_like(a) for a in uvw]
        host.updateVelocityByParticles(Ph, gh)
        host.updateMaterial(Ph, mat_h)
        phi_h = host.updateField(Ph, mat_h)
    finally:
        host.close()
    dev = ParticleSteps(dx)
    t = lambda a: torch.from_numpy(np.array(a)).cuda()   # noqa: E731
    try:
        Pd, mat_d = t(P), t(np.array(sc.mat, np.uint8))
        dev.advectParticles(Pd, mat_d, [t(a) for a in uvw], [t(a) for a in saved], 0.1)
        gd = [torch.zeros_like(t(a)) for a in uvw]
        dev.updateVelocityByParticles(Pd, gd)
        dev.updateMaterial(Pd, mat_d)
        phi_d = dev.updateField(Pd, mat_d)
    finally:
        dev.close()
    assert np.array_equal(Pd.cpu().numpy(), Ph)
    for a, b in zip(gd, gh):
        assert np.array_equal(a.cpu().numpy(), b)
    assert np.array_equal(mat_d.cpu().numpy(), mat_h)
    assert np.array_equal(phi_d.cpu().numpy(), phi_h)


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [0, 2, 6])
def test_gpu_particle_steps_on_random_masks_with_interior_solids(seed):
    """The random fluid/air/solid masks of the oracle sweep (interior solids,
    collision-heavy): advection and the material update bitwise against the
    oracle on every particle, the transfers to 1e-12."""
    import sys
    sys.path.insert(0, str(Path(__file__).parent))
    from test_oracle_sweep import _random_scene
    sc = _random_scene(seed)
    rng = np.random.default_rng(3000 + seed)
    dx = 1.0 / max(sc.ni, sc.nj, sc.nk)
    P = scenes.seed_particles(sc.mat, dx, seed=seed, jitter=0.3 * dx, vel_scale=4.0)
    extra = np.concatenate([rng.uniform(0, 1, (200, 3)) * np.array([sc.ni, sc.nj, sc.nk]) * dx,
                            rng.uniform(-4, 4, (200, 3))], 1)
    P = np.concatenate([P, extra])
    uvw = [np.clip(a, -50.0, 50.0) for a in (sc.u, sc.v, sc.w)]
    sc = scenes.Scene(sc.ni, sc.nj, sc.nk, sc.mat, *uvw)
    saved = [a + 0.1 * rng.standard_normal(a.shape) for a in uvw]
    O = oracle.Oracle()
    ref, st = O.advect_particles(sc, saved, P, 0.95, 0.08, dx, status=True)
    assert (st == 1).sum() + (st == 3).sum() > len(P) // 10
    ctx = _ctx()
    try:
        out = _gpu_advect(ctx, sc, saved, P, 0.95, 0.08, dx)
        assert np.array_equal(out, ref)
        for a, b in zip(_gpu_p2g(ctx, (sc.ni, sc.nj, sc.nk), dx, out), O.p2g((sc.ni, sc.nj, sc.nk), dx, out)):
            assert _maxrel(a, b) <= TRANSFER_TOL
        radius = 3.0 * (3 * (dx ** 3 / 8.0) / (4 * 3.141592653)) ** (1.0 / 3.0)
        phi, m = _gpu_field(ctx, sc.mat, dx, 2, radius, 0.4, out)
        phi_o, m_o = O.distance_field(sc.mat, dx, 2, radius, 0.4, out)
        assert _maxrel(phi, phi_o) <= TRANSFER_TOL and _classification_equal(m, m_o, phi_o, 2, 0.4)
        mm = np.array(sc.mat)
        ctx.check(ctx.lib.xfp_update_material(ctx.ptr, sc.ni, sc.nj, sc.nk, dx, len(out), _p(out), _p(mm)))
        assert np.array_equal(mm, O.update_material(sc.mat, dx, out))
    finally:
        ctx.close()
