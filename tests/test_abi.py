"""The C ABI (include/xfp.h) and the host-side layers, without a GPU."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    src = (ROOT / "include" / "xfp.h").read_text()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(xfp_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    from xfluid_b200 import build
    build.build()
    from xfluid_b200 import _lib
    return _lib.load()


def test_library_exports_every_declared_symbol(lib):
    names = declared_functions()
    assert "xfp_project_f32" in names and "xfp_project_backward_f64" in names
    for name in names:
        assert hasattr(lib, name), name
    from xfluid_b200 import _lib
    assert sorted(_lib.EXPORTS) == names


def test_default_options_are_the_reference_defaults(lib):
    from xfluid_b200 import _lib
    o = _lib.default_options()
    # PCGSolver() : set_solver_parameters(1e-5, 100, 0.97, 0.25)  (pcg_solver.h:229-232)
    assert (o.tol, o.max_iter, o.omega, o.min_diag_ratio) == (1e-5, 100, 0.97, 0.25)
    assert lib.xfp_version().startswith(b"xfp")


def test_product_path_fails_loudly_without_gpu(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from xfluid_b200 import _lib
    from xfluid_b200.solver import VariationalPressureSolver
    with pytest.raises(_lib.XfpError):
        VariationalPressureSolver()


def test_null_context_is_rejected(lib):
    from xfluid_b200 import _lib
    st = _lib.XfpStats()
    rc = lib.xfp_solve_f64(None, 4, 4, 4, None, None, None, None, None, None, None, None, C.byref(st))
    assert rc == _lib.XFP_ERR_ARGS


def test_particle_and_diagnostic_entry_points_reject_a_null_context(lib):
    """The particle steps and the divergence diagnostic check their context
    before touching CUDA (no GPU needed)."""
    from xfluid_b200 import _lib
    E = _lib.XFP_ERR_ARGS
    assert lib.xfp_advect_particles_f64(None, 4, 4, 4, 0.25, *[None] * 7, 0.95, 0.01, 0, None) == E
    assert lib.xfp_particles_to_grid_f64(None, 4, 4, 4, 0.25, 0, None, None, None, None) == E
    assert lib.xfp_update_material(None, 4, 4, 4, 0.25, 0, None, None) == E
    assert lib.xfp_distance_field_f64(None, 4, 4, 4, 0.25, 2, 0.2, 0.4, 0, None, None, None) == E
    assert lib.xfp_divergence_f64(None, 4, 4, 4, None, None, None, None, None) == E
    assert lib.xfp_divergence_f32(None, 4, 4, 4, None, None, None, None, None) == E


def test_particle_record_is_the_reference_layout():
    """xfp_particle is xFluid's struct Particle {Vec3d p; Vec3d v;}: six
    doubles, p first (particle.h:5-15), as include/xfp.h declares it."""
    src = (ROOT / "include" / "xfp.h").read_text()
    assert "typedef struct {\n  double p[3];\n  double v[3];\n} xfp_particle;" in src

    class Particle(C.Structure):
        _fields_ = [("p", C.c_double * 3), ("v", C.c_double * 3)]
    assert C.sizeof(Particle) == 48 and Particle.v.offset == 24


def test_scene_generators_are_seeded_and_shaped():
    from xfluid_b200 import scenes
    a = scenes.blob_scene(dims=(20, 18, 16), seed=4)
    b = scenes.blob_scene(dims=(20, 18, 16), seed=4)
    assert np.array_equal(a.mat, b.mat) and np.array_equal(a.u, b.u)
    assert a.u.shape == (16, 18, 21) and a.v.shape == (16, 19, 20) and a.w.shape == (17, 18, 20)
    assert a.u.dtype == np.float32
    # solid border ring, as FluidSimulator::setSolidBoundary requires
    for face in (a.mat[0], a.mat[-1], a.mat[:, 0], a.mat[:, -1], a.mat[:, :, 0], a.mat[:, :, -1]):
        assert np.all(face == scenes.SOLID)
    assert np.all((a.wu >= 0) & (a.wu <= 1))
    d = scenes.dam_break(dims=(24, 20, 16))
    fl = d.mat == scenes.FLUID
    assert fl.any() and not fl[:, :, 23 - 1].any()


def test_batch_scene_sizes():
    from xfluid_b200 import scenes
    bs = scenes.batch_scenes(count=5, seed=4, lo=32, hi=40)
    assert len(bs) == 5
    for s in bs:
        assert 32 <= s.ni <= 40 and 32 <= s.nj <= 40 and 32 <= s.nk <= 40
