"""Host-pointer mode with page-locked velocity arrays: only the faces that
border fluid cross PCIe (read from and written to the caller's arrays in
place).  The results must be bit-identical to the device-pointer path and to
the whole-array copies used for pageable arrays; faces away from the fluid
must keep the caller's values; the stats must report the bytes moved."""
import numpy as np
import pytest

from xfluid_b200 import scenes
from xfluid_b200.solver import VariationalPressureSolver

pytestmark = pytest.mark.gpu


def _pinned(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).pin_memory()


def _run(sc, kind, precision="mixed", dtype=np.float32, call="project"):
    """kind: 'device' (CUDA tensors), 'pinned' (page-locked host tensors),
    'pageable' (numpy).  Returns (u, v, w, p) as numpy and the call's stats."""
    import torch
    s = VariationalPressureSolver(precision=precision, tol=1e-6, max_iter=300)
    try:
        s.setSize(sc.ni, sc.nj, sc.nk)
        arrs = [np.ascontiguousarray(a, dtype) for a in (sc.u, sc.v, sc.w)]
        p = np.zeros((sc.nk, sc.nj, sc.ni), dtype)
        mat = np.ascontiguousarray(sc.mat)
        if kind == "device":
            arrs = [torch.from_numpy(a).cuda() for a in arrs]
            p, mat = torch.from_numpy(p).cuda(), torch.from_numpy(mat).cuda()
        elif kind == "pinned":
            arrs = [_pinned(a) for a in arrs]
            p, mat = _pinned(p), _pinned(mat)
        s.setMaterial(mat)
        s.setVelocityField(*arrs)
        if call == "project":
            assert s.project(p)
            st = dict(s.stats)
        else:
            s.solve(p)
            st = dict(s.stats)
            s.applyPressure(p)
        out = [a.cpu().numpy() if hasattr(a, "cpu") else a for a in (*arrs, p)]
        return out, st
    finally:
        s.close()


@pytest.mark.parametrize("scene", ["blob", "dam"])
def test_pinned_project_moves_only_fluid_faces_and_matches_device(scene):
    sc = (scenes.blob_scene(64, seed=7, dtype=np.float32) if scene == "blob"
          else scenes.dam_break(64, noise=0.5, dtype=np.float32))
    ref, st_dev = _run(sc, "device")
    pin, st_pin = _run(sc, "pinned")
    full, st_full = _run(sc, "pageable")
    for a, b, c in zip(ref, pin, full):
        assert np.array_equal(a, b)
        assert np.array_equal(a, c)
    assert st_pin["host_faces"] == 1 and st_full["host_faces"] == 0 and st_dev["host_faces"] == 0
    n = sc.ni * sc.nj * sc.nk
    faces = (sc.ni + 1) * sc.nj * sc.nk + sc.ni * (sc.nj + 1) * sc.nk + sc.ni * sc.nj * (sc.nk + 1)
    # whole arrays: material + velocities in, pressure + velocities out
    assert st_full["h2d_bytes"] == n + 4 * faces
    assert st_full["d2h_bytes"] == 4 * n + 4 * faces
    # face-sparse: the same material and pressure, and the fluid-bordering
    # spans of the velocities (equal both ways)
    sparse_in = st_pin["h2d_bytes"] - n
    assert sparse_in == st_pin["d2h_bytes"] - 4 * n
    assert 0 < sparse_in < 4 * faces
    # the span count from the material: every face row's first..last face
    # with a fluid side
    f = sc.mat == 1
    expect = 0
    for axis in range(3):
        a = np.moveaxis(f, 2 - axis, 0)          # axis of the faces first
        both = np.zeros((a.shape[0] + 1,) + a.shape[1:], bool)
        both[:-1] |= a
        both[1:] |= a                             # face borders fluid on either side
        rows = np.moveaxis(both, 0, 2 - axis).reshape(-1, (sc.ni + (axis == 0)))
        idx = np.arange(rows.shape[1])
        lo = np.where(rows, idx, rows.shape[1]).min(1)
        hi = np.where(rows, idx, -1).max(1)
        expect += int(np.where(hi >= lo, hi - lo + 1, 0).sum())
    assert sparse_in == 4 * expect


def test_pinned_solve_then_apply_matches_pageable():
    sc = scenes.blob_scene(48, seed=11, dtype=np.float32)
    pin, _ = _run(sc, "pinned", call="solve_apply")
    full, _ = _run(sc, "pageable", call="solve_apply")
    for a, b in zip(pin, full):
        assert np.array_equal(a, b)


def test_pinned_fp64_project_matches_device():
    sc = scenes.blob_scene(40, seed=5, dtype=np.float64)
    ref, _ = _run(sc, "device", precision="f64", dtype=np.float64)
    pin, st = _run(sc, "pinned", precision="f64", dtype=np.float64)
    assert st["host_faces"] == 1
    for a, b in zip(ref, pin):
        assert np.array_equal(a, b)


def test_faces_away_from_fluid_keep_the_callers_values():
    """Sentinels on faces with no fluid side survive a face-sparse call (the
    device path leaves them too: the projection does not touch them)."""
    sc = scenes.dam_break(48, noise=0.5, dtype=np.float32)
    u = np.ascontiguousarray(sc.u, np.float32).copy()
    f = sc.mat == 1
    border = np.zeros(u.shape, bool)
    border[:, :, :-1] |= f
    border[:, :, 1:] |= f
    u[~border] = 12345.0
    sc2 = scenes.Scene(sc.ni, sc.nj, sc.nk, sc.mat, u, sc.v, sc.w)
    pin, st = _run(sc2, "pinned")
    assert st["host_faces"] == 1
    assert np.all(pin[0][~border] == 12345.0)
