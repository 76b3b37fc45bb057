"""xfp_rhs_inf_noalloc_f64: |b|_inf without allocating device memory.

This entry point exists for callers that must not call cudaMalloc/cudaFree
(a real-time loop that cannot take cudaFree's device-wide synchronisation, or
an application whose allocator has reserved the device's memory).  Its only
scratch is a fixed __device__ array shared by every call, so these tests call
it several times in a row, on different scenes, and check each result against
the value the regular solve reports (xfp_solve_f64's stats.b_inf).  Both are
FP64 with the same operation order, so the tolerance is exact equality, as in
the other FP64 stage tests.

The file is named to be collected last: it runs after every other test in a
full run and passes on its own in a fresh process too.
"""
import ctypes as C

import numpy as np
import pytest

from xfluid_b200 import _lib, scenes

MAX_CELLS = 268_435_456  # the entry point's stated limit (fixed 128 KiB scratch)


def _call(lib, ni, nj, nk, ptrs, out_ptr):
    err = C.create_string_buffer(256)
    rc = lib.xfp_rhs_inf_noalloc_f64(ni, nj, nk, *ptrs, out_ptr, None, err, len(err))
    return rc, err.value.decode()


def test_rejects_grids_beyond_the_limit():
    lib = _lib.load()
    dummy = C.c_void_p(16)  # never dereferenced: sizes are checked first
    rc, msg = _call(lib, 1024, 512, 513, [dummy] * 4 + [None] * 3, dummy)
    assert rc == _lib.XFP_ERR_ARGS
    assert "no-allocation limit" in msg and str(MAX_CELLS) in msg
    rc, msg = _call(lib, 0, 4, 4, [dummy] * 4 + [None] * 3, dummy)
    assert rc == _lib.XFP_ERR_ARGS


def _scenes():
    a = scenes.blob_scene(48, seed=5, dtype=np.float64)           # fractional face weights
    b = scenes.dam_break(40, seed=2, noise=0.5)                   # xFluid's matrix (no weights)
    c = scenes.blob_scene(dims=(30, 70, 40), seed=6, fractional=False, dtype=np.float64)
    return [(a, True), (b, False), (c, False)]


@pytest.mark.gpu
def test_matches_solve_b_inf_on_calls_in_a_row():
    import torch
    from gpu_util import make_ctx, solve

    lib = _lib.load()
    expected, dev_inputs = [], []
    ctx = make_ctx("f64", tol=1e-6, max_iter=400)
    try:
        for sc, frac in _scenes():
            _, _, st = solve(ctx, sc, dtype=np.float64, fractional=frac)
            expected.append(st["b_inf"])
            t = lambda a: None if a is None else torch.from_numpy(np.ascontiguousarray(a, np.float64)).cuda()
            wts = (sc.wu, sc.wv, sc.ww) if frac else (None, None, None)
            arrs = [torch.from_numpy(np.ascontiguousarray(sc.mat, np.uint8)).cuda(),
                    *(t(a) for a in (sc.u, sc.v, sc.w)), *(t(a) for a in wts)]
            dev_inputs.append((sc, arrs))
    finally:
        ctx.close()
    assert all(e > 0 for e in expected)

    # Output buffers and inputs come from the test; the entry point itself only
    # uses its fixed array.  Each scene twice in a row, then the first again.
    outs = [torch.full((1,), -1.0, dtype=torch.float64, device="cuda") for _ in range(7)]
    order = [0, 0, 1, 1, 2, 2, 0]
    torch.cuda.synchronize()
    for n, s in enumerate(order):
        sc, arrs = dev_inputs[s]
        ptrs = [None if a is None else C.c_void_p(a.data_ptr()) for a in arrs]
        rc, msg = _call(lib, sc.ni, sc.nj, sc.nk, ptrs, C.c_void_p(outs[n].data_ptr()))
        assert rc == _lib.XFP_OK, msg
    torch.cuda.synchronize()
    got = [o.item() for o in outs]
    for n, s in enumerate(order):
        assert got[n] == expected[s], (n, s, got[n], expected[s])


@pytest.mark.gpu
def test_rejects_host_pointers():
    import torch  # noqa: F401  (initialises the CUDA context the check runs in)

    lib = _lib.load()
    sc = scenes.blob_scene(16, seed=1, dtype=np.float64, fractional=False)
    host = [np.ascontiguousarray(sc.mat, np.uint8)] + [np.ascontiguousarray(a, np.float64) for a in (sc.u, sc.v, sc.w)]
    out = np.zeros(1)
    rc, msg = _call(lib, sc.ni, sc.nj, sc.nk, [C.c_void_p(a.ctypes.data) for a in host] + [None] * 3,
                    C.c_void_p(out.ctypes.data))
    assert rc == _lib.XFP_ERR_ARGS and "device" in msg


@pytest.mark.gpu
def test_nan_in_a_face_velocity_gives_nan():
    """A field that has blown up is not reported as finite: one NaN face of a
    fluid cell makes |b|_inf NaN (a plain fmax reduction would drop it)."""
    import torch

    lib = _lib.load()
    sc = scenes.blob_scene(24, seed=3, dtype=np.float64, fractional=False)
    k, j, i = (int(x[0]) for x in np.nonzero(sc.mat == 1))
    u = np.ascontiguousarray(sc.u, np.float64).copy()
    u[k, j, i + 1] = np.nan
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    arrs = [t(np.ascontiguousarray(sc.mat, np.uint8)), t(u), t(sc.v.astype(np.float64)), t(sc.w.astype(np.float64))]
    outs = [torch.zeros(1, dtype=torch.float64, device="cuda") for _ in range(2)]
    for n, a in enumerate((arrs, [arrs[0], t(sc.u.astype(np.float64)), arrs[2], arrs[3]])):
        rc, msg = _call(lib, sc.ni, sc.nj, sc.nk, [C.c_void_p(x.data_ptr()) for x in a] + [None] * 3,
                        C.c_void_p(outs[n].data_ptr()))
        assert rc == _lib.XFP_OK, msg
    torch.cuda.synchronize()
    assert np.isnan(outs[0].item())
    assert np.isfinite(outs[1].item()) and outs[1].item() > 0
