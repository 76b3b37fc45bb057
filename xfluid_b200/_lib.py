"""ctypes binding of libxfp.so (include/xfp.h).

The library is the product's only compute path: if it is missing or no CUDA
device is present, every call raises -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libxfp.so"

XFP_OK = 0
XFP_NOT_CONVERGED = 1
XFP_ERR_ARGS = -1
XFP_ERR_CUDA = -2
XFP_ERR_TIMEOUT = -3
XFP_ERR_NOMEM = -4
XFP_ERR_BREAKDOWN = -5
XFP_ERR_UNSUPPORTED = -6

PREC = {"f64": 0, "f32": 1, "mixed": 2}
MATRIX = {"variational": 0, "normal": 1}


class XfpOptions(C.Structure):
    _fields_ = [
        ("tol", C.c_double),
        ("max_iter", C.c_int),
        ("omega", C.c_double),
        ("min_diag_ratio", C.c_double),
        ("precision", C.c_int),
        ("device_pointers", C.c_int),
        ("device", C.c_int),
        ("check_every", C.c_int),
        ("timeout_ms", C.c_double),
        ("max_refine", C.c_int),
        ("inner_tol", C.c_double),
        ("tile_k", C.c_int),
        ("stream", C.c_void_p),
        ("matrix", C.c_int),
    ]


class XfpScene(C.Structure):
    """xfp_scene: one scene of xfp_project_batch_{f32,f64}."""
    _fields_ = [
        ("ni", C.c_int), ("nj", C.c_int), ("nk", C.c_int),
        ("material", C.c_void_p),
        ("u", C.c_void_p), ("v", C.c_void_p), ("w", C.c_void_p),
        ("wu", C.c_void_p), ("wv", C.c_void_p), ("ww", C.c_void_p),
        ("pressure", C.c_void_p),
    ]


class XfpStats(C.Structure):
    _fields_ = [
        ("status", C.c_int),
        ("iterations", C.c_int),
        ("refinements", C.c_int),
        ("residual", C.c_double),
        ("rel_residual", C.c_double),
        ("b_inf", C.c_double),
        ("rows", C.c_longlong),
        ("stored", C.c_longlong),
        ("lines", C.c_longlong),
        ("ms_setup", C.c_double),
        ("ms_factor", C.c_double),
        ("ms_solve", C.c_double),
        ("ms_apply", C.c_double),
        ("ms_total", C.c_double),
        ("bytes", C.c_double),
        ("ms_sweeps", C.c_double),
        ("sweeps", C.c_int),
        ("launches", C.c_longlong),
        ("tile_k", C.c_int),
        ("graph", C.c_int),
        ("ms_vec", C.c_double * 3),
        ("vec_launches", C.c_int * 3),
        ("h2d_bytes", C.c_longlong),
        ("d2h_bytes", C.c_longlong),
        ("host_faces", C.c_int),
    ]

    def as_dict(self) -> dict:
        d = {name: getattr(self, name) for name, _ in self._fields_}
        d["ms_vec"] = list(self.ms_vec)
        d["vec_launches"] = list(self.vec_launches)
        return d


_lib = None

# every symbol include/xfp.h declares
EXPORTS = [
    "xfp_default_options", "xfp_create", "xfp_destroy", "xfp_set_options", "xfp_last_error",
    "xfp_version", "xfp_solve_f64", "xfp_solve_f32", "xfp_apply_pressure_f64",
    "xfp_apply_pressure_f32", "xfp_project_f64", "xfp_project_f32", "xfp_project_backward_f64",
    "xfp_project_backward_f32", "xfp_debug_stages", "xfp_rhs_inf_noalloc_f64",
    "xfp_project_batch_f32", "xfp_project_batch_f64", "xfp_advect_f64", "xfp_advect_f32",
    "xfp_advect_backward_f64", "xfp_advect_backward_f32", "xfp_box_loss_f64", "xfp_box_loss_f32",
    "xfp_debug_expire_next_sweep", "xfp_apply_forces_f64", "xfp_apply_forces_f32", "xfp_extrapolate_f64",
    "xfp_extrapolate_f32", "xfp_project_step_f64", "xfp_project_step_f32", "xfp_advect_particles_f64",
    "xfp_particles_to_grid_f64", "xfp_update_material", "xfp_distance_field_f64", "xfp_divergence_f64",
    "xfp_divergence_f32", "xfp_max_speed_f64",
]


def load() -> C.CDLL:
    """Load libxfp.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m xfluid_b200.build`")
    L = C.CDLL(str(LIB_PATH))
    vp = C.c_void_p
    ctx_pp = C.POINTER(C.c_void_p)
    L.xfp_default_options.argtypes = [C.POINTER(XfpOptions)]
    L.xfp_default_options.restype = None
    L.xfp_create.argtypes = [ctx_pp, C.POINTER(XfpOptions)]
    L.xfp_destroy.argtypes = [vp]
    L.xfp_set_options.argtypes = [vp, C.POINTER(XfpOptions)]
    L.xfp_last_error.argtypes = [vp]
    L.xfp_last_error.restype = C.c_char_p
    L.xfp_version.restype = C.c_char_p
    dims = [vp, C.c_int, C.c_int, C.c_int, vp]
    L.xfp_solve_f64.argtypes = dims + [vp] * 7 + [C.POINTER(XfpStats)]
    L.xfp_solve_f32.argtypes = dims + [vp] * 7 + [C.POINTER(XfpStats)]
    L.xfp_project_f64.argtypes = dims + [vp] * 7 + [C.POINTER(XfpStats)]
    L.xfp_project_f32.argtypes = dims + [vp] * 7 + [C.POINTER(XfpStats)]
    L.xfp_apply_pressure_f64.argtypes = dims + [vp] * 7
    L.xfp_apply_pressure_f32.argtypes = dims + [vp] * 7
    L.xfp_project_backward_f64.argtypes = dims + [vp] * 9 + [C.POINTER(XfpStats)]
    L.xfp_project_backward_f32.argtypes = dims + [vp] * 9 + [C.POINTER(XfpStats)]
    L.xfp_debug_stages.argtypes = dims + [vp] * 19
    L.xfp_project_batch_f32.argtypes = [vp, C.c_int, C.POINTER(XfpScene), C.POINTER(XfpStats)]
    L.xfp_project_batch_f64.argtypes = [vp, C.c_int, C.POINTER(XfpScene), C.POINTER(XfpStats)]
    for sfx in ("f64", "f32"):
        getattr(L, "xfp_advect_" + sfx).argtypes = [vp, C.c_int, C.c_int, C.c_int] + [vp] * 6 + [C.c_double]
        getattr(L, "xfp_advect_backward_" + sfx).argtypes = [vp, C.c_int, C.c_int, C.c_int] + [vp] * 9 + [C.c_double]
        getattr(L, "xfp_box_loss_" + sfx).argtypes = [vp, C.c_int, C.c_int, C.c_int] + [vp] * 3 + [
            C.POINTER(C.c_double), C.POINTER(C.c_double)] + [vp] * 3
    L.xfp_debug_expire_next_sweep.argtypes = [vp]
    d3 = C.POINTER(C.c_double)
    for sfx in ("f64", "f32"):
        getattr(L, "xfp_apply_forces_" + sfx).argtypes = [vp, C.c_int, C.c_int, C.c_int] + [vp] * 4 + [d3, C.c_double]
        getattr(L, "xfp_extrapolate_" + sfx).argtypes = [vp, C.c_int, C.c_int, C.c_int] + [vp] * 4 + [C.c_int]
        getattr(L, "xfp_project_step_" + sfx).argtypes = ([vp, C.c_int, C.c_int, C.c_int] + [vp] * 8 +
                                                          [d3, C.c_double, C.c_int, C.POINTER(XfpStats)])
    L.xfp_rhs_inf_noalloc_f64.argtypes = [C.c_int] * 3 + [vp] * 9 + [C.c_char_p, C.c_size_t]
    for sfx in ("f64", "f32"):
        getattr(L, "xfp_divergence_" + sfx).argtypes = [vp, C.c_int, C.c_int, C.c_int] + [vp] * 5
    g = [vp, C.c_int, C.c_int, C.c_int, C.c_double]
    L.xfp_advect_particles_f64.argtypes = g + [vp] * 7 + [C.c_double, C.c_double, C.c_longlong, vp]
    L.xfp_particles_to_grid_f64.argtypes = g + [C.c_longlong] + [vp] * 4
    L.xfp_update_material.argtypes = g + [C.c_longlong, vp, vp]
    L.xfp_distance_field_f64.argtypes = g + [C.c_int, C.c_double, C.c_double, C.c_longlong, vp, vp, vp]
    L.xfp_max_speed_f64.argtypes = [vp, C.c_longlong, vp, C.POINTER(C.c_double)]
    for name in EXPORTS:
        f = getattr(L, name)
        if name not in ("xfp_default_options", "xfp_last_error", "xfp_version"):
            f.restype = C.c_int
    _lib = L
    return L


def torch_stream(device: int) -> C.c_void_p:
    """Handle of torch's current CUDA stream on `device`.  For a created
    stream a context given it runs in order with torch's work there.  Torch's
    default stream has the handle NULL, which the library reads as "no stream
    given" (the context then makes its own, unordered with torch): callers
    still wait with sync_torch before the library reads torch's tensors."""
    import torch
    return C.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def sync_torch(device: int) -> None:
    """Wait for torch's current stream on `device` (CUDA tensors about to be
    read on a context stream that is not ordered after it)."""
    import torch
    torch.cuda.current_stream(device).synchronize()


def default_options() -> XfpOptions:
    o = XfpOptions()
    load().xfp_default_options(C.byref(o))
    return o


class XfpError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"xfp error {code}: {msg}")
        self.code = code


class Context:
    """Owns one xfp_ctx (device, stream, scratch)."""

    def __init__(self, opts: XfpOptions | None = None):
        self.lib = load()
        self.opts = opts if opts is not None else default_options()
        self.ptr = C.c_void_p()
        rc = self.lib.xfp_create(C.byref(self.ptr), C.byref(self.opts))
        if rc != XFP_OK:
            raise XfpError(rc, "xfp_create failed (no CUDA device?)")

    def set_options(self, opts: XfpOptions) -> None:
        rc = self.lib.xfp_set_options(self.ptr, C.byref(opts))
        if rc != XFP_OK:
            raise XfpError(rc, self.last_error())
        self.opts = opts

    def last_error(self) -> str:
        return self.lib.xfp_last_error(self.ptr).decode()

    def check(self, rc: int) -> int:
        if rc < 0:
            raise XfpError(rc, self.last_error())
        return rc

    def close(self) -> None:
        if self.ptr:
            self.lib.xfp_destroy(self.ptr)
            self.ptr = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
