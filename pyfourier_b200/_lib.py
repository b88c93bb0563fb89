"""ctypes binding of libpfb200.so (the C ABI declared in include/pfb200.h).

The shared library is built in-tree by ``pyfourier_b200._build``.  There is no
fallback: if the library is missing or fails to load, every operator raises.
"""

from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpfb200.so")

PFB_OK = 0
PFB_ERR_INVALID = 1
PFB_ERR_CUDA = 2
PFB_ERR_CUFFT = 3
PFB_ERR_NOMEM = 4
PFB_ERR_UNSUPPORTED = 5
PFB_ERR_WORKSPACE = 6
PFB_ERR_DEVICE = 7
PFB_NORM_NONE = 0
PFB_NORM_ORTHO = 1
PFB_FLAG_ACCUMULATE = 1
STAGES = {"pad": 0, "fft": 1, "interp": 2, "out": 3, "vals": 4, "spread": 5, "ifft": 6, "crop": 7,
          "transpose": 8}

# Every symbol exported by the C ABI (kept in sync with include/pfb200.h).
EXPORTS = (
    "pfb_last_error", "pfb_version", "pfb_plan_create", "pfb_plan_destroy", "pfb_plan_info", "pfb_dcf_workspace_size", "pfb_pipe_menon_dcf",
    "pfb_plan_set_tuning", "pfb_plan_set_chunk", "pfb_plan_tables", "pfb_workspace_size",
    "pfb_nufft_fwd", "pfb_nufft_adj", "pfb_spread", "pfb_interp", "pfb_deapod_pad",
    "pfb_crop_deapod", "pfb_grid_fft", "pfb_traj_grad", "pfb_gram_create", "pfb_gram_destroy",
    "pfb_gram_workspace_size", "pfb_gram_apply", "pfb_nufft_adj_noalloc",
    "pfb_grog_create", "pfb_grog_destroy", "pfb_grog_workspace_size", "pfb_grog_apply",
    "pfb_apply_workspace_size", "pfb_nufft_traj_grad", "pfb_nufft_stage", "pfb_plan_order", "pfb_spread_f64",
    "pfb_plan_check", "pfb_release_cached_memory",
)


class PfbError(RuntimeError):
    """Raised when a libpfb200 call returns a non-zero status."""

    def __init__(self, status, message):
        super().__init__(f"libpfb200 status {status}: {message}")
        self.status = status


class ApplyT(ctypes.Structure):
    _fields_ = [
        ("batch", ctypes.c_int64),
        ("ncoeff", ctypes.c_int32),
        ("nseg", ctypes.c_int32),
        ("basis", ctypes.c_void_p),
        ("weight", ctypes.c_void_p),
        ("b0_time", ctypes.c_void_p),
        ("b0_space", ctypes.c_void_p),
        ("norm", ctypes.c_int32),
        ("flags", ctypes.c_int32),
    ]


class PlanInfoT(ctypes.Structure):
    _fields_ = [
        ("ndim", ctypes.c_int32),
        ("nframes", ctypes.c_int32),
        ("total_samples", ctypes.c_int64),
        ("shape", ctypes.c_int32 * 3),
        ("os_shape", ctypes.c_int32 * 3),
        ("width", ctypes.c_int32 * 3),
        ("tile", ctypes.c_int32 * 3),
        ("scale", ctypes.c_double),
        ("n_items", ctypes.c_int32),
        ("max_bin", ctypes.c_int32),
        ("tile_offset", ctypes.c_int32 * 3),
    ]


_lib = None


def load(path=LIB_PATH):
    """Load the library (once).  Raises ImportError if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(
            f"{path} is missing: build it with `python -m pyfourier_b200._build` "
            "(pyfourier_b200 has no CPU fallback)")
    L = ctypes.CDLL(path)
    vp, i32, i64, f32 = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_float
    P = ctypes.POINTER
    sig = {
        "pfb_last_error": (ctypes.c_char_p, []),
        "pfb_version": (ctypes.c_char_p, []),
        "pfb_plan_create": (i32, [vp, i32, i32, P(ctypes.c_int64), i32, P(ctypes.c_int), P(ctypes.c_int),
                                  P(ctypes.c_int), P(ctypes.c_float), P(ctypes.c_int), P(ctypes.c_int),
                                  i32, vp, P(vp)]),
        "pfb_plan_destroy": (i32, [vp]),
        "pfb_plan_info": (i32, [vp, P(PlanInfoT)]),
        "pfb_dcf_workspace_size": (i32, [vp, P(ctypes.c_size_t)]),
        "pfb_pipe_menon_dcf": (i32, [vp, vp, i32, vp, ctypes.c_size_t, vp]),
        "pfb_plan_set_tuning": (i32, [vp, i32, i32, i32]),
        "pfb_plan_set_chunk": (i32, [vp, i32]),
        "pfb_plan_tables": (i32, [vp, i32, vp, vp, vp]),
        "pfb_plan_order": (i32, [vp, vp, vp]),
        "pfb_plan_check": (i32, [vp, vp]),
        "pfb_release_cached_memory": (i32, [i32]),
        "pfb_workspace_size": (i32, [vp, i64, P(ctypes.c_size_t)]),
        "pfb_nufft_fwd": (i32, [vp, P(ApplyT), vp, vp, vp, ctypes.c_size_t, vp]),
        "pfb_nufft_adj": (i32, [vp, P(ApplyT), vp, vp, vp, ctypes.c_size_t, vp]),
        "pfb_spread": (i32, [vp, P(ApplyT), vp, vp, i32, vp]),
        "pfb_interp": (i32, [vp, P(ApplyT), vp, vp, i32, vp]),
        "pfb_deapod_pad": (i32, [vp, P(ApplyT), vp, vp, f32, vp]),
        "pfb_crop_deapod": (i32, [vp, P(ApplyT), vp, vp, f32, vp]),
        "pfb_grid_fft": (i32, [vp, vp, i64, i32, vp, ctypes.c_size_t, vp]),
        "pfb_traj_grad": (i32, [vp, P(ApplyT), vp, vp, vp, i32, vp]),
        "pfb_spread_f64": (i32, [vp, vp, i32, vp, vp]),
        "pfb_gram_create": (i32, [i32, P(ctypes.c_int), P(ctypes.c_int), i32, i32, i32, vp, i32, vp, P(vp)]),
        "pfb_gram_destroy": (i32, [vp]),
        "pfb_gram_workspace_size": (i32, [vp, i64, P(ctypes.c_size_t)]),
        "pfb_gram_apply": (i32, [vp, vp, vp, i64, vp, vp, ctypes.c_size_t, vp]),
        "pfb_nufft_adj_noalloc": (i32, [vp, P(ApplyT), vp, vp, vp]),
        "pfb_grog_create": (i32, [vp, i64, i32, i32, i32, vp, i32, vp, P(vp)]),
        "pfb_grog_destroy": (i32, [vp]),
        "pfb_grog_workspace_size": (i32, [vp, i64, P(ctypes.c_size_t)]),
        "pfb_grog_apply": (i32, [vp, vp, vp, i64, vp, ctypes.c_size_t, vp]),
        "pfb_apply_workspace_size": (i32, [vp, P(ApplyT), P(ctypes.c_size_t)]),
        "pfb_nufft_traj_grad": (i32, [vp, P(ApplyT), vp, vp, vp, f32, vp, ctypes.c_size_t, vp]),
        "pfb_nufft_stage": (i32, [vp, P(ApplyT), i32, vp, vp, f32, vp, ctypes.c_size_t, vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def check(status):
    """Turn a non-zero status into an exception carrying pfb_last_error()."""
    if status != PFB_OK:
        msg = load().pfb_last_error().decode(errors="replace")
        if status == PFB_ERR_INVALID:
            raise ValueError(f"libpfb200: {msg}")
        if status == PFB_ERR_UNSUPPORTED:
            raise NotImplementedError(f"libpfb200: {msg}")
        raise PfbError(status, msg)


def int_array(values):
    vals = [int(v) for v in values]
    return (ctypes.c_int * len(vals))(*vals)


def float_array(values):
    vals = [float(v) for v in values]
    return (ctypes.c_float * len(vals))(*vals)
