"""ctypes binding of ``libdgc.so`` (the C ABI declared in ``include/dgc.h``).

The library is built in-tree by ``diff-geocali_b200/build.py`` into
``dgc_b200/_lib/libdgc.so``.  There is no fallback: if the library
is missing or fails to load, every operator raises ``RuntimeError``.
"""

from __future__ import annotations

import ctypes
import os
import threading
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libdgc.so"
HEADER_PATH = Path(__file__).resolve().parents[2] / "include" / "dgc.h"

_P = ctypes.c_void_p
_I = ctypes.c_int
_F = ctypes.c_float
_D = ctypes.c_double
_S = ctypes.c_size_t

_GEOM = [_P] * 8  # angles, sid, sod, det_u0, det_v0, src_x, src_y, src_z


class FpInstance(ctypes.Structure):
    """``dgc_fp_instance``: one problem of a batched projection."""

    _fields_ = [("volume", _P), ("D", _I), ("H", _I), ("W", _I),
                *[(n, _P) for n in ("angles", "sid", "sod", "det_u0", "det_v0", "src_x", "src_y",
                                    "src_z")],
                ("A", _I), ("pixel_size", _F), ("U", _I), ("V", _I), ("step_size", _F),
                ("voxel_size", _F), ("off_x", _F), ("off_y", _F), ("off_z", _F),
                ("projections", _P), ("grad_projections", _P), ("grad_volume", _P),
                ("grad_geometry", _P), ("tile_forward", _I), ("tile_backward", _I)]


class BatchPlan(ctypes.Structure):
    """``dgc_batch_plan``: a prepared batch (host-side)."""

    _fields_ = [("workspace", _P), ("n", _I), ("grid_forward", _I), ("grid_backward", _I),
                ("has_grad_volume", _I), ("backward_ready", _I),
                *[(n, ctypes.c_longlong) for n in ("items_forward", "items_backward",
                                                   "quad_blocks", "views", "fold_blocks", "rays")],
                ("grad_pad_offset", _S), ("grad_pad_bytes", _S), ("tables_bytes", _S)]


# name -> (restype, argtypes)
SIGNATURES = {
    "dgc_abi_version": (_I, []),
    "dgc_last_error": (ctypes.c_char_p, []),
    "dgc_project_workspace_bytes": (_S, [_I] * 6),
    "dgc_project": (_I, [_P, _I, _I, _I, *_GEOM, _I, _F, _I, _I, _F, _F, _F, _F, _F, _P, _P, _S, _P]),
    "dgc_project_sample_counts": (_I, [_I, _I, _I, *_GEOM, _I, _F, _I, _I, _F, _F, _F, _F, _F, _P, _P]),
    "dgc_project_backward_workspace_bytes": (_S, [_I] * 7),
    "dgc_project_backward": (_I, [_P, _P, _I, _I, _I, *_GEOM, _I, _F, _I, _I, _F, _F, _I, _F, _F, _F,
                                  *([_P] * 9), _P, _S, _P]),
    "dgc_project_mse_grad_workspace_bytes": (_S, [_I] * 6),
    "dgc_project_mse_grad": (_I, [_P, _I, _I, _I, *_GEOM, _I, _F, _I, _I, _F, _F, _F, _F, _F, _P, _P,
                                  _F, _P, _P, *([_P] * 8), _P, _S, _P]),
    "dgc_backproject_workspace_bytes": (_S, [_I] * 6),
    "dgc_backproject": (_I, [_P, _I, _I, _I, *_GEOM, _F, _I, _I, _I, _F, _F, _F, _F, _P, _P, _S, _P]),
    "dgc_backproject_backward_workspace_bytes": (_S, [_I] * 6),
    "dgc_backproject_backward": (_I, [_P, _P, _I, _I, _I, *_GEOM, _F, _I, _I, _I, _F, _F, _F, _F,
                                      *([_P] * 9), _P, _S, _P]),
    "dgc_fdk_filter_taps": (_I, [_I, _D, _D, ctypes.POINTER(_D)]),
    "dgc_fdk_filter_workspace_bytes": (_S, [_I] * 3),
    "dgc_fdk_filter": (_I, [_P, _I, _I, _I, _F, _P, _P, _F, _P, _P, _S, _P]),
    "dgc_fdk_filter_noalloc": (_I, [_P, _I, _I, _I, _F, _P, _P, _F, _P, _P]),
    "dgc_reconstruct_fdk_workspace_bytes": (_S, [_I] * 6),
    "dgc_reconstruct_fdk": (_I, [_P, _I, _I, _I, *_GEOM, _F, _I, _I, _I, _F, _F, _F, _F, _F, _P, _P,
                                 _S, _P]),
    "dgc_parker_weights": (_I, [_P, _P, _I, _I, _F, _P, _P]),
    "dgc_reconstruct_fdk_weighted": (_I, [_P, _I, _I, _I, *_GEOM, _F, _I, _I, _I, _F, _F, _F, _F, _F,
                                          _P, _F, _P, _P, _S, _P]),
    "dgc_fdk_filter_backward_workspace_bytes": (_S, [_I] * 3),
    "dgc_fdk_filter_backward": (_I, [_P, _P, _P, _I, _I, _I, _F, _P, _P, _F, _P, _P, _P, _P, _S,
                                     _P]),
    "dgc_reconstruct_fdk_partial": (_I, [_P, _I, _I, _I, *_GEOM, _F, _I, _I, _I, _F, _F, _F, _F, _F,
                                         _P, _F, _P, _P, _S, _P]),
    "dgc_fdk_filter_ex": (_I, [_P, _I, _I, _I, _F, _P, _P, _P, _P, _P, _F, _P, _P, _S, _P]),
    "dgc_fdk_filter_backward_ex": (_I, [_P, _P, _P, _I, _I, _I, _F, *([_P] * 5), _F,
                                        *([_P] * 6), _P, _S, _P]),
    "dgc_parker_weights_ex": (_I, [_P, _P, _P, _P, _I, _I, _F, _P, _P]),
    "dgc_reconstruct_fdk_ex": (_I, [_P, _I, _I, _I, *_GEOM, _F, _I, _I, _I, _F, _F, _F, _F, _F,
                                    _P, _P, _P, _P, _F, _I, _P, _P, _S, _P]),
    "dgc_clamp_volume": (_I, [_P, ctypes.c_longlong, _P]),
    "dgc_bp_add_tile_rule": (_I, [_I] * 6),
    "dgc_bp_clear_tile_rules": (_I, []),
    "dgc_bp_tiles": (_I, [_I, _I] + [ctypes.POINTER(ctypes.c_int)] * 4),
    "dgc_gemm_bf16": (_I, [_P, _P, _P, _P, _I, _I, _I, _I, _I, _I, _I, _I, _I, _F, _P, _P]),
    "dgc_im2col_nhwc_bf16": (_I, [_P, _I, _I, _I, _I, _I, _I, _I, _I, _P, _I, _P]),
    "dgc_col2im_nhwc_f32": (_I, [_P, _I, _I, _I, _I, _I, _I, _I, _I, _I, _P, _P]),
    "dgc_preprocess": (_I, [_P, _P, _P, _I, _I, _I, _I, _F, _P, _P]),
    "dgc_batch_workspace_bytes": (_S, [ctypes.POINTER(FpInstance), _I]),
    "dgc_batch_prepare": (_I, [ctypes.POINTER(FpInstance), _I, _P, _S, ctypes.POINTER(BatchPlan),
                               _P]),
    "dgc_batch_project": (_I, [ctypes.POINTER(BatchPlan), _P]),
    "dgc_batch_project_backward": (_I, [ctypes.POINTER(BatchPlan), _I, _P]),
    "dgc_trace_enable": (None, [_I]),
    "dgc_trace_count": (_I, []),
    "dgc_trace_get": (_I, [_I, ctypes.c_char_p, _I, ctypes.POINTER(_F)]),
    "dgc_trace_clear": (None, []),
    "dgc_fp_add_arm_rule": (_I, [ctypes.c_longlong, _I, _I, _I, _I]),
    "dgc_fp_clear_arm_rules": (_I, []),
    "dgc_fp_arm": (_I, [_I, _I, _I, *[ctypes.POINTER(_I)] * 4]),
    "dgc_ceiling_gather": (_I, [_P, _S, _I, _I, _I, _I, _P, ctypes.POINTER(_D), _P]),
    "dgc_ceiling_issue": (_I, [_I, _I, _P, ctypes.POINTER(_D), _P]),
}

_lib = None
_lock = threading.Lock()


def lib():
    """Load ``libdgc.so`` once; raise ``RuntimeError`` if it is unavailable."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            path = Path(os.environ.get("DGC_LIBRARY", LIB_PATH))
            if not path.exists():
                raise RuntimeError(
                    f"libdgc.so is not built ({path}). Build it with: "
                    "python diff-geocali_b200/build.py"
                )
            handle = ctypes.CDLL(str(path))
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(handle, name)
                fn.restype = res
                fn.argtypes = args
            if handle.dgc_abi_version() != 1:
                raise RuntimeError("libdgc.so ABI version mismatch")
            _lib = handle
    return _lib


class trace:
    """Context manager: CUDA-event timing of every libdgc kernel launched inside.

    ``records`` holds ``(kernel_name, milliseconds)`` after exit (the exit
    waits for the recorded events).
    """

    def __init__(self):
        self.records = []

    def __enter__(self):
        lib().dgc_trace_clear()
        lib().dgc_trace_enable(1)
        return self

    def __exit__(self, *exc):
        L = lib()
        L.dgc_trace_enable(0)
        name = ctypes.create_string_buffer(128)
        ms = ctypes.c_float()
        for i in range(L.dgc_trace_count()):
            check(L.dgc_trace_get(i, name, 128, ctypes.byref(ms)))
            self.records.append((name.value.decode(), float(ms.value)))
        L.dgc_trace_clear()
        return False


def check(status: int) -> None:
    """Turn a non-zero status into the reference's exception type (RuntimeError)."""
    if status != 0:
        msg = lib().dgc_last_error().decode("utf-8", "replace")
        raise RuntimeError(msg or f"libdgc call failed with status {status}")
