"""ctypes binding of the C ABI in include/lenseflow.h (liblenseflow.so, built in-tree).

There is no fallback: if the library is missing or cannot be loaded, every
entry point raises ``NativeLibraryError``.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liblenseflow.so")

LF_OK = 0
LF_ERR_BAD_SHAPE = 1
LF_ERR_BAD_DTYPE = 2
LF_ERR_BAD_ARG = 3
LF_ERR_SINGULAR_MAGNIFICATION = 4
LF_ERR_OOM = 5
LF_ERR_TIMEOUT = 6
LF_ERR_CUDA = 7
LF_ERR_WORKSPACE = 8

LF_F32 = 0
LF_F64 = 1
LF_PHI_MAP = 0
LF_PHI_FOURIER = 1

# Every symbol include/lenseflow.h declares, with (restype, argtypes).
_vp = ctypes.c_void_p
_i = ctypes.c_int
_sz = ctypes.c_size_t
SIGNATURES = {
    "lf_version": (_i, []),
    "lf_status_string": (ctypes.c_char_p, [_i]),
    "lf_plan_create": (_i, [ctypes.POINTER(_vp), _i, _i, ctypes.c_double, _i]),
    "lf_plan_destroy": (_i, [_vp]),
    "lf_workspace_bytes": (_sz, [_vp, _i, _i]),
    "lf_workspace_bytes_n": (_sz, [_vp, _i, _i, _i]),
    "lf_wait_timeouts": (_i, [ctypes.POINTER(ctypes.c_int), _i]),
    "lf_timeout_status": (_i, []),
    "lf_stream_check": (_i, [_vp]),
    "lf_set_wait_polls": (_i, [_i]),
    "lf_phi_planes_bytes": (_sz, [_vp, _i]),
    "lf_phi_workspace_bytes": (_sz, [_vp, _i]),
    "lf_phi_precompute": (_i, [_vp, _vp, _i, _i, _vp, _vp, _vp, _sz, _vp]),
    "lf_min_det_init": (_i, [_vp, _i, _vp]),
    "lf_decode_min_det": (ctypes.c_float, [_i]),
    "lf_lense_flow": (_i, [_vp, _vp, _i, _vp, _i, _vp, _i, _i, _i, _i, _vp, _sz, _vp]),
    "lf_pp_bytes": (_sz, [_vp, _i, _i]),
    "lf_phi_precompute_pp": (_i, [_vp, _vp, _i, _i, _vp, _vp, _i, _vp, _vp, _sz, _vp]),
    "lf_lense_flow_pp": (_i, [_vp, _vp, _i, _vp, _i, _vp, _i, _i, _i, _i, _vp, _sz, _vp]),
    "lf_fft_workspace_bytes": (_sz, [_vp, _i]),
    "lf_rfft2": (_i, [_vp, _vp, _i, _i, _vp, _vp]),
    "lf_irfft2": (_i, [_vp, _vp, _i, _vp, _i, _vp, _sz, _vp]),
    "lf_vjp_workspace_bytes": (_sz, [_vp, _i]),
    "lf_lense_flow_vjp": (_i, [_vp, _vp, _vp, _i, _vp, _i, _i, _i, _vp, _vp, _vp, _i, _vp, _sz, _vp]),
    "lf_vjp_ckpt_workspace_bytes": (_sz, [_vp, _i, _i]),
    "lf_lense_flow_vjp_ckpt": (_i, [_vp, _vp, _vp, _i, _vp, _i, _i, _i, _vp, _vp, _vp, _i, _vp, _sz, _vp]),
    "lf_modes_apply": (_i, [_vp, _i, ctypes.c_uint, _vp, _vp, _vp, _i, _i, ctypes.c_long, ctypes.c_double,
                            ctypes.c_double, _vp]),
    "lf_lense_flow_noalloc": (_i, [_i, _i, ctypes.c_double, _vp, _i, _vp, _i, _vp, _i, _i, _i, _i, _vp]),
    "lf_profile_enable": (_i, [_vp, _i]),
    "lf_profile_reset": (_i, [_vp]),
    "lf_profile_read": (_i, [_vp, _i, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(_i)]),
}

LF_NOALLOC_SCRATCH_BYTES = 24 * 1024 * 1024

LF_KIND_ROW = 0
LF_KIND_COL = 1
LF_KIND_PHI = 2
LF_KIND_PP = 3


class NativeLibraryError(RuntimeError):
    """The CUDA engine library could not be loaded."""


class LenseFlowError(RuntimeError):
    """A C ABI call returned a non-zero status."""

    def __init__(self, status, what=""):
        self.status = status
        msg = status_string(status) if _lib is not None else str(status)
        super().__init__(f"{what}: {msg} (status {status})" if what else f"{msg} (status {status})")


class SingularMagnificationError(LenseFlowError):
    """det(I + t grad grad phi) <= 0 somewhere for t in [0, 1]."""


_lib = None
_load_error = None


def load():
    """Load liblenseflow.so once; raise NativeLibraryError if it is unavailable."""
    global _lib, _load_error
    if _lib is not None:
        return _lib
    if _load_error is not None:
        raise NativeLibraryError(_load_error)
    if not os.path.exists(LIB_PATH):
        _load_error = f"{LIB_PATH} not found; build it with `python -m cmblensing_b200.build`"
        raise NativeLibraryError(_load_error)
    try:
        lib = ctypes.CDLL(LIB_PATH)
    except OSError as e:
        _load_error = f"cannot load {LIB_PATH}: {e}"
        raise NativeLibraryError(_load_error) from e
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def status_string(status):
    return load().lf_status_string(int(status)).decode()


def check(status, what=""):
    if status != LF_OK:
        if status == LF_ERR_SINGULAR_MAGNIFICATION:
            raise SingularMagnificationError(status, what)
        raise LenseFlowError(status, what)
