"""ctypes binding of libgft_b200.so (the C ABI declared in include/gft.h).

The library is built in-tree by ``gftevolver_b200/build.py``.  There is no
CPU fallback: if the shared library cannot be loaded, every entry point
raises.
"""
from __future__ import annotations

import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgft_b200.so")

GFT_OK = 0
GFT_E_INVALID = -1
GFT_E_UNSUPPORTED = -2
GFT_E_CUDA = -3
GFT_E_NOMEM = -4
GFT_E_STATE = -5
GFT_E_TIMEOUT = -6

GFT_W_ASIN_DOMAIN = 1
GFT_W_SQRT_DOMAIN = 2
GFT_W_NONFINITE = 4
GFT_W_RANGE = 16

GFT_MODEL_SM = 1
GFT_MODEL_2HDM = 2

GFT_HF_NONE = 0   # 2HDM Higgs-family gauge field: none (gaugeNum 4), U(1) (5), SU(2) (7)
GFT_HF_U1 = 1
GFT_HF_SU2 = 2
GFT_MAX_GAUSS = 7

GFT_FORM_REF = 0
GFT_FORM_FP64 = 1
GFT_FORM_MIXED = 2


class GftConfig(ctypes.Structure):
    _fields_ = [
        ("model", ctypes.c_int), ("form", ctypes.c_int), ("storage_bytes", ctypes.c_int), ("device", ctypes.c_int),
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("dz", ctypes.c_double), ("dt", ctypes.c_double),
        ("g", ctypes.c_double), ("gp", ctypes.c_double), ("div_tol", ctypes.c_double),
        ("damping", ctypes.c_double), ("nt_damped", ctypes.c_int),
        ("lam", ctypes.c_double), ("eta_sqr", ctypes.c_double),
        ("m1", ctypes.c_double), ("m2", ctypes.c_double), ("l1", ctypes.c_double), ("l2", ctypes.c_double),
        ("l3", ctypes.c_double),
        ("m12r", ctypes.c_double), ("l4p5", ctypes.c_double), ("l6r", ctypes.c_double), ("l7r", ctypes.c_double),
        ("m12i", ctypes.c_double), ("l4m5", ctypes.c_double), ("l5i", ctypes.c_double), ("l6i", ctypes.c_double),
        ("l7i", ctypes.c_double),
        ("break_son", ctypes.c_int), ("break_uhalfn", ctypes.c_int), ("apply_norm", ctypes.c_int),
        ("energy_offset", ctypes.c_double),
        ("energy_every", ctypes.c_int), ("gauss_every", ctypes.c_int),
        ("fixed_axes", ctypes.c_int),
        ("higgs_family", ctypes.c_int), ("gpp", ctypes.c_double),
        ("generator_rep", ctypes.c_int),
        ("energy_local_every", ctypes.c_int), ("gauss_local_every", ctypes.c_int),
    ]


class GftObservables(ctypes.Structure):
    _fields_ = [
        ("time_iter", ctypes.c_int), ("has_energy", ctypes.c_int), ("has_gauss", ctypes.c_int),
        ("energy", ctypes.c_double), ("potential", ctypes.c_double), ("gradient", ctypes.c_double),
        ("kinetic", ctypes.c_double), ("magnetic", ctypes.c_double), ("electric", ctypes.c_double),
        ("gauss_int", ctypes.c_double * GFT_MAX_GAUSS), ("gauss_max", ctypes.c_double * GFT_MAX_GAUSS),
        ("plaq_su2", ctypes.c_double), ("plaq_u1", ctypes.c_double), ("phi_sq", ctypes.c_double),
    ]


class GftIC(ctypes.Structure):
    _fields_ = [
        ("seed", ctypes.c_uint64),
        ("mean", ctypes.c_double * 8), ("sigma", ctypes.c_double * 8),
        ("theta_sigma", ctypes.c_double), ("eps_sigma", ctypes.c_double),
        ("wall_width", ctypes.c_double), ("wall_value", ctypes.c_double),
    ]


# int (*)(gft_handle*, int level, void* user)
EXCHANGE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p)

_FP = ctypes.POINTER(ctypes.c_float)
_DP = ctypes.POINTER(ctypes.c_double)
_H = ctypes.c_void_p

# name -> (restype, argtypes); every function declared in include/gft.h
SIGNATURES = {
    "gft_create": (ctypes.c_int, [ctypes.POINTER(GftConfig), ctypes.POINTER(_H)]),
    "gft_destroy": (None, [_H]),
    "gft_upload_f32": (ctypes.c_int, [_H, _FP, _FP, ctypes.c_int]),
    "gft_upload_f64": (ctypes.c_int, [_H, _DP, _DP, ctypes.c_int]),
    "gft_download_f32": (ctypes.c_int, [_H, _FP, _FP]),
    "gft_download_f64": (ctypes.c_int, [_H, _DP, _DP]),
    "gft_init_fields": (ctypes.c_int, [_H, ctypes.POINTER(GftIC)]),
    "gft_evolve": (ctypes.c_int, [_H, ctypes.c_int, ctypes.POINTER(GftObservables), ctypes.c_int,
                                  ctypes.POINTER(ctypes.c_int)]),
    "gft_observe": (ctypes.c_int, [_H, ctypes.POINTER(GftObservables)]),
    "gft_time_iter": (ctypes.c_int, [_H]),
    "gft_stream": (ctypes.c_void_p, [_H]),
    "gft_device_bytes": (ctypes.c_size_t, [_H]),
    "gft_upload_device_f32": (ctypes.c_int, [_H, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]),
    "gft_upload_device_f64": (ctypes.c_int, [_H, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]),
    "gft_download_device_f32": (ctypes.c_int, [_H, ctypes.c_void_p, ctypes.c_void_p]),
    "gft_download_device_f64": (ctypes.c_int, [_H, ctypes.c_void_p, ctypes.c_void_p]),
    "gft_step_kernel_ms": (ctypes.c_double, [_H, ctypes.POINTER(ctypes.c_int)]),
    "gft_step_kernel_name": (ctypes.c_char_p, [_H]),
    "gft_launch_count": (ctypes.c_longlong, [_H]),
    "gft_local_fields": (ctypes.c_int, [_H, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float),
                                        ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    "gft_selftest_math": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_double)]),
    "gft_set_kernel": (ctypes.c_int, [_H, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "gft_set_wait_limit": (ctypes.c_int, [_H, ctypes.c_ulonglong]),
    "gft_set_graphs": (ctypes.c_int, [_H, ctypes.c_int]),
    "gft_nccl_unique_id": (ctypes.c_int, [ctypes.c_char_p]),
    "gft_set_slab_nccl": (ctypes.c_int, [_H, ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_double]),
    "gft_observe_static": (ctypes.c_int, [ctypes.POINTER(GftConfig), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                          ctypes.c_void_p, ctypes.c_void_p]),
    "gft_last_error": (ctypes.c_char_p, [_H]),
    "gft_version": (ctypes.c_char_p, []),
    "gft_set_slab": (ctypes.c_int, [_H, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "gft_set_exchange": (ctypes.c_int, [_H, ctypes.c_void_p, ctypes.c_void_p]),
    "gft_level_planes": (ctypes.c_int, [_H, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p),
                                        ctypes.POINTER(ctypes.c_size_t), ctypes.c_int]),
    # ensembles
    "gft_batch_create": (ctypes.c_int, [ctypes.POINTER(GftConfig), ctypes.c_int, ctypes.POINTER(_H)]),
    "gft_batch_destroy": (None, [_H]),
    "gft_batch_size": (ctypes.c_int, [_H]),
    "gft_batch_init_fields": (ctypes.c_int, [_H, ctypes.POINTER(GftIC)]),
    "gft_batch_upload_f32": (ctypes.c_int, [_H, ctypes.c_int, _FP, _FP, ctypes.c_int]),
    "gft_batch_download_f32": (ctypes.c_int, [_H, ctypes.c_int, _FP, _FP]),
    "gft_batch_evolve": (ctypes.c_int, [_H, ctypes.c_int, ctypes.POINTER(GftObservables), ctypes.c_int,
                                        ctypes.POINTER(ctypes.c_int)]),
    "gft_batch_set_kernel": (ctypes.c_int, [_H, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "gft_batch_autotune": (ctypes.c_int, [_H, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                          ctypes.POINTER(ctypes.c_int)]),
    "gft_batch_last_ms": (ctypes.c_double, [_H]),
    "gft_batch_launch_count": (ctypes.c_longlong, [_H]),
    "gft_batch_time_iter": (ctypes.c_int, [_H]),
    "gft_batch_stream": (ctypes.c_void_p, [_H]),
    "gft_batch_device_bytes": (ctypes.c_size_t, [_H]),
    "gft_batch_last_error": (ctypes.c_char_p, [_H]),
}

_lock = threading.Lock()
_lib = None


class GftError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"gft error {code}: {msg}")
        self.code = code


def load(path: str | None = None):
    """Load libgft_b200.so (raises if it is missing: there is no fallback)."""
    global _lib
    with _lock:
        if _lib is not None and path is None:
            return _lib
        p = path or LIB_PATH
        if not os.path.exists(p):
            raise ImportError(
                f"{p} not found: build the CUDA library first (python gftevolver_b200/build.py)")
        lib = ctypes.CDLL(p)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        if path is None:
            _lib = lib
        return lib


def last_error(h=None) -> str:
    msg = load().gft_last_error(h)
    return msg.decode() if msg else ""


def check(rc: int, h=None) -> int:
    """Raise on errors (< 0); return the warning bitmask (>= 0)."""
    if rc < 0:
        raise GftError(rc, last_error(h))
    return rc


def check_batch(rc: int, b) -> int:
    """check() for gft_batch_* calls (their messages live on the batch)."""
    if rc < 0:
        msg = load().gft_batch_last_error(b) if b else None
        raise GftError(rc, (msg.decode() if msg else "") or last_error(None))
    return rc
