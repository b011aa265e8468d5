"""ctypes binding of the C ABI in include/gkm_b200.h (libgkm_b200.so).

Every product operation runs through this library on a CUDA device; there is
no CPU fallback.  A missing library or device raises at first use.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "libgkm_b200.so")

GKM_OK, GKM_ERR_INVALID, GKM_ERR_CUDA, GKM_ERR_OOM, GKM_ERR_CAPACITY, GKM_ERR_UNSUPPORTED = range(6)
PAD = 0xFFFFFFFF


class GkmError(RuntimeError):
    """A failure reported by the CUDA library."""

    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


class GkmSpec(ctypes.Structure):
    _fields_ = [
        ("l", ctypes.c_int32),
        ("include_rc", ctypes.c_int32),
        ("weighted", ctypes.c_int32),
        ("dmax", ctypes.c_int32),
        ("h", ctypes.c_double * 16),
        ("wd", ctypes.c_void_p),
        ("wd_len", ctypes.c_int32),
    ]


P = ctypes.c_void_p
I32 = ctypes.c_int32
I64 = ctypes.c_int64
D = ctypes.c_double
SPEC = ctypes.POINTER(GkmSpec)

# name -> argument types (all return int status)
# gkm_smo_solve's kernel-column provider: (count, indices, out, ctx) -> status
COLUMNS_CB = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32),
                              ctypes.POINTER(ctypes.c_double), ctypes.c_void_p)

SIGNATURES = {
    "gkm_version": [],
    "gkm_device_info": [P, P],
    "gkm_set_thread_grid_limit": [I32],
    "gkm_pack": [SPEC, P, P, I64, I64, P, P, P, P],
    "gkm_self_kernel": [SPEC, P, P, P, I64, I64, P, P, P],
    "gkm_join_pairwise": [SPEC, P, P, I64, I64, P, P, P, I64, I64, P, P, P],
    "gkm_dense_pairwise": [SPEC, P, P, I64, I64, P, P, P, I64, I64, P, P, P, P],
    "gkm_dense_set_role_wait": [I64],
    "gkm_index_create": [SPEC, P, P, P, I64, I64, P, I32, I32, P, P],
    "gkm_index_free": [P],
    "gkm_index_info": [P, P, P, P, P],
    "gkm_index_status": [P, P, I32, P],
    "gkm_index_pairwise": [P, P, P, I64, I64, I64, P, P, P],
    "gkm_index_score": [P, P, P, I64, I64, P, P, P, D, I32, D, P, P, P],
    "gkm_index_lmer_weights": [P, P, P, P],
    "gkm_index_count": [P, P, P, I64, I64, P, P],
    "gkm_index_score_noalloc": [P, P, P, I64, I64, P, P, P, D, I32, D, P, P, P],
    "gkm_lmer_table": [SPEC, P, P, I32, P, P],
    "gkm_deltasvm_table": [SPEC, P, D, I32, P, P],
    "gkm_table_score": [SPEC, P, P, P, P, I64, I64, D, I32, P, P, P, P],
    "gkm_mutant_diag": [SPEC, P, P, I64, I64, I64, P, P, P],
    "gkm_ism_table": [SPEC, P, P, P, I64, I64, I64, P, P, P, I32, P, P],
    "gkm_index_mutants_workspace": [P, I64, I64, P, P],
    "gkm_index_mutants": [P, P, P, I64, I64, I64, P, P, P, P, P, P, D, I32, P, P, I64, P],
    "gkm_raw_score": [P, I64, I64, P, P, P, D, I32, D, P, P],
    "gkm_impact": [P, I64, I64, P, P, P, D, I32, P, P],
    "gkm_explain_lmer": [SPEC, P, P, I64, I64, I64, P, P, P, P, P, I32, P, P, I32, P, P],
    "gkm_explain_table_build": [SPEC, P, P, P, P, P],
    "gkm_explain_pairs": [SPEC, P, P, I64, I64, I64, P, P, P, P, I64, I64, P, P, P, I32, I32, P, P],
    "gkm_explain_table": [SPEC, P, P, P, I64, I64, I64, P, I32, P, P],
    "gkm_smo_solve": [I32, I32, P, P, P, D, D, D, I64, I32, I32, COLUMNS_CB, P, P, P, P, I32],
    "gkm_gram_finish": [P, I64, I64, P, P, D, I32, I32, P, P],
    "gkm_lsgkm_parse_svs": [P, I64, I64, I64, P, P, P, P, P, P, P],
}

_lib = None


def load():
    """The loaded library (built by gkmsvm_lite_b200.build)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build the CUDA library first "
                "(python -m gkmsvm_lite_b200.build)")
        lib = ctypes.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = ctypes.c_int
        lib.gkm_last_error.argtypes = []
        lib.gkm_last_error.restype = ctypes.c_char_p
        _lib = lib
    return _lib


def check(status: int, what: str = "") -> None:
    if status != GKM_OK:
        msg = load().gkm_last_error().decode(errors="replace")
        if status == GKM_ERR_INVALID:
            raise ValueError(msg)
        if status == GKM_ERR_OOM:
            raise MemoryError(f"{what}: {msg}")
        raise GkmError(status, f"{what}: {msg}" if what else msg)


def call(name: str, *args) -> None:
    check(getattr(load(), name)(*args), name)


def ptr(t) -> int | None:
    """Device pointer of a torch tensor (None for None)."""
    if t is None:
        return None
    return t.data_ptr()


def stream_handle():
    import torch

    return torch.cuda.current_stream().cuda_stream


def require_cuda():
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("gkmsvm_lite_b200 needs a CUDA device (B200, sm_100a)")
    load()
