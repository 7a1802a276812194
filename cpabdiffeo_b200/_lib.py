"""ctypes binding of libcpab_b200.so (declared in include/cpab_b200.h).

The library is loaded from this package directory.  There is no fallback:
if the shared object is missing or fails to load, every GPU entry point
raises CpabLibraryError.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

_LIB_PATH = Path(__file__).resolve().parent / "libcpab_b200.so"

CPAB_OK = 0
STATUS_NAMES = {
    0: "OK", 1: "BAD_ARG", 2: "BAD_SHAPE", 3: "BAD_DTYPE", 4: "ALIAS", 5: "NO_MEMORY",
    6: "CANCELLED", 7: "TIMEOUT", 8: "NUMERIC", 9: "CUDA_ERROR", 10: "UNSUPPORTED",
}
CPAB_F64, CPAB_F32 = 0, 1
SCHEME_REF, SCHEME_SIMPLE, SCHEME_EXACT = 0, 1, 2
CNT_FAST, CNT_FALLBACK, CNT_SUBSTEPS, CNT_POINTS, CNT_FAILED, CNT_NAN, CNT_CANCELLED, CNT_CROSSINGS, CNT_N = (
    0, 1, 2, 3, 4, 5, 6, 7, 8)


class CpabLibraryError(RuntimeError):
    pass


class CpabError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"cpab status {STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


# Exported symbols and their (restype, argtypes).
_vp, _i, _i64, _d, _sz = C.c_void_p, C.c_int, C.c_int64, C.c_double, C.c_size_t
SIGNATURES = {
    "cpab_ctx_create": (_i, [C.POINTER(_vp), _i, _i, C.POINTER(_i), C.POINTER(_d)]),
    "cpab_ctx_destroy": (_i, [_vp]),
    "cpab_tess_facets": (_i, [_i, _i, C.POINTER(_i), C.POINTER(_d), _vp, _vp, C.POINTER(_i)]),
    "cpab_last_error_string": (C.c_char_p, [_vp]),
    "cpab_ctx_num_cells": (_i, [_vp]),
    "cpab_ctx_cell_len": (_i, [_vp]),
    "cpab_set_clamp": (_i, [_vp, _i, _d, _d]),
    "cpab_cancel": (_i, [_vp]),
    "cpab_clear_cancel": (_i, [_vp]),
    "cpab_cancel_requested": (_i, [_vp]),
    "cpab_set_launch": (_i, [_vp, _i, _i, _i]),
    "cpab_set_cell_sort": (_i, [_vp, _i]),
    "cpab_set_max_ctas": (_i, [_vp, _i]),
    "cpab_expm": (_i, [_vp, _vp, _i, _d, _i, _vp, _vp, _vp]),
    "cpab_theta_to_trels": (_i, [_vp, _vp, _i, _vp, _i, _d, _i, _vp, _vp, _vp, _vp]),
    "cpab_calc_cell_idx": (_i, [_vp, _vp, _vp, _i64, _vp]),
    "cpab_calc_v": (_i, [_vp, _vp, _vp, _vp, _i64, _vp]),
    "cpab_calc_T": (_i, [_vp, _vp, _vp, _vp, _vp, _i64, _i, _i, _d, _i, _i, _vp, _vp]),
    "cpab_batched_workspace_bytes": (_sz, [_i]),
    "cpab_calc_T_batched": (_i, [_vp, _vp, _vp, _vp, _vp, _i, _vp, _i64, _vp, _sz, _i, _i, _d, _i, _i, _vp, _vp]),
    "cpab_calc_trajectory": (_i, [_vp, _vp, _vp, _vp, _vp, _i64, _d, _i, _i, _vp]),
    "cpab_calc_T_batched_noalloc": (_i, [_vp, _vp, _vp, _vp, _vp, _i, _vp, _i64, _i, _i, _d, _i, _i, _vp, _vp]),
    "cpab_remap_workspace_bytes": (_sz, [_i, _i, _i]),
    "cpab_remap_ssd": (_i, [_vp, _vp, _i, _vp, _vp, _i, _i, _i, _d, _d, _d, _d, _d, _vp, _vp, _vp, _sz, _vp]),
    "cpab_register_workspace_bytes": (_sz, [_vp, _i, _i, _i]),
    "cpab_register_ll": (_i, [_vp, _vp, _vp, _i, _vp, _vp, _i, _i, _d, _i, _d, _i, _i, _vp, _vp, _vp, _sz, _vp,
                              _vp]),
    "cpab_remap3d_workspace_bytes": (_sz, [_i, _i, _i, _i]),
    "cpab_remap3d_ssd": (_i, [_vp, _vp, _i, _vp, _vp, _i, _i, _i, _i, _d, _d, _d, _d, _d, _d, _d, _vp, _vp, _vp,
                              _sz, _vp]),
    "cpab_register3d_workspace_bytes": (_sz, [_vp, _i, _i, _i, _i]),
    "cpab_register3d_ll": (_i, [_vp, _vp, _vp, _i, _vp, _vp, _i, _i, _i, _d, _i, _d, _i, _i, _vp, _vp, _vp, _sz,
                                _vp, _vp]),
    "cpab_landmark_workspace_bytes": (_sz, [_vp, _i, _i]),
    "cpab_landmark_ll": (_i, [_vp, _vp, _vp, _i, _vp, _i64, _vp, _i64, _i, _d, _i, _d, _i, _i, _vp, _vp, _vp, _sz,
                              _vp, _vp]),
    "cpab_mcmc_propose": (_i, [_vp, _i, _i, _vp, _vp, _d, C.c_uint64, _vp, _vp, _vp]),
    "cpab_mcmc_propose_local": (_i, [_vp, _i, _i, _vp, _i, _vp, _vp, _vp, _d, C.c_uint64, _vp, _vp, _vp]),
    "cpab_mcmc_accept": (_i, [_vp, _i, _i, _vp, _vp, _vp, _vp, _d, _vp, _d, _vp, _i, C.c_uint64, _vp, _vp, _vp]),
    "cpab_mcmc_run_workspace_bytes": (_sz, [_vp, _i, _i, _i, _i]),
    "cpab_mcmc_run": (_i, [_vp, _vp, _i, _i, _vp, _vp, _d, _vp, _vp, _i, _i, _d, _i, _d, _i, _i, _d, _i, C.c_uint64,
                           _vp, _i, _vp, _vp, _vp, _sz, _vp]),
    "cpab_grad_workspace_bytes": (_sz, [_vp, _i, _i64, _i, _i]),
    "cpab_grad_theta": (_i, [_vp, _vp, _i, _vp, _i, _vp, _i64, _vp, _d, _i, _i, _i, _i, _vp, _vp, _vp, _vp, _vp,
                             _sz, _vp]),
    "cpab_grad_ref_workspace_bytes": (_sz, [_vp, _i, _i64, _i, _i]),
    "cpab_grad_theta_ref": (_i, [_vp, _vp, _i, _vp, _vp, _i, _vp, _i64, _vp, _i, _d, _i, _i, _i, _i, _vp, _vp, _vp,
                                 _vp, _vp, _sz, _vp]),
}
NOALLOC_MAX_INSTANCES = 65536

_lib = None


def lib_path() -> Path:
    return _LIB_PATH


def load() -> C.CDLL:
    """Load (once) and return the library; raise CpabLibraryError if absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not _LIB_PATH.exists():
        raise CpabLibraryError(
            f"{_LIB_PATH} is missing: build it with `python -m cpabdiffeo_b200.build` "
            "(there is no CPU fallback)")
    try:
        lib = C.CDLL(str(_LIB_PATH), mode=os.RTLD_NOW | os.RTLD_LOCAL)
    except OSError as e:
        raise CpabLibraryError(f"cannot load {_LIB_PATH}: {e}") from e
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(status: int, ctx=None) -> None:
    if status != CPAB_OK:
        msg = load().cpab_last_error_string(ctx)
        raise CpabError(status, msg.decode() if msg else "")


def ptr(t) -> int | None:
    """Device pointer of a torch tensor (None for None)."""
    return None if t is None else t.data_ptr()


def stream_ptr(stream=None) -> int | None:
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream or None
