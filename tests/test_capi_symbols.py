"""libcpab_b200.so loads and exports every function include/cpab_b200.h declares;
no compute calls (no GPU needed).  Also checks host-side argument validation
paths that return before any CUDA call."""
import ctypes as C
import re
from pathlib import Path

import pytest

from cpabdiffeo_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]


def declared():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names |= set(re.findall(r"\b(cpab_\w+)\s*\(", text))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared()
    assert "cpab_calc_T" in names and "cpab_ctx_create" in names
    assert len(names) >= 15


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_bindings_cover_header():
    assert set(declared()) <= set(_lib.SIGNATURES)


def test_ctx_create_validation():
    lib = _lib.load()
    h = C.c_void_p()
    nCs = (C.c_int * 3)(4, 4, 1)
    incs = (C.c_double * 3)(0.25, 0.25, 1.0)
    assert lib.cpab_ctx_create(C.byref(h), 4, 1, nCs, incs) == 1          # bad dim
    assert b"dim" in lib.cpab_last_error_string(None)
    assert lib.cpab_ctx_create(C.byref(h), 1, 1, nCs, incs) == 1          # 1D tess I
    bad = (C.c_double * 3)(0.0, 0.25, 1.0)
    assert lib.cpab_ctx_create(C.byref(h), 2, 1, nCs, bad) == 1           # inc 0
    assert lib.cpab_ctx_create(C.byref(h), 2, 1, nCs, incs) == 0
    assert lib.cpab_ctx_num_cells(h) == 64 and lib.cpab_ctx_cell_len(h) == 6
    # argument checks that return before any CUDA call
    assert lib.cpab_calc_T(h, None, None, None, None, 10, 0, 0, 0.02, 50, 100, None, None) == 1
    assert lib.cpab_calc_T(h, 8, 8, 16, 16, 10, 5, 0, 0.02, 50, 100, None, None) == 3   # dtype
    assert lib.cpab_calc_T(h, 8, 8, 16, 16, 10, 0, 0, 0.02, 50, 0, None, None) == 1     # nStepsODE
    # pts and out overlap -> ALIAS (reference raises, cpab/cpaNd/_CpaCalcs.py:388)
    assert lib.cpab_calc_T(h, 8, 8, 4096, 4096 + 64, 10, 0, 0, 0.02, 50, 100, None, None) == 4
    assert b"same memory" in lib.cpab_last_error_string(h)
    # the 2D/3D exact scheme needs the facet tables a context gets on a device
    assert lib.cpab_calc_T(h, 8, 8, 16, 16, 10, 0, 2, 0.02, 50, 100, None, None) == 10
    assert b"facet" in lib.cpab_last_error_string(h)
    assert lib.cpab_set_launch(h, 48, 0, 0) == 1
    assert lib.cpab_set_max_ctas(h, -1) == 1
    assert lib.cpab_set_max_ctas(h, 37) == 0 and lib.cpab_set_max_ctas(h, 0) == 0
    assert lib.cpab_ctx_destroy(h) == 0


def test_misaligned_pointers_are_rejected_before_launch():
    """A device pointer that is not aligned to its element size returns
    CPAB_BAD_ARG naming the argument (a misaligned access would fault the GPU)."""
    lib = _lib.load()
    h = C.c_void_p()
    nCs = (C.c_int * 3)(4, 4, 1)
    incs = (C.c_double * 3)(0.25, 0.25, 1.0)
    assert lib.cpab_ctx_create(C.byref(h), 2, 1, nCs, incs) == 0
    base = 1 << 20
    # FP64 points at a 4-byte offset
    assert lib.cpab_calc_T(h, base, base, base + 4096 + 4, base + 8192, 10, 0, 0, 0.02, 50, 100, None, None) == 1
    assert b"pts is not aligned" in lib.cpab_last_error_string(h)
    # FP32 points at a 4-byte offset are fine up to the table check; the tables must be 8-aligned
    assert lib.cpab_calc_T(h, base + 4, base, base + 4096, base + 8192, 10, 1, 0, 0.02, 50, 100, None, None) == 1
    assert b"signedA is not aligned" in lib.cpab_last_error_string(h)
    # cell index output at an odd address
    assert lib.cpab_calc_cell_idx(h, base, base + 4096 + 2, 10, None) == 1
    assert b"cell_idx is not aligned" in lib.cpab_last_error_string(h)
    # remap with a float64 map on a 4-byte boundary
    assert lib.cpab_remap_ssd(h, base + 4, 0, base + 4096, None, 1, 8, 8, 1.0, 0.0, 1.0, 0.0, 1.0,
                              base + 8192, None, None, 0, None) == 1
    assert b"map is not aligned" in lib.cpab_last_error_string(h)
    assert lib.cpab_ctx_destroy(h) == 0



def test_mcmc_run_validation_before_launch():
    """cpab_mcmc_run checks its arguments before enqueueing anything."""
    lib = _lib.load()
    h = C.c_void_p()
    nCs = (C.c_int * 3)(2, 2, 2)
    incs = (C.c_double * 3)(0.5, 0.5, 0.5)
    assert lib.cpab_ctx_create(C.byref(h), 3, 1, nCs, incs) == 0
    base = 1 << 20
    args = [h, base, 10, 4, base, base, 0.05, base, base, 8, 8, 0.05, 0, 0.02, 50, 100, 1 / 64, 0, 1, base, 5, base,
            None, base, 1 << 20, None]
    assert lib.cpab_mcmc_run(*args) == 10                      # 3D space: UNSUPPORTED
    assert lib.cpab_ctx_destroy(h) == 0
    nCs2 = (C.c_int * 3)(4, 4, 1)
    incs2 = (C.c_double * 3)(0.25, 0.25, 1.0)
    assert lib.cpab_ctx_create(C.byref(h), 2, 1, nCs2, incs2) == 0
    args[0] = h
    bad = list(args)
    bad[4] = None                                              # theta NULL
    assert lib.cpab_mcmc_run(*bad) == 1
    small = list(args)
    small[24] = 16                                             # workspace too small
    assert lib.cpab_mcmc_run(*small) == 5
    assert b"workspace" in lib.cpab_last_error_string(h)
    assert lib.cpab_ctx_destroy(h) == 0


def test_grad_ref_validation_before_launch():
    """cpab_grad_theta_ref checks its arguments (and sizes its workspace) before enqueueing anything."""
    lib = _lib.load()
    h = C.c_void_p()
    nCs = (C.c_int * 3)(4, 4, 1)
    incs = (C.c_double * 3)(0.25, 0.25, 1.0)
    assert lib.cpab_ctx_create(C.byref(h), 2, 1, nCs, incs) == 0
    N, n, nT, ck = 3, 100, 50, 5
    ws = lib.cpab_grad_ref_workspace_bytes(h, N, n, nT, ck)
    # checkpoints (10 x 300 points x 2 doubles) + dLoss/dTrels and dLoss/d(sub-step map)
    # (3 x 64 cells x 6 doubles each), each 256-aligned
    assert ws == 48128 + 2 * 9216
    assert lib.cpab_grad_workspace_bytes(h, N, n, nT, ck) == 48128
    base = 1 << 20
    args = [h, base, 62, base, base, N, base, n, base, 0, 0.02, nT, 100, 1, ck, None, None, base, base, base, ws, None]
    bad = list(args)
    bad[4] = None                                              # Trels NULL
    assert lib.cpab_grad_theta_ref(*bad) == 1
    assert b"Trels" in lib.cpab_last_error_string(h)
    bad = list(args)
    bad[13] = 0                                                # sign 0
    assert lib.cpab_grad_theta_ref(*bad) == 1
    bad = list(args)
    bad[12] = 300                                              # more sub-steps than the adjoint replays
    assert lib.cpab_grad_theta_ref(*bad) != 0
    small = list(args)
    small[20] = ws - 8                                         # workspace too small
    assert lib.cpab_grad_theta_ref(*small) == 5
    assert b"workspace" in lib.cpab_last_error_string(h)
    bad = list(args)
    bad[9] = 7                                                 # unknown precision
    assert lib.cpab_grad_theta_ref(*bad) == 3
    assert lib.cpab_ctx_destroy(h) == 0
