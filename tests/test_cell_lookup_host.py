"""The device cell lookup (cpabdiffeo_b200/csrc/cpab_cell.cuh) compiled as host
code must reproduce the reference's lookup bit for bit (exact family) and stay
within one neighbouring cell of it (float family).  CPU only."""
import ctypes as C
import subprocess
from pathlib import Path

import numpy as np
import pytest

from cpabdiffeo_b200.space import build_space

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def host_lib(tmp_path_factory):
    out = tmp_path_factory.mktemp("cell") / "libcellhost.so"
    cxx = "/usr/bin/g++" if Path("/usr/bin/g++").exists() else "g++"
    cmd = [cxx, "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", "-fno-fast-math",
           "-I", str(ROOT / "cpabdiffeo_b200" / "csrc"), str(ROOT / "tests" / "cell_lookup_host.cpp"), "-o", str(out)]
    subprocess.run(cmd, check=True, capture_output=True)
    return C.CDLL(str(out))


def _tess(lib, geo):
    buf = C.create_string_buffer(lib.host_tess_size())
    nCs = (C.c_int * 3)(*(list(geo.nCs) + [1] * (3 - geo.dim)))
    incs = (C.c_double * 3)(*(list(geo.incs) + [1.0] * (3 - geo.dim)))
    assert lib.host_make_tess(geo.dim, geo.tess_code, nCs, incs, buf) == 1
    return buf


def _adversarial(rng, dim, geo, n):
    inc = np.asarray(geo.incs)
    k = rng.integers(-2, np.asarray(geo.nCs) + 3, size=(n, dim))
    base = k * inc
    # exact multiples, one ulp either side, tiny offsets, random
    choice = rng.integers(0, 5, size=(n, dim))
    ulp = np.spacing(np.abs(base) + 1e-300)
    jitter = np.select([choice == 0, choice == 1, choice == 2, choice == 3],
                       [0.0, ulp, -ulp, rng.uniform(-1e-10, 1e-10, size=(n, dim))],
                       rng.uniform(0, 1, size=(n, dim)) * inc)
    return base + jitter


CASES = [(1, (100,), "II"), (1, (7,), "II"), (2, (4, 4), "I"), (2, (3, 5), "I"), (2, (4, 4), "II"),
         (2, (6, 3), "II"), (3, (4, 4, 4), "I"), (3, (3, 2, 5), "I"), (3, (2, 2, 2), "II"), (3, (3, 4, 2), "II")]


@pytest.mark.parametrize("dim,nCs,tess", CASES)
def test_exact_lookup_matches_oracle(host_lib, oracle_mod, dim, nCs, tess):
    O = oracle_mod
    geo = build_space(dim, nCs, tess) if (dim, nCs) != (3, (3, 2, 5)) and (dim, nCs) != (3, (3, 4, 2)) else None
    if geo is None:
        # geometry only (no basis needed): a throwaway object with the fields used
        from cpabdiffeo_b200.space import compute_incs, create_cells, SpaceGeometry
        cells = create_cells(dim, nCs, (0.0,) * dim, (1.0,) * dim, tess)
        geo = SpaceGeometry(dim, tess, nCs, (0.0,) * dim, (1.0,) * dim, (True,) * dim, cells,
                            compute_incs(cells, dim, tess, nCs), np.zeros((0, 0)))
    rng = np.random.default_rng(7)
    pts = np.concatenate([rng.uniform(-0.3, 1.3, size=(200000, dim)), _adversarial(rng, dim, geo, 200000),
                          np.full((3, dim), np.nan), np.full((2, dim), np.inf), -np.full((2, dim), np.inf)])
    pts = np.ascontiguousarray(pts)
    t = O.tess_struct(dim, geo.tess_code, nCs, geo.incs)
    want = O.calc_cell_idx(t, pts)
    got = np.empty_like(want)
    buf = _tess(host_lib, geo)
    host_lib.host_exact_cells(buf, pts.ctypes.data_as(C.c_void_p), got.ctypes.data_as(C.c_void_p),
                              C.c_long(pts.shape[0]))
    bad = np.flatnonzero(got != want)
    assert bad.size == 0, f"{bad.size} mismatches, e.g. {pts[bad[:5]]} got {got[bad[:5]]} want {want[bad[:5]]}"


@pytest.mark.parametrize("dim,nCs,tess", [c for c in CASES if c[1] not in ((3, 2, 5), (3, 4, 2))])
def test_fast_lookup_close_to_oracle(host_lib, oracle_mod, dim, nCs, tess):
    O = oracle_mod
    geo = build_space(dim, nCs, tess)
    rng = np.random.default_rng(11)
    pts = rng.uniform(0, 1, size=(100000, dim)).astype(np.float32)
    t = O.tess_struct(dim, geo.tess_code, nCs, geo.incs)
    want = O.calc_cell_idx(t, pts.astype(np.float64))
    got = np.empty_like(want)
    buf = _tess(host_lib, geo)
    host_lib.host_fast_cells(buf, pts.ctypes.data_as(C.c_void_p), got.ctypes.data_as(C.c_void_p),
                             C.c_long(pts.shape[0]))
    # float rounding may move points within ~1 ulp of a cell boundary
    assert (got != want).mean() < 1e-4
