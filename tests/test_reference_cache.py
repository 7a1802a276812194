"""Reading the reference's subspace cache (cpab/cpaNd/_CpaSpace.py:224-230,
written by cpab/cpa2d/CpaSpace.py:173-178): a Python 2 pickle of a dict with
B, nConstraints, nEdges and cont_constraints_are_separable.  No Python 2
exists here, so the test writes such a file opcode by opcode as Python 2's
pickle protocol 2 writes it -- byte strings as BINSTRING, numpy arrays
through numpy.core.multiarray._reconstruct with their raw data as a byte
string -- holding a B that spans the space's subspace in another basis (a
rotation of this package's B, as a different SVD would give).  CPU only."""
import struct

import numpy as np
import pytest
import torch

from cpabdiffeo_b200.space import (build_space, basis_from_reference_cache, load_reference_subspace,
                                   reference_subspace_string)


def _str(b: bytes) -> bytes:
    return (b"U" + bytes([len(b)]) + b) if len(b) < 256 else (b"T" + struct.pack("<i", len(b)) + b)


def _int(i: int) -> bytes:
    return b"J" + struct.pack("<i", i)


def _global(mod: str, name: str) -> bytes:
    return b"c" + mod.encode() + b"\n" + name.encode() + b"\n"


def _ndarray_f8(a: np.ndarray) -> bytes:
    a = np.ascontiguousarray(a, dtype="<f8")
    dtype = (_global("numpy", "dtype") + _str(b"f8") + b"\x89\x88\x87R" +
             b"(" + b"K\x03" + _str(b"<") + b"NNN" + _int(-1) + _int(-1) + b"K\x00" + b"tb")
    shape = b"(" + b"".join(_int(n) for n in a.shape) + b"t"
    state = b"(" + b"K\x01" + shape + dtype + b"\x89" + _str(a.tobytes()) + b"t"
    return (_global("numpy.core.multiarray", "_reconstruct") + _global("numpy", "ndarray") + b"K\x00\x85" +
            _str(b"b") + b"\x87R" + state + b"b")


def py2_subspace_pickle(B: np.ndarray, n_constraints: int, n_edges: int) -> bytes:
    items = (_str(b"B") + _ndarray_f8(B) + _str(b"nConstraints") + _int(n_constraints) + _str(b"nEdges") +
             _int(n_edges) + _str(b"cont_constraints_are_separable") + b"\x89")
    return b"\x80\x02}(" + items + b"u."


def test_subspace_string_matches_reference_format():
    assert reference_subspace_string(2, "I", [0, 0], [1, 1], [4, 4], [True, True]) == \
        "tessI_R2toR2_MINS_0_0_MAXS_1_1_nc_4_4_Xbdr_0_0_ext_0"
    assert reference_subspace_string(1, "II", [0], [1], [100], [True]) == "R1toR1_MINS_0_MAXS_1_nc_100_Xbdr_0"
    assert reference_subspace_string(3, "II", [0, 0, 0], [1, 1, 1], [2, 2, 2], [True, False, True]) == \
        "tessII_R3toR3_MINS_0_0_0_MAXS_1_1_1_nc_2_2_2_Xbdr_0_1_0"


@pytest.mark.parametrize("dim,nCs,tess", [(1, (20,), "II"), (2, (4, 4), "I"), (3, (2, 2, 2), "II")])
def test_reads_python2_subspace_pickle(tmp_path, dim, nCs, tess):
    geo = build_space(dim, nCs, tess)
    rng = np.random.default_rng(3)
    Q, _ = np.linalg.qr(rng.standard_normal((geo.d, geo.d)))
    B_ref = geo.B @ Q                                       # the same subspace, another orthonormal basis
    d = tmp_path / f"{dim}d" / reference_subspace_string(dim, tess, geo.xmins, geo.xmaxs, nCs,
                                                         geo.zero_v_across_bdry)
    d.mkdir(parents=True)
    (d / "subspace.pkl").write_bytes(py2_subspace_pickle(B_ref, 123, 45))
    z = load_reference_subspace(d / "subspace.pkl")
    assert z["nConstraints"] == 123 and z["nEdges"] == 45 and z["cont_constraints_are_separable"] is False
    np.testing.assert_array_equal(z["B"], B_ref)
    np.testing.assert_array_equal(basis_from_reference_cache(geo, tmp_path), B_ref)


def test_rejects_a_cache_of_another_subspace(tmp_path):
    geo = build_space(2, (4, 4), "I")
    wrong = np.linalg.qr(np.random.default_rng(1).standard_normal(geo.B.shape))[0]
    d = tmp_path / "2d" / reference_subspace_string(2, "I", geo.xmins, geo.xmaxs, (4, 4), geo.zero_v_across_bdry)
    d.mkdir(parents=True)
    (d / "subspace.pkl").write_bytes(py2_subspace_pickle(wrong, 1, 1))
    with pytest.raises(ValueError):
        basis_from_reference_cache(geo, tmp_path)
    assert basis_from_reference_cache(build_space(2, (2, 2), "I"), tmp_path) is None   # absent file


def test_cpaspace_uses_the_reference_basis(tmp_path):
    """CpaSpace(reference_cache=...) adopts the cached B, so a theta from the
    reference's runs gives the same A = B theta."""
    from cpabdiffeo_b200.cpa_space import CpaSpace
    geo = build_space(2, (4, 4), "I")
    Q, _ = np.linalg.qr(np.random.default_rng(4).standard_normal((geo.d, geo.d)))
    d = tmp_path / "2d" / reference_subspace_string(2, "I", geo.xmins, geo.xmaxs, (4, 4), geo.zero_v_across_bdry)
    d.mkdir(parents=True)
    (d / "subspace.pkl").write_bytes(py2_subspace_pickle(geo.B @ Q, 1, 1))
    sp = CpaSpace([0, 0], [1, 1], (4, 4), tess="I", device="cpu", reference_cache=tmp_path)
    np.testing.assert_array_equal(sp.B_host, geo.B @ Q)
    assert build_space(2, (4, 4), "I").B is geo.B           # the shared geometry is untouched
