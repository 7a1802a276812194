"""The oracle's Philox4x32-10 against the published known-answer vectors of the
Random123 distribution (Salmon et al., SC 2011: kat_vectors, philox4x32 10 rounds).
CPU only."""
import numpy as np


def test_philox_known_answers(oracle_mod):
    O = oracle_mod
    cases = [
        ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
        ((0xFFFFFFFF,) * 4, (0xFFFFFFFF, 0xFFFFFFFF), (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
        ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
         (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
    ]
    for c, k, want in cases:
        got = O.philox4x32_10(np.asarray([c], dtype=np.uint64), k)[0]
        assert tuple(int(x) for x in got) == want


def test_normals_are_standard(oracle_mod):
    z = oracle_mod.mcmc_normals(seed=7, step=3, C=2000, d=63)
    assert abs(z.mean()) < 0.01 and abs(z.std() - 1) < 0.01
