"""Generate the golden fixtures in tests/golden/ from the reference's own code.

The reference (freifeld/cpabDiffeo) is Python 2 + pycuda and cannot run here,
but its kernel sources (cpab/gpu/calc_{1Dto1D,2Dto2D,3Dto3D}.cu and the expm
kernel strings in cpab/gpu/expm/expm_affine_by_series_{2D,3D}.py) compile as
host C++ through oracle/ref_shim.h; oracle/Makefile builds them into
oracle/_ref/libcpab_ref.so from the reference checkout.  This script feeds
seeded inputs through that build and stores inputs and outputs as .npz.

Run (where the reference checkout exists):
    make -C oracle && python tests/golden/make_golden.py

Inputs: per-cell matrices A = B theta with theta from the Gaussian prior of
each space (length scale 0.1, variance 1), points uniform in the domain plus
the edge cases the cell lookup distinguishes (grid vertices, box centres,
points on the triangle diagonals and tetrahedron planes, domain corners, and
points outside the domain on every side).
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from cpabdiffeo_b200.space import Prior, build_space  # noqa: E402
from oracle import oracle as O  # noqa: E402

OUT = Path(__file__).resolve().parent

CONFIGS = [
    # name, dim, nCs, tess, n_random
    ("d1_nc100", 1, (100,), "II", 3000),
    ("d2_tessI_4x4", 2, (4, 4), "I", 3000),
    ("d2_tessII_4x4", 2, (4, 4), "II", 1500),
    ("d3_tessI_4x4x4", 3, (4, 4, 4), "I", 2000),
    ("d3_tessII_2x2x2", 3, (2, 2, 2), "II", 1000),
]
DT, NT, NODE = 0.02, 50, 100


def edge_points(dim: int, nCs) -> np.ndarray:
    g = [np.linspace(0, 1, n + 1) for n in nCs]
    h = [(np.arange(n) + 0.5) / n for n in nCs]
    pts = []
    if dim == 1:
        pts += [[x] for x in g[0]] + [[x] for x in h[0]]
        pts += [[-0.3], [-1e-12], [-0.0], [1.0 + 1e-12], [1.4], [0.5 - 1e-17], [0.5 + 1e-16]]
    elif dim == 2:
        for x in np.concatenate([g[0], h[0]]):
            for y in np.concatenate([g[1], h[1]]):
                pts.append([x, y])
        # on the diagonals of each box (triangle boundaries)
        for t in np.linspace(0.01, 0.99, 7):
            pts.append([t * 0.25, t * 0.25])
            pts.append([t * 0.25, 0.25 - t * 0.25])
            pts.append([0.5 + t * 0.25, 0.75 - t * 0.25])
        # outside, all sides and corners
        for x in (-0.2, -1e-9, 0.3, 1.0, 1.0 + 1e-9, 1.2):
            for y in (-0.25, -1e-9, 0.6, 1.0, 1.0 + 1e-9, 1.3):
                pts.append([x, y])
        pts += [[-0.1, -0.05], [-0.05, -0.1], [1.1, -0.05], [1.05, -0.1], [-0.1, 1.05], [-0.05, 1.1],
                [1.1, 1.05], [1.05, 1.1]]
    else:
        for x in g[0]:
            for y in g[1]:
                for z in g[2]:
                    pts.append([x, y, z])
        for x in h[0]:
            for y in h[1]:
                for z in h[2]:
                    pts.append([x, y, z])
        rng = np.random.default_rng(123)
        # points on the planes -x-y+z=0 etc. inside box (0,0,0) (local coords)
        inc = 1.0 / np.asarray(nCs)
        for _ in range(30):
            u, w = rng.uniform(0, 1, 2)
            pts.append([u * inc[0], w * inc[1], min(u + w, 1.0) * inc[2]])
            pts.append([u * inc[0], w * inc[1], max(u + w - 2 + 1, 0.0) * inc[2]])
        for x in (-0.2, 0.4, 1.0, 1.2):
            for y in (-0.1, 0.3, 1.0, 1.1):
                for z in (-0.3, 0.7, 1.0, 1.05):
                    pts.append([x, y, z])
    return np.asarray(pts, dtype=np.float64)


def main() -> None:
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libcpab_ref.so is missing: run `make -C oracle` where the reference exists")
    for seed, (name, dim, nCs, tess, n) in enumerate(CONFIGS):
        rng = np.random.default_rng(1000 + seed)
        geo = build_space(dim, nCs, tess)
        prior = Prior.create(geo, length_scale=0.1, variance=1.0)
        theta = prior.sample(1, rng)[0]
        A = (geo.B @ theta).reshape(geo.nC, -1)
        tc = geo.tess_code
        pts = np.concatenate([rng.uniform(0, 1, size=(n, dim)), edge_points(dim, nCs)])
        pts_wide = np.concatenate([rng.uniform(-0.5, 1.5, size=(n // 2, dim)), edge_points(dim, nCs)])
        rec = dict(dim=dim, tess=tc, nCs=np.asarray(nCs), incs=geo.incs, A=A, pts=pts, pts_wide=pts_wide,
                   dt=DT, nT=NT, nODE=NODE)
        rec["cell_idx"] = O.ref_calc_cell_idx(dim, tc, nCs, geo.incs, pts_wide, geo.nC)
        rec["v"] = O.ref_calc_v(dim, tc, nCs, geo.incs, A, pts, geo.nC)
        for sign, tag in ((1, "fwd"), (-1, "inv")):
            sA = -A if sign < 0 else A.copy()
            M = sA * DT
            Tr = O.ref_expm_1d(M) if dim == 1 else O.ref_expm(dim, M)
            rec[f"Trels_{tag}"] = Tr
            out = O.ref_calc_T(dim, tc, nCs, geo.incs, Tr, sA, pts, DT, NT, NODE, geo.nC)
            if dim == 1:
                out = O.clamp_1d(out)
            rec[f"T_{tag}"] = out
        sA = A.copy()
        rec["T_simple"] = O.ref_calc_T(dim, tc, nCs, geo.incs, rec["Trels_fwd"], sA, pts[:500], DT, NT, NODE,
                                       geo.nC, simple=True)
        rec["traj"] = O.ref_calc_trajectory(dim, tc, nCs, geo.incs, rec["Trels_fwd"], sA, pts[:200], DT, NT,
                                            NODE, geo.nC)
        np.savez_compressed(OUT / f"{name}.npz", **rec)
        print(name, {k: np.shape(v) for k, v in rec.items()})


if __name__ == "__main__":
    main()
