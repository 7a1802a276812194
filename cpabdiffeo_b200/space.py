"""Host-side construction of a CPA space: tessellation, continuity and
boundary constraints, the orthonormal basis B of the constrained subspace,
and the Gaussian prior.  Setup work, done once per configuration and cached;
the GPU path consumes the arrays built here.

Follows freifeld/cpabDiffeo:
  * cells and their vertex order: cpab/cpa1d/Tessellation.py:34-52,
    cpab/cpa2d/Tessellation.py:73-138, cpab/cpa3d/Tessellation.py:62-200
  * box sizes ("incs"): cpab/cpaNd/_CpaSpace.py:278-294
  * continuity constraints: cpab/cpa2d/utils/constraints/_create_cont_constraint_mat.py:11-103
    (A_i v = A_j v at every vertex v of a facet shared by cells i and j)
  * zero velocity across the boundary: cpab/cpa2d/Tessellation.py:532-580,
    cpab/cpa3d/Tessellation.py:540-588 (the velocity component normal to a
    boundary face vanishes at every vertex on that face)
  * B = orthonormal basis of null(L) by SVD: cpab/cpaNd/utils/_null.py:23-80
  * prior: cpab/distributions/create_joint_algebra_cov.py:14-172 and
    cpab/distributions/CpaCovs.py:100-121 (Sigma_CPA = B^T Sigma_PA B)

The basis is only defined up to a rotation of theta; the distribution of
A = B theta under the prior does not depend on that choice.
"""
from __future__ import annotations

import hashlib
import os
import pickle
from dataclasses import dataclass, field
from functools import lru_cache
from pathlib import Path
from typing import Sequence

import numpy as np

TESS_I, TESS_II = "I", "II"


def _tess_code(tess: str) -> int:
    """The reference's TESS_TYPE macro: 2 for 'II', 1 for 'I' (cpab/gpu/Calcs.py:159-162)."""
    return 2 - [TESS_II, TESS_I].index(tess)


# --------------------------------------------------------------------------- cells


def create_cells(dim: int, nCs: Sequence[int], xmins: Sequence[float], xmaxs: Sequence[float],
                 tess: str) -> np.ndarray:
    """Vertices of every cell in homogeneous coordinates, [nC, nV, dim+1],
    in the reference's cell and vertex order (which compute_cell_idx relies on)."""
    V = [np.linspace(xmins[k], xmaxs[k], int(nCs[k]) + 1) for k in range(dim)]
    cells = []
    if dim == 1:
        for i in range(int(nCs[0])):
            cells.append(((V[0][i], 1.0), (V[0][i + 1], 1.0)))
    elif dim == 2:
        Vx, Vy = V
        nCx, nCy = map(int, nCs)
        for i in range(nCy):
            for j in range(nCx):
                ul = (Vx[j], Vy[i], 1.0)
                ur = (Vx[j + 1], Vy[i], 1.0)
                ll = (Vx[j], Vy[i + 1], 1.0)
                lr = (Vx[j + 1], Vy[i + 1], 1.0)
                if tess == TESS_II:
                    cells.append((ul, ur, lr, ll))
                else:
                    center = ((Vx[j] + Vx[j + 1]) / 2, (Vy[i] + Vy[i + 1]) / 2, 1.0)
                    cells.append((center, ul, ur))   # 0: top
                    cells.append((center, ur, lr))   # 1: right
                    cells.append((center, lr, ll))   # 2: bottom
                    cells.append((center, ll, ul))   # 3: left
    elif dim == 3:
        Vx, Vy, Vz = V
        nCx, nCy, nCz = map(int, nCs)
        for k in range(nCz):
            for i in range(nCy):
                for j in range(nCx):
                    ul0 = (Vx[j], Vy[i], Vz[k], 1.0)
                    ur0 = (Vx[j + 1], Vy[i], Vz[k], 1.0)
                    ll0 = (Vx[j], Vy[i + 1], Vz[k], 1.0)
                    lr0 = (Vx[j + 1], Vy[i + 1], Vz[k], 1.0)
                    ul1 = (Vx[j], Vy[i], Vz[k + 1], 1.0)
                    ur1 = (Vx[j + 1], Vy[i], Vz[k + 1], 1.0)
                    ll1 = (Vx[j], Vy[i + 1], Vz[k + 1], 1.0)
                    lr1 = (Vx[j + 1], Vy[i + 1], Vz[k + 1], 1.0)
                    if tess == TESS_II:
                        cells.append((ul0, ur0, lr0, ll0, ul1, ur1, lr1, ll1))
                        continue
                    # checkerboard flip (cpab/cpa3d/Tessellation.py:160-170)
                    if (i + j + k) % 2 == 1:
                        ul0, ur0, lr0, ll0 = ur0, lr0, ll0, ul0
                        ul1, ur1, lr1, ll1 = ur1, lr1, ll1, ul1
                    cells.append((ll1, ur1, ul0, lr0))  # central tetrahedron
                    cells.append((ul1, ur1, ll1, ul0))
                    cells.append((lr1, ur1, ll1, lr0))
                    cells.append((ll0, ul0, lr0, ll1))
                    cells.append((ur0, ul0, lr0, ur1))
    else:
        raise NotImplementedError(dim)
    return np.asarray(cells, dtype=np.float64)


def box_centers(cells: np.ndarray, dim: int, tess: str) -> np.ndarray:
    if dim == 2 and tess == TESS_I:
        return cells[::4][:, 0].copy()
    if dim == 3 and tess == TESS_I:
        return cells[::5].mean(axis=1)
    return cells.mean(axis=1)


def compute_incs(cells: np.ndarray, dim: int, tess: str, nCs: Sequence[int]) -> np.ndarray:
    """Box size per axis as the reference derives it from the box centres."""
    cols = box_centers(cells, dim, tess).T[:-1]
    incs = []
    for k in range(dim):
        u = np.unique(cols[k])
        incs.append(np.diff(u)[0] if nCs[k] > 1 else 2 * u[0])
    incs = np.asarray(incs, dtype=np.float64)
    if (incs <= 0).any():
        raise ValueError(incs)
    return incs


# --------------------------------------------------------------------------- constraints


def constraint_matrix(cells: np.ndarray, dim: int, xmins, xmaxs,
                      zero_v_across_bdry: Sequence[bool]) -> np.ndarray:
    """Rows of L with L . Avees = 0 for continuous, boundary-respecting fields."""
    nC, nV, nh = cells.shape
    ne = dim * nh
    ncols = nC * ne
    vert_cells: dict[tuple, list[int]] = {}
    for c in range(nC):
        for v in cells[c]:
            vert_cells.setdefault(tuple(v), []).append(c)
    shared: dict[tuple[int, int], list[tuple]] = {}
    for v, cs in vert_cells.items():
        for a in range(len(cs)):
            for b in range(a + 1, len(cs)):
                i, j = (cs[a], cs[b]) if cs[a] < cs[b] else (cs[b], cs[a])
                if i != j:
                    shared.setdefault((i, j), []).append(v)
    rows = []
    for (i, j), verts in shared.items():
        if len(verts) < dim:  # neighbours through a lower-dimensional face only
            continue
        for v in verts:
            v = np.asarray(v)
            for k in range(dim):
                r = np.zeros(ncols)
                r[i * ne + k * nh:i * ne + (k + 1) * nh] = v
                r[j * ne + k * nh:j * ne + (k + 1) * nh] = -v
                rows.append(r)
    seen = set()
    for v, cs in vert_cells.items():
        c = cs[0]
        va = np.asarray(v)
        for k in range(dim):
            if zero_v_across_bdry[k] and (v[k] == xmins[k] or v[k] == xmaxs[k]) and (v, k) not in seen:
                seen.add((v, k))
                r = np.zeros(ncols)
                r[c * ne + k * nh:c * ne + (k + 1) * nh] = va
                rows.append(r)
    if not rows:
        return np.zeros((0, ncols))
    return np.asarray(rows)


def null_space(L: np.ndarray, n: int, eps: float = 1e-6) -> np.ndarray:
    """Orthonormal basis of null(L) (columns): singular values below eps
    (cpab/cpaNd/utils/_null.py:23-80)."""
    if L.shape[0] == 0:
        return np.eye(n)
    if n <= 4096:
        _, s, vh = np.linalg.svd(L, full_matrices=True)
        s_full = np.zeros(n)
        s_full[:s.size] = s
        B = vh.T[:, s_full < eps]
    else:
        # large spaces: eigen-decomposition of L^T L, relative threshold
        w, V = np.linalg.eigh(L.T @ L)
        B = V[:, w < 1e-10 * w.max()]
    # deterministic sign: first non-negligible entry of each column positive
    for j in range(B.shape[1]):
        nz = np.flatnonzero(np.abs(B[:, j]) > 1e-12)
        if nz.size and B[nz[0], j] < 0:
            B[:, j] *= -1
    return np.ascontiguousarray(B)


# --------------------------------------------------------------------------- space


def _cache_dir() -> Path | None:
    d = os.environ.get("CPAB_B200_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "cpabdiffeo_b200"))
    if d in ("", "0", "off"):
        return None
    return Path(d)


@dataclass
class SpaceGeometry:
    dim: int
    tess: str
    nCs: tuple
    xmins: tuple
    xmaxs: tuple
    zero_v_across_bdry: tuple
    cells: np.ndarray = field(repr=False)
    incs: np.ndarray = field(repr=False)
    B: np.ndarray = field(repr=False)

    @property
    def nC(self) -> int:
        return self.cells.shape[0]

    @property
    def nHomoCoo(self) -> int:
        return self.dim + 1

    @property
    def lengthAvee(self) -> int:
        return self.dim * (self.dim + 1)

    @property
    def D(self) -> int:
        return self.nC * self.lengthAvee

    @property
    def d(self) -> int:
        return self.B.shape[1]

    @property
    def tess_code(self) -> int:
        return _tess_code(self.tess)

    @property
    def subspace_string(self) -> str:
        s = f"tess{self.tess}_R{self.dim}toR{self.dim}_MINS_{self.xmins}_MAXS_{self.xmaxs}"
        s += f"_nc_{self.nCs}_Xbdr_{tuple(int(not z) for z in self.zero_v_across_bdry)}"
        return s.replace(" ", "").replace(",", "_").replace("(", "").replace(")", "")


@lru_cache(maxsize=32)
def build_space(dim: int, nCs: tuple, tess: str = TESS_II, xmins: tuple | None = None,
                xmaxs: tuple | None = None, zero_v_across_bdry: tuple | None = None) -> SpaceGeometry:
    """Build (or load from the cache) the geometry and basis of a CPA space."""
    nCs = tuple(int(n) for n in nCs)
    if len(nCs) != dim:
        raise ValueError(f"len(nCs) = {len(nCs)} != dim = {dim}")
    if tess not in (TESS_I, TESS_II):
        raise ValueError(tess)
    if dim == 1 and tess == TESS_I:
        raise ValueError("1D spaces use tess 'II'")
    xmins = tuple(float(x) for x in (xmins or (0.0,) * dim))
    xmaxs = tuple(float(x) for x in (xmaxs or (1.0,) * dim))
    if zero_v_across_bdry is None:
        zero_v_across_bdry = (True,) * dim
    zero_v_across_bdry = tuple(bool(z) for z in zero_v_across_bdry)
    cells = create_cells(dim, nCs, xmins, xmaxs, tess)
    incs = compute_incs(cells, dim, tess, nCs)
    geo = SpaceGeometry(dim, tess, nCs, xmins, xmaxs, zero_v_across_bdry, cells, incs, np.zeros((0, 0)))
    key = hashlib.sha1(geo.subspace_string.encode()).hexdigest()[:16]
    cdir = _cache_dir()
    path = cdir / f"B_{key}.npz" if cdir else None
    if path is not None and path.exists():
        try:
            with np.load(path) as z:
                if str(z["subspace"]) == geo.subspace_string:
                    geo.B = z["B"]
                    return geo
        except Exception:
            pass
    L = constraint_matrix(cells, dim, xmins, xmaxs, zero_v_across_bdry)
    geo.B = null_space(L, cells.shape[0] * dim * (dim + 1))
    if geo.B.shape[1] == 0:
        raise ValueError(f"dim = 0 (no degrees of freedom): {geo.subspace_string}")
    if path is not None:
        try:
            path.parent.mkdir(parents=True, exist_ok=True)
            tmp = path.with_suffix(f".{os.getpid()}.tmp.npz")
            np.savez(tmp, B=geo.B, subspace=np.asarray(geo.subspace_string))
            os.replace(tmp, path)
        except OSError:
            pass
    return geo


# --------------------------------------------------------------------------- the reference's subspace cache


def reference_subspace_string(dim: int, tess: str, xmins, xmaxs, nCs, zero_v_across_bdry,
                              valid_outside: bool = False) -> str:
    """The name of the reference's cached subspace for a zero-boundary space
    without volume preservation, zero values or wrap-around
    (create_subspace_string, cpab/cpaNd/_CpaSpace.py:525-566): numpy
    integer arrays printed as "[a b]", then brackets dropped and blanks
    turned into "_"."""
    def arr(v):
        return "[" + " ".join(str(int(x)) for x in v) + "]"
    xbdry = [0 if z else 1 for z in zero_v_across_bdry]
    s = ""
    if dim > 1:
        s += "tess" + str(tess) + "_"
    s += f"R{dim}toR{dim}"
    s += f"_MINS_{arr(xmins)}_MAXS_{arr(xmaxs)}"
    s += f"_nc_{arr(nCs)}"
    s += f"_Xbdr_{arr(xbdry)}"
    s = s.replace("[", "").replace("]", "").replace(" ", "_")
    if tess == TESS_I and dim == 2:
        s += f"_ext_{int(bool(valid_outside))}"
    return s


class _Py2Unpickler(pickle.Unpickler):
    """Python 2 pickles of numpy / scipy objects: the module paths of those
    releases mapped to today's."""
    RENAMES = {"copy_reg": "copyreg", "__builtin__": "builtins", "numpy.core.multiarray": "numpy._core.multiarray",
               "numpy.core.numeric": "numpy._core.numeric"}

    def find_class(self, module, name):
        return super().find_class(self.RENAMES.get(module, module), name)


def load_reference_subspace(path) -> dict:
    """The reference's cached subspace, <cache>/<dim>d/<subspace string>/subspace.pkl
    (cpab/cpaNd/_CpaSpace.py:224-230; written by cpab/cpa2d/CpaSpace.py:
    173-178 and its 1D/3D twins: a dict with B, nConstraints, nEdges or
    nSides, constraintMat, cont_constraints_are_separable).  The files are
    Python 2 pickles: strings are read as latin-1, which also restores numpy
    arrays' raw data."""
    with open(path, "rb") as f:
        d = _Py2Unpickler(f, encoding="latin1").load()
    if not isinstance(d, dict) or "B" not in d:
        raise ValueError(f"{path}: not a cpabDiffeo subspace file")
    d["B"] = np.ascontiguousarray(np.asarray(d["B"], dtype=np.float64))
    return d


def basis_from_reference_cache(geo: "SpaceGeometry", cache_dir) -> np.ndarray | None:
    """B from the reference's cache directory for this space, or None when the
    file is absent.  The cached B must span the same subspace as this
    package's construction (checked); using it keeps theta interchangeable
    with the reference's runs (B is defined only up to a rotation)."""
    path = Path(cache_dir) / f"{geo.dim}d" / reference_subspace_string(
        geo.dim, geo.tess, geo.xmins, geo.xmaxs, geo.nCs, geo.zero_v_across_bdry) / "subspace.pkl"
    if not path.exists():
        return None
    B = load_reference_subspace(path)["B"]
    if B.shape != geo.B.shape:
        raise ValueError(f"{path}: B has shape {B.shape}, the space needs {geo.B.shape}")
    if np.abs(B.T @ B - np.eye(B.shape[1])).max() > 1e-8:
        raise ValueError(f"{path}: B is not orthonormal")
    if np.abs(geo.B @ (geo.B.T @ B) - B).max() > 1e-8:
        raise ValueError(f"{path}: B spans a different subspace")
    return B


# --------------------------------------------------------------------------- prior


def joint_algebra_cov(geo: SpaceGeometry, scale_spatial: float = 1.0, scale_value: float = 0.1,
                      left_blk_rel_scale: float = 1.0, right_vec_scale: float = 1.0) -> np.ndarray:
    """Sigma_PA, [D, D] (create_joint_algebra_cov, cpab/distributions/create_joint_algebra_cov.py:14-172).

    Between cells i != j, the same entry of A_i and A_j has covariance
    exp(-dist_ij / (scale_spatial * d0))**2 * var_entry, where d0 is the
    distance between the centroids of cells 0 and 1; within a cell the entries
    are independent with std right_vec_std for the translation column and
    right_vec_std * left_blk_rel_scale for the linear block.  All times
    scale_value**2."""
    centers = geo.cells.mean(axis=1)
    nC, L = geo.nC, geo.lengthAvee
    if nC > 1:
        d0 = np.linalg.norm(centers[0] - centers[1])
        ss = d0 * scale_spatial
    else:
        ss = scale_spatial
    extent = np.asarray(geo.xmaxs) - np.asarray(geo.xmins)
    right = right_vec_scale * (abs(extent[0]) if geo.dim == 1 else np.sqrt(np.prod(extent)))
    left = right * left_blk_rel_scale
    var = np.full(L, left ** 2)
    for k in range(geo.dim):
        var[(geo.dim + 1) * (k + 1) - 1] = right ** 2
    diff = centers[:, None, :] - centers[None, :, :]
    dists = np.sqrt((diff ** 2).sum(-1))
    C = np.zeros((nC, nC))
    if ss > 1e-12 and nC > 1:
        C = np.exp(-(dists / ss)) ** 2
    np.fill_diagonal(C, 1.0)
    # block (i, j) = C[i, j] * diag(var): Kronecker structure
    cov = np.kron(C, np.diag(var))
    cov *= scale_value ** 2
    return cov


@dataclass
class Prior:
    """Gaussian prior theta ~ N(0, Sigma_CPA) of one space."""
    geo: SpaceGeometry
    cov_pa: np.ndarray = field(repr=False)
    cov_cpa: np.ndarray = field(repr=False)

    @classmethod
    def create(cls, geo: SpaceGeometry, length_scale: float = 0.1, variance: float = 1.0,
               left_blk_rel_scale: float | None = None, right_vec_scale: float = 1.0) -> "Prior":
        """length_scale is in domain units: scale_spatial = length_scale / d0
        so that the reference's kernel exp(-r/(scale_spatial*d0))**2 uses it."""
        if left_blk_rel_scale is None:
            # 1D TransformWrapper uses 1; 2D/3D use 1/100 (cpab/cpa2d/TransformWrapper.py:114-116)
            left_blk_rel_scale = 1.0 if geo.dim == 1 else 0.01
        centers = geo.cells.mean(axis=1)
        d0 = np.linalg.norm(centers[0] - centers[1]) if geo.nC > 1 else 1.0
        cov_pa = joint_algebra_cov(geo, scale_spatial=length_scale / d0, scale_value=np.sqrt(variance),
                                   left_blk_rel_scale=left_blk_rel_scale, right_vec_scale=right_vec_scale)
        cov_cpa = geo.B.T @ cov_pa @ geo.B
        cov_cpa = 0.5 * (cov_cpa + cov_cpa.T)
        return cls(geo, cov_pa, cov_cpa)

    def sample(self, n: int, rng: np.random.Generator) -> np.ndarray:
        """n draws of theta, [n, d]."""
        w, V = np.linalg.eigh(self.cov_cpa)
        w = np.clip(w, 0, None)
        z = rng.standard_normal((n, self.geo.d))
        return z @ (V * np.sqrt(w)).T


# --------------------------------------------------------------------------- host helpers


def theta2Avees(geo: SpaceGeometry, theta: np.ndarray) -> np.ndarray:
    """A = B theta (CpaSpace.theta2Avees, cpab/cpaNd/_CpaSpace.py:366-376); theta [..., d] -> [..., D]."""
    return np.asarray(theta) @ geo.B.T


def Avees2As(geo: SpaceGeometry, Avees: np.ndarray) -> np.ndarray:
    return np.asarray(Avees).reshape(*np.shape(Avees)[:-1], geo.nC, geo.dim, geo.dim + 1)


def vertices_1d(geo: SpaceGeometry) -> np.ndarray:
    if geo.dim != 1:
        raise ValueError
    return np.linspace(geo.xmins[0], geo.xmaxs[0], geo.nCs[0] + 1)


def pixel_centers(H: int, W: int) -> np.ndarray:
    """[H*W, 2] points ((col+0.5)/W, (row+0.5)/H), row-major (row outer)."""
    ys, xs = np.meshgrid((np.arange(H) + 0.5) / H, (np.arange(W) + 0.5) / W, indexing="ij")
    return np.stack([xs.ravel(), ys.ravel()], axis=1)


# --------------------------------------------------------------------------- local proposal


@dataclass(frozen=True)
class LocalProposalTables:
    """The linear maps behind the local (vertex-velocity) proposal of
    cpab/cpaNd/inference/Proposal.py:65-130.  With velTess the velocities at
    the tessellation's vertices (cpa_space.Avees2velTess / velTess2Avees):
      E[k] (dim x d): velocity at vertex k of theta, v_k = E[k] theta;
      G[k] (d x dim): theta change for a velocity change dv at vertex k alone,
                      B^T (A(velTess + e_k dv) - A(velTess)) = G[k] dv,
                      velTess2Avees then Avees2theta (B^T, :377-390);
      bdry[k]:        vertex k on the domain boundary (the reference then sets
                      its velocity to 0, :104-120).
    Simplicial tessellations only (1D, or type I), as in the reference (:73-74)."""
    vertices: np.ndarray   # [nV, dim]
    E: np.ndarray          # [nV, dim, d]
    G: np.ndarray          # [nV, d, dim]
    bdry: np.ndarray       # [nV] bool


def local_proposal_tables(geo: SpaceGeometry) -> LocalProposalTables:
    dim, nC, ne = geo.dim, geo.nC, geo.lengthAvee
    if dim != 1 and geo.tess != TESS_I:
        raise NotImplementedError("the local proposal needs a simplicial tessellation (1D or type I)")
    V_all = geo.cells[:, :, :dim].reshape(-1, dim)
    key = np.round(V_all * 2 ** 30).astype(np.int64)
    uniq, inv = np.unique(key, axis=0, return_inverse=True)
    inv = inv.reshape(nC, dim + 1)
    nV = uniq.shape[0]
    verts = np.zeros((nV, dim))
    verts[inv.ravel()] = V_all
    B = geo.B.reshape(nC, dim, dim + 1, -1)                # A_c[r, j] = B[c, r, j, :] theta
    d = B.shape[-1]
    E = np.zeros((nV, dim, d))
    G = np.zeros((nV, d, dim))
    for c in range(nC):
        Vh = np.concatenate([geo.cells[c, :, :dim], np.ones((dim + 1, 1))], axis=1).T   # [dim+1, dim+1], columns [v_i; 1]
        Vinv = np.linalg.inv(Vh)
        for i in range(dim + 1):
            k = inv[c, i]
            if not E[k].any():
                E[k] = np.einsum("rjd,j->rd", B[c], Vh[:, i])     # v_k = A_c [v_k; 1]
            # A_c = Vel Vh^-1: a change dv at vertex i changes A_c by dv (x) Vh^-1[i, :]
            for r in range(dim):
                G[k, :, r] += np.einsum("jd,j->d", B[c, r], Vinv[i, :])
    lo, hi = np.asarray(geo.xmins), np.asarray(geo.xmaxs)
    bdry = np.any(np.isclose(verts, lo[None]) | np.isclose(verts, hi[None]), axis=1)
    if not any(geo.zero_v_across_bdry):
        bdry[:] = False
    return LocalProposalTables(verts, E, G, bdry)
