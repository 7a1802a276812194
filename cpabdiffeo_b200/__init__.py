"""cpabdiffeo_b200 -- the CPAB transform hot path of freifeld/cpabDiffeo,
rebuilt for NVIDIA B200 (sm_100a).

Public surface (mirrors the reference):
    CpaSpace          calc_T_fwd / calc_T_inv / calc_T_simple / calc_v /
                      calc_trajectory / calc_cell_idx / theta2Avees / update_pat
    build_space, Prior  host-side basis and Gaussian prior
Compute runs in libcpab_b200.so (hand-written CUDA behind a C ABI,
include/cpab_b200.h); there is no CPU fallback.
"""
from .space import Prior, SpaceGeometry, build_space, pixel_centers  # noqa: F401


def __getattr__(name):
    if name in ("CpaSpace", "PAT"):
        from . import cpa_space
        return getattr(cpa_space, name)
    raise AttributeError(name)
