"""cpab_calc_T_batched_noalloc -- the ragged batch for callers that cannot
allocate device memory (a host that owns the whole device pool and passes a
plugin only its inputs and outputs, or a latency-critical loop that cannot
afford cudaMalloc's implicit synchronisation).  Its bookkeeping lives in a
fixed array inside the library instead of caller scratch.

Checked through the C ABI against cpab_calc_T_batched (same kernel, so the
tolerance is the suite's bit-exact one for the REF scheme) on two calls in a
row with different batches, since every call reuses the same array.  This file
is collected last so that a run stopping at the first failure has run every
other test already; it also passes alone in a fresh process.
"""
import numpy as np
import pytest
import torch

from cpabdiffeo_b200 import _lib
from cpabdiffeo_b200.cpa_space import CpaSpace
from cpabdiffeo_b200.space import Prior

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
DT, NT, NODE = 0.02, 50, 100


def _batch(sp, rng, n_theta, max_pts, dtype):
    theta = Prior.create(sp.geo, 0.1, 1.0).sample(n_theta, rng)
    tables = sp.tables_from_theta(torch.as_tensor(theta, device=DEV), DT, 1)
    sizes = rng.integers(0, max_pts, size=n_theta)
    sizes[0] = 0                                   # an empty instance
    offs = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    x = torch.as_tensor(rng.uniform(0, 1, size=(int(offs[-1]), sp.dim)), dtype=dtype, device=DEV)
    return tables, torch.as_tensor(offs, device=DEV), x


def _with_workspace(sp, tables, offs, x, prec):
    out = torch.empty_like(x)
    sp.calc_T_batched(tables, x, out, offsets=offs, dt=DT, nTimeSteps=NT, nStepsODEsolver=NODE)
    return out


def _noalloc(sp, tables, offs, x, prec):
    sA, Tr = tables
    out = torch.full_like(x, float("nan"))
    c = sp._ctx
    c.check(c.lib.cpab_calc_T_batched_noalloc(c.h, _lib.ptr(sA), _lib.ptr(Tr), _lib.ptr(x), _lib.ptr(out),
                                              sA.shape[0], _lib.ptr(offs), 0, prec, _lib.SCHEME_REF, DT, NT,
                                              NODE, None, _lib.stream_ptr()))
    return out


@pytest.mark.parametrize("dim,nCs,tess,dtype", [(1, (100,), "II", torch.float32), (2, (4, 4), "I", torch.float64)])
def test_noalloc_matches_workspace_entry_point_twice(dim, nCs, tess, dtype):
    sp = CpaSpace([0.0] * dim, [1.0] * dim, nCs, tess=tess, device=DEV, precision=dtype)
    prec = _lib.CPAB_F64 if dtype == torch.float64 else _lib.CPAB_F32
    rng = np.random.default_rng(2024)
    first = _batch(sp, rng, 300, 2000, dtype)     # call 1: 300 instances
    second = _batch(sp, rng, 17, 9000, dtype)     # call 2: fewer, larger instances
    got1 = _noalloc(sp, *first, prec)
    got2 = _noalloc(sp, *second, prec)
    torch.cuda.synchronize()
    want1 = _with_workspace(sp, *first, prec)
    want2 = _with_workspace(sp, *second, prec)
    torch.cuda.synchronize()
    assert torch.equal(got1, want1)
    assert torch.equal(got2, want2)


def test_noalloc_at_the_maximum_and_uniform():
    """A ragged call at exactly NOALLOC_MAX_INSTANCES (most instances empty)
    and a uniform call (offsets NULL, which needs no scratch) both equal the
    workspace entry point."""
    sp = CpaSpace([0.0], [1.0], (100,), device=DEV, precision=torch.float32)
    rng = np.random.default_rng(7)
    n = _lib.NOALLOC_MAX_INSTANCES
    theta = Prior.create(sp.geo, 0.1, 1.0).sample(n, rng)
    tables = sp.tables_from_theta(torch.as_tensor(theta, device=DEV), DT, 1)
    sizes = np.zeros(n, dtype=np.int64)
    busy = rng.choice(n, size=64, replace=False)
    sizes[busy] = rng.integers(1, 700, size=busy.size)
    sizes[-1] = 5                                   # the last instance is not empty
    offs = torch.as_tensor(np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64), device=DEV)
    x = torch.as_tensor(rng.uniform(0, 1, size=(int(sizes.sum()), 1)), dtype=torch.float32, device=DEV)
    got = _noalloc(sp, tables, offs, x, _lib.CPAB_F32)
    want = _with_workspace(sp, tables, offs, x, _lib.CPAB_F32)
    torch.cuda.synchronize()
    assert torch.equal(got, want)

    sA, Tr = (t[:9].contiguous() for t in tables)
    xu = torch.as_tensor(rng.uniform(0, 1, size=(9 * 333, 1)), dtype=torch.float32, device=DEV)
    out = torch.full_like(xu, float("nan"))
    c = sp._ctx
    c.check(c.lib.cpab_calc_T_batched_noalloc(c.h, _lib.ptr(sA), _lib.ptr(Tr), _lib.ptr(xu), _lib.ptr(out), 9,
                                              None, 333, _lib.CPAB_F32, _lib.SCHEME_REF, DT, NT, NODE, None,
                                              _lib.stream_ptr()))
    want_u = torch.empty_like(xu)
    sp.calc_T_batched((sA, Tr), xu, want_u, dt=DT, nTimeSteps=NT, nStepsODEsolver=NODE)
    torch.cuda.synchronize()
    assert torch.equal(out, want_u)


def test_noalloc_rejects_too_many_instances():
    sp = CpaSpace([0.0], [1.0], (100,), device=DEV, precision=torch.float32)
    c = sp._ctx
    n = _lib.NOALLOC_MAX_INSTANCES + 1
    st = c.lib.cpab_calc_T_batched_noalloc(c.h, None, None, None, None, n, None, 0, _lib.CPAB_F32,
                                           _lib.SCHEME_REF, DT, NT, NODE, None, None)
    assert st == 2  # CPAB_BAD_SHAPE
    assert str(_lib.NOALLOC_MAX_INSTANCES).encode() in c.lib.cpab_last_error_string(c.h)
