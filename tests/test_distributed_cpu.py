"""Multi-process sharding logic on CPU: world size 2 over gloo.  Each rank
transforms its shard of a ragged 1D batch with the CPU oracle; the gathered
result equals the single-process result, and the timing reduction is the max
over ranks."""
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from cpabdiffeo_b200.distributed import gather_to_rank0, max_over_ranks, shard, shard_ragged


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _problem():
    from cpabdiffeo_b200.space import Prior, build_space
    geo = build_space(1, (20,), "II")
    rng = np.random.default_rng(0)
    theta = Prior.create(geo, 0.1, 1.0).sample(9, rng)
    sizes = rng.integers(0, 400, size=9)
    offs = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    x = rng.uniform(0, 1, size=(int(offs[-1]), 1))
    return geo, theta, offs, x


def _transform(geo, theta, offs, x, a, b):
    from oracle import oracle as O
    t = O.tess_struct(1, 2, geo.nCs, geo.incs)
    outs = []
    for i in range(a, b):
        sA, Tr = O.expm_cells(1, geo.B @ theta[i], 0.02, 1)
        y, _ = O.calc_T(t, Tr, sA, x[offs[i]:offs[i + 1]], 0.02, 50, 100)
        outs.append(O.clamp_1d(y))
    return np.concatenate(outs) if outs else np.zeros((0, 1))


def _worker(rank, size, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=size)
    try:
        geo, theta, offs, x = _problem()
        a, b = shard_ragged(offs, rank, size)
        local = torch.as_tensor(_transform(geo, theta, offs, x, a, b))
        full = gather_to_rank0(local)
        t = max_over_ranks(float(rank + 1))
        if rank == 0:
            q.put((full.numpy(), t))
    finally:
        dist.destroy_process_group()


def test_shard_covers_range():
    for n in (0, 1, 7, 100):
        for size in (1, 2, 3, 8):
            parts = [shard(n, r, size) for r in range(size)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            assert all(parts[i][1] == parts[i + 1][0] for i in range(size - 1))


def test_shard_ragged_covers_instances():
    offs = np.concatenate([[0], np.cumsum([5, 0, 100, 3, 50, 50, 1])])
    for size in (1, 2, 3, 5):
        parts = [shard_ragged(offs, r, size) for r in range(size)]
        assert parts[0][0] == 0 and parts[-1][1] == len(offs) - 1
        assert all(parts[i][1] == parts[i + 1][0] for i in range(size - 1))


def test_two_ranks_gloo_equal_single_process():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    full, tmax = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    geo, theta, offs, x = _problem()
    np.testing.assert_array_equal(full, _transform(geo, theta, offs, x, 0, len(offs) - 1))
    assert tmax == 2.0
