"""The autotuner times its candidates on whole instances of the caller's batch
(each with its own points), so the pick carries over to the full launch."""
import numpy as np

from cpabdiffeo_b200.autotune import sample_extent


def test_uniform_batch_keeps_points_per_instance():
    # 4096 instances x 8192 points: as many whole instances as the sample holds
    assert sample_extent(4096, 4096 * 8192, None, 4_000_000) == (488, 488 * 8192)
    n_inst, n_pts = sample_extent(4096, 4096 * 8192, None, 1 << 22)
    assert n_pts == n_inst * 8192 and n_inst == 512


def test_uniform_batch_smaller_than_sample_or_one_huge_instance():
    assert sample_extent(10, 10 * 100, None, 1 << 22) == (10, 1000)
    # one instance larger than the sample: still one whole instance
    assert sample_extent(3, 3 * 5_000_000, None, 1 << 22) == (1, 5_000_000)


def test_ragged_batch_whole_instances():
    sizes = np.array([1000, 50_000, 3, 0, 200_000, 7])
    offs = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    for sp, want in ((10, 2), (1000, 2), (1001, 3), (51_000, 3), (60_000, 6), (10 ** 9, 6)):
        n_inst, n_pts = sample_extent(len(sizes), int(offs[-1]), offs, sp)
        assert n_inst == want, (sp, n_inst)
        assert n_pts == offs[n_inst]                  # ends on an instance boundary
        assert n_pts >= min(sp, offs[-1])             # holds the requested points
