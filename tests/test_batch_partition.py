"""Host logic of the pipelined batch (ae_mpm_batch_partition, no GPU): consecutive groups, none
empty, of about equal particle capacity."""
import numpy as np
import pytest

import ae_mpm as M


def check(caps, groups):
    first = M.batch_partition(caps, groups)
    n = len(caps)
    g = min(max(groups, 1), n)
    assert len(first) == g + 1 and first[0] == 0 and first[-1] == n
    assert all(a < b for a, b in zip(first, first[1:]))  # no empty group
    return first


@pytest.mark.parametrize("groups", [0, 1, 2, 3, 4, 8, 16, 511, 512, 513, 1000])
def test_groups_cover_the_scenes_in_order(groups):
    rng = np.random.default_rng(groups)
    caps = rng.integers(2048, 65536, 512)
    first = check(caps, groups)
    if 1 < groups <= 16:  # balanced: no group above the mean by more than the largest scene
        sums = [int(caps[a:b].sum()) for a, b in zip(first, first[1:])]
        assert max(sums) <= caps.sum() / len(sums) + caps.max()


def test_lopsided_and_empty_capacities():
    check([100, 1, 1, 1], 4)
    check([1, 1, 1, 100], 4)
    assert check([0, 0, 0, 0, 0], 3) == [0, 1, 2, 5]
    assert check([5], 8) == [0, 1]
    huge = [2 ** 62, 2 ** 62, 1, 2 ** 62]  # no overflow in the running sums
    check(huge, 3)
    assert M.batch_partition([], 4) == []
