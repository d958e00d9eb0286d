"""Host logic of the batching paths, no GPU: the pipelined batch's grouping
(ae_mpm_batch_partition: consecutive groups, none empty, of about equal particle capacity) and the
server's slot size classes (ae_mpm_server_slot_class)."""
import numpy as np
import pytest

import ae_mpm as M
import ae_mpm_scenes as S


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


# ------------------------------------------------------------------ server slot classes

@pytest.mark.parametrize("n", [1, 255, 256, 1024, 1025, 3000, 17_913, 65_536, 1 << 20, 3_000_001])
def test_server_slot_classes(n):
    sc, _ = S.tiny_scene(64, 32)
    sc.n = (33, 16, 100)
    grid, cap, mats = M.server_slot_class(sc, n)
    assert grid == (48, 16, 112)
    assert cap >= n and cap % 256 == 0 and cap >= 1024
    assert cap <= max(1024, 1.19 * n + 256)  # the next quarter-octave step
    assert mats == 4
    # monotone: a larger request never gets a smaller class
    assert M.server_slot_class(sc, n + 1)[1] >= cap


def test_server_slot_class_materials_and_small_grids():
    sc, _ = S.tiny_scene(64, 8)
    sc.materials = [S.jelly()] * 5
    grid, _, mats = M.server_slot_class(sc, 100)
    assert grid == (16, 16, 16) and mats == 8
