"""CPU checks of the engine-call workloads bench.py times: the population's LOD shells, the index lists
the engine would pass (ascending, the near set at the LOD cap) and that every selected particle lies
inside its grid, so the drop-in call sees the shapes the reference's own measurement had."""
import numpy as np

import bench as B


def test_midfield_population_matches_the_reference_measurement():
    p, idx, grid, cfg = B.midfield_setup(0xAE06)
    assert p.n == B.MID["n_near"] + B.MID["n_mid"] + B.MID["n_far"] == 1000055
    assert idx.size == 490045
    assert np.all(np.diff(idx.astype(np.int64)) > 0)  # ascending: the whole-array device gather applies
    assert 4 * idx.size >= p.n
    r = np.linalg.norm(p.pos[idx.astype(np.int64)].astype(np.float64), axis=1)
    assert r.min() >= B.MID["near"] - 1e-3 and r.max() <= B.MID["mid"] + 1e-3
    lo = np.asarray(grid.origin, np.float64)
    hi = lo + grid.dx * np.array([grid.nx, grid.ny, grid.nz], np.float64)
    sel = p.pos[idx.astype(np.int64)]
    assert np.all(sel >= lo) and np.all(sel <= hi)
    assert cfg.substeps == 1 and (grid.nx, grid.ny, grid.nz) == (32, 32, 32)


def test_near_population_is_the_lod_cap_of_the_same_buffer():
    p, idx, grid, cfg, mats, models = B.near_setup(0xAE07)
    assert idx.size == 10000
    assert np.all(np.diff(idx.astype(np.int64)) > 0)
    assert 4 * idx.size < p.n  # a sparse list: the host gather path
    sel = p.pos[idx.astype(np.int64)].astype(np.float64)
    assert np.linalg.norm(sel, axis=1).max() < B.MID["near"]
    half = grid.nx * grid.dx / 2
    assert np.all(np.abs(sel) < half)
    assert len(mats) == len(models) == 4 and set(np.unique(p.mat)) <= {0, 1, 2, 3}


def test_dominant_kernel_times_the_fused_kernel_without_the_snow_clamp():
    import bench as B

    fused = {"sort": 6.0, "p2g": 2.6, "grid": 9.0, "g2p": 98.0, "substep": 116.0, "g2p_kernel": 91.0}
    assert B.dominant_kernel(fused) == ("g2p2g", 91.0)
    plain = {"sort": 6.0, "p2g": 58.0, "grid": 9.0, "g2p": 60.0, "substep": 133.0, "g2p_kernel": 56.0}
    assert B.dominant_kernel(plain) == ("p2g", 58.0)
    old = {"sort": 6.0, "p2g": 2.6, "grid": 9.0, "g2p": 98.0, "substep": 116.0}  # five-stage timings
    assert B.dominant_kernel(old) == ("g2p2g", 98.0)
    assert B.KERNEL_BYTES["g2p2g"] == (260, 32)  # P2G 104 + G2P 156 B per particle, 16 + 16 B per node


def test_batched_shards_deal_one_scene_list():
    import bench as B

    a = B.shard(list(range(10)), 0, 3)
    b = B.shard(list(range(10)), 1, 3)
    c = B.shard(list(range(10)), 2, 3)
    assert sorted(a + b + c) == list(range(10)) and a == [0, 3, 6, 9]


def test_substep_roofline_counts_the_scope_bytes():
    import bench as B

    r = B.substep_roofline(1000, 100, {"substep": 1.0}, 1000.0)
    assert r["substep_bytes"] == 260 * 1000 + 80 * 100
    assert abs(r["substep_achieved"] - 268.0) < 1e-9 and abs(r["substep_frac"] - 0.268) < 1e-12
