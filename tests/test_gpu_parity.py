"""GPU parity tests: the CUDA library, called through the C ABI, against the CPU oracle.

Tolerances (floating point; stated per check):
  * f32 GPU vs f64 oracle, positions: max |dx| / max |x| <= 1e-5 after tens of substeps
  * f64 GPU vs f64 oracle, positions: <= 1e-10 relative (only summation order differs)
  * reference mode f32 GPU vs f32 oracle: <= 2e-5 relative (FMA contraction and atomic order)
  * integer work (radix sort permutation, keys): bit-exact
"""
import os
import subprocess

import numpy as np
import pytest

import ae_mpm as M
import ae_mpm_scenes as S
import oracle as O

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def rel(a, b, floor=1e-12):
    return float(np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64)).max() /
                 max(float(np.abs(np.asarray(b, np.float64)).max()), floor))


def run_gpu(ctx, sc, p, substeps, **opts):
    f64 = p.dtype == np.float64
    w = M.World(ctx, [sc], M.exec_opts(precision=64 if f64 else 32, **opts))
    w.upload(0, p)
    w.step(substeps)
    w.sync()
    out = w.download(0, p.n)
    w.close()
    return out


# ------------------------------------------------------------------ radix sort (bit-exact)
@pytest.mark.parametrize("n,bits,kind", [
    (1, 8, "random"), (7, 3, "random"), (2048, 16, "random"), (2049, 21, "random"), (100000, 32, "random"),
    (300001, 24, "nearly_sorted"), (65536, 18, "equal"), (50000, 1, "random"), (1 << 21, 21, "nearly_sorted"),
    (4095, 12, "random"), (4096, 22, "nearly_sorted"), (4097, 22, "random"), (3000001, 32, "random"),
])
def test_radix_sort_matches_stable_cpu_sort(ctx, n, bits, kind):
    rng = np.random.default_rng(n + bits)
    if kind == "random":
        keys = rng.integers(0, 1 << bits, n, dtype=np.uint64).astype(np.uint32)
    elif kind == "equal":
        keys = np.full(n, 12345 & ((1 << bits) - 1), np.uint32)
    else:
        keys = np.sort(rng.integers(0, 1 << bits, n, dtype=np.uint64)).astype(np.uint32)
        swap = rng.integers(0, n - 1, n // 20)
        keys[swap], keys[swap + 1] = keys[swap + 1].copy(), keys[swap].copy()
    sk, perm = ctx.radix_sort(keys, bits)
    ref = np.argsort(keys, kind="stable").astype(np.uint32)
    assert np.array_equal(perm, ref)
    assert np.array_equal(sk, keys[ref])


def test_radix_sort_repeated_sorts_of_changing_sizes(ctx):
    # every sort reuses the context's look-back status array; entries left by earlier sorts (other
    # sizes, other digit widths) must read as not yet written
    rng = np.random.default_rng(77)
    for n, bits in ((40000, 22), (9000, 8), (123457, 22), (4096, 32), (40000, 22), (250000, 14)):
        keys = rng.integers(0, 1 << bits, n, dtype=np.uint64).astype(np.uint32)
        sk, perm = ctx.radix_sort(keys, bits)
        ref = np.argsort(keys, kind="stable").astype(np.uint32)
        assert np.array_equal(perm, ref), (n, bits)
        assert np.array_equal(sk, keys[ref]), (n, bits)


def test_radix_sort_empty(ctx):
    sk, perm = ctx.radix_sort(np.zeros(0, np.uint32), 8)
    assert sk.size == 0 and perm.size == 0


# the grouping sort of non-deterministic worlds with keys of at most 16 bits: keys ascending and
# bit-exact, the permutation a permutation that reproduces them (equal keys in any order)
@pytest.mark.parametrize("n,bits,kind", [
    (1, 4, "random"), (16384, 15, "random"), (16385, 15, "random"), (490045, 15, "random"), (490045, 15, "sorted"),
    (100000, 16, "random"), (100003, 16, "equal"), (200000, 1, "random"), (65536, 9, "random"),
    (2000001, 16, "sorted"), (30000, 3, "random"),
])
def test_counting_sort_groups_keys(ctx, n, bits, kind):
    rng = np.random.default_rng(3 * n + bits)
    if kind == "equal":
        keys = np.full(n, 54321 & ((1 << bits) - 1), np.uint32)
    else:
        keys = rng.integers(0, 1 << bits, n, dtype=np.uint64).astype(np.uint32)
        if kind == "sorted":
            keys = np.sort(keys)
    keys |= np.uint32(0xA5A50000)  # bits above key_bits are carried, not compared
    sk, perm = ctx.counting_sort(keys, bits)
    mask = np.uint32((1 << bits) - 1)
    assert np.array_equal(np.sort(perm), np.arange(n, dtype=np.uint32))
    assert np.array_equal(sk, keys[perm])
    assert np.array_equal(sk & mask, np.sort(keys & mask))


def test_counting_sort_rejects_wide_keys(ctx):
    with pytest.raises(M.MpmError):
        ctx.counting_sort(np.zeros(100000, np.uint32), 17)


# ------------------------------------------------------------------ physics mode parity
@pytest.mark.parametrize("variant", [M.P2G_TILE, M.P2G_WARP_AGG, M.P2G_GLOBAL, M.P2G_LANES])
def test_physics_jelly_matches_fp64_oracle(ctx, variant):
    sc, p = S.tiny_scene(4096, 32, S.jelly(), v=(0.7, -0.2, 0.3))
    ref = p.astype(np.float64)
    O.run(sc, ref, 30)
    g = run_gpu(ctx, sc, p, 30, p2g_variant=variant)
    assert rel(g.pos, ref.pos) <= 1e-5
    assert rel(g.vel, ref.vel) <= 1e-3
    assert rel(g.F, ref.F) <= 1e-4
    assert np.array_equal(g.mat, p.mat) and np.array_equal(g.mass, p.mass)


def test_physics_dense_small_grid_matches_fp64_oracle(ctx):
    # 40 000 particles on a 32^3 grid: 15-bit cell keys over more than one CTA's worth of particles,
    # so the non-deterministic world groups them with the counting sort (the deterministic one
    # keeps the stable radix sort); both held to the FP64 oracle
    sc, p = S.tiny_scene(40000, 32, S.jelly(), v=(0.7, -0.2, 0.3))
    ref = p.astype(np.float64)
    O.run(sc, ref, 20)
    for det in (0, 1):
        g = run_gpu(ctx, sc, p, 20, deterministic=det)
        assert rel(g.pos, ref.pos) <= 1e-5, det
        assert rel(g.vel, ref.vel) <= 1e-3, det
        assert rel(g.F, ref.F) <= 1e-4, det


def test_physics_fp64_kernels_match_fp64_oracle(ctx):
    sc, p = S.tiny_scene(4096, 32, S.jelly(), v=(0.7, -0.2, 0.3))
    ref = p.astype(np.float64)
    O.run(sc, ref, 30)
    g = run_gpu(ctx, sc, p.astype(np.float64), 30)
    assert rel(g.pos, ref.pos) <= 1e-10
    assert rel(g.vel, ref.vel) <= 1e-8
    # C is ~1e-15 here (uniform motion), so bound it on the scale of a velocity difference per cell
    assert np.abs(g.C - ref.C).max() <= 1e-9 * np.abs(ref.vel).max() / sc.dx
    assert rel(g.F, ref.F) <= 1e-10


@pytest.mark.parametrize("mat", ["snow", "water"])
def test_physics_materials_match_fp64_oracle(ctx, mat):
    m = S.snow() if mat == "snow" else S.water()
    sc, p = S.tiny_scene(8192, 32, m, v=(1.5, 0.0, -1.0))
    ref = p.astype(np.float64)
    O.run(sc, ref, 40)
    g = run_gpu(ctx, sc, p, 40)
    assert rel(g.pos, ref.pos) <= 1e-5
    assert rel(g.J, ref.J) <= 1e-4
    g64 = run_gpu(ctx, sc, p.astype(np.float64), 40)
    assert rel(g64.pos, ref.pos) <= 1e-10
    assert rel(g64.J, ref.J) <= 1e-9


def test_snow_collision_through_plastic_flow_matches_fp64_oracle(ctx):
    # two snow boxes collide: most particles reach the clamp band and take the SVD return mapping
    # (and its FP64 redo near degenerate pairs) every substep.  Tolerances: f32 GPU vs f64 oracle
    # 1e-5 in positions, 2e-4 in F and J_p (the f32 oracle itself is 2e-6 / 2e-5 from f64 here);
    # f64 GPU vs f64 oracle 1e-10 / 1e-9.
    sc, p = S.snow_collision_small()
    ref = p.astype(np.float64)
    O.run(sc, ref, 80)
    lo, hi = 1 - 2.5e-2, 1 + 7.5e-3
    s = np.linalg.svd(ref.F.reshape(-1, 3, 3), compute_uv=False)
    assert ((np.abs(s - lo) < 1e-9) | (np.abs(s - hi) < 1e-9)).any(1).mean() > 0.5  # the clamp is active
    g = run_gpu(ctx, sc, p, 80)
    assert rel(g.pos, ref.pos) <= 1e-5
    assert rel(g.F, ref.F) <= 2e-4
    assert rel(g.J, ref.J) <= 2e-4
    g64 = run_gpu(ctx, sc, p.astype(np.float64), 80)
    assert rel(g64.pos, ref.pos) <= 1e-10
    assert rel(g64.F, ref.F) <= 1e-9
    assert rel(g64.J, ref.J) <= 1e-9


@pytest.mark.parametrize("interval", [2, 5, 32])
def test_sort_interval_does_not_change_results(ctx, interval):
    sc, p = S.tiny_scene(4096, 32, S.jelly(), v=(0.5, 0.5, 0.0))
    a = run_gpu(ctx, sc, p, 25, sort_interval=1)
    b = run_gpu(ctx, sc, p, 25, sort_interval=interval)
    assert rel(b.pos, a.pos) <= 1e-6


def test_split_steps_and_upload_mid_run_agree_with_one_run(ctx):
    # World state carried between step() calls (buffer parity, sort phase, cell keys, graph
    # replays) must give the same trajectory as one call, eager and graph alike; an upload
    # mid-run must restart cleanly; the LANES and TILE P2G variants must agree.  Snow exercises the
    # clamp kernel.  Tolerance: f32, only atomic summation order differs: 1e-6 relative in positions.
    sc, p = S.tiny_scene(8192, 32, S.snow(), v=(1.0, -0.5, 0.25))
    one = run_gpu(ctx, sc, p, 24, p2g_variant=M.P2G_LANES, use_graph=1)
    for graph in (0, 1):
        w = M.World(ctx, [sc], M.exec_opts(p2g_variant=M.P2G_LANES, use_graph=graph, sort_interval=4))
        w.upload(0, p)
        for k in (5, 11, 8):
            w.step(k)
        w.sync()
        split = w.download(0, p.n)
        w.upload(0, p)  # back to the start: the pending scatter of the stepped state must go
        w.step(24)
        w.sync()
        again = w.download(0, p.n)
        w.close()
        assert rel(split.pos, one.pos) <= 1e-6, graph
        assert rel(again.pos, one.pos) <= 1e-6, graph
        assert rel(again.F, one.F) <= 1e-5, graph
    unfused = run_gpu(ctx, sc, p, 24, p2g_variant=M.P2G_TILE)
    assert rel(unfused.pos, one.pos) <= 1e-6
    assert rel(unfused.F, one.F) <= 1e-5


def test_graph_and_eager_paths_agree(ctx):
    sc, p = S.tiny_scene(4096, 32, S.snow(), v=(0.5, 0.5, 0.0))
    a = run_gpu(ctx, sc, p, 16, use_graph=0, deterministic=1)
    b = run_gpu(ctx, sc, p, 16, use_graph=1, deterministic=1)
    assert np.array_equal(a.pos, b.pos) and np.array_equal(a.F, b.F)


# ------------------------------------------------------------------ deterministic mode
def test_deterministic_mode_is_bitwise_reproducible(ctx):
    sc, p = S.tiny_scene(8192, 32, S.snow(), v=(1.0, -0.5, 0.25))
    a = run_gpu(ctx, sc, p, 30, deterministic=1)
    b = run_gpu(ctx, sc, p, 30, deterministic=1)
    for f in ("pos", "vel", "F", "J", "C"):
        assert np.array_equal(getattr(a, f), getattr(b, f)), f
    fast = run_gpu(ctx, sc, p, 30)
    assert rel(a.pos, fast.pos) <= 1e-5


def test_deterministic_fp64_matches_oracle(ctx):
    sc, p = S.tiny_scene(4096, 32, S.water(), v=(1.0, 0.0, 0.0))
    ref = p.astype(np.float64)
    O.run(sc, ref, 20)
    g = run_gpu(ctx, sc, p.astype(np.float64), 20, deterministic=1)
    assert rel(g.pos, ref.pos) <= 1e-10


# ------------------------------------------------------------------ batched = alone
def test_batched_world_matches_scenes_alone(ctx):
    rng = S.Rng(0xBEEF)
    pairs = [S.batched_scene(rng) for _ in range(6)]
    scenes = [s for s, _ in pairs]
    w = M.World(ctx, scenes, M.exec_opts(deterministic=1))
    for i, (_, p) in enumerate(pairs):
        w.upload(i, p)
    w.step(12)
    w.sync()
    for i, (s, p) in enumerate(pairs):
        got = w.download(i, p.n)
        alone = run_gpu(ctx, s, p, 12, deterministic=1)
        for f in ("pos", "vel", "F", "J", "C"):
            assert np.array_equal(getattr(got, f), getattr(alone, f)), (i, f)
    w.close()


def test_batched_world_with_atomics_matches_fp64_oracle_per_scene(ctx):
    # the default (fused G2P + P2G) path on a world of several scenes of different grids and
    # materials, snow included: the clamp kernel's scatter takes queue entries of several scenes in
    # one warp.  Each scene against the FP64 oracle run alone: 1e-5 of the largest |x|.
    rng = S.Rng(0xF05E)
    pairs = [S.batched_scene(rng) for _ in range(9)]
    pairs.append(S.snow_collision_small(n_box=2048, grid=32))
    scenes = [sc for sc, _ in pairs]
    w = M.World(ctx, scenes, M.exec_opts(p2g_variant=M.P2G_LANES, block_threads=128, sort_interval=4))
    for i, (_, p) in enumerate(pairs):
        w.upload(i, p)
    w.step(40)
    assert w.sync(raise_on_error=False) == M.OK
    clamped = 0
    for i, (sc, p) in enumerate(pairs):
        got = w.download(i, p.n)
        ref = p.astype(np.float64)
        cnt = O.run(sc, ref, 40)
        assert rel(got.pos, ref.pos) <= 1e-5, i
        assert rel(got.F, ref.F) <= 2e-4, i
        if sc.materials[0].model == M.PHYS_SNOW:  # J carries the plastic J_p for snow
            clamped += int(np.sum(np.abs(ref.J - 1.0) > 1e-9))
    assert clamped > 1000  # snow particles took the return mapping (and the clamp kernel's scatter)
    w.close()


# ------------------------------------------------------------------ reference mode (drop-in)
def _ref_setup(n=3000, grid=32, dx=0.05, origin=(0.0, 0.0, 0.0), models=(M.NEO_HOOKEAN,), seed=5):
    rng = np.random.default_rng(seed)
    p = M.Particles.empty(n)
    lo = np.asarray(origin) + np.array([0.2, 0.3, 0.2]) * grid * dx
    p.pos[:] = lo + rng.random((n, 3)) * 0.4 * grid * dx
    p.vel[:] = rng.normal(0, 0.3, (n, 3))
    p.mass[:] = 0.001
    p.mat[:] = rng.integers(0, len(models) + 1, n)
    p.J[:] = 1.0
    cfg = M.Config(grid_dx=dx, grid_size=(grid, grid, grid), substeps=4, gravity=(0, -9.81, 0), damping=0.995)
    g = M.Grid(grid, grid, grid, dx, origin)
    mats = [M.material(young_modulus=1e4, poisson_ratio=0.25, yield_stress=50.0, density=1000.0,
                       friction_angle=30.0, cohesion=10.0) for _ in models]
    return p, g, cfg, mats, list(models)


@pytest.mark.parametrize("models", [
    (M.NEO_HOOKEAN,), (M.NEWTONIAN_FLUID,), (M.DRUCKER_PRAGER,), (M.VON_MISES,), (M.COROTATED,),
    (M.FIXED_COROTATED,), (M.RIGID,),
    (M.NEO_HOOKEAN, M.NEWTONIAN_FLUID, M.DRUCKER_PRAGER, M.VON_MISES),
])
def test_dropin_step_parallel_with_grid_matches_oracle(ctx, models):
    p, g, cfg, mats, mods = _ref_setup(models=models)
    idx = np.arange(0, p.n, 2, dtype=np.uint64)  # every other particle, like the LOD index list
    a, b = p.copy(), p.copy()
    ctx.step_parallel_with_grid(a, g, cfg, mats, mods, 0.016, idx)
    assert O.step_parallel_with_grid(b, g, cfg, mats, mods, 0.016, idx) == 0
    assert rel(a.pos, b.pos) <= 2e-5
    assert rel(a.vel, b.vel) <= 1e-3
    assert rel(a.F, b.F) <= 1e-4
    untouched = np.arange(1, p.n, 2)
    assert np.array_equal(a.pos[untouched], p.pos[untouched])


def test_dropin_parallel_path_rules_with_moving_window(ctx):
    # >= 50 000 indices switch to the parallel path, whose x/z walls are offset by the origin
    p, g, cfg, mats, mods = _ref_setup(n=60000, grid=64, dx=0.1, origin=(-3.2, 0.0, -3.2),
                                       models=(M.NEO_HOOKEAN, M.NEWTONIAN_FLUID))
    idx = np.arange(p.n, dtype=np.uint64)
    a, b = p.copy(), p.copy()
    ctx.step_parallel_with_grid(a, g, cfg, mats, mods, 0.016, idx)
    assert O.step_parallel_with_grid(b, g, cfg, mats, mods, 0.016, idx, threads=4) == 0
    assert rel(a.pos, b.pos) <= 2e-5


# index lists: ascending and a quarter or more of the buffer take the whole-array device gather; sparse
# or unordered lists take the host gather
INDEX_PATTERNS = {
    "all": lambda n: np.arange(n),
    "every_other": lambda n: np.arange(0, n, 2),
    "sparse": lambda n: np.arange(3, n, 7),
    "descending": lambda n: np.arange(n)[::-1],
}


@pytest.mark.parametrize("pattern", sorted(INDEX_PATTERNS))
def test_dropin_velocity_only_matches_oracle(ctx, pattern):
    p, g, cfg, mats, mods = _ref_setup(n=5000, grid=16, dx=25.0)
    idx = INDEX_PATTERNS[pattern](p.n).astype(np.uint64)
    a, b = p.copy(), p.copy()
    ctx.step_velocity_only_parallel(a, g, cfg, 0.2, idx)
    assert O.step_velocity_only_parallel(b, g, cfg, 0.2, idx) == 0
    assert rel(a.pos, b.pos) <= 2e-5
    assert rel(a.vel, b.vel) <= 1e-4
    assert np.array_equal(a.F, p.F) and np.array_equal(a.C, p.C) and np.array_equal(a.J, p.J)
    untouched = np.setdiff1d(np.arange(p.n), idx.astype(np.int64))
    assert np.array_equal(a.pos[untouched], p.pos[untouched]) and np.array_equal(a.vel[untouched], p.vel[untouched])


def test_dropin_velocity_only_at_mid_field_size_matches_oracle(ctx):
    # the engine's mid-field call at full size: 490 045 mid particles of a 1 000 055-particle buffer
    # on a 32^3 grid (15-bit keys: the call groups particles with the counting sort)
    import bench as B

    p, idx, g, cfg = B.midfield_setup(0xAE06)
    a, b = p.copy(), p.copy()
    ctx.step_velocity_only_parallel(a, g, cfg, 0.2, idx)
    assert O.step_velocity_only_parallel(b, g, cfg, 0.2, idx, threads=os.cpu_count() or 1) == 0
    ii = idx.astype(np.int64)
    assert rel(a.pos[ii], b.pos[ii]) <= 2e-5
    assert rel(a.vel[ii], b.vel[ii]) <= 1e-4
    rest = np.setdiff1d(np.arange(p.n), ii)
    assert np.array_equal(a.pos[rest], p.pos[rest]) and np.array_equal(a.vel[rest], p.vel[rest])


@pytest.mark.parametrize("pattern", ["every_other", "sparse", "descending"])
def test_dropin_reference_index_patterns_match_oracle(ctx, pattern):
    p, g, cfg, mats, mods = _ref_setup(n=4000, models=(M.NEO_HOOKEAN, M.NEWTONIAN_FLUID))
    idx = INDEX_PATTERNS[pattern](p.n).astype(np.uint64)
    a, b = p.copy(), p.copy()
    ctx.step_parallel_with_grid(a, g, cfg, mats, mods, 0.016, idx)
    assert O.step_parallel_with_grid(b, g, cfg, mats, mods, 0.016, idx) == 0
    assert rel(a.pos, b.pos) <= 2e-5
    assert rel(a.F, b.F) <= 1e-4
    assert rel(a.J, b.J) <= 1e-4
    untouched = np.setdiff1d(np.arange(p.n), idx.astype(np.int64))
    for f in ("pos", "vel", "F", "J", "C", "mass", "mat"):
        assert np.array_equal(getattr(a, f)[untouched], getattr(p, f)[untouched]), f


@pytest.mark.parametrize("order", ["ascending", "descending"])
def test_dropin_counts_change_within_a_capacity_bucket(ctx, order):
    # the drop-in world is cached per power-of-two particle bucket: counts that grow and shrink inside
    # one bucket (the engine's near set from tick to tick) reuse it, on both data paths
    p, g, cfg, mats, mods = _ref_setup(n=9000, models=(M.NEO_HOOKEAN, M.NEWTONIAN_FLUID))
    for m in (3000, 3500, 2100, 4096):
        idx = np.arange(m, dtype=np.uint64)
        if order == "descending":
            idx = idx[::-1].copy()
        a, b = p.copy(), p.copy()
        ctx.step_parallel_with_grid(a, g, cfg, mats, mods, 0.016, idx)
        assert O.step_parallel_with_grid(b, g, cfg, mats, mods, 0.016, idx) == 0
        assert rel(a.pos, b.pos) <= 2e-5, m
        v1, v2 = p.copy(), p.copy()
        ctx.step_velocity_only_parallel(v1, g, cfg, 0.016, idx)
        assert O.step_velocity_only_parallel(v2, g, cfg, 0.016, idx) == 0
        assert rel(v1.pos, v2.pos) <= 2e-5, m


def test_dropin_empty_and_invalid_calls(ctx):
    p, g, cfg, mats, mods = _ref_setup(n=10)
    a = p.copy()
    ctx.step_parallel_with_grid(a, g, cfg, mats, mods, 0.016, np.zeros(0, np.uint64))
    assert np.array_equal(a.pos, p.pos)
    with pytest.raises(M.MpmError) as e:
        ctx.step_parallel_with_grid(a, g, cfg, [], mods, 0.016, np.arange(3, dtype=np.uint64))
    assert e.value.code == M.EINVAL
    with pytest.raises(M.MpmError):
        ctx.step_parallel_with_grid(a, g, cfg, mats, mods, 0.016, np.array([10], np.uint64))


# ------------------------------------------------------------------ C++ host mirror
def test_host_mirror_reference_unit_tests():
    exe = os.path.join(ROOT, "ae-engine_b200", "_build", "test_host_mirror")
    r = subprocess.run([exe], stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True, timeout=600)
    assert r.returncode == 0, r.stdout
    assert "ALL HOST-MIRROR TESTS PASSED" in r.stdout
