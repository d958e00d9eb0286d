"""GPU tests of the features around the substep: scene updates, error words and host-side fault
injection, FP64 totals and conservation, the autotuner, the continuous-batching server, and the
benchmark configurations at (or near) full size.

Tolerances are stated per check.  Faults are injected on the host only (NaN and out-of-domain
inputs, oversize requests, cancellation); nothing here faults, traps or hangs the GPU.
"""
import time

import numpy as np
import pytest

import ae_mpm as M
import ae_mpm_scenes as S
import oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b, floor=1e-12):
    return float(np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64)).max() /
                 max(float(np.abs(np.asarray(b, np.float64)).max()), floor))


def world_of(ctx, scenes, parts, **opts):
    f64 = parts[0].dtype == np.float64
    w = M.World(ctx, scenes, M.exec_opts(precision=64 if f64 else 32, **opts))
    for i, p in enumerate(parts):
        w.upload(i, p)
    return w


# ------------------------------------------------------------------ scene updates
def test_set_scene_changes_dt_mid_run_like_the_oracle(ctx):
    sc, p = S.tiny_scene(4096, 32, S.snow(), v=(1.0, -0.5, 0.0))
    ref = p.astype(np.float64)
    w = world_of(ctx, [sc], [p.astype(np.float64)])
    O.run(sc, ref, 10)
    w.step(10)
    sc2 = S.tiny_scene(4096, 32, S.snow(E=2.0e5))[0]
    sc2.dt = 5e-5
    sc2.gravity = (0.0, -5.0, 0.0)
    w.set_scene(0, sc2)
    O.run(sc2, ref, 10)
    w.step(10)
    got = w.download(0, p.n)
    assert rel(got.pos, ref.pos) <= 1e-10
    assert rel(got.F, ref.F) <= 1e-10
    assert np.abs(got.C - ref.C).max() <= 1e-8 * np.abs(ref.vel).max() / sc.dx


def test_set_scene_rejects_grid_or_mode_changes(ctx):
    sc, p = S.tiny_scene(512, 16)
    w = world_of(ctx, [sc], [p])
    bad = S.tiny_scene(512, 32)[0]
    with pytest.raises(M.MpmError):
        w.set_scene(0, bad)
    bad2 = S.tiny_scene(512, 16)[0]
    bad2.mode = M.MODE_REFERENCE
    with pytest.raises(M.MpmError):
        w.set_scene(0, bad2)


# ------------------------------------------------------------------ error words (host-side injection)
def test_nan_position_raises_enan(ctx):
    sc, p = S.tiny_scene(512, 16)
    p.pos[7] = (np.nan, 0.5, 0.5)
    w = world_of(ctx, [sc], [p])
    w.step(2)
    assert w.sync(raise_on_error=False) == M.ENAN
    word, _ = w.errors(0)
    assert word & 1


def test_out_of_domain_particles_are_clamped_and_reported(ctx):
    # 40 m/s for 100 substeps of 1e-4 s carries the block 0.4 m, past the domain edge (14/16)
    sc, p = S.tiny_scene(512, 16, v=(40.0, 0.0, 0.0))
    sc.wall_mode = M.WALL_SLIP
    sc.wall_margin = 1
    sc.restitution = 1.0
    w = world_of(ctx, [sc], [p])
    w.step(100)
    assert w.sync(raise_on_error=False) == M.EDOMAIN
    got = w.download(0, p.n)
    assert (got.pos <= (sc.n[0] - 2) * sc.dx + 1e-6).all() and (got.pos >= sc.dx - 1e-6).all()
    word, counters = w.errors(0)
    assert word & 2 and counters[1] > 0


def test_upload_rejects_bad_requests(ctx):
    sc, p = S.tiny_scene(512, 16)
    w = world_of(ctx, [sc], [p])
    with pytest.raises(M.MpmError) as e:
        w.upload(0, S.tiny_scene(600, 16)[1])
    assert e.value.code == M.EINVAL
    with pytest.raises(TypeError):
        w.upload(0, p.astype(np.float64))
    with pytest.raises(M.MpmError):
        M.World(ctx, [S.tiny_scene(64, 2)[0]])  # physics grids need >= 4 nodes per axis


# ------------------------------------------------------------------ totals and conservation
def test_totals_and_momentum_conservation(ctx):
    # conservation_test.rs:141 (mass) and :209 (x/z momentum without gravity on those axes)
    sc, p = S.tiny_scene(8192, 32, S.jelly(E=500.0))
    sc.gravity = (0.0, 0.0, 0.0)
    half = p.n // 2
    p.vel[:half] = (0.6, 0.0, 0.1)
    p.vel[half:] = (-0.6, 0.0, -0.1)
    w = world_of(ctx, [sc], [p])
    t0 = w.totals(0)
    w.step(60)
    t1 = w.totals(0)
    # particle masses are carried, not recomputed; the FP64 sum only changes order with the sort
    assert abs(t1[0] - t0[0]) <= 1e-12 * t0[0]
    assert abs(t1[1] - t0[1]) < 1e-5 * t0[0] and abs(t1[3] - t0[3]) < 1e-5 * t0[0]
    ref = O.totals(w.download(0, p.n))
    assert np.allclose(ref, t1, rtol=1e-12, atol=1e-15)


# ------------------------------------------------------------------ autotuner
def test_autotune_picks_a_valid_choice_and_restores_state(ctx):
    sc, p = S.tiny_scene(8192, 32, S.water(), v=(0.5, 0.0, 0.0))
    w = world_of(ctx, [sc], [p], deterministic=0)
    before = w.download(0, p.n)
    r = w.autotune(4)
    assert r.p2g_variant in (M.P2G_TILE, M.P2G_WARP_AGG, M.P2G_GLOBAL, M.P2G_LANES)
    assert r.block_threads in (128, 256) and r.sort_interval in (1, 2, 4, 8, 16, 32) and r.us_per_substep > 0
    after = w.download(0, p.n)
    assert np.array_equal(before.pos, after.pos) and np.array_equal(before.F, after.F)


def test_stage_times_split_the_g2p_kernel_from_the_snow_clamp(ctx):
    sc, p = S.tiny_scene(8192, 32, S.snow(), v=(1.5, 0.0, -1.0))
    w = world_of(ctx, [sc], [p])
    w.step(3)
    t = w.stage_times(6)
    assert all(t[k] >= 0 for k in t) and t["substep"] > 0
    assert 0 < t["g2p_kernel"] <= t["g2p"] + 1e-3
    assert t["sort"] + t["p2g"] + t["grid"] + t["g2p"] <= t["substep"] + 1e-3


# ------------------------------------------------------------------ many-scene transfers
def test_upload_many_and_download_many_equal_scene_by_scene(ctx):
    # the batched transfer calls (every copy through one staging area, one wait) move the same
    # particles as one upload / download per scene: deterministic mode, bitwise after 9 substeps,
    # with views both in the one-copy staging layout and as separate arrays
    rng = S.Rng(0x3A9)
    pairs = [S.batched_scene(rng) for _ in range(7)]
    scenes = [sc for sc, _ in pairs]
    parts = [p for _, p in pairs]
    a = M.World(ctx, scenes, M.exec_opts(deterministic=1))
    b = M.World(ctx, scenes, M.exec_opts(deterministic=1))
    a.upload_many(list(range(len(parts))), parts)
    for i, p in enumerate(parts):
        b.upload(i, p)
    for w in (a, b):
        w.step(9)
        assert w.sync(raise_on_error=False) == M.OK
    outs = [M.Particles.empty(p.n) for p in parts]
    order = list(range(len(parts)))[::-1]  # any scene order
    a.download_many(order, [outs[i] for i in order])
    for i, p in enumerate(parts):
        ref = b.download(i, p.n)
        for f in ("pos", "vel", "F", "J", "C", "mass", "mat"):
            assert np.array_equal(getattr(outs[i], f), getattr(ref, f)), (i, f)
    # a round trip without substeps returns the inputs
    c = M.World(ctx, scenes, M.exec_opts())
    c.upload_many(list(range(len(parts))), parts)
    back = [M.Particles.empty(p.n) for p in parts]
    c.download_many(list(range(len(parts))), back)
    for p, q in zip(parts, back):
        assert np.array_equal(p.pos, q.pos) and np.array_equal(p.F, q.F) and np.array_equal(p.mat, q.mat)
        assert np.allclose(p.C, q.C, rtol=1e-5, atol=1e-6)  # C travels as A = m C - k tau and back
    for w in (a, b, c):
        w.close()


def test_pipelined_batch_equals_one_world_of_all_scenes(ctx):
    # the pipelined batch (groups of scenes in worlds of their own, copies on their own streams,
    # groups computing one after another) gives every scene the results one world of all scenes
    # gives it: deterministic mode, bitwise, over two runs (the second in place)
    rng = S.Rng(0xBA7C)
    pairs = [S.batched_scene(rng) for _ in range(11)]
    scenes = [sc for sc, _ in pairs]
    parts = [p for _, p in pairs]
    det = M.exec_opts(deterministic=1)
    b = M.Batch(ctx, scenes, det, groups=3)
    first = b.groups()
    assert len(first) == 4 and first[0] == 0 and first[-1] == len(scenes)
    assert all(x < y for x, y in zip(first, first[1:]))
    w = M.World(ctx, scenes, det)
    ids = list(range(len(parts)))
    outs = [M.Particles.empty(p.n) for p in parts]
    assert b.run(parts, 12, out=outs, raise_on_error=False) == M.OK
    w.upload_many(ids, parts)
    w.step(12)
    ref = [M.Particles.empty(p.n) for p in parts]
    w.download_many(ids, ref)
    for i in ids:
        for f in ("pos", "vel", "F", "J", "C", "mass", "mat"):
            assert np.array_equal(getattr(outs[i], f), getattr(ref[i], f)), (i, f)
    assert not np.array_equal(outs[0].pos, parts[0].pos)
    # in place; the world takes the same host state (C crosses the boundary as m C - k tau and
    # back, so a round trip through the host is not the resident state to the last bit)
    assert b.run(outs, 5, raise_on_error=False) == M.OK
    w.upload_many(ids, ref)
    w.step(5)
    w.download_many(ids, ref)
    for i in ids:
        assert np.array_equal(outs[i].pos, ref[i].pos) and np.array_equal(outs[i].F, ref[i].F), i
    b.close()
    w.close()
    # more groups than scenes: one scene per group; FP64 batches are refused
    b2 = M.Batch(ctx, scenes[:2], M.exec_opts(), groups=8)
    assert b2.groups() == [0, 1, 2]
    b2.close()
    with pytest.raises(M.MpmError):
        M.Batch(ctx, scenes[:2], M.exec_opts(precision=64), groups=2)


# ------------------------------------------------------------------ server
def test_server_results_equal_running_alone(ctx):
    rng = S.Rng(0x5E4E)
    reqs = [S.batched_scene(rng) for _ in range(5)]
    substeps = [20, 35, 10, 50, 25]
    srv = M.Server(ctx, hbm_budget_bytes=4 << 30, substeps_per_tick=7, exec_options=M.exec_opts(deterministic=1))
    ids = []
    for (sc, p), k in zip(reqs, substeps):
        ids.append(srv.submit(sc, p, k))
        time.sleep(0.002)  # arrivals while earlier requests are on the device
    assert srv.drain(120.0) == M.OK
    done = {}
    for _ in range(100):
        for rid, st, t0, ta, td, out in srv.poll():
            done[rid] = (st, out, t0, ta, td)
        if len(done) == len(ids):
            break
        time.sleep(0.01)
    assert len(done) == len(ids)
    stats = srv.stats()
    srv.close()
    for rid, (sc, p), k in zip(ids, reqs, substeps):
        st, out, t0, ta, td = done[rid]
        assert st == M.OK and t0 <= ta <= td
        w = world_of(ctx, [sc], [p], deterministic=1)
        w.step(k)
        alone = w.download(0, p.n)
        w.close()
        for f in ("pos", "vel", "F", "J", "C"):
            assert np.array_equal(getattr(out, f), getattr(alone, f)), (rid, f)
    assert stats["particle_substeps"] >= sum(p.n * k for (_, p), k in zip(reqs, substeps))


def _served(srv, reqs, substeps):
    ids = [srv.submit(sc, p, k) for (sc, p), k in zip(reqs, substeps)]
    assert srv.drain(120.0) == M.OK
    done = {}
    for _ in range(100):
        for rid, st, t0, ta, td, out in srv.poll(1024):
            done[rid] = (st, out)
        if len(done) == len(ids):
            break
        time.sleep(0.01)
    assert len(done) == len(ids)
    return [done[i] for i in ids]


def test_server_reuses_slots_in_place_and_results_equal_running_alone(ctx):
    # at most 3 resident scenes: later requests take the slots that finished ones vacate while the
    # others keep running; slots are assigned by size class, so scenes of different grids and
    # particle counts share them.  Deterministic mode: every result bitwise the scene run alone.
    rng = S.Rng(0x5107)
    reqs = [S.batched_scene(rng) for _ in range(8)]
    substeps = [12, 30, 7, 18, 25, 9, 14, 21]
    srv = M.Server(ctx, hbm_budget_bytes=4 << 30, substeps_per_tick=5, max_scenes=3,
                   exec_options=M.exec_opts(deterministic=1))
    res = _served(srv, reqs, substeps)
    srv.close()
    for (st, out), (sc, p), k in zip(res, reqs, substeps):
        assert st == M.OK
        w = world_of(ctx, [sc], [p], deterministic=1)
        w.step(k)
        alone = w.download(0, p.n)
        w.close()
        for f in ("pos", "vel", "F", "J", "C"):
            assert np.array_equal(getattr(out, f), getattr(alone, f)), f


def test_server_default_path_results_match_running_alone(ctx):
    # the default options (fused G2P + P2G with float atomics, snow clamp kernel): a scene's result
    # in the mix equals the scene run alone up to the order of the atomic sums: positions within
    # 1e-5 of the largest |x|, F within 1e-4
    rng = S.Rng(0x5108)
    reqs = [S.batched_scene(rng) for _ in range(10)]
    substeps = [15, 40, 8, 22, 31, 12, 17, 26, 9, 35]
    srv = M.Server(ctx, hbm_budget_bytes=4 << 30, substeps_per_tick=6, max_scenes=4)
    res = _served(srv, reqs, substeps)
    srv.close()
    for (st, out), (sc, p), k in zip(res, reqs, substeps):
        assert st == M.OK
        w = world_of(ctx, [sc], [p], p2g_variant=M.P2G_LANES, block_threads=256, sort_interval=4, use_graph=0)
        w.step(k)
        alone = w.download(0, p.n)
        w.close()
        assert rel(out.pos, alone.pos) <= 1e-5
        assert rel(out.F, alone.F) <= 1e-4


def test_server_budget_and_cancel(ctx):
    sc, p = S.batched_scene(S.Rng(7))
    srv = M.Server(ctx, hbm_budget_bytes=1 << 20, substeps_per_tick=5)
    with pytest.raises(M.MpmError) as e:
        srv.submit(sc, p, 10)
    assert e.value.code == M.EBUDGET
    srv.close()
    srv = M.Server(ctx, hbm_budget_bytes=4 << 30, substeps_per_tick=5)
    rid = srv.submit(sc, p, 100000)
    time.sleep(0.05)
    assert srv.cancel(rid) == M.OK
    assert srv.drain(60.0) == M.OK
    res = srv.poll()
    assert len(res) == 1 and res[0][1] == M.EINVAL
    srv.close()


# ------------------------------------------------------------------ the benchmark configurations
def test_config1_fp32_vs_fp64_after_200_substeps(ctx):
    # target: <= 1e-4 relative position error against the FP64 kernels after 200 substeps
    sc, p = S.config1_jelly()
    w32 = world_of(ctx, [sc], [p])
    w64 = world_of(ctx, [sc], [p.astype(np.float64)])
    w32.step(200)
    w64.step(200)
    a, b = w32.download(0, p.n), w64.download(0, p.n)
    err = rel(a.pos, b.pos)
    assert err <= 1e-4, err
    ref = p.astype(np.float64)
    O.run(sc, ref, 200, threads=8)
    assert rel(b.pos, ref.pos) <= 1e-9


def test_config2_full_size_properties(ctx):
    sc, p = S.config2_snow()
    w32 = world_of(ctx, [sc], [p])
    w64 = world_of(ctx, [sc], [p.astype(np.float64)])
    t0 = w64.totals(0)
    w32.step(100)
    w64.step(100)
    assert w32.sync(raise_on_error=False) == M.OK
    a, b = w32.download(0, p.n), w64.download(0, p.n)
    assert rel(a.pos, b.pos) <= 1e-4
    t1 = w64.totals(0)
    assert abs(t1[1] - t0[1]) < 1e-6 * t0[0] and abs(t1[3] - t0[3]) < 1e-6 * t0[0]  # symmetric x collision


def test_config3_deterministic_runs_are_bitwise_equal(ctx):
    sc, p = S.config3_dam(scale=0.125)
    outs = []
    for _ in range(2):
        w = world_of(ctx, [sc], [p], deterministic=1)
        w.step(20)
        outs.append(w.download(0, p.n))
        w.close()
    for f in ("pos", "vel", "F", "J", "C"):
        assert np.array_equal(getattr(outs[0], f), getattr(outs[1], f)), f


# ------------------------------------------------------------------ chunking of the particle slots
@pytest.mark.parametrize("spare", [0, 61, 700])
@pytest.mark.parametrize("threads", [128, 256])
def test_one_scene_chunks_equal_the_chunk_table(ctx, spare, threads):
    # a world of one scene derives its CTA chunks arithmetically; a world of several reads them
    # from a table.  With spare capacity the last live chunk is partial and later chunks hold only
    # dead slots.  In deterministic mode scene 0 must come out bitwise the same either way.
    import dataclasses
    sc, p = S.tiny_scene(3001, 32, S.snow(), v=(1.0, -0.5, 0.25))
    sc = dataclasses.replace(sc, max_particles=p.n + spare)
    opts = dict(deterministic=1, block_threads=threads)
    one = world_of(ctx, [sc], [p], **opts)
    two = world_of(ctx, [sc, dataclasses.replace(sc)], [p, p], **opts)
    for w in (one, two):
        w.step(24)
        assert w.sync(raise_on_error=False) == M.OK
    a, b = one.download(0, p.n), two.download(0, p.n)
    one.close()
    two.close()
    for f in ("pos", "vel", "F", "J", "C"):
        assert np.array_equal(getattr(a, f), getattr(b, f)), f
    assert np.isfinite(a.pos).all() and not np.array_equal(a.pos, p.pos)
    # the atomic path (LANES P2G, chunked G2P): against the FP64 oracle, 1e-5 relative in positions
    ref = p.astype(np.float64)
    O.run(sc, ref, 24)
    fast = world_of(ctx, [sc], [p], p2g_variant=M.P2G_LANES, block_threads=threads, sort_interval=4)
    fast.step(24)
    assert fast.sync(raise_on_error=False) == M.OK
    g = fast.download(0, p.n)
    fast.close()
    assert rel(g.pos, ref.pos) <= 1e-5
