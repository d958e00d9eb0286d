"""GPU parity of the engine tick's particle passes (ae_engine/src/managers/simulation.rs):
LOD classification (:495-532), far-field update (:612-679), coarse temperature field (:877-966),
through the C ABI, against the CPU oracle.

Tolerances: none.  The kernels restate the reference's f32 arithmetic with explicitly rounded
operations, index lists are integers, and the coarse field sums each cell's particles in index
order, so every comparison is bit-exact.  The one freedom is the order of the capped near list,
which the reference (select_nth_unstable_by) leaves unspecified: the library returns ascending
index order, and the near lists are compared as sets.
"""
import numpy as np
import pytest

import ae_mpm as M
import oracle as O

pytestmark = pytest.mark.gpu
f32 = np.float32


def population(n, seed, cluster=0, inactive=0.1):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(-400, 400, (n, 3))
    if cluster:
        pos[:cluster] = rng.uniform(-35, 35, (cluster, 3))
        pos = pos[rng.permutation(n)]
    pos = pos.astype(f32)
    active = (rng.uniform(size=n) > inactive).astype(np.uint8)
    return pos, active


@pytest.mark.parametrize("n,cluster,max_near", [
    (1, 0, 10), (2047, 0, 10000), (2048, 300, 100), (2049, 300, 10000), (100000, 20000, 10000),
    (1000000, 30000, 10000), (50000, 0, 0),
])
def test_lod_classify_matches_oracle(ctx, n, cluster, max_near):
    pos, active = population(n, n + cluster, cluster)
    player = np.array([5.0, -3.0, 7.5], f32)
    ref = O.lod_classify(pos, active, player, 50.0, 200.0, max_near)
    got = ctx.lod_classify(pos, active, player, 50.0, 200.0, max_near)
    rn, rm, rf = ref
    gn, gm, gf = got
    assert (gn.size, gm.size, gf.size) == (rn.size, rm.size, rf.size)
    assert np.array_equal(gn, np.sort(rn))
    assert np.array_equal(gf, rf)
    # mid: the mid particles in index order, then the culled near ones (as a set; ascending here)
    d = pos - player
    d2 = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
    n_mid_proper = int(np.count_nonzero(active.astype(bool) & (d2 >= f32(2500.0)) & (d2 < f32(40000.0))))
    assert np.array_equal(gm[:n_mid_proper], rm[:n_mid_proper])
    assert np.array_equal(gm[n_mid_proper:], np.sort(rm[n_mid_proper:]))


def test_lod_classify_ties_at_the_cap_keep_the_lower_index(ctx):
    # lattice points at equal distances: 8 of the 12 particles at distance 10 fit under the cap
    pos = np.array([[10, 0, 0], [-10, 0, 0], [0, 10, 0], [0, -10, 0], [0, 0, 10], [0, 0, -10]] * 2, f32)
    pos = np.concatenate([np.array([[1, 0, 0], [0, 2, 0]], f32), pos])
    near, mid, far = ctx.lod_classify(pos, None, np.zeros(3, f32), 50.0, 200.0, 10)
    assert near.tolist() == list(range(10)) and mid.tolist() == [10, 11, 12, 13] and far.size == 0


def test_lod_classify_all_inactive_and_empty(ctx):
    pos, _ = population(5000, 7)
    near, mid, far = ctx.lod_classify(pos, np.zeros(5000, np.uint8), np.zeros(3, f32), 50.0, 200.0, 100)
    assert near.size == mid.size == far.size == 0
    near, mid, far = ctx.lod_classify(np.zeros((0, 3), f32), None, np.zeros(3, f32), 50.0, 200.0, 100)
    assert near.size == mid.size == far.size == 0


def far_case(n, seed, frac=2):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(-500, 500, (n, 3)).astype(f32)
    vel = rng.normal(0, 5, (n, 3)).astype(f32)
    temp = rng.uniform(250, 600, n).astype(f32)
    coarse = rng.uniform(270, 330, 16 ** 3).astype(f32)
    origin = np.array([-400.0, -400.0, -400.0], f32)
    idx = np.sort(rng.choice(n, max(n // frac, 1), replace=False)).astype(np.uint64)
    return pos, vel, temp, coarse, origin, idx


# half the particles far: the host path copies whole arrays and gathers on the device; an eighth:
# it gathers the far particles on the host
@pytest.mark.parametrize("frac", [2, 8])
@pytest.mark.parametrize("n", [1, 3001, 200000])
def test_far_field_update_matches_oracle_bitwise(ctx, n, frac):
    pos, vel, temp, coarse, origin, idx = far_case(n, n, frac)
    a = [pos.copy(), vel.copy(), temp.copy()]
    b = [pos.copy(), vel.copy(), temp.copy()]
    ctx.far_field_update(*a, idx, coarse, 50.0, origin, 1.0)
    O.far_field_update(*b, idx, coarse, 50.0, origin, 1.0)
    for x, y in zip(a, b):
        assert np.array_equal(x.view(np.uint32), y.view(np.uint32))


def test_far_field_rejects_out_of_range_indices(ctx):
    pos, vel, temp, coarse, origin, _ = far_case(100, 3)
    with pytest.raises(M.MpmError) as e:
        ctx.far_field_update(pos, vel, temp, np.array([5, 100], np.uint64), coarse, 50.0, origin, 1.0)
    assert e.value.code == M.EINVAL


@pytest.mark.parametrize("n_near,cn", [(0, 16), (1, 4), (10000, 16), (120000, 16), (5000, 33)])
def test_coarse_field_update_matches_oracle_bitwise(ctx, n_near, cn):
    rng = np.random.default_rng(n_near + cn)
    n = max(n_near, 1) * 2
    pos = rng.uniform(-420, 420, (n, 3)).astype(f32)
    pos[: n // 3] = rng.uniform(-50, 50, (n // 3, 3))  # many particles in a few cells
    mass = rng.uniform(0, 3, n).astype(f32)
    mass[::97] = 0.0
    temp = rng.uniform(250, 1200, n).astype(f32)
    active = (rng.uniform(size=n) > 0.15).astype(np.uint8)
    idx = np.sort(rng.choice(n, n_near, replace=False)).astype(np.uint64)
    coarse = rng.uniform(280, 300, cn ** 3).astype(f32)
    origin = np.array([-400.0, -400.0, -400.0], f32)
    a, b = coarse.copy(), coarse.copy()
    ctx.coarse_field_update(pos, mass, temp, active, idx, a, 50.0, origin, 1.0)
    O.coarse_field_update(pos, mass, temp, active, idx, b, 50.0, origin, 1.0)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_device_pointers_give_the_host_results(ctx):
    torch = pytest.importorskip("torch")
    pos, active = population(300000, 11, cluster=20000)
    player = np.array([1.0, 2.0, 3.0], f32)
    host = ctx.lod_classify(pos, active, player, 50.0, 200.0, 10000)
    dpos = torch.from_numpy(pos).cuda()
    dact = torch.from_numpy(active).cuda()
    outs = [torch.empty(pos.shape[0], dtype=torch.int64, device="cuda") for _ in range(3)]
    cnt = [M.C.c_uint64(0) for _ in range(3)]
    pl = player.copy()
    ctx.check(ctx.lib.ae_mpm_lod_classify(ctx.h, dpos.data_ptr(), dact.data_ptr(), pos.shape[0], pl.ctypes.data, 50.0,
                                          200.0, 10000, outs[0].data_ptr(), M.C.byref(cnt[0]), outs[1].data_ptr(),
                                          M.C.byref(cnt[1]), outs[2].data_ptr(), M.C.byref(cnt[2])))
    torch.cuda.synchronize()
    for h, o, c in zip(host, outs, cnt):
        assert np.array_equal(h, o[: c.value].cpu().numpy().astype(np.uint64))
    # far field in place on device arrays, then the coarse field from the near list
    vel = np.random.default_rng(12).normal(0, 2, pos.shape).astype(f32)
    temp = np.random.default_rng(13).uniform(250, 500, pos.shape[0]).astype(f32)
    mass = np.ones(pos.shape[0], f32)
    coarse = np.full(16 ** 3, 288.15, f32)
    origin = np.array([-400.0, -400.0, -400.0], f32)
    hp, hv, ht, hc = pos.copy(), vel.copy(), temp.copy(), coarse.copy()
    ctx.far_field_update(hp, hv, ht, host[2], hc, 50.0, origin, 1.0)
    ctx.coarse_field_update(hp, mass, ht, active, host[0], hc, 50.0, origin, 1.0)
    dp, dv, dt_, dc = (torch.from_numpy(x.copy()).cuda() for x in (pos, vel, temp, coarse))
    dm = torch.from_numpy(mass).cuda()
    far_d = outs[2][: cnt[2].value]
    near_d = outs[0][: cnt[0].value]
    o = origin.copy()
    ctx.check(ctx.lib.ae_mpm_far_field_update(ctx.h, dp.data_ptr(), dv.data_ptr(), dt_.data_ptr(), pos.shape[0],
                                              far_d.data_ptr(), far_d.numel(), dc.data_ptr(), 16, 50.0, o.ctypes.data,
                                              1.0))
    ctx.check(ctx.lib.ae_mpm_coarse_field_update(ctx.h, dp.data_ptr(), dm.data_ptr(), dt_.data_ptr(), dact.data_ptr(),
                                                 pos.shape[0], near_d.data_ptr(), near_d.numel(), dc.data_ptr(), 16,
                                                 50.0, o.ctypes.data, 1.0))
    torch.cuda.synchronize()
    for h, d in ((hp, dp), (hv, dv), (ht, dt_), (hc, dc)):
        assert np.array_equal(h.view(np.uint32), d.cpu().numpy().view(np.uint32))


def test_engine_tick_sequence_matches_oracle(ctx):
    # one reclassify + far-field + coarse-field tick, as simulation.rs runs them, on both sides
    pos, active = population(400000, 21, cluster=25000)
    rng = np.random.default_rng(22)
    vel = rng.normal(0, 2, pos.shape).astype(f32)
    temp = rng.uniform(250, 500, pos.shape[0]).astype(f32)
    mass = rng.uniform(0.5, 2, pos.shape[0]).astype(f32)
    player = np.array([12.0, 0.5, -8.0], f32)
    origin = (player - f32(400.0)).astype(f32)
    coarse = np.full(16 ** 3, 288.15, f32)
    g = [pos.copy(), vel.copy(), temp.copy(), coarse.copy()]
    r = [pos.copy(), vel.copy(), temp.copy(), coarse.copy()]
    gn, gm, gf = ctx.lod_classify(g[0], active, player, 50.0, 200.0, 10000)
    rn, rm, rf = O.lod_classify(r[0], active, player, 50.0, 200.0, 10000)
    assert np.array_equal(gf, rf) and np.array_equal(gn, np.sort(rn))
    ctx.far_field_update(g[0], g[1], g[2], gf, g[3], 50.0, origin, 1.0)
    O.far_field_update(r[0], r[1], r[2], rf, r[3], 50.0, origin, 1.0)
    # the oracle's near list is in select_nth order; the coarse-field sums follow the list order,
    # so the oracle gets the same (sorted) list for a bit-exact comparison
    ctx.coarse_field_update(g[0], mass, g[2], active, gn, g[3], 50.0, origin, 1.0)
    O.coarse_field_update(r[0], mass, r[2], active, np.sort(rn), r[3], 50.0, origin, 1.0)
    for x, y in zip(g, r):
        assert np.array_equal(x.view(np.uint32), y.view(np.uint32))


# ---------------------------------------------------------------- MpssBuffer housekeeping
def housekeeping_case(n, seed):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(-1200, 1200, (n, 3)).astype(f32)
    vel = rng.normal(0, 10, (n, 3)).astype(f32)
    temp = rng.uniform(-100, 9000, n).astype(f32)
    temp[::53] = np.nan
    temp[1::61] = np.inf
    pos[2::71, 1] = np.nan
    phase = rng.integers(0, 8, n).astype(np.uint8)
    mat = rng.choice([0, 1, 2, 3, 3, 1, 5], n).astype(np.uint16)
    active = (rng.uniform(size=n) > 0.1).astype(np.uint8)
    return pos, vel, temp, phase, mat, active


@pytest.mark.parametrize("n,passes", [(1, 7), (1000, 7), (1000003, 7), (200000, 1), (200000, 2), (200000, 4),
                                      (200000, 5)])
def test_housekeeping_matches_oracle_bitwise(ctx, n, passes):
    lo, hi = np.array([-1000, -50, -1000], f32), np.array([1000, 900, 1000], f32)
    a = housekeeping_case(n, n + passes)
    b = tuple(x.copy() for x in a)
    ca = ctx.mpss_housekeeping(a[0], a[1], a[2], a[3], a[4], a[5], lo, hi, 10.0, 8000.0, passes)
    cb = O.mpss_housekeeping(b[0], b[1], b[2], b[3], b[4], b[5], lo, hi, 10.0, 8000.0, passes)
    assert ca == cb
    for x, y in zip(a[:4], b[:4]):
        assert np.array_equal(x.view(np.uint8), y.view(np.uint8))


def test_housekeeping_reference_phase_cases_and_device_pointers(ctx):
    import json
    import os
    torch = pytest.importorskip("torch")
    cases = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "phase_cases.json")))
    temps = np.array(sum((c["temps"] for c in cases), []), f32)
    mats = np.array(sum(([c["material"]] * len(c["temps"]) for c in cases), []), np.uint16)
    expected = sum((c["expected"] for c in cases), [])
    n = temps.size
    pos, vel = np.zeros((n, 3), f32), np.zeros((n, 3), f32)
    phase = np.zeros(n, np.uint8)
    ctx.mpss_housekeeping(pos, vel, temps.copy(), phase, mats, None, [-1e9] * 3, [1e9] * 3, 10.0, 8000.0, 4)
    assert phase.tolist() == expected
    # device pointers: the same pass in place on device arrays
    a = housekeeping_case(300000, 77)
    b = tuple(x.copy() for x in a)
    d = [torch.from_numpy(x.copy()).cuda() for x in a]
    lo, hi = np.array([-1000, -50, -1000], f32), np.array([1000, 900, 1000], f32)
    tr = M.C.c_uint32(0)
    ctx.check(ctx.lib.ae_mpm_mpss_housekeeping(ctx.h, d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(),
                                               d[3].data_ptr(), d[4].data_ptr(), d[5].data_ptr(), a[0].shape[0],
                                               lo.ctypes.data, hi.ctypes.data, 10.0, 8000.0, 7, M.C.byref(tr)))
    torch.cuda.synchronize()
    cb = O.mpss_housekeeping(b[0], b[1], b[2], b[3], b[4], b[5], lo, hi, 10.0, 8000.0, 7)
    assert tr.value == cb
    for x, y in zip(d[:4], b[:4]):
        assert np.array_equal(x.cpu().numpy().view(np.uint8), y.view(np.uint8))
