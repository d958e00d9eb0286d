"""CPU tests of the oracle for the engine tick's particle passes (ae_engine/src/managers/simulation.rs):
LOD classification (:495-532), far-field update (:612-679) and coarse temperature field (:877-966).

The oracle is pinned against an independent numpy restatement of the same lines: numpy float32
scalar arithmetic rounds every operation (no fused multiply-add), like Rust's f32, so the two must
agree bit for bit.  The reference has no unit tests for these passes.
"""
import numpy as np

import oracle as O

f32 = np.float32


def as_isize(v):  # Rust `f32 as isize`
    v = float(v)
    if v != v:
        return 0
    return int(v)  # truncation toward zero (values here are far from the saturation range)


def np_far_field(pos, vel, temp, idx, coarse, dx, origin, dt):
    n = round(coarse.size ** (1 / 3))
    for i in idx:
        vel[i, 1] = f32(vel[i, 1] - f32(f32(9.81) * dt))
        pos[i, 1] = f32(pos[i, 1] + f32(vel[i, 1] * dt))
        g = [as_isize(f32(f32(pos[i, a] - origin[a]) / dx)) for a in range(3)]
        if all(0 <= g[a] < n for a in range(3)):
            field = coarse[g[0] + g[1] * n + g[2] * n * n]
            temp[i] = f32(temp[i] + f32(f32(f32(field - temp[i]) * f32(0.02)) * dt))


def np_coarse_field(pos, mass, temp, active, idx, coarse, dx, origin, dt):
    n = round(coarse.size ** (1 / 3))
    inv = f32(f32(1.0) / dx)
    ta = np.zeros(n ** 3, f32)
    ma = np.zeros(n ** 3, f32)
    for i in idx:
        if active is not None and not active[i]:
            continue
        g = [as_isize(f32(f32(pos[i, a] - origin[a]) * inv)) for a in range(3)]
        if any(v < 0 or v >= n for v in g):
            continue
        gid = g[0] + g[1] * n + g[2] * n * n
        m = f32(max(mass[i], f32(1e-6)))
        ta[gid] = f32(ta[gid] + f32(temp[i] * m))
        ma[gid] = f32(ma[gid] + m)
    blend = f32(min(f32(f32(0.1) * dt), f32(1.0)))
    for c in range(n ** 3):
        if ma[c] > f32(1e-6):
            coarse[c] = f32(coarse[c] + f32(f32(f32(ta[c] / ma[c]) - coarse[c]) * blend))
    coef = f32(min(f32(f32(f32(10.0) * dt) / f32(dx * dx)), f32(0.16)))
    old = coarse.copy()
    for k in range(n):
        for j in range(n):
            for i in range(n):
                g = i + j * n + k * n * n
                lap, cnt = f32(0.0), 0
                for ok, o in ((i > 0, -1), (i + 1 < n, 1), (j > 0, -n), (j + 1 < n, n), (k > 0, -n * n),
                              (k + 1 < n, n * n)):
                    if ok:
                        lap = f32(lap + old[g + o])
                        cnt += 1
                if cnt:
                    avg = f32(lap / f32(cnt))
                    coarse[g] = f32(old[g] + f32(f32(coef * f32(avg - old[g])) * f32(cnt)))


def test_far_field_oracle_matches_numpy_restatement_bitwise():
    rng = np.random.default_rng(1)
    n = 300
    pos = (rng.uniform(-500, 500, (n, 3))).astype(f32)
    vel = rng.normal(0, 3, (n, 3)).astype(f32)
    temp = rng.uniform(250, 400, n).astype(f32)
    coarse = rng.uniform(270, 320, 4 ** 3).astype(f32)
    origin = np.array([-100.0, -100.0, -100.0], f32)
    idx = rng.choice(n, 200, replace=False).astype(np.uint32)
    a = (pos.copy(), vel.copy(), temp.copy())
    b = (pos.copy(), vel.copy(), temp.copy())
    O.far_field_update(*a, idx, coarse, f32(50.0), origin, f32(1.0))
    np_far_field(*b, idx, coarse, f32(50.0), origin, f32(1.0))
    for x, y in zip(a, b):
        assert np.array_equal(x.view(np.uint32), y.view(np.uint32))
    # particles within one cell below the origin truncate to cell 0, as Rust's `as isize` does
    assert any(-50.0 < p[0] - origin[0] < 0.0 for p in a[0][idx])


def test_coarse_field_oracle_matches_numpy_restatement_bitwise():
    rng = np.random.default_rng(2)
    n = 500
    pos = rng.uniform(-60, 260, (n, 3)).astype(f32)
    mass = rng.uniform(0, 2, n).astype(f32)
    mass[:10] = 0.0  # below the 1e-6 floor
    temp = rng.uniform(250, 900, n).astype(f32)
    active = (rng.uniform(size=n) > 0.2).astype(np.uint8)
    coarse = np.full(5 ** 3, 288.15, f32)
    coarse[7] = 500.0
    origin = np.array([-50.0, -50.0, -50.0], f32)
    idx = np.arange(n, dtype=np.uint32)
    a, b = coarse.copy(), coarse.copy()
    O.coarse_field_update(pos, mass, temp, active, idx, a, f32(50.0), origin, f32(1.0))
    np_coarse_field(pos, mass, temp, active, idx, b, f32(50.0), origin, f32(1.0))
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert not np.array_equal(a, coarse)


def test_lod_oracle_partitions_by_distance_and_caps_near():
    rng = np.random.default_rng(3)
    # a spread-out population plus a dense cluster around the player, so the near cap binds
    pos = np.concatenate([rng.uniform(-300, 300, (20000, 3)), rng.uniform(-30, 40, (3000, 3))]).astype(f32)
    n = pos.shape[0]
    active = (rng.uniform(size=n) > 0.1).astype(np.uint8)
    player = np.array([10.0, -5.0, 3.0], f32)
    near, mid, far = O.lod_classify(pos, active, player, 50.0, 200.0, 100)
    d = pos - player
    d2 = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
    act = np.flatnonzero(active)
    assert len(near) == 100 and len(near) + len(mid) + len(far) == act.size
    assert np.array_equal(np.sort(np.concatenate([near, mid, far])), act)
    within = act[d2[act] < f32(2500.0)]
    assert set(near.tolist()) <= set(within.tolist())
    culled = np.setdiff1d(within, near)
    assert d2[near].max() <= d2[culled].min()  # the kept ones are the closest
    mid_proper = act[(d2[act] >= f32(2500.0)) & (d2[act] < f32(40000.0))]
    assert np.array_equal(mid[:mid_proper.size], mid_proper)  # index order, then the culled ones
    assert np.array_equal(np.sort(mid[mid_proper.size:]), culled)
    assert np.array_equal(far, act[d2[act] >= f32(40000.0)])
    # under the cap the near list keeps index order
    near2, _, _ = O.lod_classify(pos, active, player, 50.0, 200.0, 10 ** 9)
    assert np.array_equal(near2, within)
