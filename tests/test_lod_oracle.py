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


# ---------------------------------------------------------------- MpssBuffer housekeeping
import json  # noqa: E402
import os  # noqa: E402

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "phase_cases.json")


def test_phase_transitions_match_the_reference_scenario_cases():
    # game/src/bin/scenario_test.rs:217-265, extracted by tests/golden/extract_phase_cases.py
    cases = json.load(open(GOLDEN))
    assert len(cases) == 3
    for c in cases:
        n = len(c["temps"])
        pos = np.zeros((n, 3), f32)
        vel = np.zeros((n, 3), f32)
        temp = np.array(c["temps"], f32)
        phase = np.full(n, c["start"], np.uint8)
        mat = np.full(n, c["material"], np.uint16)
        changed = O.mpss_housekeeping(pos, vel, temp, phase, mat, None, [-1e9] * 3, [1e9] * 3, 0.0, 1e9, passes=4)
        assert phase.tolist() == c["expected"], c["name"]
        assert changed == sum(e != c["start"] for e in c["expected"])


def np_housekeeping(pos, vel, temp, phase, mat, active, lo, hi, tmin, tmax, passes):
    n = pos.shape[0]
    arms = [(1, 0, ">=", 273.0, 1), (1, 1, ">=", 373.0, 2), (1, 2, "<", 373.0, 1), (1, 1, "<", 273.0, 0),
            (3, 0, ">=", 1811.0, 1), (3, 1, ">=", 3134.0, 2), (3, 2, "<", 3134.0, 1), (3, 1, "<", 1811.0, 0),
            (0, 0, ">=", 500.0, 2), (2, 0, ">=", 1923.0, 2)]
    changed = 0
    for i in range(n):
        if active is not None and not active[i]:
            continue
        if passes & 1:
            for d in range(3):
                if pos[i, d] < lo[d]:
                    pos[i, d] = lo[d]
                    if vel[i, d] < 0:
                        vel[i, d] = f32(-vel[i, d] * f32(0.5))
                elif pos[i, d] > hi[d]:
                    pos[i, d] = hi[d]
                    if vel[i, d] > 0:
                        vel[i, d] = f32(-vel[i, d] * f32(0.5))
        if passes & 2:
            if temp[i] > tmax:
                temp[i] = tmax
            elif temp[i] < tmin:
                temp[i] = tmin
        if passes & 4:
            cur = int(phase[i])
            for _ in range(3):
                nxt = cur
                for m, p, op, th, to in arms:
                    if mat[i] == m and cur == p and ((temp[i] >= th) if op == ">=" else (temp[i] < th)):
                        nxt = to
                        break
                if nxt == cur:
                    break
                cur = nxt
            if cur != phase[i]:
                phase[i] = cur
                changed += 1
    return changed


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


def test_housekeeping_oracle_matches_numpy_restatement_bitwise():
    lo, hi = np.array([-1000, -50, -1000], f32), np.array([1000, 900, 1000], f32)
    for passes in (7, 1, 2, 4, 6):
        a = housekeeping_case(3000, passes)
        b = tuple(x.copy() for x in a)
        ca = O.mpss_housekeeping(a[0], a[1], a[2], a[3], a[4], a[5], lo, hi, 10.0, 8000.0, passes)
        cb = np_housekeeping(b[0], b[1], b[2], b[3], b[4], b[5], lo, hi, f32(10.0), f32(8000.0), passes)
        assert ca == cb, passes
        for x, y in zip(a[:4], b[:4]):
            assert np.array_equal(x.view(np.uint8), y.view(np.uint8)), passes
