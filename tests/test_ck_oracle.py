"""CPU tests of the CK-MPM oracle (oracle/ck_oracle.cpp), the restatement of CkMpmSolver
(ae_compute/src/ck_mpm.rs).

* The reference's own unit tests (ck_mpm.rs:510-781), scenario for scenario, as the properties
  they assert.  The reference ships no numeric golden vectors for this solver; these tests and
  the known-answer kinetic energy are what pins the oracle.
* The oracle against an independent numpy restatement of one step, bit for bit: numpy float32
  scalar arithmetic rounds every operation (no fused multiply-add) like Rust's f32, and f32::ln
  is the C library's logf, called here through ctypes.
"""
import ctypes as C
import math

import numpy as np

import ae_mpm as M
import oracle as O

f32 = np.float32
_libm = C.CDLL("libm.so.6")
_libm.logf.restype = C.c_float
_libm.logf.argtypes = [C.c_float]


def run(cfg, particles, steps):
    p = np.array(particles, np.float32, order="C")  # a copy: the caller's records stay as they were
    O.ck_step(p, cfg, steps)
    return p


def det_cols(r):
    x, y, z = r[15:18].astype(np.float64), r[18:21].astype(np.float64), r[21:24].astype(np.float64)
    return float(np.dot(z, np.cross(x, y)))


# ---------------------------------------------------------------- the reference's unit tests
def test_config_default():  # test_ckmpm_config_default (:514-521)
    c = M.ck_config()
    assert c.dt > 0 and c.grid_h > 0 and c.grid_n > 0 and c.density > 0
    assert math.isclose(c.dt, 1 / 240, rel_tol=1e-7) and c.grid_n == 32 and c.dual_grid == 1
    assert list(c.gravity) == [0.0, f32(-9.81), 0.0]


def test_config_default_matches_the_library():
    # ae_mpm_ck_config_default is host code: it runs without a GPU
    lib = M.load()
    a, b = M.CkConfig(), M.ck_config()
    lib.ae_mpm_ck_config_default(C.byref(a))
    assert bytes(a) == bytes(b)


def test_particle_creation():  # test_ckmpm_particle_creation (:523-529)
    p = M.ck_particles([[0.5, 0.5, 0.5]], 1.0, 0.001)[0]
    assert list(p[0:3]) == [0.5, 0.5, 0.5] and p[25] == 1.0
    assert list(p[15:24]) == [1, 0, 0, 0, 1, 0, 0, 0, 1] and not p[3:15].any()


def test_weight_zero_outside_support():  # :538-544
    assert O.ck_weight(0.15, 0.1) == 0.0 and O.ck_weight(-0.15, 0.1) == 0.0
    assert O.ck_weight_grad(0.15, 0.1) == 0.0


def test_weight_nonzero_inside():  # :546-553
    w = O.ck_weight(0.0, 0.1)
    w2 = O.ck_weight(0.05, 0.1)
    assert w > 0 and 0 < w2 < w
    assert O.ck_weight_grad(0.05, 0.1) < 0 < O.ck_weight_grad(-0.05, 0.1)


def test_single_particle_no_crash():  # :555-562
    p = run(M.ck_config(grid_n=16, grid_h=0.1), M.ck_particles([[0.5, 0.5, 0.5]], 1.0, 0.001), 1)
    assert p.shape == (1, 26) and np.isfinite(p).all()


def test_particle_falls_under_gravity():  # :564-580
    cfg = M.ck_config(dt=0.01, grid_n=16, grid_h=0.1, gravity=(0, -9.81, 0), bounds_min=(-2, -2, -2),
                      bounds_max=(2, 2, 2))
    p0 = M.ck_particles([[0.8, 1.5, 0.8]], 1.0, 0.001)
    p = run(cfg, p0, 1)
    assert p[0, 1] < p0[0, 1]


def test_boundary_collision():  # :582-601
    cfg = M.ck_config(dt=0.01, grid_n=32, grid_h=0.05, gravity=(0, -20, 0), bounds_min=(0, 0, 0),
                      bounds_max=(1.6, 1.6, 1.6))
    p = run(cfg, M.ck_particles([[0.8, 1.5, 0.8]], 1.0, 0.001), 300)
    assert -0.1 <= p[0, 1] < 0.5


def test_volume_ratio_finite():  # :603-612
    p = run(M.ck_config(), M.ck_particles([[0.5, 0.5, 0.5]], 1.0, 0.001), 10)
    _, _, ratio = O.ck_stats(p)
    assert np.isfinite(ratio)


def block(n, origin, spacing, mass, vol):
    g = np.arange(n, dtype=np.float32) * f32(spacing)
    pts = [(f32(origin[0]) + g[i], f32(origin[1]) + g[j], f32(origin[2]) + g[k])
           for i in range(n) for j in range(n) for k in range(n)]
    return M.ck_particles(pts, mass, vol)


def test_multiple_particles():  # :614-646
    cfg = M.ck_config(grid_n=16, grid_h=0.1, bounds_min=(-1, -1, -1), bounds_max=(2, 2, 2))
    p = run(cfg, block(3, (0.5, 0.5, 0.5), 0.05, 1.0, 0.0001), 20)
    assert np.isfinite(p[:, 0]).all() and np.isfinite(p[:, 3]).all()
    assert all(np.isfinite(det_cols(r)) for r in p)


def test_kinetic_energy():  # :648-658
    p = M.ck_particles([[0.5, 0.5, 0.5]], 2.0, 0.001, velocity=[[1.0, 0.0, 0.0]])
    ke, v, _ = O.ck_stats(p)
    assert abs(ke - 1.0) < 1e-4 and list(v) == [1.0, 0.0, 0.0]


def test_apic_affine():  # :660-684 (the reference asserts only that the step runs)
    cfg = M.ck_config(dt=0.005, grid_n=16, grid_h=0.1, bounds_min=(-1, -1, -1), bounds_max=(2, 2, 2))
    pts = [(0.5 + i * 0.05, 1.0, 0.5) for i in range(3)]
    p = run(cfg, M.ck_particles(pts, 1.0, 0.0001), 1)
    assert np.isfinite(p).all()
    assert np.abs(p[:, 6:15]).max() > 1e-10  # gravity leaves a velocity gradient on the grid


def test_elastic_deformation():  # :686-722
    cfg = M.ck_config(dt=0.001, grid_n=16, grid_h=0.1, youngs_modulus=1e4, bounds_min=(-1, -1, -1),
                      bounds_max=(2, 2, 2))
    p = run(cfg, block(4, (0.6, 0.6, 0.6), 0.04, 0.01, 0.0001), 50)
    f1 = det_cols(p[0])
    assert np.isfinite(f1) and abs(f1) < 100


def test_dual_grid_flag():  # :724-737
    outs = []
    for dual in (1, 0):
        p = run(M.ck_config(grid_n=16, grid_h=0.1, dual_grid=dual), M.ck_particles([[0.5, 0.5, 0.5]], 1.0, 0.001), 1)
        assert np.isfinite(p[0, 0])
        outs.append(p)
    assert np.array_equal(outs[0], outs[1])  # the flag is read by no step


def test_no_nan_long_run():  # :739-779
    cfg = M.ck_config(dt=0.002, grid_n=24, grid_h=0.05, youngs_modulus=1e3, bounds_min=(0, 0, 0),
                      bounds_max=(1.2, 1.2, 1.2))
    p = block(3, (0.5, 0.8, 0.5), 0.03, 0.01, 0.0001)
    for _ in range(4):
        p = run(cfg, p, 50)
        assert np.isfinite(p[:, 0]).all() and np.isfinite(p[:, 3]).all()


def test_empty_solver():
    p = np.zeros((0, 26), np.float32)
    O.ck_step(p, M.ck_config(), 3)
    ke, v, ratio = O.ck_stats(p)
    assert ke == 0 and not v.any() and ratio == 1.0  # average_volume_ratio of no particles is 1


# ---------------------------------------------------------------- independent numpy restatement
def np_weight(x, h):
    r = f32(abs(x) / h)
    if r >= 1:
        return f32(0)
    a = f32(f32(1) - f32(r * r))
    return f32(f32(f32(a * a) * a) / h)


def np_weight_grad(x, h):
    r = f32(abs(x) / h)
    if r >= 1:
        return f32(0)
    a = f32(f32(1) - f32(r * r))
    return f32(f32(f32(f32(-6) * x) * f32(a * a)) / f32(f32(h * h) * h))


def mv(m, v):  # glam Mat3 x Vec3; m[c] is column c
    return [f32(f32(f32(m[0][i] * v[0]) + f32(m[1][i] * v[1])) + f32(m[2][i] * v[2])) for i in range(3)]


def cross(a, b):
    return [f32(a[1] * b[2]) - f32(b[1] * a[2]), f32(a[2] * b[0]) - f32(b[2] * a[0]),
            f32(a[0] * b[1]) - f32(b[0] * a[1])]


def dot(a, b):
    return f32(f32(f32(a[0] * b[0]) + f32(a[1] * b[1])) + f32(a[2] * b[2]))


def length(a):
    return f32(np.sqrt(dot(a, a)))


def det(m):
    return dot(m[2], cross(m[0], m[1]))


def transpose(m):
    return [[m[0][0], m[1][0], m[2][0]], [m[0][1], m[1][1], m[2][1]], [m[0][2], m[1][2], m[2][2]]]


def inverse(m):
    t0, t1, t2 = cross(m[1], m[2]), cross(m[2], m[0]), cross(m[0], m[1])
    inv = f32(f32(1) / dot(m[2], t2))
    return transpose([[f32(x * inv) for x in t] for t in (t0, t1, t2)])


def cols(r, o):
    return [[r[o], r[o + 1], r[o + 2]], [r[o + 3], r[o + 4], r[o + 5]], [r[o + 6], r[o + 7], r[o + 8]]]


def finite(v):
    return all(np.isfinite(x) for x in v)


def np_step(ps, cfg, cr_ln=False):
    """One CkMpmSolver::step (ck_mpm.rs:187-480) on (n, 26) float32 records, in place.  cr_ln: the
    correctly rounded logarithm instead of the C library's logf."""
    h, dt, gn = f32(cfg.grid_h), f32(cfg.dt), int(cfg.grid_n)
    grid = {}

    def nodes(pos):
        c = [int(np.floor(f32(pos[a] / h))) for a in range(3)]
        for dk in (0, 1):
            for dj in (0, 1):
                for di in (0, 1):
                    i, j, k = c[0] + di, c[1] + dj, c[2] + dk
                    if min(i, j, k) < 0 or max(i, j, k) >= gn:
                        continue
                    npos = [f32(f32(f32(t) + f32(0.5)) * h) for t in (i, j, k)]
                    yield (i, j, k), [f32(npos[a] - pos[a]) for a in range(3)]

    for r in ps:  # P2G
        pos, vel, B, m = r[0:3], r[3:6], cols(r, 6), r[25]
        for key, d in nodes(pos):
            w = f32(f32(np_weight(d[0], h) * np_weight(d[1], h)) * np_weight(d[2], h))
            g = grid.setdefault(key, [f32(0), [f32(0)] * 3, [f32(0)] * 3])
            g[0] = f32(g[0] + f32(w * m))
            bd = mv(B, d)
            vg = [f32(vel[a] + bd[a]) for a in range(3)]
            wm = f32(w * m)
            g[1] = [f32(g[1][a] + f32(vg[a] * wm)) for a in range(3)]
    for g in grid.values():  # momentum -> velocity
        g[1] = [f32(x / g[0]) for x in g[1]] if g[0] > f32(1e-10) else [f32(0)] * 3
    E, nu = f32(cfg.youngs_modulus), f32(cfg.poissons_ratio)
    mu = f32(E / f32(f32(2) * f32(f32(1) + nu)))
    lam = f32(f32(E * nu) / f32(f32(f32(1) + nu) * f32(f32(1) - f32(f32(2) * nu))))
    for r in ps:  # forces
        pos, F = r[0:3], cols(r, 15)
        fdet = max(det(F), f32(1e-10))
        fit = inverse(transpose(F))
        ln = f32(np.log(np.float64(fdet))) if cr_ln else f32(_libm.logf(float(fdet)))
        P = [[f32(f32(f32(F[c][i] - fit[c][i]) * mu) + f32(fit[c][i] * f32(lam * ln))) for i in range(3)]
             for c in range(3)]
        coeff = f32(-r[24])
        for key, d in nodes(pos):
            wx, wy, wz = (np_weight(d[a], h) for a in range(3))
            gx, gy, gz = (np_weight_grad(d[a], h) for a in range(3))
            grad = [f32(f32(gx * wy) * wz), f32(f32(wx * gy) * wz), f32(f32(wx * wy) * gz)]
            force = [f32(x * coeff) for x in mv(P, grad)]
            fl = length(force)
            if fl > f32(1e4):
                force = [f32(x * f32(f32(1e4) / fl)) for x in force]
            g = grid[key]
            g[2] = [f32(g[2][a] + force[a]) for a in range(3)]
    lo, hi, rest = [f32(x) for x in cfg.bounds_min], [f32(x) for x in cfg.bounds_max], f32(cfg.restitution)
    grav = [f32(x) for x in cfg.gravity]
    for key, g in grid.items():  # grid update and boundaries
        if g[0] > f32(1e-10):
            acc = [f32(f32(g[2][a] / g[0]) + grav[a]) for a in range(3)]
            nv = [f32(g[1][a] + f32(acc[a] * dt)) for a in range(3)]
            if not finite(nv):
                nv = [f32(0)] * 3
            vl = length(nv)
            if vl > f32(50):
                nv = [f32(x * f32(f32(50) / vl)) for x in nv]
            g[1] = nv
        if not g[0] < f32(1e-10):
            for a in range(3):
                npos = f32(f32(f32(key[a]) + f32(0.5)) * h)
                if npos < lo[a] and g[1][a] < 0:
                    g[1][a] = f32(g[1][a] * -rest)
                elif npos > hi[a] and g[1][a] > 0:
                    g[1][a] = f32(g[1][a] * -rest)
    d_inv = f32(f32(4) / f32(h * h))
    for r in ps:  # G2P
        pos = r[0:3].copy()
        nv = [f32(0)] * 3
        nb = [[f32(0)] * 3 for _ in range(3)]
        for key, d in nodes(pos):
            w = f32(f32(np_weight(d[0], h) * np_weight(d[1], h)) * np_weight(d[2], h))
            v = grid[key][1]
            nv = [f32(nv[a] + f32(v[a] * w)) for a in range(3)]
            for c in range(3):
                s = f32(d[c] * d_inv)
                nb[c] = [f32(nb[c][a] + f32(f32(v[a] * s) * w)) for a in range(3)]
        if not finite(nv):
            nv = [f32(0)] * 3
        vl = length(nv)
        if vl > f32(50):
            nv = [f32(x * f32(f32(50) / vl)) for x in nv]
        r[3:6] = nv
        r[6:15] = np.array(nb, np.float32).ravel()
        gv = [[f32(x * d_inv) for x in c] for c in nb]
        gnorm = max(max(length([abs(x) for x in gv[0]]), length([abs(x) for x in gv[1]])),
                    length([abs(x) for x in gv[2]]))
        gs = f32(f32(100) / gnorm) if gnorm > f32(100) else f32(1)
        A = [[f32(f32(1 if a == c else 0) + f32(f32(gv[c][a] * gs) * dt)) for a in range(3)] for c in range(3)]
        F = cols(r, 15)
        fn = [mv(A, F[c]) for c in range(3)]
        fd = det(fn)
        if np.isfinite(fd) and abs(fd) > f32(1e-10) and abs(fd) < f32(100):
            r[15:24] = np.array(fn, np.float32).ravel()
        npos = [f32(pos[a] + f32(nv[a] * dt)) for a in range(3)]
        if finite(npos):
            r[0:3] = npos
    for r in ps:  # particle bounds
        for a in range(3):
            if r[a] < lo[a]:
                r[a] = lo[a]
                if r[3 + a] < 0:
                    r[3 + a] = f32(-r[3 + a] * rest)
            elif r[a] > hi[a]:
                r[a] = hi[a]
                if r[3 + a] > 0:
                    r[3 + a] = f32(-r[3 + a] * rest)


def test_oracle_matches_numpy_restatement_bitwise():
    rng = np.random.default_rng(11)
    n = 40
    pos = rng.uniform(0.3, 0.9, (n, 3)).astype(np.float32)
    pos[0] = (-0.03, 0.5, 0.5)        # below the grid on x: only the i = 0 node exists
    pos[1] = (1.58, 1.57, 0.2)        # at the top edge of a 32-node grid
    p = M.ck_particles(pos, 0.01, 1e-4, velocity=rng.normal(0, 1, (n, 3)))
    p[:, 6:15] = rng.normal(0, 0.5, (n, 9))                       # APIC matrices
    p[:, 15:24] += rng.normal(0, 0.05, (n, 9)).astype(np.float32)  # sheared / stretched F
    p[2, 15:24] = (1, 0, 0, 0, -1, 0, 0, 0, 1)                    # inverted: det clamps to 1e-10
    cfg = M.ck_config(dt=0.002, bounds_min=(0, 0, 0), bounds_max=(1.6, 1.6, 1.6))
    a, b = p.copy(), p.copy()
    for _ in range(3):
        O.ck_step(a, cfg, 1)
        np_step(b, cfg)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert not np.array_equal(a, p)


def test_oracle_with_correctly_rounded_ln_matches_numpy_restatement_bitwise():
    # the oracle's checker option for the device's deterministic mode: only f32::ln changes
    rng = np.random.default_rng(12)
    n = 30
    p = M.ck_particles(rng.uniform(0.3, 0.9, (n, 3)), 0.01, 1e-4, velocity=rng.normal(0, 1, (n, 3)))
    p[:, 15:24] += rng.normal(0, 0.05, (n, 9)).astype(np.float32)
    cfg = M.ck_config(dt=0.002, bounds_min=(0, 0, 0), bounds_max=(1.6, 1.6, 1.6))
    a, b = p.copy(), p.copy()
    for _ in range(2):
        O.ck_step(a, cfg, 1, correctly_rounded_ln=True)
        np_step(b, cfg, cr_ln=True)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))

