"""CPU tests of the oracle (oracle/mpm_oracle.cpp) against the reference's own known answers and
property tests.  These pin the oracle before it is trusted as the checker of the CUDA library.

Sources of every check (reference project paths):
  tests/golden/known_answers.json    b_spline / quadratic_weight values (mpm_solver.rs:1595-1609,
                                     mpm_compute.rs:1103-1132), extracted from the Rust tests
  partition of unity                 mpm_compute.rs:1134-1151
  constitutive known answers         constitutive.rs:619-665
  sandpile / water / steel           mpm_solver.rs:1611-1745
  mass conservation, fall, floor     mpm_compute.rs:1223-1301
  conservation harness thresholds    game/src/bin/conservation_test.rs:141,209
"""
import json
import math
import os

import numpy as np
import pytest

import ae_mpm as M
import ae_mpm_scenes as S
import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))


def known_answers():
    with open(os.path.join(HERE, "golden", "known_answers.json")) as f:
        return json.load(f)


@pytest.mark.parametrize("row", known_answers(), ids=lambda r: "%s(%g)@%s" % (r["function"], r["arg"], r["source"]))
def test_kernel_known_answers(row):
    f = getattr(O, row["function"])
    assert abs(f(row["arg"]) - row["expected"]) < row["tol"]


def test_known_answer_fixture_is_complete():
    rows = known_answers()
    assert len(rows) == 19
    assert {r["function"] for r in rows} == {"b_spline", "b_spline_deriv", "quadratic_weight", "quadratic_weight_grad"}


def test_partition_of_unity():
    # mpm_compute.rs:1134-1151: weights of the 3-node stencil sum to 1 for fx in [0.5, 1.5]
    for i in range(101):
        fx = 0.5 + i / 100.0
        s = O.quadratic_weight(fx) + O.quadratic_weight(fx - 1.0) + O.quadratic_weight(fx - 2.0)
        assert abs(s - 1.0) < 1e-5


def test_reference_stencil_partition_defect():
    # the ae_particle stencil (nodes g..g+2 with fx in [0,1)) sums to 0.875 at fx = 0: the
    # documented reference inconsistency that reference mode reproduces
    s = O.b_spline(0.0) + O.b_spline(1.0) + O.b_spline(2.0)
    assert abs(s - 0.875) < 1e-7


def test_lame_constants_match_material_params():
    m = M.material(young_modulus=1e6, poisson_ratio=0.3)
    mu, lam, k = O.lame(m)
    assert math.isclose(mu, 1e6 / 2.6, rel_tol=1e-6)
    assert math.isclose(lam, 1e6 * 0.3 / (1.3 * 0.4), rel_tol=1e-6)
    assert math.isclose(k, 1e6 / (3 * 0.4), rel_tol=1e-6)
    # poisson_ratio clamped to 0.4999 (constitutive.rs:61-63): finite at nu = 0.5
    assert all(math.isfinite(x) for x in O.lame(M.material(poisson_ratio=0.5)))


I3 = np.eye(3, dtype=np.float32).reshape(9)


def test_neo_hookean_identity_is_stress_free():  # constitutive.rs:623-631
    st, _, _ = O.compute_stress(M.NEO_HOOKEAN, M.material(), I3, 1.0)
    assert np.abs(st).max() < 1e-4


def test_newtonian_fluid_signs():  # constitutive.rs:633-648
    st, _, _ = O.compute_stress(M.NEWTONIAN_FLUID, M.material(), I3, 1.0)
    assert np.abs(st[[0, 4, 8]]).max() < 1e-4
    st, _, _ = O.compute_stress(M.NEWTONIAN_FLUID, M.material(), I3, 0.9)
    assert st[0] < 0


def test_sand_yields_under_shear():  # constitutive.rs:650-658
    F = I3.copy()
    F[1] = 0.5
    sand = M.material(young_modulus=5e7, poisson_ratio=0.2, yield_stress=1e4, hardening=0.005, density=1600,
                      friction_angle=35.0, cohesion=0.0)
    _, _, plastic = O.compute_stress(M.DRUCKER_PRAGER, sand, F, 1.0)
    assert plastic


def test_steel_elastic_at_identity():  # constitutive.rs:660-665
    steel = M.material(young_modulus=2e11, poisson_ratio=0.3, yield_stress=2.5e8, hardening=0.01, density=7850,
                       friction_angle=0.0)
    _, _, plastic = O.compute_stress(M.VON_MISES, steel, I3, 1.0)
    assert not plastic


def test_rigid_returns_identity_stress():  # constitutive.rs:370-373
    st, _, _ = O.compute_stress(M.RIGID, M.material(), I3 * 1.1, 1.0)
    assert np.allclose(st, I3)


def test_polar_decomposition_reproduces_reference_sign_iteration():
    # The reference's inv_transpose (constitutive.rs:306-324) returns the inverse, not the inverse
    # transpose, so its "Newton polar" iteration R <- (R + R^-1)/2 (:284-304) is the matrix sign
    # iteration: R -> I whenever F's eigenvalues have positive real part, and S = R^T F = F.
    th = 0.3
    R = np.array([[math.cos(th), -math.sin(th), 0], [math.sin(th), math.cos(th), 0], [0, 0, 1]])
    F = R @ np.diag([1.1, 0.95, 1.02])
    Rg, Sg = O.polar_decomp(F.reshape(9))
    assert np.allclose(Rg.reshape(3, 3), np.eye(3), atol=1e-5)
    assert np.allclose(Sg.reshape(3, 3), F, atol=1e-5)
    # a rotation past 90 degrees has eigenvalues with negative real part: sign(F) != I there
    th = 2.5
    R2 = np.array([[math.cos(th), -math.sin(th), 0], [math.sin(th), math.cos(th), 0], [0, 0, 1]])
    Rg2, _ = O.polar_decomp(R2.reshape(9))
    assert not np.allclose(Rg2.reshape(3, 3), np.eye(3), atol=1e-2)


@pytest.mark.parametrize("seed", range(20))
def test_svd3_reconstructs_and_is_proper(seed):
    rng = np.random.default_rng(seed)
    F = np.eye(3) + rng.normal(0, 0.3 if seed % 2 else 0.01, (3, 3))
    for f64 in (False, True):
        U, s, V, _ = O.svd3(F, f64=f64)
        tol = 1e-12 if f64 else 2e-6
        assert np.abs(U @ np.diag(s) @ V.T - F).max() <= tol * max(1.0, np.abs(F).max()) * 10
        assert abs(np.linalg.det(U) - 1) < 1e-5 and abs(np.linalg.det(V) - 1) < 1e-5
        assert np.allclose(np.abs(s), np.linalg.svd(F)[1], rtol=1e-5, atol=1e-6)
        assert s[0] >= s[1] >= abs(s[2]) - 1e-6


def test_svd3_fp64_fallback_only_where_a_degenerate_pair_straddles_a_threshold():
    lo, hi = 1 - 2.5e-2, 1 + 7.5e-3
    # sigma_0 ~ sigma_1 on both sides of the stretch threshold hi: their clamped values differ
    F = np.diag([hi + 5e-5, hi - 5e-5, 0.999]).astype(np.float32)
    assert O.svd3(F, allow_fallback=True, lo=lo, hi=hi)[3]
    # near-degenerate but on the same side (both clamped to hi): FP32 suffices
    F = np.diag([1.02, 1.02 + 1e-6, 0.999]).astype(np.float32)
    assert not O.svd3(F, allow_fallback=True, lo=lo, hi=hi)[3]
    # well separated
    assert not O.svd3(np.diag([1.2, 1.0, 0.8]).astype(np.float32), allow_fallback=True, lo=lo, hi=hi)[3]


def test_clamp_identity_fast_path_is_exact():
    lo, hi = 1 - 2.5e-2, 1 + 7.5e-3
    rng = np.random.default_rng(7)
    for _ in range(200):
        F = np.eye(3) + rng.normal(0, 4e-3, (3, 3))
        s = np.linalg.svd(F)[1]
        inside = s.min() >= lo and s.max() <= hi and np.linalg.det(F) > 0
        if O.clamp_is_identity(F, lo, hi):
            assert inside  # the bound never claims a clamp-free F that would be clamped
    th = 0.4
    R = np.array([[math.cos(th), -math.sin(th), 0], [math.sin(th), math.cos(th), 0], [0, 0, 1]])
    assert O.clamp_is_identity(R, lo, hi)  # pure rotations need no SVD


def rotation(rng):
    q, r = np.linalg.qr(rng.normal(size=(3, 3)))
    q = q * np.sign(np.diag(r))
    return q if np.linalg.det(q) > 0 else -q


def test_clamp_identity_is_tight_for_rotated_f():
    # F = R1 diag(s) R2^T with the singular values spread across the band: the test is exact, so
    # every such F whose singular values are inside by a margin skips the SVD, whatever its rotations
    # (a Gershgorin bound on F^T F rejects most of them), and every F with one outside takes it
    lo, hi = 1 - 2.5e-2, 1 + 7.5e-3
    rng = np.random.default_rng(11)
    margin = 1e-5
    for _ in range(400):
        R1, R2 = rotation(rng), rotation(rng)
        s = rng.uniform(lo + margin, hi - margin, 3)
        F = (R1 @ np.diag(s) @ R2.T).astype(np.float32)
        assert O.clamp_is_identity(F, lo, hi), s
        k = rng.integers(0, 3)
        t = s.copy()
        t[k] = rng.choice([rng.uniform(lo - 0.02, lo - margin), rng.uniform(hi + margin, hi + 0.02)])
        G = (R1 @ np.diag(t) @ R2.T).astype(np.float32)
        assert not O.clamp_is_identity(G, lo, hi), t
        assert not O.clamp_is_identity((R1 @ np.diag(s * [1, 1, -1]) @ R2.T).astype(np.float32), lo, hi)
    assert not O.clamp_is_identity(np.diag([1.0, 1.0, -1.0]), lo, hi)  # inverted


def test_snow_collision_oracle_f32_tracks_f64_through_plastic_flow():
    # the scene the GPU parity test uses for the SVD return mapping: most particles reach the
    # clamp band, J_p falls well below 1, and the f32 oracle stays close to the f64 one (pos 1.8e-6,
    # F 1.6e-5, J 1.3e-5 relative after 80 substeps), which bounds what f32 rounding alone does here
    sc, p = S.snow_collision_small()
    r64 = p.astype(np.float64)
    O.run(sc, r64, 80)
    r32 = S.concat([p])
    O.run(sc, r32, 80)
    lo, hi = 1 - 2.5e-2, 1 + 7.5e-3
    s = np.linalg.svd(r64.F.reshape(-1, 3, 3), compute_uv=False)
    assert ((np.abs(s - lo) < 1e-9) | (np.abs(s - hi) < 1e-9)).any(1).mean() > 0.5
    assert r64.J.min() < 0.9
    rel = lambda a, b: float(np.abs(a.astype(np.float64) - b).max() / np.abs(b).max())
    assert rel(r32.pos, r64.pos) <= 1e-5
    assert rel(r32.F, r64.F) <= 1e-4
    assert rel(r32.J, r64.J) <= 1e-4


def _velocity_only_substep_np(pos, vel, mass, idx, grid, dt, gravity, damping):
    """mpm_substep_velocity_only (ae_particle/src/mpm_solver.rs:1353-1572) restated with numpy float32
    scalars, one IEEE single rounding per operation: serial P2G in index order, the dense grid update
    (Grid::update_parallel :112-139 without forces), G2P of velocity only with the NaN and |v| <= 50
    guards, the mixed wall rules and damping."""
    f = np.float32
    nx, ny, nz = grid.nx, grid.ny, grid.nz
    dx = f(grid.dx)
    inv_dx = f(1.0) / dx
    org = [f(o) for o in grid.origin]
    gmass = np.zeros(nx * ny * nz, np.float32)
    gvel = np.zeros((nx * ny * nz, 3), np.float32)

    def bs(x):
        ax = abs(x)
        if ax < f(0.5):
            return f(0.75) - ax * ax
        if ax < f(1.5):
            t = f(1.5) - ax
            return f(0.5) * t * t
        return f(0.0)

    def stencil(p):
        g, fr = [], []
        for a in range(3):
            q = (p[a] - org[a]) * inv_dx - f(0.5)
            gi = int(np.floor(q))
            fr.append((p[a] - org[a]) * inv_dx - f(0.5) - f(gi))
            g.append(max(gi, 0))
        w = [[bs(f(k) - fr[a]) for k in range(3)] for a in range(3)]
        return g, w

    for i in idx:
        p = pos[i]
        g, w = stencil(p)
        wm = mass[i]
        for dk in range(3):
            if w[2][dk] < f(1e-10) or g[2] + dk >= nz:
                continue
            for dj in range(3):
                if w[1][dj] < f(1e-10) or g[1] + dj >= ny:
                    continue
                wyz = w[1][dj] * w[2][dk]
                for di in range(3):
                    ww = w[0][di] * wyz
                    if ww < f(1e-10) or g[0] + di >= nx:
                        continue
                    gid = (g[0] + di) + (g[1] + dj) * nx + (g[2] + dk) * nx * ny
                    gmass[gid] += ww * wm
                    for a in range(3):
                        gvel[gid, a] += ww * wm * vel[i, a]
    grav = [f(x) for x in gravity]
    for gid in range(nx * ny * nz):
        m = gmass[gid]
        if m > f(1e-12):
            for a in range(3):
                gvel[gid, a] = gvel[gid, a] / m + (grav[a] + f(0.0) / m) * dt
            if (gid % (nx * ny)) // nx == 0:
                gvel[gid, 1] = max(gvel[gid, 1], f(0.0))
                gvel[gid, 0] *= f(0.9)
                gvel[gid, 2] *= f(0.9)
    gmax_x = f(nx - 1) * dx
    gmax_z = f(nz - 1) * dx
    for i in idx:
        p = pos[i].copy()
        g, w = stencil(p)
        nv = [f(0.0)] * 3
        for dk in range(3):
            if w[2][dk] < f(1e-10) or g[2] + dk >= nz:
                continue
            for dj in range(3):
                if w[1][dj] < f(1e-10) or g[1] + dj >= ny:
                    continue
                wyz = w[1][dj] * w[2][dk]
                for di in range(3):
                    ww = w[0][di] * wyz
                    if ww < f(1e-10) or g[0] + di >= nx:
                        continue
                    gid = (g[0] + di) + (g[1] + dj) * nx + (g[2] + dk) * nx * ny
                    if gmass[gid] < f(1e-12):
                        continue
                    nv = [nv[a] + ww * gvel[gid, a] for a in range(3)]
        if not all(np.isfinite(nv)):
            nv = [f(0.0)] * 3
        nv = [min(max(v, f(-50.0)), f(50.0)) for v in nv]
        npos = [p[a] + nv[a] * dt for a in range(3)]
        if not all(np.isfinite(npos)):
            npos, nv = list(p), [f(0.0)] * 3
        if npos[1] < f(0.0):
            npos[1], nv[1] = f(0.0), max(nv[1], f(0.0)) * f(0.5)
        if npos[0] < f(0.0):
            npos[0], nv[0] = f(0.0), max(nv[0], f(0.0)) * f(0.5)
        elif npos[0] > gmax_x + org[0]:
            npos[0], nv[0] = gmax_x + org[0], min(nv[0], f(0.0)) * f(0.5)
        if npos[2] < f(0.0):
            npos[2], nv[2] = f(0.0), max(nv[2], f(0.0)) * f(0.5)
        elif npos[2] > gmax_z + org[2]:
            npos[2], nv[2] = gmax_z + org[2], min(nv[2], f(0.0)) * f(0.5)
        pos[i] = npos
        vel[i] = [v * f(damping) for v in nv]


@pytest.mark.parametrize("origin", [(0.0, 0.0, 0.0), (-0.4, 0.0, -0.4)])
def test_velocity_only_oracle_matches_a_numpy_restatement(origin):
    # the oracle's mpm_step_velocity_only_parallel against an independent float32 restatement of the
    # reference's substep, bit for bit; particles near the walls exercise the mixed wall rules
    rng = np.random.default_rng(3)
    n, grid_n, dx = 400, 8, 0.1
    p = M.Particles.empty(n)
    lo = np.asarray(origin) + 0.05
    p.pos[:] = (lo + rng.random((n, 3)) * (grid_n - 1) * dx).astype(np.float32)
    p.vel[:] = rng.normal(0, 2.0, (n, 3)).astype(np.float32)
    p.mass[:] = rng.uniform(0.5, 2.0, n).astype(np.float32)
    g = M.Grid(grid_n, grid_n, grid_n, dx, origin)
    cfg = M.Config(grid_dx=dx, grid_size=(grid_n,) * 3, substeps=2, gravity=(0, -9.81, 0), damping=0.995)
    idx = np.sort(rng.choice(n, 300, replace=False)).astype(np.uint64)
    a = p.copy()
    assert O.step_velocity_only_parallel(a, g, cfg, 0.02, idx) == 0
    pos, vel = p.pos.copy(), p.vel.copy()
    sub_dt = np.float32(0.02) / np.float32(cfg.substeps)
    for _ in range(cfg.substeps):
        _velocity_only_substep_np(pos, vel, p.mass, idx.astype(np.int64), g, sub_dt, (0, -9.81, 0), 0.995)
    assert np.array_equal(a.pos, pos) and np.array_equal(a.vel, vel)
    untouched = np.setdiff1d(np.arange(n), idx.astype(np.int64))
    assert np.array_equal(a.pos[untouched], p.pos[untouched])


# ---- float32 restatement of the reference's constitutive models (constitutive.rs), one IEEE single
# rounding per operation; sin, cos and ln from the C library as Rust's f32 methods
import ctypes  # noqa: E402

_LIBM = ctypes.CDLL("libm.so.6")
logf, sinf, cosf = _LIBM.logf, _LIBM.sinf, _LIBM.cosf
for _fn in (logf, sinf, cosf):
    _fn.restype, _fn.argtypes = ctypes.c_float, [ctypes.c_float]
f = np.float32


def _lame_np(m):
    nu = min(max(f(m.poisson_ratio), f(-0.999)), f(0.4999))
    e = f(m.young_modulus)
    return e / (f(2.0) * (f(1.0) + nu)), e * nu / ((f(1.0) + nu) * (f(1.0) - f(2.0) * nu)), \
        e / (f(3.0) * (f(1.0) - f(2.0) * nu))


def _mm_np(a, b):
    return [a[r * 3 + 0] * b[0 * 3 + c] + a[r * 3 + 1] * b[1 * 3 + c] + a[r * 3 + 2] * b[2 * 3 + c]
            for r in range(3) for c in range(3)]

def _inv_t_np(q):  # constitutive.rs:306-324 (the adjugate over the determinant: the inverse)
    det = q[0] * (q[4] * q[8] - q[5] * q[7]) - q[1] * (q[3] * q[8] - q[5] * q[6]) + q[2] * (q[3] * q[7] - q[4] * q[6])
    if abs(det) < f(1e-15):
        return [f(1), f(0), f(0), f(0), f(1), f(0), f(0), f(0), f(1)]
    i = f(1.0) / det
    return [(q[4] * q[8] - q[5] * q[7]) * i, -(q[1] * q[8] - q[2] * q[7]) * i, (q[1] * q[5] - q[2] * q[4]) * i,
            -(q[3] * q[8] - q[5] * q[6]) * i, (q[0] * q[8] - q[2] * q[6]) * i, -(q[0] * q[5] - q[2] * q[3]) * i,
            (q[3] * q[7] - q[4] * q[6]) * i, -(q[0] * q[7] - q[1] * q[6]) * i, (q[0] * q[4] - q[1] * q[3]) * i]

def _polar_np(F):  # constitutive.rs:284-304
    r = list(F)
    for _ in range(8):
        ri = _inv_t_np(r)
        nr = [f(0.5) * (r[i] + ri[i]) for i in range(9)]
        diff = f(0.0)
        for i in range(9):
            diff = diff + abs(nr[i] - r[i])
        r = nr
        if diff < f(1e-10):
            break
    rt = [r[0], r[3], r[6], r[1], r[4], r[7], r[2], r[5], r[8]]
    return r, _mm_np(rt, F)

def _deviatoric_np(m, F):  # the shared trial of constitutive.rs:443-600
    mu, la, _ = _lame_np(m)
    _, sm = _polar_np(F)
    eps = [sm[0] - f(1), sm[1], sm[2], sm[3], sm[4] - f(1), sm[5], sm[6], sm[7], sm[8] - f(1)]
    tr = eps[0] + eps[4] + eps[8]
    tr3 = tr / f(3.0)
    for i in (0, 4, 8):
        eps[i] = eps[i] - tr3
    sd = [f(2.0) * mu * e for e in eps]
    sn = np.sqrt(f(0.5) * (sd[0] * sd[0] + sd[4] * sd[4] + sd[8] * sd[8] + f(2.0) * (
        sd[1] * sd[1] + sd[2] * sd[2] + sd[3] * sd[3] + sd[5] * sd[5] + sd[6] * sd[6] + sd[7] * sd[7])))
    return sd, sn, -la * tr

def _ref_stress_np(model, m, F, J):
    mu, la, k = _lame_np(m)
    if model == M.NEWTONIAN_FLUID:
        sd = k * (J - f(1.0))
        return [sd, f(0), f(0), f(0), sd, f(0), f(0), f(0), sd]
    if model == M.RIGID:  # constitutive.rs:370-373
        return [f(1), f(0), f(0), f(0), f(1), f(0), f(0), f(0), f(1)]
    if model in (M.COROTATED, M.FIXED_COROTATED):  # constitutive.rs:395-442
        r, _ = _polar_np(F)
        if model == M.COROTATED:
            out = [f(2.0) * mu * (F[i] - r[i]) for i in range(9)]
            for i in (0, 4, 8):
                out[i] = out[i] + la * (J - f(1.0))
            return out
        rt = [r[0], r[3], r[6], r[1], r[4], r[7], r[2], r[5], r[8]]
        dr = _mm_np([F[i] - r[i] for i in range(9)], rt)
        out = [f(2.0) * mu * dr[i] for i in range(9)]
        for i in (0, 4, 8):
            out[i] = out[i] + la * (J - f(1.0)) * J
        return out
    if model in (M.DRUCKER_PRAGER, M.VON_MISES):
        sd, sn, pressure = _deviatoric_np(m, F)
        if model == M.DRUCKER_PRAGER:
            phi = f(m.friction_angle) * (f(math.pi) / f(180.0))  # f32::to_radians
            sphi, cphi, s3 = f(sinf(phi)), f(cosf(phi)), np.sqrt(f(3.0))
            alpha = (f(2.0) * sphi) / (s3 * (f(3.0) - sphi))
            kk = (f(6.0) * f(m.cohesion) * cphi) / (s3 * (f(3.0) - sphi))
            if sn + alpha * pressure - kk > f(0.0):
                sc = max(kk - alpha * pressure, f(0.0)) / max(sn, f(1e-10))
                sd = [x * sc for x in sd]
        else:
            thr = f(m.yield_stress) / np.sqrt(f(3.0))
            if sn > thr:
                sc = thr / sn
                sd = [x * sc for x in sd]
        for i in (0, 4, 8):
            sd[i] = sd[i] - pressure
        return sd
    b = [F[r * 3 + 0] * F[c * 3 + 0] + F[r * 3 + 1] * F[c * 3 + 1] + F[r * 3 + 2] * F[c * 3 + 2]
         for r in range(3) for c in range(3)]
    p_term = la * f(logf(J)) / J if J > f(0.0) else f(0.0)
    scale = mu / max(J, f(1e-10))
    return [scale * ((b[i] - f(1.0) + p_term / scale) if i % 4 == 0 else b[i]) for i in range(9)]


def _serial_substep_np(p, idx, grid, dt, gravity, damping, mats, models, parallel=False):
    """mpm_substep_serial_active (ae_particle/src/mpm_solver.rs:812-1054) with the neo-Hookean and
    Newtonian-fluid stresses (constitutive.rs:375-393, 603-617) restated with numpy float32 scalars,
    one IEEE single rounding per operation, ln from the C library as Rust's f32::ln."""
    nx, ny, nz = grid.nx, grid.ny, grid.nz
    dx = f(grid.dx)
    inv_dx = f(1.0) / dx
    org = [f(o) for o in grid.origin]
    n_nodes = nx * ny * nz
    gm = np.zeros(n_nodes, np.float32)
    gv = np.zeros((n_nodes, 3), np.float32)
    gf = np.zeros((n_nodes, 3), np.float32)

    def bs(x):
        ax = abs(x)
        if ax < f(0.5):
            return f(0.75) - ax * ax
        if ax < f(1.5):
            t = f(1.5) - ax
            return f(0.5) * t * t
        return f(0.0)

    def dbs(x):
        ax = abs(x)
        if ax < f(0.5):
            return f(-2.0) * x
        if ax < f(1.5):
            return -(f(1.5) - ax) * f(math.copysign(1.0, float(x)))
        return f(0.0)

    def base(x):
        g, fr = [], []
        for a in range(3):
            gi = int(np.floor((x[a] - org[a]) * inv_dx - f(0.5)))
            fr.append((x[a] - org[a]) * inv_dx - f(0.5) - f(gi))
            g.append(max(gi, 0))
        return g, fr

    def stencil(g, fr):
        for dk in range(3):
            for dj in range(3):
                for di in range(3):
                    w = bs(f(di) - fr[0]) * bs(f(dj) - fr[1]) * bs(f(dk) - fr[2])
                    if w < f(1e-10):
                        continue
                    X, Y, Z = g[0] + di, g[1] + dj, g[2] + dk
                    if X >= nx or Y >= ny or Z >= nz:
                        continue
                    dw = [dbs(f(di) - fr[0]) * inv_dx, dbs(f(dj) - fr[1]) * inv_dx, dbs(f(dk) - fr[2]) * inv_dx]
                    d = [(f(X) + f(0.5)) * dx + org[0], (f(Y) + f(0.5)) * dx + org[1], (f(Z) + f(0.5)) * dx + org[2]]
                    yield X + Y * nx + Z * nx * ny, w, dw, d

    for i in idx:
        mi = int(p.mat[i])
        m = mats[mi] if mi < len(mats) else mats[0]
        model = models[mi] if mi < len(models) else M.NEO_HOOKEAN
        sig = _ref_stress_np(model, m, list(p.F[i]), p.J[i])
        vol = p.mass[i] / f(m.density)
        sv = [vol * x for x in sig]
        g, fr = base(p.pos[i])
        c, v, x, mass = p.C[i], p.vel[i], p.pos[i], p.mass[i]
        for gid, w, dw, d in stencil(g, fr):
            dg = [d[a] - x[a] for a in range(3)]
            vv = [v[r] + c[3 * r] * dg[0] + c[3 * r + 1] * dg[1] + c[3 * r + 2] * dg[2] for r in range(3)]
            gm[gid] += w * mass
            for r in range(3):
                gv[gid, r] += w * mass * vv[r]
            for r in range(3):
                gf[gid, r] += sv[3 * r] * dw[0] + sv[3 * r + 1] * dw[1] + sv[3 * r + 2] * dw[2]
    grav = [f(a) for a in gravity]
    for gid in range(n_nodes):
        mm = gm[gid]
        if mm > f(1e-12):
            for r in range(3):
                gv[gid, r] = gv[gid, r] / mm + (grav[r] + gf[gid, r] / mm) * dt
            if (gid % (nx * ny)) // nx == 0:
                gv[gid, 1] = max(gv[gid, 1], f(0.0))
                gv[gid, 0] *= f(0.9)
                gv[gid, 2] *= f(0.9)
    gmax_x, gmax_z = f(nx - 1) * dx, f(nz - 1) * dx
    for i in idx:
        x = list(p.pos[i])
        g, fr = base(x)
        nv, nc, gr = [f(0)] * 3, [f(0)] * 9, [f(0)] * 9
        for gid, w, dw, d in stencil(g, fr):
            if gm[gid] < f(1e-12):
                continue
            u = gv[gid]
            dg = [d[a] - x[a] for a in range(3)]
            nv = [nv[r] + w * u[r] for r in range(3)]
            sc = f(4.0) * inv_dx * inv_dx * w
            nc = [nc[3 * r + a] + sc * u[r] * dg[a] for r in range(3) for a in range(3)]
            gr = [gr[3 * r + a] - w * u[r] * dw[a] for r in range(3) for a in range(3)]
        if not all(np.isfinite(nv)):
            nv, nc = [f(0)] * 3, [f(0)] * 9
        nv = [min(max(a, f(-50.0)), f(50.0)) for a in nv]
        npos = [x[a] + nv[a] * dt for a in range(3)]
        if not all(np.isfinite(npos)):
            npos, nv = [f(6.0), f(5.0), f(6.0)], [f(0)] * 3
        if npos[1] < f(0.0):
            npos[1], nv[1] = f(0.0), max(nv[1], f(0.0)) * f(0.5)
        # the serial path's x/z walls are [0, (n-1) dx]; the parallel path's (mpm_solver.rs:1282-1287)
        # are offset by the grid origin
        x_lo, z_lo = (org[0], org[2]) if parallel else (f(0.0), f(0.0))
        x_hi, z_hi = (gmax_x + org[0], gmax_z + org[2]) if parallel else (gmax_x, gmax_z)
        if npos[0] < x_lo:
            npos[0], nv[0] = x_lo, max(nv[0], f(0.0)) * f(0.5)
        elif npos[0] > x_hi:
            npos[0], nv[0] = x_hi, min(nv[0], f(0.0)) * f(0.5)
        if npos[2] < z_lo:
            npos[2], nv[2] = z_lo, max(nv[2], f(0.0)) * f(0.5)
        elif npos[2] > z_hi:
            npos[2], nv[2] = z_hi, min(nv[2], f(0.0)) * f(0.5)
        F = p.F[i]
        nf = []
        for r in range(3):
            for c2 in range(3):
                acc = f(0.0)
                for k in range(3):
                    acc = acc + ((f(1.0) if r == k else f(0.0)) + gr[3 * r + k] * dt) * F[3 * k + c2]
                nf.append(acc)
        if all(np.isfinite(nf)) and all(abs(a) <= f(1e3) for a in nf):
            J = nf[0] * (nf[4] * nf[8] - nf[5] * nf[7]) - nf[1] * (nf[3] * nf[8] - nf[5] * nf[6]) + \
                nf[2] * (nf[3] * nf[7] - nf[4] * nf[6])
            fin, jn = nf, min(max(J, f(0.1)), f(10.0))
        else:
            fin, jn = [f(1), f(0), f(0), f(0), f(1), f(0), f(0), f(0), f(1)], f(1.0)
        p.vel[i] = [a * f(damping) for a in nv]
        p.C[i] = nc
        p.pos[i] = npos
        p.F[i] = fin
        p.J[i] = jn


ENGINE_TABLE = (  # ae_engine/src/managers/simulation.rs:251-294
    dict(young_modulus=1.0e6, poisson_ratio=0.3, yield_stress=1.0e4, hardening=0.01, density=1000.0,
         friction_angle=35.0, cohesion=0.0),
    dict(young_modulus=2.0e6, poisson_ratio=0.45, yield_stress=0.0, hardening=0.0, density=1000.0,
         friction_angle=0.0, cohesion=0.0),
    dict(young_modulus=5.0e7, poisson_ratio=0.3, yield_stress=0.0, hardening=0.0, density=1600.0,
         friction_angle=35.0, cohesion=0.0),
    dict(young_modulus=2.0e11, poisson_ratio=0.3, yield_stress=2.5e8, hardening=0.01, density=7850.0,
         friction_angle=0.0, cohesion=0.0))


def test_reference_parallel_path_oracle_matches_a_numpy_restatement():
    # 50 000 indices take the parallel path (mpm_solver.rs:1077): one fold adds into an empty grid
    # exactly, so the serial summation order stands, and the x/z walls follow the grid origin
    rng = np.random.default_rng(12)
    n, grid_n, dx = 50000, 16, 0.1
    origin = (-1.2, 0.0, -1.2)
    p = M.Particles.empty(n)
    p.pos[:] = (np.asarray(origin) + 0.15 + rng.random((n, 3)) * 1.3).astype(np.float32)
    p.vel[:] = rng.normal(0, 0.5, (n, 3)).astype(np.float32)
    p.pos[:300, 0], p.vel[:300, 0] = np.float32(origin[0] + 0.001), -3.0  # into the x wall at the origin
    p.pos[300:600, 2], p.vel[300:600, 2] = np.float32(origin[2] + 1.499), 3.0  # into the upper z wall
    p.F[:] = (np.eye(3).reshape(9) + rng.normal(0, 0.01, (n, 9))).astype(np.float32)
    p.J[:] = np.linalg.det(p.F.reshape(-1, 3, 3).astype(np.float64)).astype(np.float32)
    p.mass[:] = np.float32(1e-4)
    p.mat[:] = rng.integers(0, 2, n).astype(np.uint16)
    mats = [M.material(young_modulus=1e4, poisson_ratio=0.25, density=1000.0),
            M.material(young_modulus=2e4, poisson_ratio=0.45, density=1000.0)]
    models = [M.NEO_HOOKEAN, M.NEWTONIAN_FLUID]
    g = M.Grid(grid_n, grid_n, grid_n, dx, origin)
    cfg = M.Config(grid_dx=dx, grid_size=(grid_n,) * 3, substeps=1, gravity=(0, -9.81, 0), damping=0.995)
    idx = np.arange(n, dtype=np.uint64)
    a = p.copy()
    assert O.step_parallel_with_grid(a, g, cfg, mats, models, 0.002, idx, threads=1) == 0
    b = p.copy()
    _serial_substep_np(b, idx.astype(np.int64), g, np.float32(0.002), (0, -9.81, 0), 0.995, mats, models,
                       parallel=True)
    for fld in ("pos", "vel", "F", "J", "C"):
        assert np.array_equal(getattr(a, fld), getattr(b, fld)), fld
    assert (a.pos[:300, 0] == np.float32(origin[0])).sum() > 0
    assert (a.pos[300:600, 2] == np.float32(15 * dx) + np.float32(origin[2])).sum() > 0


@pytest.mark.parametrize("model,params", [
    (M.NEO_HOOKEAN, ENGINE_TABLE[0]), (M.NEWTONIAN_FLUID, ENGINE_TABLE[1]), (M.DRUCKER_PRAGER, ENGINE_TABLE[2]),
    (M.DRUCKER_PRAGER, dict(ENGINE_TABLE[2], cohesion=1e5)), (M.VON_MISES, ENGINE_TABLE[3]),
    (M.VON_MISES, dict(ENGINE_TABLE[0], yield_stress=2e3)), (M.COROTATED, ENGINE_TABLE[0]),
    (M.FIXED_COROTATED, ENGINE_TABLE[2]), (M.RIGID, ENGINE_TABLE[3])])
def test_constitutive_oracle_matches_a_numpy_restatement(model, params):
    # compute_stress of the oracle against the float32 restatement of constitutive.rs, bit for bit,
    # on deformed F that put about half of the plastic models' samples past their yield surface
    rng = np.random.default_rng(1)
    m = M.material(**params)
    for _ in range(200):
        F = (np.eye(3).reshape(9) + rng.normal(0, 0.03, 9)).astype(np.float32)
        J = np.float32(np.linalg.det(F.reshape(3, 3).astype(np.float64)))
        r = O.compute_stress(model, m, F, float(J))
        a = np.asarray(r[0] if isinstance(r, tuple) else r, np.float32)
        assert np.array_equal(a, np.asarray(_ref_stress_np(model, m, list(F), J), np.float32))


@pytest.mark.parametrize("table", ["neo_fluid", "engine", "all_models"])
def test_reference_serial_oracle_matches_a_numpy_restatement(table):
    # the oracle's drop-in substep (below 50 000 indices: mpm_substep_serial_active) against an
    # independent float32 restatement, bit for bit: the neo-Hookean and fluid models, or the engine's
    # own 4-material table (NeoHookean, NewtonianFluid, DruckerPrager, VonMises); a material index past
    # the tables (material_table[0] with NeoHookean), deformed F and a nonzero C
    rng = np.random.default_rng(9)
    n, grid_n, dx = 300, 12, 0.05
    p = M.Particles.empty(n)
    p.pos[:] = (0.08 + rng.random((n, 3)) * 0.44).astype(np.float32)
    p.vel[:] = rng.normal(0, 0.5, (n, 3)).astype(np.float32)
    p.F[:] = (np.eye(3).reshape(9) + rng.normal(0, 0.03, (n, 9))).astype(np.float32)
    p.J[:] = np.linalg.det(p.F.reshape(-1, 3, 3).astype(np.float64)).astype(np.float32)
    p.C[:] = rng.normal(0, 0.5, (n, 9)).astype(np.float32)
    p.mass[:] = rng.uniform(0.5e-3, 2e-3, n).astype(np.float32)
    p.mat[:] = rng.integers(0, 3, n).astype(np.uint16)
    p.pos[:20, 0], p.vel[:20, 0] = 0.001, -3.0  # into the x = 0 wall
    p.pos[20:40, 1], p.vel[20:40, 1] = 0.001, -3.0  # into the floor
    if table == "engine":
        mats = [M.material(**kw) for kw in ENGINE_TABLE]
        models = [M.NEO_HOOKEAN, M.NEWTONIAN_FLUID, M.DRUCKER_PRAGER, M.VON_MISES]
        p.mat[:] = rng.integers(0, 5, n).astype(np.uint16)
    elif table == "all_models":  # the seven ConstitutiveModel variants, softer materials
        models = [M.NEO_HOOKEAN, M.DRUCKER_PRAGER, M.VON_MISES, M.NEWTONIAN_FLUID, M.COROTATED,
                  M.FIXED_COROTATED, M.RIGID]
        mats = [M.material(young_modulus=1e4 * (k + 1), poisson_ratio=0.3, yield_stress=50.0, density=1000.0,
                           friction_angle=30.0, cohesion=10.0) for k in range(7)]
        p.mat[:] = rng.integers(0, 8, n).astype(np.uint16)
    else:
        mats = [M.material(young_modulus=1e4, poisson_ratio=0.25, density=1000.0),
                M.material(young_modulus=2e4, poisson_ratio=0.45, density=1000.0)]
        models = [M.NEO_HOOKEAN, M.NEWTONIAN_FLUID]
    g = M.Grid(grid_n, grid_n, grid_n, dx, (0.0, 0.0, 0.0))
    cfg = M.Config(grid_dx=dx, grid_size=(grid_n,) * 3, substeps=2, gravity=(0, -9.81, 0), damping=0.995)
    idx = np.sort(rng.choice(n, 240, replace=False)).astype(np.uint64)
    a = p.copy()
    assert O.step_parallel_with_grid(a, g, cfg, mats, models, 0.004, idx) == 0
    b = p.copy()
    sub_dt = np.float32(0.004) / np.float32(cfg.substeps)
    for _ in range(cfg.substeps):
        _serial_substep_np(b, idx.astype(np.int64), g, sub_dt, (0, -9.81, 0), 0.995, mats, models)
    for fld in ("pos", "vel", "F", "J", "C"):
        assert np.array_equal(getattr(a, fld), getattr(b, fld)), fld
    assert not np.array_equal(a.pos, p.pos) and not np.array_equal(a.F, p.F)
    sel = idx.astype(np.int64)
    assert (a.pos[sel, 0] == 0).sum() > 0 and (a.pos[sel, 1] == 0).sum() > 0  # the wall rules ran


def test_svd3_reflection_gives_negative_last_singular_value():
    F = np.diag([1.1, 0.9, -1.0])
    U, s, V, _ = O.svd3(F, f64=True)
    assert s[2] < 0 and np.abs(U @ np.diag(s) @ V.T - F).max() < 1e-12


# ---------------------------------------------------------------- reference-mode property tests
def _ref_buffer(positions, mass, material=0, J=1.0):
    p = M.Particles.empty(len(positions))
    p.pos[:] = np.asarray(positions, np.float32)
    p.mass[:] = mass
    p.mat[:] = material
    p.J[:] = J
    return p


def test_oracle_sandpile_static_angle():  # mpm_solver.rs:1611-1657
    pos = [(x * 0.05, y * 0.05 + 0.5, z * 0.05) for x in range(10) for y in range(10) for z in range(10)]
    p = _ref_buffer(pos, 0.001)
    cfg = M.Config(grid_dx=1.6, grid_size=(16, 16, 16), substeps=8, gravity=(0, -9.81, 0), damping=0.995)
    g = M.Grid(16, 16, 16, 1.6, (0, 0, 0))
    mats = [M.material(young_modulus=1e4, poisson_ratio=0.2, yield_stress=1e3, hardening=0.005, density=1600,
                       friction_angle=35.0, cohesion=0.0)]
    idx = np.arange(p.n, dtype=np.uint64)
    for _ in range(60):
        assert O.step_parallel_with_grid(p, g, cfg, mats, [M.DRUCKER_PRAGER], 0.016, idx) == 0
    assert (p.pos[:, 1] >= 0).all()


def test_oracle_water_pressure():  # mpm_solver.rs:1659-1711
    pos = [(x * 0.05, y * 0.05 + 0.1, z * 0.05) for y in range(10) for x in range(5) for z in range(5)]
    p = _ref_buffer(pos, 0.001, J=0.95)
    cfg = M.Config(grid_dx=0.05, grid_size=(32, 32, 32), substeps=8, gravity=(0, -9.81, 0), damping=0.995)
    g = M.Grid(32, 32, 32, 0.05, (0, 0, 0))
    mats = [M.material(young_modulus=1e3, poisson_ratio=0.499, yield_stress=0, hardening=0, density=1000,
                       friction_angle=0, cohesion=0)]
    assert O.step_parallel_with_grid(p, g, cfg, mats, [M.NEWTONIAN_FLUID], 0.016, np.arange(p.n)) == 0
    assert np.isfinite(p.J).all() and (p.J > 0).all() and (p.J < 100).all()


def test_oracle_steel_rigid_fall():  # mpm_solver.rs:1713-1745
    p = _ref_buffer([(0.2, 0.5, 0.2)], 0.01)
    cfg = M.Config(grid_dx=0.02, grid_size=(32, 32, 32), substeps=8, gravity=(0, -9.81, 0), damping=0.995)
    g = M.Grid(32, 32, 32, 0.02, (0, 0, 0))
    mats = [M.material(young_modulus=1e5, poisson_ratio=0.3, yield_stress=1e4, hardening=0.01, density=7850,
                       friction_angle=0, cohesion=0)]
    for _ in range(30):
        assert O.step_parallel_with_grid(p, g, cfg, mats, [M.VON_MISES], 0.016, [0]) == 0
    assert 0.0 <= p.pos[0, 1] < 0.5


def test_oracle_grid_export_is_the_reference_grid_after_the_call():
    # Grid the reference leaves behind after mpm_step_parallel_with_grid (mpm_solver.rs:73-176):
    # one stress-free particle (F = I) at a known position, one substep.  P2G puts m*N(fx)N(fy)N(fz)
    # on nodes g..g+2 per axis with g = floor((x-o)/dx - 0.5) (:161-175, :863-875); the update turns
    # momentum into v + g*dt on nodes above the 1e-12 mass threshold (:112-139).  Everything else is 0.
    x = np.array([0.537, 0.611, 0.449])
    p = _ref_buffer([tuple(x)], 2.0)
    p.vel[0] = (0.3, -0.2, 0.1)
    n, dx, o = 16, 0.0625, np.array([-0.1, 0.0, -0.05], np.float32)
    cfg = M.Config(grid_dx=dx, grid_size=(n, n, n), substeps=1, gravity=(0, -9.81, 0), damping=0.995)
    g = M.Grid(n, n, n, dx, tuple(o))
    dt = 0.004
    gm, gv = O.step_parallel_with_grid_grid(p, g, cfg, [M.material(young_modulus=1e4, density=1000)],
                                            [M.NEO_HOOKEAN], dt, [0])
    q = (x - o.astype(np.float64)) / dx - 0.5
    base = np.floor(q).astype(int)
    fx = q - base
    want = np.zeros(n ** 3)
    for di in range(3):
        for dj in range(3):
            for dk in range(3):
                w = np.prod([O.b_spline(float(fx[a] - d)) for a, d in zip(range(3), (di, dj, dk))])
                i, j, k = base + (di, dj, dk)
                want[i + j * n + k * n * n] += 2.0 * w
    assert np.allclose(gm, want, rtol=1e-5, atol=1e-7)
    live = gm > 1e-12
    assert live.sum() >= 8 and np.all(gm[~live] == 0) and np.all(gv[~live] == 0)
    v = np.array([0.3, -0.2 - 9.81 * dt, 0.1])
    assert np.allclose(gv[live], v, rtol=0, atol=1e-5)


def test_oracle_parallel_path_matches_serial_fold_order():
    # thread-local grids merged in order (rayon fold/reduce shape) agree with the serial path
    rng = np.random.default_rng(3)
    p = _ref_buffer(rng.random((4000, 3)) * 0.6 + 0.2, 0.001)
    p.vel[:] = rng.normal(0, 0.2, (4000, 3))
    sc = M.Scene(n=(32, 32, 32), dx=1.0 / 32, dt=1e-3, materials=[M.material(young_modulus=1e4, density=1000)],
                 mode=M.MODE_REFERENCE, wall_origin=1)
    a, b = p.copy(), p.copy()
    O.run(sc, a, 5, threads=1)
    O.run(sc, b, 5, threads=4)
    assert np.abs(a.pos - b.pos).max() <= 1e-6


# ---------------------------------------------------------------- physics-mode property tests
def test_physics_mass_conserved_and_falls():  # mpm_compute.rs:1223-1274
    sc, p = S.tiny_scene(1000, 32, S.jelly())
    sc.wall_mode = M.WALL_SLIP
    m0 = O.totals(p)[0]
    y0 = p.pos[:, 1].mean()
    q = p.copy()
    O.run(sc, q, 10)
    assert abs(O.totals(q)[0] - m0) < 1e-5 * max(m0, 1)
    assert q.pos[:, 1].mean() < y0


def test_physics_floor_not_penetrated():  # mpm_compute.rs:1276-1301
    sc, p = S.tiny_scene(64, 32, S.jelly(), box=(0.45, 0.55))
    sc.wall_mode = M.WALL_SLIP
    sc.gravity = (0.0, -20.0, 0.0)
    sc.dt = 1e-3
    O.run(sc, p, 200)
    assert (p.pos[:, 1] >= 0).all() and p.pos[:, 1].max() < 0.5


def test_physics_compressed_block_expands():
    # force sign: a compressed elastic block pushes outward (the reference's ae_compute force is
    # sign-flipped, mpm_compute.rs:328-335; physics mode uses the physically correct sign)
    sc, p = S.tiny_scene(4096, 32, S.jelly(E=1e3), box=(0.4, 0.6))
    sc.gravity = (0.0, 0.0, 0.0)
    p.F[:, [0, 4, 8]] = 0.95
    c0 = p.pos.mean(0)
    spread0 = np.abs(p.pos - c0).mean()
    O.run(sc, p, 30)
    assert np.abs(p.pos - p.pos.mean(0)).mean() > spread0


def test_physics_momentum_conserved_without_gravity():
    # conservation_test.rs:209 style: free-flight momentum of a colliding pair is conserved
    sc, p = S.tiny_scene(2048, 32, S.jelly(E=500.0))
    sc.gravity = (0.0, 0.0, 0.0)
    half = p.n // 2
    p.vel[:half] = (0.5, 0.0, 0.0)
    p.vel[half:] = (-0.5, 0.0, 0.0)
    t0 = O.totals(p)
    O.run(sc, p, 50)
    t1 = O.totals(p)
    assert abs(t1[1] - t0[1]) < 1e-6 and abs(t1[3] - t0[3]) < 1e-6


def test_physics_fp32_oracle_tracks_fp64():
    sc, p = S.config1_jelly()
    sub = p.subset(np.arange(0, p.n, 8))
    a = sub.copy()
    b = sub.astype(np.float64)
    O.run(sc, a, 40)
    O.run(sc, b, 40)
    assert np.abs(a.pos - b.pos).max() / np.abs(b.pos).max() < 1e-6


def test_physics_snow_clamps_singular_values():
    sc, p = S.tiny_scene(2048, 32, S.snow())
    p.F[:, [0, 4, 8]] = (1.1, 0.9, 1.0)  # beyond theta_s / theta_c
    O.run(sc, p, 1)
    for k in range(0, p.n, 97):
        s = np.linalg.svd(p.F[k].reshape(3, 3).astype(np.float64))[1]
        assert s.max() <= 1 + 7.5e-3 + 1e-4 and s.min() >= 1 - 2.5e-2 - 1e-4
    assert (p.J != 1.0).all()  # plastic J_p absorbed the clamped part


def _physics_substep_np(p, sc):
    """One physics-mode (MLS-MPM) substep in float64, vectorised over particles, restated from the
    formulas rather than from the oracle's loops: quadratic B-spline stencil based at floor(X - 1/2);
    A = m C - (4 dt V0 / dx^2) tau with the neo-Hookean Kirchhoff stress mu (F F^T - I) + lambda ln(Jc) I
    (ae_physics/src/mpm.rs:443-452) or the fluid's K (J - 1) I; grid v = p / m + dt g with sticky walls
    in the margin; G2P v, C = 4 / dx^2 sum w v (x) d, advect and keep the stencil inside the grid;
    F <- (I + dt C) F and J = det F, or J <- J (1 + dt tr C) for the fluid (mpm_compute.rs:244-459)."""
    f32 = np.float32
    n = np.array(sc.n)
    # the scene descriptor carries dx, dt, origin and gravity as float32
    dx, dt = float(f32(sc.dx)), float(f32(sc.dt))
    org = np.array(sc.origin, np.float32).astype(np.float64)
    g = np.array(sc.gravity, np.float32).astype(np.float64)
    inv_dx = 1.0 / dx
    x, v, C, F, J, m = p.pos, p.vel, p.C.reshape(-1, 3, 3), p.F.reshape(-1, 3, 3), p.J, p.mass
    mat = p.mat.astype(np.int64)
    nm = len(sc.materials)
    mu = np.zeros(nm)
    la = np.zeros(nm)
    bulk = np.zeros(nm)
    rho = np.zeros(nm)
    fluid = np.zeros(nm, bool)
    snow = np.zeros(nm, bool)
    xi = np.zeros(nm)
    band = np.zeros((nm, 2))
    for k, mt in enumerate(sc.materials):
        snow[k] = mt.model == M.PHYS_SNOW
        xi[k] = f32(mt.hardening_xi)
        band[k] = (1.0 - float(f32(mt.theta_c)), 1.0 + float(f32(mt.theta_s)))
        nu = min(max(f32(mt.poisson_ratio), f32(-0.999)), f32(0.4999))
        e = f32(mt.young_modulus)
        mu[k] = e / (f32(2.0) * (f32(1.0) + nu))
        la[k] = e * nu / ((f32(1.0) + nu) * (f32(1.0) - f32(2.0) * nu))
        bulk[k] = f32(mt.bulk_modulus) if mt.bulk_modulus > 0 else e / (f32(3.0) * (f32(1.0) - f32(2.0) * nu))
        rho[k] = f32(mt.density)
        fluid[k] = mt.model == M.PHYS_FLUID
    mat = np.where(mat < nm, mat, 0)
    isf = fluid[mat]
    iss = snow[mat]
    # stress (snow: Stomakhin hardening exp(xi (1 - J_p)), capped to [0.1, 5], on both Lame parameters)
    h = np.where(iss, np.clip(np.exp(xi[mat] * (1.0 - J)), 0.1, 5.0), 1.0)
    detF = np.linalg.det(F)
    lnJ = np.log(np.clip(detF, 0.01, 100.0))
    tau = (h * mu[mat])[:, None, None] * (F @ np.transpose(F, (0, 2, 1)) - np.eye(3)) + \
        (h * la[mat] * lnJ)[:, None, None] * np.eye(3)
    tau[isf] = (bulk[mat][isf] * (J[isf] - 1.0))[:, None, None] * np.eye(3)
    kst = 4.0 * dt * (m / rho[mat]) * inv_dx * inv_dx
    A = m[:, None, None] * C - kst[:, None, None] * tau
    # stencil
    X = (x - org) * inv_dx
    base = np.floor(X - 0.5).astype(np.int64)
    fx = X - base
    w = np.stack([0.5 * (1.5 - fx) ** 2, 0.75 - (fx - 1.0) ** 2, 0.5 * (fx - 0.5) ** 2], -1)  # (N, axis, k)
    d = (np.arange(3)[None, None, :] - fx[:, :, None]) * dx
    offs = np.array([(a, b, c) for c in range(3) for b in range(3) for a in range(3)])
    node = base[:, None, :] + offs[None, :, :]  # (N, 27, 3)
    inside = np.all((node >= 0) & (node < n), axis=2)
    ww = w[:, 0, offs[:, 0]] * w[:, 1, offs[:, 1]] * w[:, 2, offs[:, 2]]
    dd = np.stack([d[:, 0, offs[:, 0]], d[:, 1, offs[:, 1]], d[:, 2, offs[:, 2]]], -1)  # (N, 27, 3)
    gid = node[..., 0] + n[0] * (node[..., 1] + n[1] * node[..., 2])
    mom = ww[..., None] * (m[:, None, None] * v[:, None, :] + np.einsum("nrk,njk->njr", A, dd))
    gm = np.zeros(int(np.prod(n)))
    gp = np.zeros((int(np.prod(n)), 3))
    np.add.at(gm, gid[inside], (ww * m[:, None])[inside])
    np.add.at(gp, gid[inside], mom[inside])
    # grid
    live = gm > 0
    gv = np.zeros_like(gp)
    gv[live] = gp[live] / gm[live][:, None] + dt * g
    ijk = np.stack([np.arange(gm.size) % n[0], (np.arange(gm.size) // n[0]) % n[1], np.arange(gm.size) // (n[0] * n[1])], 1)
    mg = sc.wall_margin
    wall = np.any((ijk < mg) | (ijk >= n - mg), axis=1)
    gv[wall] = 0.0
    # G2P
    vg = np.where(inside[..., None], gv[np.where(inside, gid, 0)], 0.0)
    nv = np.einsum("nj,njr->nr", ww, vg)
    B = np.einsum("nj,njr,njk->nrk", ww, vg, dd)
    Cn = 4.0 * inv_dx * inv_dx * B
    xn = np.clip(x + dt * nv, org + dx, org + (n - 2) * dx)
    Fn = (np.eye(3) + dt * Cn) @ F
    Jn = np.where(isf, np.maximum(J * (1.0 + dt * np.trace(Cn, axis1=1, axis2=2)), 0.01), np.linalg.det(Fn))
    # snow: singular values clamped to [1 - theta_c, 1 + theta_s], J_p scaled by prod(s) / prod(s_clamped)
    # (ae_physics/src/mpm.rs:565-606 with Stomakhin's J_p); F inside the band is left as it is
    if iss.any():
        U, sg, Vt = np.linalg.svd(Fn[iss])
        lo, hi = band[mat][iss, 0], band[mat][iss, 1]
        inband = np.all((sg > lo[:, None]) & (sg < hi[:, None]), axis=1) & (np.linalg.det(Fn[iss]) > 0)
        sc_ = np.clip(sg, lo[:, None], hi[:, None])
        Fc = U @ (sc_[:, :, None] * Vt)
        Jp = J[iss] * (np.prod(sg, axis=1) / np.prod(sc_, axis=1))
        Fs = np.where(inband[:, None, None], Fn[iss], Fc)
        Fn[iss] = Fs
        Jn[iss] = np.where(inband, J[iss], Jp)
    p.pos[:] = xn
    p.vel[:] = nv
    p.C[:] = Cn.reshape(-1, 9)
    p.F[:] = np.where(isf[:, None, None], F, Fn).reshape(-1, 9)
    p.J[:] = Jn


def test_physics_oracle_matches_a_vectorised_restatement():
    # jelly and water in one f64 scene, against the formulas restated independently; only the
    # summation order differs (measured: 2e-16 to 2e-14 relative after 12 substeps)
    sc, p = S.tiny_scene(2048, 16, S.jelly(E=2e4), v=(0.8, -0.4, 0.3))
    sc.materials = [S.jelly(E=2e4), S.water()]
    p.mat[1::2] = 1
    rng = np.random.default_rng(4)
    p.F[:] = (np.eye(3).reshape(9) + rng.normal(0, 0.02, (p.n, 9))).astype(np.float32)
    ref = p.astype(np.float64)
    mine = p.astype(np.float64)
    O.run(sc, ref, 12)
    for _ in range(12):
        _physics_substep_np(mine, sc)
    scale = lambda a: float(np.abs(a).max())
    assert np.abs(mine.pos - ref.pos).max() <= 1e-14 * scale(ref.pos)
    assert np.abs(mine.vel - ref.vel).max() <= 1e-13 * scale(ref.vel)
    assert np.abs(mine.F - ref.F).max() <= 1e-13 * scale(ref.F)
    assert np.abs(mine.J - ref.J).max() <= 1e-13 * scale(ref.J)
    assert np.abs(mine.C - ref.C).max() <= 1e-12 * scale(ref.C)
    assert not np.allclose(ref.pos, p.pos)


def test_physics_snow_oracle_matches_a_vectorised_restatement():
    # the colliding snow boxes in f64, 40 % of the particles on the yield surface by the end: the
    # restatement's LAPACK SVD and the oracle's Jacobi SVD give the same return mapping to roundoff
    # (measured: F 5.5e-14, J_p 1.3e-14 relative after 40 substeps)
    sc, p = S.snow_collision_small(n_box=1024)
    ref = p.astype(np.float64)
    mine = p.astype(np.float64)
    O.run(sc, ref, 40)
    for _ in range(40):
        _physics_substep_np(mine, sc)
    s = np.linalg.svd(ref.F.reshape(-1, 3, 3), compute_uv=False)
    assert ((np.abs(s - (1 - 2.5e-2)) < 1e-9) | (np.abs(s - (1 + 7.5e-3)) < 1e-9)).any(1).mean() > 0.3
    scale = lambda a: float(np.abs(a).max())
    assert np.abs(mine.pos - ref.pos).max() <= 1e-14 * scale(ref.pos)
    assert np.abs(mine.F - ref.F).max() <= 1e-12 * scale(ref.F)
    assert np.abs(mine.J - ref.J).max() <= 1e-12 * scale(ref.J)


def test_physics_threads_agree():
    sc, p = S.tiny_scene(4096, 32, S.water(), v=(1, 0, 0))
    a, b = p.copy(), p.copy()
    O.run(sc, a, 10, threads=1)
    O.run(sc, b, 10, threads=3)
    assert np.abs(a.pos - b.pos).max() <= 1e-6
