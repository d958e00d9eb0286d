"""GPU parity of the drop-in at the settings of the engine's own call.

SimulationManager::update_fields_and_particles calls mpm_step_parallel_with_grid every tick on the
near set (ae_engine/src/managers/simulation.rs:570-583): the 10 000 nearest particles of the whole
MpssBuffer, a 64^3 grid at dx 1.6 m whose origin follows the player (:541-549), one substep of
dt = 1/60 s, and the engine's 4-entry material table with its model table (:251-294): rubber-like
neo-Hookean, Newtonian fluid, Drucker-Prager sand and 2e11 Pa von Mises steel.  Here the 1 000 055-
particle buffer of the engine-call benchmark (bench.near_setup) goes through the C ABI and through
the oracle, call by call, and the Grid the call leaves behind is read back with
ae_mpm_grid_download (the reference's Grid::mass / Grid::vel, mpm_solver.rs:73-86).

At these settings the reference is ill-conditioned after its first call: the steel's stress on a
deformed F drives most particles into the |v| <= 50 clamp and the J clamp, and one ulp of input
position moves single-call outputs by up to 5 cm (the oracle against itself).  So:
  * call 1 (from the buffer's rest state F = I, as on the engine's first tick) is held to the
    drop-in tolerances of the other parity tests: positions 2e-5 of the largest |x|, F and J 1e-4,
    and the grid's mass and velocity to 1e-5 / 1e-4 of their largest values;
  * calls 2-4 start from the oracle's own state after the previous call (so differences cannot
    accumulate) and are held to the oracle's rounding envelope at that state: the oracle run again
    with every selected input position moved by one ulp.  The device's per-particle differences
    must stay within 10x that envelope at the 50th, 90th and 99th percentiles (plus a floor of
    1e-6 of the field's scale), and the grid likewise; grid velocities, which span 15 decades at
    these settings, are also held per node to 1e-4 relative at the 99th percentile.
The position update x + v dt is rounded as Rust rounds it (product, then sum): an earlier wall
clamp leaves particles at exactly 50 dt above the floor, and a fused multiply-add there turns
the reference's 0 into -4e-9, takes the floor branch and zeroes the velocity that the reference
keeps (found by this test at call 3).
Unselected particles must come back bit-unchanged after every call.
"""
import numpy as np
import pytest

import bench as B
import oracle as O

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0
FIELDS = ("pos", "vel", "F", "J")


def _diff(a, b, f, ii):
    A = getattr(a, f)[ii].astype(np.float64).reshape(len(ii), -1)
    Bv = getattr(b, f)[ii].astype(np.float64).reshape(len(ii), -1)
    return np.abs(A - Bv).max(1), float(np.abs(Bv).max())


def _rel(a, b, floor=1e-12):
    return float(np.abs(np.asarray(a, np.float64) - b).max() / max(float(np.abs(b).max()), floor))


def _within_envelope(dev, env, scale, name):
    floor = 1e-6 * scale
    for q in (50, 90, 99):
        got, lim = np.percentile(dev, q), 10.0 * np.percentile(env, q) + floor
        print("%s p%d: device %.3g, limit %.3g" % (name, q, got, lim))
        assert got <= lim, "%s p%d: device %.3g > 10 x envelope + floor %.3g" % (name, q, got, lim)


def test_engine_near_call_and_grid_readback_match_oracle_call_by_call(ctx):
    p, idx, grid, cfg, mats, models = B.near_setup(0xAE07)
    ii = idx.astype(np.int64)
    rest = np.setdiff1d(np.arange(p.n), ii)
    nn = grid.nx * grid.ny * grid.nz
    state = p.copy()
    for call in range(4):
        dev = state.copy()
        ctx.step_parallel_with_grid(dev, grid, cfg, mats, models, DT, idx)
        gm_dev, gv_dev = ctx.grid_download(grid.nx, grid.ny, grid.nz)
        ref = state.copy()
        gm, gv = O.step_parallel_with_grid_grid(ref, grid, cfg, mats, models, DT, idx)
        assert gm.size == nn and gm_dev.size == nn
        for f in ("pos", "vel", "F", "J", "C", "mass", "mat"):
            assert np.array_equal(getattr(dev, f)[rest], getattr(state, f)[rest]), (call, f)
        live = gm > 1e-12
        if call == 0:
            print("call 1: pos %.3g F %.3g J %.3g vel %.3g grid mass %.3g grid vel %.3g" % (
                _rel(dev.pos[ii], ref.pos[ii]), _rel(dev.F[ii], ref.F[ii]), _rel(dev.J[ii], ref.J[ii]),
                _rel(dev.vel[ii], ref.vel[ii]), _rel(gm_dev, gm), _rel(gv_dev[live], gv[live])))
            assert _rel(dev.pos[ii], ref.pos[ii]) <= 2e-5
            assert _rel(dev.F[ii], ref.F[ii]) <= 1e-4
            assert _rel(dev.J[ii], ref.J[ii]) <= 1e-4
            assert _rel(dev.vel[ii], ref.vel[ii]) <= 1e-3
            assert _rel(gm_dev, gm) <= 1e-5
            # velocities of nodes above the reference's mass threshold (below it the reference keeps
            # raw momentum sums, the device zero)
            assert _rel(gv_dev[live], gv[live]) <= 1e-4
            assert np.abs(gm_dev[~live]).max(initial=0.0) <= 1e-12
        else:
            env = state.copy()
            env.pos[ii] = np.nextafter(env.pos[ii], np.float32(np.inf))
            gm_e, gv_e = O.step_parallel_with_grid_grid(env, grid, cfg, mats, models, DT, idx)
            for f in FIELDS:
                d_dev, scale = _diff(dev, ref, f, ii)
                d_env, _ = _diff(env, ref, f, ii)
                _within_envelope(d_dev, d_env, scale, "call %d %s" % (call + 1, f))
            _within_envelope(np.abs(gm_dev - gm.astype(np.float64)), np.abs(gm_e - gm.astype(np.float64)),
                             float(np.abs(gm).max()), "call %d grid mass" % (call + 1))
            both = live & (gm_e > 1e-12) & (gm_dev > 1e-12)
            _within_envelope(np.abs(gv_dev[both] - gv[both].astype(np.float64)).max(1),
                             np.abs(gv_e[both] - gv[both].astype(np.float64)).max(1),
                             float(np.abs(gv[both]).max()), "call %d grid velocity" % (call + 1))
            # grid velocities span 15 decades here, so also per node: the 99th percentile of
            # |v_dev - v_ref| / |v_ref| within 1e-4 (the device's atomic order and folded force)
            rel_node = (np.abs(gv_dev[both] - gv[both].astype(np.float64)).max(1) /
                        np.maximum(np.abs(gv[both].astype(np.float64)).max(1), 1e-30))
            print("call %d grid velocity per-node relative p99 %.3g" % (call + 1, np.percentile(rel_node, 99)))
            assert np.percentile(rel_node, 99) <= 1e-4
        assert np.isfinite(dev.pos[ii]).all()
        state = ref
