"""ctypes binding of the CPU oracle (oracle/mpm_oracle.cpp).  TEST INFRASTRUCTURE ONLY.

Imported by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg to check or time
the CUDA library against a CPU restatement of the reference's MPM substep.  The product path
(ae-engine_b200/) never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "ae-engine_b200"))
import ae_mpm as M  # noqa: E402  (struct definitions shared with the C ABI)

LIB_PATH = os.path.join(HERE, "_build", "libae_mpm_oracle.so")
_lib = None


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("oracle library not built (%s)" % LIB_PATH)
    lib = C.CDLL(LIB_PATH)
    f = C.c_float
    for name in ("oracle_b_spline", "oracle_b_spline_deriv", "oracle_quadratic_weight",
                 "oracle_quadratic_weight_grad"):
        getattr(lib, name).restype = f
        getattr(lib, name).argtypes = [f]
    lib.oracle_material_lame.argtypes = [C.POINTER(M.Material), C.POINTER(f)]
    lib.oracle_compute_stress.restype = C.c_int
    lib.oracle_compute_stress.argtypes = [C.c_int32, C.POINTER(M.Material), C.POINTER(f), f, C.POINTER(f),
                                          C.POINTER(f)]
    lib.oracle_polar_decomp.argtypes = [C.POINTER(f)] * 3
    lib.oracle_svd3_f32.restype = C.c_int
    lib.oracle_svd3_f32.argtypes = [C.POINTER(f)] * 4 + [C.c_int32, f, f]
    lib.oracle_clamp_is_identity_f32.restype = C.c_int
    lib.oracle_clamp_is_identity_f32.argtypes = [C.POINTER(f), f, f]
    d = C.c_double
    lib.oracle_svd3_f64.argtypes = [C.POINTER(d)] * 4
    lib.oracle_phys_tau_f64.argtypes = [C.POINTER(M.Material), C.POINTER(d), d, C.POINTER(d)]
    for name in ("oracle_run_f32", "oracle_run_f64"):
        g = getattr(lib, name)
        g.restype = C.c_int
        g.argtypes = [C.POINTER(M.SceneDesc), C.POINTER(M.ParticlesView), C.c_uint64, C.c_uint32, C.c_int32,
                      C.c_int32, C.POINTER(C.c_uint64)]
    lib.oracle_totals_f32.argtypes = [C.POINTER(M.ParticlesView), C.c_uint64, C.POINTER(d)]
    lib.oracle_totals_f64.argtypes = [C.POINTER(M.ParticlesView), C.c_uint64, C.POINTER(d)]
    lib.oracle_mpm_step_parallel_with_grid.restype = C.c_int
    lib.oracle_mpm_step_parallel_with_grid.argtypes = [
        C.POINTER(M.ParticlesView), C.c_uint64, C.POINTER(M.Grid), C.POINTER(M.Config), C.POINTER(M.Material),
        C.c_uint32, C.POINTER(C.c_int32), C.c_uint32, f, C.POINTER(C.c_uint64), C.c_uint64, C.c_int32]
    lib.oracle_mpm_step_parallel_with_grid_export.restype = C.c_int
    lib.oracle_mpm_step_parallel_with_grid_export.argtypes = [
        C.POINTER(M.ParticlesView), C.c_uint64, C.POINTER(M.Grid), C.POINTER(M.Config), C.POINTER(M.Material),
        C.c_uint32, C.POINTER(C.c_int32), C.c_uint32, f, C.POINTER(C.c_uint64), C.c_uint64, C.c_int32,
        C.c_void_p, C.c_void_p]
    lib.oracle_mpm_step_velocity_only_parallel.restype = C.c_int
    lib.oracle_mpm_step_velocity_only_parallel.argtypes = [
        C.POINTER(M.ParticlesView), C.c_uint64, C.POINTER(M.Grid), C.POINTER(M.Config), f,
        C.POINTER(C.c_uint64), C.c_uint64, C.c_int32]
    V = C.c_void_p
    lib.oracle_lod_classify.argtypes = [V, V, C.c_uint64, V, f, f, C.c_uint64, V, C.POINTER(C.c_uint64), V,
                                        C.POINTER(C.c_uint64), V, C.POINTER(C.c_uint64)]
    lib.oracle_far_field_update.argtypes = [V, V, V, V, C.c_uint64, V, C.c_uint64, f, V, f]
    lib.oracle_coarse_field_update.argtypes = [V, V, V, V, V, C.c_uint64, V, C.c_uint64, f, V, f]
    lib.oracle_ck_step.argtypes = [V, C.c_uint64, C.POINTER(M.CkConfig), C.c_uint32]
    lib.oracle_ck_step_ln.argtypes = [V, C.c_uint64, C.POINTER(M.CkConfig), C.c_uint32, C.c_int]
    lib.oracle_ck_weight.restype = f
    lib.oracle_ck_weight.argtypes = [f, f]
    lib.oracle_ck_weight_grad.restype = f
    lib.oracle_ck_weight_grad.argtypes = [f, f]
    lib.oracle_mpss_housekeeping.restype = C.c_uint32
    lib.oracle_mpss_housekeeping.argtypes = [V, V, V, V, V, V, C.c_uint64, V, V, f, f, C.c_uint32]
    _lib = lib
    return lib


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def run(scene: M.Scene, p: M.Particles, substeps: int, threads: int = 1, svd_fallback: bool = True):
    """Steps `p` in place; returns [svd fallbacks, domain clamps, NaN positions]."""
    lib = load()
    d = scene.desc()
    v = p.view()
    cnt = (C.c_uint64 * 3)()
    fn = lib.oracle_run_f64 if p.dtype == np.float64 else lib.oracle_run_f32
    rc = fn(C.byref(d), C.byref(v), p.n, substeps, threads, 1 if svd_fallback else 0, cnt)
    if rc != 0:
        raise RuntimeError("oracle run failed: %d" % rc)
    return [int(x) for x in cnt]


def totals(p: M.Particles) -> np.ndarray:
    lib = load()
    out = (C.c_double * 5)()
    v = p.view()
    (lib.oracle_totals_f64 if p.dtype == np.float64 else lib.oracle_totals_f32)(C.byref(v), p.n, out)
    return np.array(out[:])


def step_parallel_with_grid(p: M.Particles, grid: M.Grid, config: M.Config, materials, models, total_dt, indices,
                            threads: int = 1) -> int:
    lib = load()
    mats = (M.Material * max(len(materials), 1))(*materials)
    mods = (C.c_int32 * max(len(models), 1))(*models)
    idx = np.ascontiguousarray(np.asarray(indices, np.uint64))
    v = p.view()
    return lib.oracle_mpm_step_parallel_with_grid(C.byref(v), p.n, C.byref(grid), C.byref(config), mats,
                                                  len(materials), mods, len(models), total_dt,
                                                  idx.ctypes.data_as(C.POINTER(C.c_uint64)), idx.size, threads)


def step_parallel_with_grid_grid(p: M.Particles, grid: M.Grid, config: M.Config, materials, models, total_dt, indices,
                                 threads: int = 1):
    """step_parallel_with_grid, returning the Grid the reference leaves behind: (mass (nx*ny*nz,),
    vel (nx*ny*nz, 3)) after the last substep's grid update, dense in i + j*nx + k*nx*ny order."""
    lib = load()
    mats = (M.Material * max(len(materials), 1))(*materials)
    mods = (C.c_int32 * max(len(models), 1))(*models)
    idx = np.ascontiguousarray(np.asarray(indices, np.uint64))
    nn = int(grid.nx * grid.ny * grid.nz)
    gm = np.zeros(nn, np.float32)
    gv = np.zeros((nn, 3), np.float32)
    v = p.view()
    rc = lib.oracle_mpm_step_parallel_with_grid_export(C.byref(v), p.n, C.byref(grid), C.byref(config), mats,
                                                       len(materials), mods, len(models), total_dt,
                                                       idx.ctypes.data_as(C.POINTER(C.c_uint64)), idx.size, threads,
                                                       gm.ctypes.data, gv.ctypes.data)
    if rc != 0:
        raise RuntimeError("oracle step failed: %d" % rc)
    return gm, gv


def step_velocity_only_parallel(p: M.Particles, grid: M.Grid, config: M.Config, total_dt, indices,
                                threads: int = 1) -> int:
    lib = load()
    idx = np.ascontiguousarray(np.asarray(indices, np.uint64))
    v = p.view()
    return lib.oracle_mpm_step_velocity_only_parallel(C.byref(v), p.n, C.byref(grid), C.byref(config), total_dt,
                                                      idx.ctypes.data_as(C.POINTER(C.c_uint64)), idx.size,
                                                      threads)


def b_spline(x):
    return load().oracle_b_spline(x)


def b_spline_deriv(x):
    return load().oracle_b_spline_deriv(x)


def quadratic_weight(x):
    return load().oracle_quadratic_weight(x)


def quadratic_weight_grad(x):
    return load().oracle_quadratic_weight_grad(x)


def compute_stress(model: int, params: M.Material, F, J: float):
    F = np.ascontiguousarray(np.asarray(F, np.float32).reshape(9))
    st = np.zeros(9, np.float32)
    nf = np.zeros(9, np.float32)
    plastic = load().oracle_compute_stress(model, C.byref(params), _fp(F), J, _fp(st), _fp(nf))
    return st, nf, bool(plastic)


def lame(params: M.Material):
    out = (C.c_float * 3)()
    load().oracle_material_lame(C.byref(params), out)
    return tuple(out[:])


def polar_decomp(F):
    F = np.ascontiguousarray(np.asarray(F, np.float32).reshape(9))
    R = np.zeros(9, np.float32)
    S = np.zeros(9, np.float32)
    load().oracle_polar_decomp(_fp(F), _fp(R), _fp(S))
    return R, S


def clamp_is_identity(F, lo: float, hi: float) -> bool:
    F = np.ascontiguousarray(np.asarray(F, np.float32).reshape(9))
    return bool(load().oracle_clamp_is_identity_f32(_fp(F), lo, hi))


def svd3(F, f64: bool = False, allow_fallback: bool = True, lo: float = 1 - 2.5e-2, hi: float = 1 + 7.5e-3):
    if f64:
        F = np.ascontiguousarray(np.asarray(F, np.float64).reshape(9))
        U, s, V = np.zeros(9), np.zeros(3), np.zeros(9)
        load().oracle_svd3_f64(_dp(F), _dp(U), _dp(s), _dp(V))
        return U.reshape(3, 3), s, V.reshape(3, 3), False
    F = np.ascontiguousarray(np.asarray(F, np.float32).reshape(9))
    U, s, V = np.zeros(9, np.float32), np.zeros(3, np.float32), np.zeros(9, np.float32)
    fb = load().oracle_svd3_f32(_fp(F), _fp(U), _fp(s), _fp(V), 1 if allow_fallback else 0, lo, hi)
    return U.reshape(3, 3), s, V.reshape(3, 3), bool(fb)


# ---------------------------------------------------------------- engine tick passes (simulation.rs)
def lod_classify(pos, active, player, near_dist, mid_dist, max_near):
    """simulation.rs:495-532: (near, mid, far) index arrays; near in the order select_nth leaves it."""
    pos = np.ascontiguousarray(pos, np.float32)
    n = pos.shape[0]
    act = None if active is None else np.ascontiguousarray(active, np.uint8)
    outs = [np.empty(max(n, 1), np.uint32) for _ in range(3)]
    cnt = [C.c_uint64(0) for _ in range(3)]
    pl = np.ascontiguousarray(player, np.float32)
    load().oracle_lod_classify(pos.ctypes.data, None if act is None else act.ctypes.data, n, pl.ctypes.data,
                               near_dist, mid_dist, max_near, outs[0].ctypes.data, C.byref(cnt[0]),
                               outs[1].ctypes.data, C.byref(cnt[1]), outs[2].ctypes.data, C.byref(cnt[2]))
    return tuple(o[:c.value].astype(np.uint64) for o, c in zip(outs, cnt))


def far_field_update(pos, vel, temperature, far_idx, coarse, coarse_dx, origin, far_dt):
    """simulation.rs:612-679, in place on float32 arrays."""
    idx = np.ascontiguousarray(far_idx, np.uint32)
    coarse = np.ascontiguousarray(coarse, np.float32)
    cn = int(round(coarse.size ** (1.0 / 3.0)))
    o = np.ascontiguousarray(origin, np.float32)
    load().oracle_far_field_update(pos.ctypes.data, vel.ctypes.data, temperature.ctypes.data, idx.ctypes.data,
                                   idx.size, coarse.ctypes.data, cn, coarse_dx, o.ctypes.data, far_dt)


def coarse_field_update(pos, mass, temperature, active, near_idx, coarse, coarse_dx, origin, dt):
    """simulation.rs:877-966, coarse (float32, n^3) in place."""
    idx = np.ascontiguousarray(near_idx, np.uint32)
    cn = int(round(coarse.size ** (1.0 / 3.0)))
    o = np.ascontiguousarray(origin, np.float32)
    act = None if active is None else np.ascontiguousarray(active, np.uint8)
    load().oracle_coarse_field_update(np.ascontiguousarray(pos, np.float32).ctypes.data,
                                      np.ascontiguousarray(mass, np.float32).ctypes.data,
                                      np.ascontiguousarray(temperature, np.float32).ctypes.data,
                                      None if act is None else act.ctypes.data, idx.ctypes.data, idx.size,
                                      coarse.ctypes.data, cn, coarse_dx, o.ctypes.data, dt)


def mpss_housekeeping(pos, vel, temperature, phase, material_idx, active, bounds_min, bounds_max, min_temp, max_temp,
                      passes=7):
    """ae_engine/src/lib.rs:347-358 (mpss.rs serial forms), in place; returns the transition count."""
    mat = np.ascontiguousarray(material_idx, np.uint16)
    act = None if active is None else np.ascontiguousarray(active, np.uint8)
    lo = np.ascontiguousarray(bounds_min, np.float32)
    hi = np.ascontiguousarray(bounds_max, np.float32)
    return load().oracle_mpss_housekeeping(pos.ctypes.data, vel.ctypes.data, temperature.ctypes.data,
                                           phase.ctypes.data, mat.ctypes.data, None if act is None else act.ctypes.data,
                                           pos.shape[0], lo.ctypes.data, hi.ctypes.data, min_temp, max_temp, passes)


# ---------------------------------------------------------------- CK-MPM (ae_compute/src/ck_mpm.rs)
def ck_step(particles: np.ndarray, config: M.CkConfig, steps: int = 1, correctly_rounded_ln: bool = False) -> None:
    """`steps` x CkMpmSolver::step (ck_mpm.rs:187-480) in place on (n, 26) float32 records.
    correctly_rounded_ln replaces the C library's logf (the reference's f32::ln) by the correctly
    rounded logarithm, for checking the device's deterministic mode bit for bit."""
    if particles.dtype != np.float32 or not particles.flags.c_contiguous or particles.shape[-1] != M.CK_RECORD:
        raise ValueError("particles must be a C-contiguous (n, 26) float32 array")
    load().oracle_ck_step_ln(particles.ctypes.data if particles.size else None, particles.shape[0], C.byref(config),
                             steps, 1 if correctly_rounded_ln else 0)


def ck_weight(x: float, h: float) -> float:
    return load().oracle_ck_weight(x, h)


def ck_weight_grad(x: float, h: float) -> float:
    return load().oracle_ck_weight_grad(x, h)


def ck_stats(particles: np.ndarray):
    """kinetic_energy, average_velocity, average_volume_ratio (ck_mpm.rs:484-503): sequential f32
    sums in particle order, as the reference's iterator sums."""
    p = np.asarray(particles, np.float32)
    n = p.shape[0]
    if n == 0:
        return np.float32(0.0), np.zeros(3, np.float32), np.float32(1.0)
    ke = np.float32(0.0)
    vs = np.zeros(3, np.float32)
    ds = np.float32(0.0)
    f32 = np.float32
    for r in p:
        v = r[3:6]
        lsq = f32(f32(v[0] * v[0]) + f32(v[1] * v[1])) + f32(v[2] * v[2])
        ke = f32(ke + f32(f32(f32(0.5) * r[25]) * lsq))
        vs = (vs + v).astype(np.float32)
        x, y, z = r[15:18], r[18:21], r[21:24]
        cx = np.array([f32(x[1] * y[2]) - f32(y[1] * x[2]), f32(x[2] * y[0]) - f32(y[2] * x[0]),
                       f32(x[0] * y[1]) - f32(y[0] * x[1])], np.float32)
        ds = f32(ds + (f32(f32(z[0] * cx[0]) + f32(z[1] * cx[1])) + f32(z[2] * cx[2])))
    return ke, (vs / f32(n)).astype(np.float32), f32(ds / f32(n))
