"""ctypes binding of libae_mpm.so (include/ae_mpm.h) for tests, benchmarks and Python callers.

Particle state crosses the boundary in the reference's MpssBuffer layout
(ae_particle/src/mpss.rs:105-157): pos/vel as [f32;3], strain (F) and c (APIC C) as row-major
[f32;9], jacobian and mass as f32, material_idx as u16.  `Particles` holds those arrays as numpy.

There is no CPU fallback: if the library is missing or no CUDA device is usable, the calls
raise.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libae_mpm.so")

OK, EINVAL, ENOMEM, ENAN, ETIMEOUT, EBUDGET, ECUDA, EDOMAIN, ENOTFOUND, EAGAIN = range(10)
STATUS = {OK: "OK", EINVAL: "EINVAL", ENOMEM: "ENOMEM", ENAN: "ENAN", ETIMEOUT: "ETIMEOUT", EBUDGET: "EBUDGET",
          ECUDA: "ECUDA", EDOMAIN: "EDOMAIN", ENOTFOUND: "ENOTFOUND", EAGAIN: "EAGAIN"}

# ConstitutiveModel (ae_particle/src/constitutive.rs:12-27) and the physics-mode materials
NEO_HOOKEAN, DRUCKER_PRAGER, VON_MISES, NEWTONIAN_FLUID, COROTATED, FIXED_COROTATED, RIGID = range(7)
PHYS_JELLY, PHYS_SNOW, PHYS_FLUID = 16, 17, 18
MODE_PHYSICS, MODE_REFERENCE, MODE_VELOCITY_ONLY = 0, 1, 2
WALL_STICKY, WALL_SLIP = 0, 1
P2G_AUTO, P2G_TILE, P2G_WARP_AGG, P2G_GLOBAL, P2G_LANES = 0, 1, 2, 3, 4


class MpmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__("%s: %s" % (STATUS.get(code, code), msg))
        self.code = code


class Material(C.Structure):
    _fields_ = [("young_modulus", C.c_float), ("poisson_ratio", C.c_float), ("yield_stress", C.c_float),
                ("hardening", C.c_float), ("density", C.c_float), ("friction_angle", C.c_float),
                ("cohesion", C.c_float), ("model", C.c_int32), ("theta_c", C.c_float), ("theta_s", C.c_float),
                ("hardening_xi", C.c_float), ("bulk_modulus", C.c_float)]


class Config(C.Structure):
    _fields_ = [("grid_dx", C.c_float), ("grid_size", C.c_uint64 * 3), ("substeps", C.c_uint64),
                ("gravity", C.c_float * 3), ("damping", C.c_float), ("enable_plasticity", C.c_uint8),
                ("enable_contact", C.c_uint8), ("use_sparse_grid", C.c_uint8)]


class Grid(C.Structure):
    _fields_ = [("nx", C.c_uint64), ("ny", C.c_uint64), ("nz", C.c_uint64), ("dx", C.c_float),
                ("origin", C.c_float * 3)]


class ParticlesView(C.Structure):
    _fields_ = [("pos", C.c_void_p), ("vel", C.c_void_p), ("strain", C.c_void_p), ("jacobian", C.c_void_p),
                ("c", C.c_void_p), ("mass", C.c_void_p), ("material_idx", C.c_void_p)]


class SceneDesc(C.Structure):
    _fields_ = [("mode", C.c_int32), ("n", C.c_uint32 * 3), ("dx", C.c_float), ("origin", C.c_float * 3),
                ("gravity", C.c_float * 3), ("dt", C.c_float), ("wall_mode", C.c_int32),
                ("wall_margin", C.c_int32), ("restitution", C.c_float), ("damping", C.c_float),
                ("wall_origin", C.c_int32), ("n_materials", C.c_uint32), ("materials", C.POINTER(Material)),
                ("max_particles", C.c_uint64)]


class ExecOpts(C.Structure):
    _fields_ = [("precision", C.c_int32), ("deterministic", C.c_int32), ("sort_interval", C.c_int32),
                ("p2g_variant", C.c_int32), ("block_threads", C.c_int32), ("use_graph", C.c_int32),
                ("track_totals", C.c_int32), ("svd_fp64_fallback", C.c_int32)]


class TuneResult(C.Structure):
    _fields_ = [("p2g_variant", C.c_int32), ("block_threads", C.c_int32), ("sort_interval", C.c_int32),
                ("us_per_substep", C.c_float)]


class ServerOpts(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_uint64), ("substeps_per_tick", C.c_uint32), ("max_scenes", C.c_uint32),
                ("exec", ExecOpts)]


class RequestResult(C.Structure):
    _fields_ = [("request_id", C.c_uint64), ("status", C.c_int32), ("submit_s", C.c_double),
                ("admit_s", C.c_double), ("done_s", C.c_double)]


class CkConfig(C.Structure):
    """ae_mpm_ck_config: CkMpmConfig (ae_compute/src/ck_mpm.rs:41-59)."""
    _fields_ = [("dt", C.c_float), ("grid_h", C.c_float), ("grid_n", C.c_uint32), ("gravity", C.c_float * 3),
                ("youngs_modulus", C.c_float), ("poissons_ratio", C.c_float), ("density", C.c_float),
                ("bounds_min", C.c_float * 3), ("bounds_max", C.c_float * 3), ("restitution", C.c_float),
                ("dual_grid", C.c_uint8), ("pad", C.c_uint8 * 3)]


class CkStats(C.Structure):
    _fields_ = [("kinetic_energy", C.c_float), ("average_velocity", C.c_float * 3),
                ("average_volume_ratio", C.c_float)]


CK_RECORD = 26  # floats per CkMpmParticle record: position, velocity, affine, deformation, rest_volume, mass


def ck_config(**overrides) -> CkConfig:
    """CkMpmConfig::default() (ck_mpm.rs:61-77) with `overrides` applied, like the reference's
    `CkMpmConfig { grid_n: 16, ..CkMpmConfig::default() }`."""
    c = CkConfig()
    c.dt = 1.0 / 240.0
    c.grid_h = 0.05
    c.grid_n = 32
    c.gravity[:] = (0.0, -9.81, 0.0)
    c.youngs_modulus = 1e5
    c.poissons_ratio = 0.3
    c.density = 1000.0
    c.bounds_min[:] = (-1.0, -1.0, -1.0)
    c.bounds_max[:] = (1.0, 1.0, 1.0)
    c.restitution = 0.3
    c.dual_grid = 1
    for k, v in overrides.items():
        if k in ("gravity", "bounds_min", "bounds_max"):
            getattr(c, k)[:] = tuple(float(x) for x in v)
        else:
            setattr(c, k, v)
    return c


def ck_particles(positions, mass, rest_volume, velocity=None) -> np.ndarray:
    """(n, 26) float32 CkMpmParticle records as CkMpmParticle::new (ck_mpm.rs:97-108) makes them:
    zero velocity and affine matrix, identity deformation gradient."""
    pos = np.asarray(positions, np.float32).reshape(-1, 3)
    n = pos.shape[0]
    r = np.zeros((n, CK_RECORD), np.float32)
    r[:, 0:3] = pos
    if velocity is not None:
        r[:, 3:6] = np.asarray(velocity, np.float32).reshape(-1, 3)
    r[:, 15] = r[:, 19] = r[:, 23] = 1.0
    r[:, 24] = rest_volume
    r[:, 25] = mass
    return r


# every function include/ae_mpm.h declares: name -> (restype, argtypes)
_P = C.c_void_p
SIGNATURES = {
    "ae_mpm_abi_version": (C.c_int, []),
    "ae_mpm_exec_opts_default": (None, [C.POINTER(ExecOpts)]),
    "ae_mpm_ctx_create": (C.c_int, [C.c_int, C.POINTER(_P)]),
    "ae_mpm_ctx_destroy": (None, [_P]),
    "ae_mpm_last_error": (C.c_char_p, [_P]),
    "ae_mpm_step_parallel_with_grid": (C.c_int, [_P, C.POINTER(ParticlesView), C.c_uint64, C.POINTER(Grid),
                                                 C.POINTER(Config), C.POINTER(Material), C.c_uint32,
                                                 C.POINTER(C.c_int32), C.c_uint32, C.c_float,
                                                 C.POINTER(C.c_uint64), C.c_uint64]),
    "ae_mpm_step_velocity_only_parallel": (C.c_int, [_P, C.POINTER(ParticlesView), C.c_uint64, C.POINTER(Grid),
                                                     C.POINTER(Config), C.c_float, C.POINTER(C.c_uint64),
                                                     C.c_uint64]),
    "ae_mpm_grid_download": (C.c_int, [_P, _P, _P, C.c_uint64]),
    "ae_mpm_world_create": (C.c_int, [_P, C.POINTER(SceneDesc), C.c_uint32, C.POINTER(ExecOpts), C.POINTER(_P)]),
    "ae_mpm_world_destroy": (C.c_int, [_P]),
    "ae_mpm_world_upload": (C.c_int, [_P, C.c_uint32, C.POINTER(ParticlesView), C.c_uint64]),
    "ae_mpm_world_upload_f64": (C.c_int, [_P, C.c_uint32, C.POINTER(ParticlesView), C.c_uint64]),
    "ae_mpm_world_step": (C.c_int, [_P, C.c_uint32]),
    "ae_mpm_world_set_scene": (C.c_int, [_P, C.c_uint32, C.POINTER(SceneDesc)]),
    "ae_mpm_world_sync": (C.c_int, [_P]),
    "ae_mpm_world_download": (C.c_int, [_P, C.c_uint32, C.POINTER(ParticlesView)]),
    "ae_mpm_world_download_f64": (C.c_int, [_P, C.c_uint32, C.POINTER(ParticlesView)]),
    "ae_mpm_world_upload_many": (C.c_int, [_P, C.c_uint32, _P, _P, _P]),
    "ae_mpm_world_download_many": (C.c_int, [_P, C.c_uint32, _P, _P]),
    "ae_mpm_batch_create": (C.c_int, [_P, C.POINTER(SceneDesc), C.c_uint32, C.POINTER(ExecOpts), C.c_uint32,
                                      C.POINTER(_P)]),
    "ae_mpm_batch_run": (C.c_int, [_P, _P, _P, _P, C.c_uint32]),
    "ae_mpm_batch_groups": (C.c_uint32, [_P, _P]),
    "ae_mpm_batch_destroy": (C.c_int, [_P]),
    "ae_mpm_batch_partition": (C.c_uint32, [_P, C.c_uint32, C.c_uint32, _P]),
    "ae_mpm_world_totals": (C.c_int, [_P, C.c_uint32, C.POINTER(C.c_double)]),
    "ae_mpm_world_errors": (C.c_int, [_P, C.c_uint32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint64)]),
    "ae_mpm_world_launch_count": (C.c_int, [_P, C.POINTER(C.c_uint64)]),
    "ae_mpm_world_stage_times": (C.c_int, [_P, C.c_uint32, C.POINTER(C.c_double)]),
    "ae_mpm_world_stage_times_split": (C.c_int, [_P, C.c_uint32, C.POINTER(C.c_double)]),
    "ae_mpm_world_stream": (_P, [_P]),
    "ae_mpm_world_particles": (C.c_uint64, [_P]),
    "ae_mpm_world_scene_particles": (C.c_uint64, [_P, C.c_uint32]),
    "ae_mpm_radix_sort_keys": (C.c_int, [_P, _P, C.c_uint64, C.c_uint32, _P, _P]),
    "ae_mpm_radix_sort_keys_noalloc": (C.c_int, [_P, _P, C.c_uint64, C.c_uint32, _P, _P, _P]),
    "ae_mpm_counting_sort_keys": (C.c_int, [_P, _P, C.c_uint64, C.c_uint32, _P, _P]),
    "ae_mpm_lod_classify": (C.c_int, [_P, _P, _P, C.c_uint64, _P, C.c_float, C.c_float, C.c_uint64, _P,
                                      C.POINTER(C.c_uint64), _P, C.POINTER(C.c_uint64), _P, C.POINTER(C.c_uint64)]),
    "ae_mpm_far_field_update": (C.c_int, [_P, _P, _P, _P, C.c_uint64, _P, C.c_uint64, _P, C.c_uint32, C.c_float, _P,
                                          C.c_float]),
    "ae_mpm_coarse_field_update": (C.c_int, [_P, _P, _P, _P, _P, C.c_uint64, _P, C.c_uint64, _P, C.c_uint32,
                                             C.c_float, _P, C.c_float]),
    "ae_mpm_mpss_housekeeping": (C.c_int, [_P, _P, _P, _P, _P, _P, _P, C.c_uint64, _P, _P, C.c_float, C.c_float,
                                           C.c_uint32, C.POINTER(C.c_uint32)]),
    "ae_mpm_ck_config_default": (None, [C.POINTER(CkConfig)]),
    "ae_mpm_ck_step": (C.c_int, [_P, _P, C.c_uint64, C.POINTER(CkConfig), C.c_uint32]),
    "ae_mpm_ck_step_timed": (C.c_int, [_P, _P, C.c_uint64, C.POINTER(CkConfig), C.c_uint32, C.POINTER(C.c_double)]),
    "ae_mpm_ck_step_deterministic": (C.c_int, [_P, _P, C.c_uint64, C.POINTER(CkConfig), C.c_uint32]),
    "ae_mpm_ck_stats_compute": (C.c_int, [_P, _P, C.c_uint64, C.POINTER(CkStats)]),
    "ae_mpm_ck_weights": (C.c_int, [_P, _P, C.c_uint64, C.c_float, _P, _P]),
    "ae_mpm_world_autotune": (C.c_int, [_P, C.c_uint32, C.POINTER(TuneResult)]),
    "ae_mpm_server_create": (C.c_int, [_P, C.POINTER(ServerOpts), C.POINTER(_P)]),
    "ae_mpm_server_submit": (C.c_int, [_P, C.POINTER(SceneDesc), C.POINTER(ParticlesView), C.c_uint64, C.c_uint32,
                                       C.POINTER(ParticlesView), C.POINTER(C.c_uint64)]),
    "ae_mpm_server_cancel": (C.c_int, [_P, C.c_uint64]),
    "ae_mpm_server_poll": (C.c_int, [_P, C.POINTER(RequestResult), C.c_uint32, C.POINTER(C.c_uint32)]),
    "ae_mpm_server_drain": (C.c_int, [_P, C.c_double]),
    "ae_mpm_server_stats": (C.c_int, [_P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint32), C.POINTER(C.c_uint64),
                                      C.POINTER(C.c_uint64)]),
    "ae_mpm_server_destroy": (C.c_int, [_P]),
    "ae_mpm_server_slot_class": (C.c_int, [C.POINTER(SceneDesc), C.c_uint64, _P, C.POINTER(C.c_uint64),
                                           C.POINTER(C.c_uint32)]),
}

_lib = None


def load(path: str = LIB_PATH):
    """Loads the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError("libae_mpm.so is not built (%s): run __graft_entry__.build()" % path)
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def batch_partition(capacities, groups: int):
    """ae_mpm_batch_partition: the first scene of every group of a pipelined batch, then the
    scene count (host only)."""
    caps = np.ascontiguousarray(capacities, np.uint64)
    first = np.zeros(caps.size + 1, np.uint32)
    g = load().ae_mpm_batch_partition(caps.ctypes.data, caps.size, groups, first.ctypes.data)
    return [int(x) for x in first[:g + 1]] if g else []


def server_slot_class(scene: "Scene", n_particles: int):
    """ae_mpm_server_slot_class: (grid axes, particle capacity, material count) of the server slot
    a request takes (host only)."""
    d = scene.desc()
    g = np.zeros(3, np.uint32)
    cap, mats = C.c_uint64(), C.c_uint32()
    rc = load().ae_mpm_server_slot_class(C.byref(d), n_particles, g.ctypes.data, C.byref(cap), C.byref(mats))
    if rc != OK:
        raise MpmError(rc, "slot class")
    return tuple(int(x) for x in g), int(cap.value), int(mats.value)


def exec_opts(**kw) -> ExecOpts:
    o = ExecOpts()
    load().ae_mpm_exec_opts_default(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def material(young_modulus=1e6, poisson_ratio=0.3, yield_stress=1e4, hardening=0.01, density=1000.0,
             friction_angle=35.0, cohesion=0.0, model=NEO_HOOKEAN, theta_c=2.5e-2, theta_s=7.5e-3,
             hardening_xi=10.0, bulk_modulus=0.0) -> Material:
    return Material(young_modulus, poisson_ratio, yield_stress, hardening, density, friction_angle, cohesion,
                    model, theta_c, theta_s, hardening_xi, bulk_modulus)


@dataclass
class Particles:
    """Particle arrays in the reference layout (float32 or float64)."""
    pos: np.ndarray
    vel: np.ndarray
    F: np.ndarray
    J: np.ndarray
    C: np.ndarray
    mass: np.ndarray
    mat: np.ndarray

    @staticmethod
    def empty(n: int, dtype=np.float32) -> "Particles":
        F = np.zeros((n, 9), dtype)
        F[:, [0, 4, 8]] = 1
        return Particles(np.zeros((n, 3), dtype), np.zeros((n, 3), dtype), F, np.ones(n, dtype),
                         np.zeros((n, 9), dtype), np.ones(n, dtype), np.zeros(n, np.uint16))

    @property
    def n(self) -> int:
        return int(self.pos.shape[0])

    @property
    def dtype(self):
        return self.pos.dtype

    def astype(self, dtype) -> "Particles":
        return Particles(*(np.ascontiguousarray(a.astype(dtype)) for a in
                           (self.pos, self.vel, self.F, self.J, self.C, self.mass)), self.mat.copy())

    def copy(self) -> "Particles":
        return Particles(self.pos.copy(), self.vel.copy(), self.F.copy(), self.J.copy(), self.C.copy(),
                         self.mass.copy(), self.mat.copy())

    def subset(self, idx) -> "Particles":
        return Particles(self.pos[idx].copy(), self.vel[idx].copy(), self.F[idx].copy(), self.J[idx].copy(),
                         self.C[idx].copy(), self.mass[idx].copy(), self.mat[idx].copy())

    def check(self) -> None:
        for name in ("pos", "vel", "F", "J", "C", "mass", "mat"):
            a = getattr(self, name)
            if not a.flags["C_CONTIGUOUS"]:
                setattr(self, name, np.ascontiguousarray(a))

    def view(self) -> ParticlesView:
        self.check()
        return ParticlesView(self.pos.ctypes.data, self.vel.ctypes.data, self.F.ctypes.data, self.J.ctypes.data,
                             self.C.ctypes.data, self.mass.ctypes.data, self.mat.ctypes.data)


@dataclass
class Scene:
    """Python form of ae_mpm_scene_desc."""
    n: tuple
    dx: float
    dt: float
    materials: list
    mode: int = MODE_PHYSICS
    origin: tuple = (0.0, 0.0, 0.0)
    gravity: tuple = (0.0, -9.8, 0.0)
    wall_mode: int = WALL_STICKY
    wall_margin: int = 3
    restitution: float = 0.0
    damping: float = 0.995
    wall_origin: int = 1
    max_particles: int = 0
    _mats: object = field(default=None, repr=False)

    def desc(self) -> SceneDesc:
        arr = (Material * len(self.materials))(*self.materials)
        self._mats = arr
        return SceneDesc(self.mode, (C.c_uint32 * 3)(*self.n), self.dx, (C.c_float * 3)(*self.origin),
                         (C.c_float * 3)(*self.gravity), self.dt, self.wall_mode, self.wall_margin,
                         self.restitution, self.damping, self.wall_origin, len(self.materials),
                         C.cast(arr, C.POINTER(Material)), self.max_particles)


class Context:
    def __init__(self, device: int = 0):
        lib = load()
        h = C.c_void_p()
        rc = lib.ae_mpm_ctx_create(device, C.byref(h))
        if rc != OK:
            raise MpmError(rc, "ae_mpm_ctx_create(%d) failed (no usable CUDA device?)" % device)
        self.h = h
        self.lib = lib

    def close(self):
        if self.h:
            self.lib.ae_mpm_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check(self, rc: int) -> int:
        if rc != OK:
            raise MpmError(rc, self.lib.ae_mpm_last_error(self.h).decode())
        return rc

    # -- drop-in entry points ----------------------------------------------------------------
    def step_parallel_with_grid(self, p: Particles, grid: Grid, config: Config, materials, models, total_dt,
                                indices) -> None:
        mats = (Material * max(len(materials), 1))(*materials)
        mods = (C.c_int32 * max(len(models), 1))(*models)
        idx = np.ascontiguousarray(np.asarray(indices, np.uint64))
        v = p.view()
        self.check(self.lib.ae_mpm_step_parallel_with_grid(
            self.h, C.byref(v), p.n, C.byref(grid), C.byref(config), mats, len(materials), mods, len(models),
            total_dt, idx.ctypes.data_as(C.POINTER(C.c_uint64)), idx.size))

    def step_velocity_only_parallel(self, p: Particles, grid: Grid, config: Config, total_dt, indices) -> None:
        idx = np.ascontiguousarray(np.asarray(indices, np.uint64))
        v = p.view()
        self.check(self.lib.ae_mpm_step_velocity_only_parallel(
            self.h, C.byref(v), p.n, C.byref(grid), C.byref(config), total_dt,
            idx.ctypes.data_as(C.POINTER(C.c_uint64)), idx.size))

    def grid_download(self, nx, ny, nz):
        m = np.zeros(nx * ny * nz, np.float32)
        v = np.zeros((nx * ny * nz, 3), np.float32)
        self.check(self.lib.ae_mpm_grid_download(self.h, m.ctypes.data, v.ctypes.data, m.size))
        return m, v

    # engine tick passes around the substep (simulation.rs): numpy arrays in MpssBuffer layout
    # (pos, vel: (count, 3) f32; mass, temperature: (count,) f32; active: (count,) bool/u8 or None)
    def lod_classify(self, pos, active, player, near_dist, mid_dist, max_near):
        pos = np.ascontiguousarray(pos, np.float32)
        n = pos.shape[0]
        act = None if active is None else np.ascontiguousarray(active, np.uint8)
        outs = [np.empty(max(n, 1), np.uint64) for _ in range(3)]
        cnt = [C.c_uint64(0) for _ in range(3)]
        pl = np.ascontiguousarray(player, np.float32)
        self.check(self.lib.ae_mpm_lod_classify(self.h, pos.ctypes.data, None if act is None else act.ctypes.data, n,
                                                pl.ctypes.data, near_dist, mid_dist, max_near,
                                                outs[0].ctypes.data, C.byref(cnt[0]), outs[1].ctypes.data,
                                                C.byref(cnt[1]), outs[2].ctypes.data, C.byref(cnt[2])))
        return tuple(o[:c.value].copy() for o, c in zip(outs, cnt))

    def far_field_update(self, pos, vel, temperature, far_idx, coarse, coarse_dx, origin, far_dt):
        """Updates pos, vel and temperature (float32 arrays) in place."""
        idx = np.ascontiguousarray(far_idx, np.uint64)
        coarse = np.ascontiguousarray(coarse, np.float32)
        cn = int(round(coarse.size ** (1.0 / 3.0)))
        o = np.ascontiguousarray(origin, np.float32)
        self.check(self.lib.ae_mpm_far_field_update(self.h, pos.ctypes.data, vel.ctypes.data, temperature.ctypes.data,
                                                    pos.shape[0], idx.ctypes.data, idx.size, coarse.ctypes.data, cn,
                                                    coarse_dx, o.ctypes.data, far_dt))

    def coarse_field_update(self, pos, mass, temperature, active, near_idx, coarse, coarse_dx, origin, dt):
        """Updates coarse (float32, n^3) in place."""
        pos = np.ascontiguousarray(pos, np.float32)
        mass = np.ascontiguousarray(mass, np.float32)
        temperature = np.ascontiguousarray(temperature, np.float32)
        act = None if active is None else np.ascontiguousarray(active, np.uint8)
        idx = np.ascontiguousarray(near_idx, np.uint64)
        cn = int(round(coarse.size ** (1.0 / 3.0)))
        o = np.ascontiguousarray(origin, np.float32)
        self.check(self.lib.ae_mpm_coarse_field_update(self.h, pos.ctypes.data, mass.ctypes.data, temperature.ctypes.data,
                                                       None if act is None else act.ctypes.data, pos.shape[0],
                                                       idx.ctypes.data, idx.size, coarse.ctypes.data, cn, coarse_dx,
                                                       o.ctypes.data, dt))

    def mpss_housekeeping(self, pos, vel, temperature, phase, material_idx, active, bounds_min, bounds_max,
                          min_temp, max_temp, passes=7):
        """ae_engine/src/lib.rs:347-358 in place on pos, vel (float32 (n,3)), temperature (float32),
        phase (uint8); returns the number of phase transitions."""
        mat = np.ascontiguousarray(material_idx, np.uint16)
        act = None if active is None else np.ascontiguousarray(active, np.uint8)
        lo = np.ascontiguousarray(bounds_min, np.float32)
        hi = np.ascontiguousarray(bounds_max, np.float32)
        tr = C.c_uint32(0)
        self.check(self.lib.ae_mpm_mpss_housekeeping(self.h, pos.ctypes.data, vel.ctypes.data, temperature.ctypes.data,
                                                     phase.ctypes.data, mat.ctypes.data,
                                                     None if act is None else act.ctypes.data, pos.shape[0],
                                                     lo.ctypes.data, hi.ctypes.data, min_temp, max_temp, passes,
                                                     C.byref(tr)))
        return tr.value

    # CK-MPM solver (ae_compute/src/ck_mpm.rs): particles are (n, 26) float32 records
    def ck_step(self, particles: np.ndarray, config: CkConfig, steps: int = 1, deterministic: bool = False) -> None:
        """`steps` x CkMpmSolver::step, in place.  deterministic: node sums in particle order
        (bitwise reproducible, the reference's summation order)."""
        if particles.dtype != np.float32 or not particles.flags.c_contiguous or particles.shape[-1] != CK_RECORD:
            raise ValueError("particles must be a C-contiguous (n, 26) float32 array")
        fn = self.lib.ae_mpm_ck_step_deterministic if deterministic else self.lib.ae_mpm_ck_step
        self.check(fn(self.h, particles.ctypes.data, particles.shape[0], C.byref(config), steps))

    def ck_stats(self, particles: np.ndarray):
        """(kinetic_energy, average_velocity (3,), average_volume_ratio)."""
        p = np.ascontiguousarray(particles, np.float32)
        st = CkStats()
        self.check(self.lib.ae_mpm_ck_stats_compute(self.h, p.ctypes.data if p.size else None, p.shape[0],
                                                    C.byref(st)))
        return st.kinetic_energy, np.array(st.average_velocity[:], np.float32), st.average_volume_ratio

    def ck_weights(self, x, h: float):
        """CkMpmSolver::weight / weight_grad evaluated on the device."""
        x = np.ascontiguousarray(x, np.float32).ravel()
        w = np.empty_like(x)
        dw = np.empty_like(x)
        self.check(self.lib.ae_mpm_ck_weights(self.h, x.ctypes.data, x.size, h, w.ctypes.data, dw.ctypes.data))
        return w, dw

    def radix_sort(self, keys: np.ndarray, key_bits: int):
        keys = np.ascontiguousarray(keys, np.uint32)
        sk = np.empty_like(keys)
        perm = np.empty_like(keys)
        self.check(self.lib.ae_mpm_radix_sort_keys(self.h, keys.ctypes.data, keys.size, key_bits,
                                                   sk.ctypes.data, perm.ctypes.data))
        return sk, perm

    def counting_sort(self, keys: np.ndarray, key_bits: int):
        """Grouping sort of keys of at most 16 bits: ascending keys, equal keys in no defined order."""
        keys = np.ascontiguousarray(keys, np.uint32)
        sk = np.empty_like(keys)
        perm = np.empty_like(keys)
        self.check(self.lib.ae_mpm_counting_sort_keys(self.h, keys.ctypes.data, keys.size, key_bits,
                                                      sk.ctypes.data, perm.ctypes.data))
        return sk, perm


class World:
    """Device-resident scenes stepped in lockstep (batched path; one scene = plain path)."""

    def __init__(self, ctx: Context, scenes, opts: ExecOpts | None = None):
        self.ctx = ctx
        self.scenes = list(scenes)
        descs = (SceneDesc * len(self.scenes))(*[s.desc() for s in self.scenes])
        self._descs = descs
        h = C.c_void_p()
        ctx.check(ctx.lib.ae_mpm_world_create(ctx.h, descs, len(self.scenes),
                                              C.byref(opts) if opts is not None else None, C.byref(h)))
        self.h = h
        self.f64 = opts is not None and opts.precision == 64

    def close(self):
        if self.h:
            self.ctx.lib.ae_mpm_world_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, scene: int, p: Particles) -> None:
        want = np.float64 if self.f64 else np.float32
        if p.dtype != want:
            raise TypeError("world precision needs %s particles" % np.dtype(want).name)
        v = p.view()
        fn = self.ctx.lib.ae_mpm_world_upload_f64 if self.f64 else self.ctx.lib.ae_mpm_world_upload
        self.ctx.check(fn(self.h, scene, C.byref(v), p.n))
        self._keep = p

    def scene_particles(self, scene: int) -> int:
        return int(self.ctx.lib.ae_mpm_world_scene_particles(self.h, scene))

    def _room(self, scene: int, n: int) -> None:
        have = self.scene_particles(scene)
        if n < have:
            raise ValueError("scene %d holds %d particles; room for %d" % (scene, have, n))

    def download(self, scene: int, n: int) -> Particles:
        self._room(scene, n)
        p = Particles.empty(n, np.float64 if self.f64 else np.float32)
        v = p.view()
        fn = self.ctx.lib.ae_mpm_world_download_f64 if self.f64 else self.ctx.lib.ae_mpm_world_download
        self.ctx.check(fn(self.h, scene, C.byref(v)))
        return p

    def download_into(self, scene: int, p: Particles) -> None:
        self._room(scene, p.n)
        v = p.view()
        fn = self.ctx.lib.ae_mpm_world_download_f64 if self.f64 else self.ctx.lib.ae_mpm_world_download
        self.ctx.check(fn(self.h, scene, C.byref(v)))

    def upload_many(self, scenes, parts) -> None:
        """ae_mpm_world_upload_many: parts[i] (float32 Particles) into scene scenes[i]."""
        k = len(parts)
        views = (ParticlesView * max(k, 1))(*[p.view() for p in parts])
        ids = np.ascontiguousarray(scenes, np.uint32)
        counts = np.ascontiguousarray([p.n for p in parts], np.uint64)
        self._keep_many = parts
        self.ctx.check(self.ctx.lib.ae_mpm_world_upload_many(self.h, k, ids.ctypes.data, C.addressof(views),
                                                             counts.ctypes.data))

    def download_many(self, scenes, parts) -> None:
        """ae_mpm_world_download_many: scene scenes[i] into parts[i] (float32 Particles)."""
        for sc, p in zip(scenes, parts):
            self._room(sc, p.n)
        k = len(parts)
        views = (ParticlesView * max(k, 1))(*[p.view() for p in parts])
        ids = np.ascontiguousarray(scenes, np.uint32)
        self.ctx.check(self.ctx.lib.ae_mpm_world_download_many(self.h, k, ids.ctypes.data, C.addressof(views)))

    def step(self, n: int) -> None:
        self.ctx.check(self.ctx.lib.ae_mpm_world_step(self.h, n))

    def set_scene(self, index: int, scene: "Scene") -> None:
        d = scene.desc()
        self.ctx.check(self.ctx.lib.ae_mpm_world_set_scene(self.h, index, C.byref(d)))
        self.scenes[index] = scene

    def sync(self, raise_on_error: bool = True) -> int:
        rc = self.ctx.lib.ae_mpm_world_sync(self.h)
        if raise_on_error:
            self.ctx.check(rc)
        return rc

    def totals(self, scene: int) -> np.ndarray:
        out = (C.c_double * 5)()
        self.ctx.check(self.ctx.lib.ae_mpm_world_totals(self.h, scene, out))
        return np.array(out[:])

    def errors(self, scene: int):
        w = C.c_uint32()
        c = (C.c_uint64 * 3)()
        self.ctx.check(self.ctx.lib.ae_mpm_world_errors(self.h, scene, C.byref(w), c))
        return int(w.value), [int(x) for x in c]

    def launches(self) -> int:
        n = C.c_uint64()
        self.ctx.check(self.ctx.lib.ae_mpm_world_launch_count(self.h, C.byref(n)))
        return int(n.value)

    def stage_times(self, n: int) -> dict:
        """Mean per-substep device time of each stage (us), measured with CUDA events; "g2p" includes
        the snow clamp, "g2p_kernel" is the G2P (or fused G2P + P2G) kernel alone."""
        out = (C.c_double * 6)()
        self.ctx.check(self.ctx.lib.ae_mpm_world_stage_times_split(self.h, n, out))
        return dict(zip(("sort", "p2g", "grid", "g2p", "substep", "g2p_kernel"), out[:]))

    def stream(self) -> int:
        return int(self.ctx.lib.ae_mpm_world_stream(self.h) or 0)

    def particles(self) -> int:
        return int(self.ctx.lib.ae_mpm_world_particles(self.h))

    def autotune(self, substeps_per_trial: int = 8) -> TuneResult:
        r = TuneResult()
        self.ctx.check(self.ctx.lib.ae_mpm_world_autotune(self.h, substeps_per_trial, C.byref(r)))
        return r


class ViewArray:
    """Views of a list of float32 Particles for the many-scene calls, built once: callers that
    pass the same buffers call after call save rebuilding them.  Holds the particles alive; the
    views stay valid while their arrays are not replaced (in-place writes are fine)."""

    def __init__(self, parts):
        self.parts = list(parts)
        k = len(self.parts)
        self.arr = (ParticlesView * max(k, 1))(*[p.view() for p in self.parts])
        self.counts = np.ascontiguousarray([p.n for p in self.parts], np.uint64)

    def __len__(self):
        return len(self.parts)


class Batch:
    """Pipelined batch (ae_mpm_batch_*): scenes in host memory advanced n substeps per run, in
    `groups` consecutive groups whose PCIe copies overlap the other groups' substeps."""

    def __init__(self, ctx: Context, scenes, opts: ExecOpts | None = None, groups: int = 4):
        self.ctx = ctx
        self.scenes = list(scenes)
        descs = (SceneDesc * len(self.scenes))(*[s.desc() for s in self.scenes])
        h = C.c_void_p()
        ctx.check(ctx.lib.ae_mpm_batch_create(ctx.h, descs, len(self.scenes),
                                              C.byref(opts) if opts is not None else None, groups, C.byref(h)))
        self.h = h

    def groups(self):
        """First scene of every group, then the scene count."""
        n = self.ctx.lib.ae_mpm_batch_groups(self.h, None)
        first = np.zeros(n + 1, np.uint32)
        self.ctx.lib.ae_mpm_batch_groups(self.h, first.ctypes.data)
        return [int(x) for x in first]

    def run(self, parts, n_substeps: int, out=None, raise_on_error: bool = True) -> int:
        """Scene i takes parts[i] (float32 Particles, or a ViewArray of them), runs n_substeps and
        lands in out[i] (parts itself when out is None).  Returns the status code (raises on
        errors unless told not to; every result is written either way)."""
        vin = parts if isinstance(parts, ViewArray) else ViewArray(parts)
        vout = vin if out is None else (out if isinstance(out, ViewArray) else ViewArray(out))
        if len(vin) != len(self.scenes) or len(vout) != len(self.scenes):
            raise ValueError("one input and one output per scene")
        if vout is not vin and any(o.n < i.n for i, o in zip(vin.parts, vout.parts)):
            raise ValueError("an output holds fewer particles than its input")
        if any(p.dtype != np.float32 for p in vin.parts + vout.parts):
            raise TypeError("a batch moves float32 particles")
        rc = self.ctx.lib.ae_mpm_batch_run(self.h, C.addressof(vin.arr), vin.counts.ctypes.data,
                                           C.addressof(vout.arr), n_substeps)
        if rc != OK and (raise_on_error or rc not in (ENAN, EDOMAIN)):
            self.ctx.check(rc)
        return rc

    def close(self):
        if self.h:
            self.ctx.lib.ae_mpm_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous-batching server (ae_mpm_server_*)."""

    def __init__(self, ctx: Context, hbm_budget_bytes=0, substeps_per_tick=10, max_scenes=4096,
                 exec_options: ExecOpts | None = None):
        self.ctx = ctx
        o = ServerOpts(hbm_budget_bytes, substeps_per_tick, max_scenes, exec_options or exec_opts())
        h = C.c_void_p()
        ctx.check(ctx.lib.ae_mpm_server_create(ctx.h, C.byref(o), C.byref(h)))
        self.h = h
        self._pending = {}

    def submit(self, scene: Scene, p: Particles, substeps: int, out: Particles | None = None) -> int:
        """Queues `substeps` substeps of `scene` starting from `p`; the results arrive in `out`
        (allocated here when not given) and are returned by poll()."""
        if out is None:
            out = Particles(*(np.empty_like(a) for a in (p.pos, p.vel, p.F, p.J, p.C, p.mass, p.mat)))
        vin, vout = p.view(), out.view()
        d = scene.desc()
        rid = C.c_uint64()
        self.ctx.check(self.ctx.lib.ae_mpm_server_submit(self.h, C.byref(d), C.byref(vin), p.n, substeps,
                                                         C.byref(vout), C.byref(rid)))
        self._pending[int(rid.value)] = (out, scene)
        return int(rid.value)

    def cancel(self, rid: int) -> int:
        return self.ctx.lib.ae_mpm_server_cancel(self.h, rid)

    def poll(self, max_n: int = 256):
        res = (RequestResult * max_n)()
        n = C.c_uint32()
        rc = self.ctx.lib.ae_mpm_server_poll(self.h, res, max_n, C.byref(n))
        out = []
        for i in range(n.value if rc == OK else 0):
            r = res[i]
            parts, _ = self._pending.pop(int(r.request_id), (None, None))
            out.append((int(r.request_id), int(r.status), r.submit_s, r.admit_s, r.done_s, parts))
        return out

    def drain(self, timeout_s: float = 60.0) -> int:
        return self.ctx.lib.ae_mpm_server_drain(self.h, timeout_s)

    def stats(self):
        rb, rs, tk, ps = C.c_uint64(), C.c_uint32(), C.c_uint64(), C.c_uint64()
        self.ctx.check(self.ctx.lib.ae_mpm_server_stats(self.h, C.byref(rb), C.byref(rs), C.byref(tk), C.byref(ps)))
        return dict(resident_bytes=rb.value, resident_scenes=rs.value, ticks=tk.value, particle_substeps=ps.value)

    def close(self):
        if self.h:
            self.ctx.lib.ae_mpm_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
