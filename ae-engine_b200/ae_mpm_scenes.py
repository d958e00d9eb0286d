"""Seeded synthetic MPM scenes.

The reference publishes no benchmark scenes (its MPM inputs are placed on unseeded lattices,
ae_compute/src/mpm_compute.rs:193-216, ae_physics/src/mpm.rs:179-210), so every workload here is
generated: SplitMix64 (Steele, Lea & Flood 2014) in counter form, seed 0xAE00 + config number.

  config1_jelly     64^3 grid, 32 768 neo-Hookean particles jittered in [0.3,0.5]^3, dt 1e-4
  config2_snow      128^3 grid, 1 048 576 Stomakhin-snow particles in two 0.2^3 boxes at +-2 m/s
  config3_dam       256^3 grid, 8 388 608 particles: 60% fluid, 25% elastic cubes, 15% snow
  config4_batched   512 scenes: grid in {32,48,64}^3, log-uniform 2k..64k particles, one of
                    jelly/snow/water each, box velocity in [-1,1]^3 m/s
  config5_request   one served request: a config4 scene, or (5%) a 128^3 scene of 1M snow
                    particles, with 100..2000 substeps

The sizes are as stated even where they disagree with "8 particles per cell": config 1's box is
12.8^3 cells for 32 768 particles (15.6 per cell) and config 2's boxes give 31 per cell.
"""
from __future__ import annotations

import math

import numpy as np

import ae_mpm as M

GAMMA = np.uint64(0x9E3779B97F4A7C15)
M1 = np.uint64(0xBF58476D1CE4E5B9)
M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed: int, n: int, offset: int = 0) -> np.ndarray:
    """Outputs offset+1 .. offset+n of a SplitMix64 stream started at `seed`."""
    with np.errstate(over="ignore"):
        z = np.uint64(seed & 0xFFFFFFFFFFFFFFFF) + np.arange(offset + 1, offset + n + 1, dtype=np.uint64) * GAMMA
        z = (z ^ (z >> np.uint64(30))) * M1
        z = (z ^ (z >> np.uint64(27))) * M2
        return z ^ (z >> np.uint64(31))


class Rng:
    """Sequential uniform draws from one SplitMix64 stream."""

    def __init__(self, seed: int):
        self.seed = seed
        self.pos = 0

    def uniform(self, n: int) -> np.ndarray:
        u = (splitmix64(self.seed, n, self.pos) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
        self.pos += n
        return u

    def scalar(self) -> float:
        return float(self.uniform(1)[0])


def jelly(E=1e4, nu=0.2, rho=1.0) -> M.Material:
    return M.material(young_modulus=E, poisson_ratio=nu, density=rho, model=M.PHYS_JELLY)


def snow(E=1.4e5, nu=0.2, rho=400.0, theta_c=2.5e-2, theta_s=7.5e-3, xi=10.0) -> M.Material:
    return M.material(young_modulus=E, poisson_ratio=nu, density=rho, model=M.PHYS_SNOW, theta_c=theta_c,
                      theta_s=theta_s, hardening_xi=xi)


def water(K=1e4, rho=1.0) -> M.Material:
    return M.material(young_modulus=K, poisson_ratio=0.2, density=rho, model=M.PHYS_FLUID, bulk_modulus=K)


def jittered_box(rng: Rng, lo, hi, n: int) -> np.ndarray:
    """n positions in the box: a stratified lattice of m^3 sub-cells with k = n/m^3 jittered
    points each when n factors that way, else uniform."""
    lo = np.asarray(lo, np.float64)
    hi = np.asarray(hi, np.float64)
    m = int(round(n ** (1.0 / 3.0)))
    while m > 1 and n % (m ** 3) != 0:
        m -= 1
    k = n // (m ** 3) if m > 1 else 0
    if m > 1 and k >= 1 and k * m ** 3 == n:
        g = np.stack(np.meshgrid(np.arange(m), np.arange(m), np.arange(m), indexing="ij"), -1).reshape(-1, 3)
        g = np.repeat(g, k, axis=0)
        u = rng.uniform(3 * n).reshape(n, 3)
        x = lo + (g + u) * ((hi - lo) / m)
    else:
        u = rng.uniform(3 * n).reshape(n, 3)
        x = lo + u * (hi - lo)
    return x


def make_particles(x: np.ndarray, v, mass: float, mat_idx) -> M.Particles:
    n = x.shape[0]
    p = M.Particles.empty(n)
    p.pos[:] = x.astype(np.float32)
    p.vel[:] = np.asarray(v, np.float32)
    p.mass[:] = np.float32(mass)
    p.mat[:] = mat_idx
    return p


def concat(ps) -> M.Particles:
    return M.Particles(*(np.ascontiguousarray(np.concatenate([getattr(p, f) for p in ps]))
                         for f in ("pos", "vel", "F", "J", "C", "mass", "mat")))


def config1_jelly(seed: int = 0xAE01):
    rng = Rng(seed)
    n = 32768
    x = jittered_box(rng, (0.3, 0.3, 0.3), (0.5, 0.5, 0.5), n)
    mats = [jelly()]
    p = make_particles(x, (0, 0, 0), 1.0 * 0.2 ** 3 / n, 0)
    p.J[:] = 1.0
    sc = M.Scene(n=(64, 64, 64), dx=1.0 / 64, dt=1e-4, materials=mats, max_particles=n)
    return sc, p


def config2_snow(seed: int = 0xAE02):
    rng = Rng(seed)
    n_box = 524288
    mats = [snow()]
    rho = 400.0
    a = jittered_box(rng, (0.28, 0.40, 0.40), (0.48, 0.60, 0.60), n_box)
    b = jittered_box(rng, (0.52, 0.40, 0.40), (0.72, 0.60, 0.60), n_box)
    m = rho * 0.2 ** 3 / n_box
    p = concat([make_particles(a, (2, 0, 0), m, 0), make_particles(b, (-2, 0, 0), m, 0)])
    p.J[:] = 1.0  # plastic J_p starts at 1
    sc = M.Scene(n=(128, 128, 128), dx=1.0 / 128, dt=5e-5, materials=mats, max_particles=2 * n_box)
    return sc, p


def snow_collision_small(n_box: int = 4096, grid: int = 32, seed: int = 0xAE22, v: float = 2.0):
    """Config 2 in miniature for parity tests: two snow boxes 0.2 x 0.2 x 0.2 half a cell apart,
    closing at 2v, so the Stomakhin clamp is active from the first tens of substeps."""
    rng = Rng(seed)
    dx = 1.0 / grid
    w, c, gap = 0.2, 0.5, 0.5 * dx
    a = jittered_box(rng, (c - gap / 2 - w, 0.4, 0.4), (c - gap / 2, 0.6, 0.6), n_box)
    b = jittered_box(rng, (c + gap / 2, 0.4, 0.4), (c + gap / 2 + w, 0.6, 0.6), n_box)
    m = 400.0 * w ** 3 / n_box
    p = concat([make_particles(a, (v, 0, 0), m, 0), make_particles(b, (-v, 0, 0), m, 0)])
    p.J[:] = 1.0
    sc = M.Scene(n=(grid, grid, grid), dx=dx, dt=1e-4, materials=[snow()], max_particles=2 * n_box)
    return sc, p


def config3_dam(seed: int = 0xAE03, scale: float = 1.0):
    """Mixed dam break.  `scale` < 1 shrinks the particle counts (same boxes) for tests."""
    rng = Rng(seed)
    total = int(8388608 * scale)
    nw, ne = int(total * 0.60), int(total * 0.25)
    ns = total - nw - ne
    dx = 1.0 / 256
    base = 4 * dx
    mats = [water(K=1e4, rho=1000.0), jelly(E=1e5, nu=0.3, rho=1000.0), snow()]
    w_hi = (base + 0.5, base + 0.375, base + 0.2)
    pw = make_particles(jittered_box(rng, (base, base, base), w_hi, nw), (0, 0, 0), 1000.0 * 0.5 * 0.375 * 0.2 / nw, 0)
    side = 0.198
    c1 = jittered_box(rng, (0.6, base, 0.1), (0.6 + side, base + side, 0.1 + side), ne // 2)
    c2 = jittered_box(rng, (0.6, base, 0.5), (0.6 + side, base + side, 0.5 + side), ne - ne // 2)
    pe = concat([make_particles(c1, (0, 0, 0), 1000.0 * side ** 3 / (ne // 2), 1),
                 make_particles(c2, (0, 0, 0), 1000.0 * side ** 3 / (ne - ne // 2), 1)])
    sside = 0.21
    s = jittered_box(rng, (0.3, 0.5, 0.3), (0.3 + sside, 0.5 + sside, 0.3 + sside), ns)
    psn = make_particles(s, (0, -1.0, 0), 400.0 * sside ** 3 / ns, 2)
    p = concat([pw, pe, psn])
    p.J[:] = 1.0
    sc = M.Scene(n=(256, 256, 256), dx=dx, dt=2e-5, materials=mats, max_particles=p.n)
    return sc, p


def batched_scene(rng: Rng, large: bool = False):
    if large:
        n, grid = 1048576, 128
        kind = 1
    else:
        grid = (32, 48, 64)[min(2, int(rng.scalar() * 3))]
        n = int(round(math.exp(math.log(2048) + rng.scalar() * (math.log(65536) - math.log(2048)))))
        kind = min(2, int(rng.scalar() * 3))
    dx = 1.0 / grid
    mat = [jelly(), snow(), water()][kind]
    rho = [1.0, 400.0, 1.0][kind]
    side_cells = (n / 8.0) ** (1.0 / 3.0)
    side = side_cells * dx
    lo_c = 4.0
    hi_c = grid - 4.0 - side_cells
    off = np.array([lo_c + rng.scalar() * max(hi_c - lo_c, 0.0) for _ in range(3)]) * dx
    x = jittered_box(rng, off, off + side, n)
    v = np.array([rng.scalar() * 2 - 1 for _ in range(3)])
    p = make_particles(x, v, rho * side ** 3 / n, 0)
    p.J[:] = 1.0
    sc = M.Scene(n=(grid, grid, grid), dx=dx, dt=1e-4 if not large else 5e-5, materials=[mat], max_particles=n)
    return sc, p


def config4_batched(n_scenes: int = 512, seed: int = 0xAE04):
    rng = Rng(seed)
    return [batched_scene(rng) for _ in range(n_scenes)]


def config5_request(rng: Rng):
    large = rng.scalar() < 0.05
    sc, p = batched_scene(rng, large)
    substeps = 100 + int(rng.scalar() * 1901)
    return sc, p, substeps


def tiny_scene(n_particles: int = 512, grid: int = 16, material=None, seed: int = 0xAE10, v=(0, 0, 0),
               box=(0.35, 0.6)):
    """Small physics-mode scene for parity tests."""
    rng = Rng(seed)
    mat = material if material is not None else jelly()
    lo, hi = box
    x = jittered_box(rng, (lo, lo, lo), (hi, hi, hi), n_particles)
    rho = mat.density
    p = make_particles(x, v, rho * (hi - lo) ** 3 / n_particles, 0)
    p.J[:] = 1.0
    sc = M.Scene(n=(grid, grid, grid), dx=1.0 / grid, dt=1e-4, materials=[mat], max_particles=n_particles)
    return sc, p
