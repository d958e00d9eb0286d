#!/usr/bin/env python
"""MPM particle-updates/s on B200, batched vs plain, with p50/p99 scene latency.

Default workload ("batched"): 512 independent scenes, grid per scene drawn from
{32,48,64}^3, particle count log-uniform in [2k, 64k] (9.7 M particles in all), material jelly,
snow or water, box velocities in [-1,1]^3 m/s, f32.  One bench step = one MPM substep of every
scene (radix sort by cell key, P2G, grid update, G2P), all scenes in one world: one launch of each
kernel per substep serves every scene.  The particle state (2 x 112 B x 9.7 M = 2.2 GB) exceeds
the 126 MB L2, so no flush is needed between steps.

  value            particle-updates/s of the batched world with every scene resident in HBM
                   (CUDA events on the world's stream around K substeps; max over ranks)
  batched_vs_plain the same kernels stepping one world per scene, one scene after another, over
                   every scene (device-resident and end to end)
  scene_latency_s  p50/p99 scene completion latency of a full run (200 substeps per scene, every
                   scene submitted at once) through the C ABI, batched and plain
  e2e              the metric through the public C ABI with host buffers: upload every scene from
                   pinned host memory, 200 substeps, download every scene, per call
  error_vs_fp64    per-particle position error of that run against the FP64 instantiation of the
                   same kernels after the same substeps
  roofline         the dominant kernel: algorithmic bytes / its mean event-timed duration
  cpu_baseline     the CPU restatement of the reference substep (oracle/) on this host's cores

--impl reference times that CPU restatement alone on the same scenes (the reference is Rust, and
no Rust toolchain is available to build it).  --gpus N deals a scene list of N x 512 scenes
round-robin to the ranks (weak scaling, no data-path collective).  Other workloads:
--workload snow|jelly|dam|served|tick|ck|midfield|near.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "ae-engine_b200"))

import numpy as np  # noqa: E402

# Algorithmic bytes of each kernel per particle-substep and per active grid node, for the f32
# particle state x 12, v 12, C 36, F 36, J_p 4, mass/material 4 B: P2G reads all of it (104 B);
# G2P reads x, F, J_p and the material (56 B) and writes x, v, C, F, J_p (100 B); each touches
# 16 B per active node; the grid update reads and writes 64 B per active node.  (The kernels'
# own layout moves 64 B per particle in P2G and 180 B in G2P: P2G reads an affine matrix that
# G2P folds the stress into, instead of F.)
KERNEL_BYTES = {"p2g": (104, 16), "g2p": (156, 16), "grid": (0, 64), "g2p2g": (104 + 156, 16 + 16)}


def dominant_kernel(stages):
    """The kernel the roofline is quoted on, from a world's stage times.  A world whose P2G is
    fused into G2P (physics mode, column-lane P2G) reports no stand-alone P2G: its G2P stage is the
    fused kernel, which moves the bytes of both; "g2p_kernel" times it without the snow clamp."""
    g2p = stages.get("g2p_kernel") or stages["g2p"]  # the kernel alone, without the snow clamp
    if stages["p2g"] < 0.1 * stages["g2p"]:
        return "g2p2g", g2p
    alone = {"p2g": stages["p2g"], "g2p": g2p, "grid": stages["grid"]}
    k = max(alone, key=lambda k: alone[k])
    return k, alone[k]


def substep_roofline(n_particles, active_nodes, stages, peak):
    """The whole substep against HBM with the scope's per-substep bytes: 260 B per particle (P2G
    104, G2P 156) and 80 B per active node (clear 16, P2G write 16, update 32, G2P read 16), over
    the event-timed substep of the same state as the kernel figures."""
    b = 260 * n_particles + 80 * active_nodes
    us = stages["substep"]
    ach = b / (us * 1e-6) / 1e9
    return {"substep_bytes": b, "substep_us": us, "substep_achieved": ach, "substep_frac": ach / peak}


def l2_note(n_particles):
    """How the timed region relates to the 126 MB L2: the particle state (two 112-byte copies per
    particle, read and written every substep) either exceeds it, or the scene is L2-resident."""
    mb = 2 * 112 * n_particles / 1e6
    if mb > 126:
        return "inputs larger than L2 (%.0f MB particle state), no flush" % mb
    return "inputs fit in L2 (%.1f MB particle state), no flush: an L2-resident scene" % mb


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps; default: the workload's run length in substeps (RUN_LENGTH), else 200")
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="batched", choices=["snow", "jelly", "dam", "batched", "served", "tick", "ck", "midfield", "near"])
    ap.add_argument("--ck-h", type=float, default=1.0,
                    help="ck: grid spacing (the scene scales with it); 1 takes the exact power-of-two division path")
    ap.add_argument("--e2e-reps", type=int, default=3)
    ap.add_argument("--e2e-groups", type=int, default=8,
                    help="batched workload: groups of the pipelined batch call that the headline e2e times")
    ap.add_argument("--e2e-substeps", type=int, default=None,
                    help="substeps per end-to-end call; default: the workload's run length")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 error reference run")
    ap.add_argument("--no-plain", action="store_true", help="batched: skip the plain (one world per scene) arm")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--variant", choices=["lanes", "tile", "warp_agg", "global"],
                    help="fixed P2G variant (with --block-threads and --sort-interval: no autotune)")
    ap.add_argument("--block-threads", type=int, choices=[128, 256])
    ap.add_argument("--sort-interval", type=int)
    ap.add_argument("--scenes", type=int, default=512, help="batched: number of scenes")
    ap.add_argument("--rates", default="50,100,200,500,1000,2000", help="served: Poisson arrival rates (scenes/s)")
    ap.add_argument("--served-seconds", type=float, default=1.5, help="served: arrival window per rate")
    ap.add_argument("--served-max", type=int, default=800, help="served: cap on requests per rate")
    return ap.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.tmp = None

    def start(self):
        try:
            self.tmp = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.tmp, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except Exception:
            self.proc.kill()
        self.tmp.flush()
        self.tmp.seek(0)
        rows = [r.split(",") for r in self.tmp.read().strip().splitlines() if r.strip()]
        os.unlink(self.tmp.name)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
                for k, nm in enumerate(names):
                    if r[5 + k].strip().lower() == "active":
                        reasons.add(nm)
            except Exception:
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "samples": len(sm), "reasons": sorted(reasons)}


def dist_setup(args):
    world_size = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world_size > 1:
        import datetime

        import torch
        import torch.distributed as dist

        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
        pg = dist
    return rank, local, world_size, pg


def max_over_ranks(pg, x: float) -> float:
    if pg is None:
        return x
    import torch

    dev = "cuda" if pg.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(pg, x: float) -> float:
    if pg is None:
        return x
    import torch

    dev = "cuda" if pg.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.SUM)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


def shard(items, rank: int, world_size: int):
    """Scenes of a batched workload dealt round-robin to ranks (scenes are independent)."""
    return list(items[rank::world_size])


def workload(name: str, rank: int, n_scenes: int, world_size: int = 1):
    """Scenes of a workload for one rank.  Single-scene workloads run one replica per rank (seed
    offset by rank); the batched workload draws one list of world_size x n_scenes scenes and deals
    it round-robin, so every rank steps n_scenes scenes of one seeded population."""
    import ae_mpm_scenes as S

    if name == "served":
        return [], [], {"workload": "served"}
    single = {"parallelism": "replicas" if world_size > 1 else "single GPU"}
    if name == "snow":
        sc, p = S.config2_snow(0xAE02 + 1000 * rank)
        single["l2"] = l2_note(p.n)
        return [sc], [p], dict({"workload": "snow collision 128^3, 1048576 Stomakhin snow particles, dt 5e-5",
                                "grid": 128, "particles": p.n}, **single)
    if name == "jelly":
        sc, p = S.config1_jelly(0xAE01 + 1000 * rank)
        single["l2"] = l2_note(p.n)
        return [sc], [p], dict({"workload": "jelly 64^3, 32768 neo-Hookean particles, dt 1e-4", "grid": 64,
                                "particles": p.n}, **single)
    if name == "dam":
        sc, p = S.config3_dam(0xAE03 + 1000 * rank)
        single["l2"] = l2_note(p.n)
        return [sc], [p], dict({"workload": "mixed dam break 256^3, 8388608 particles (60% fluid, 25% jelly, 15% snow)",
                                "grid": 256, "particles": p.n}, **single)
    pairs = shard(S.config4_batched(n_scenes * world_size, 0xAE04), rank, world_size)
    n = int(sum(b.n for _, b in pairs))
    return [a for a, _ in pairs], [b for _, b in pairs], {
        "workload": "%d independent scenes, grids {32,48,64}^3, 2k-64k particles, jelly/snow/water, 200-substep runs"
                    % n_scenes, "scenes": len(pairs), "particles": n, "l2": l2_note(n),
        "parallelism": "%d scenes per GPU, dealt round-robin from one list of %d" % (len(pairs), n_scenes * world_size)
        if world_size > 1 else "single GPU"}


def fixed_options(args) -> dict:
    """Execution options fixed on the command line (--variant, --block-threads, --sort-interval);
    any of them turns the autotuner off."""
    import ae_mpm as M

    fixed = {}
    if args.variant:
        fixed["p2g_variant"] = {"tile": M.P2G_TILE, "warp_agg": M.P2G_WARP_AGG, "global": M.P2G_GLOBAL,
                                "lanes": M.P2G_LANES}[args.variant]
    if args.block_threads:
        fixed["block_threads"] = args.block_threads
    if args.sort_interval:
        fixed["sort_interval"] = args.sort_interval
    return fixed


def hold_stream(torch, stream, ms: float = 10.0):
    """Queues a bounded busy kernel (torch.cuda._sleep, a fixed number of clock cycles) on `stream`
    ahead of a timed region, so that the region's work is all submitted before the device reaches
    its start event: a host scheduling gap during submission then does not count as device time."""
    with torch.cuda.stream(stream):
        torch.cuda._sleep(int(ms * 1e-3 * 1.965e9))


def timed_range(torch, begin: bool):
    """NVTX range "timed" around the timed substeps, so a profiler can select exactly their launches
    (ncu --nvtx --nvtx-include "timed/")."""
    if begin:
        torch.cuda.nvtx.range_push("timed")
    else:
        torch.cuda.nvtx.range_pop()


def traffic_record(workload_name: str, kernel: str):
    """DRAM bytes per launch of `kernel` (dram__bytes_read.sum + dram__bytes_write.sum) from the
    committed ncu capture of this workload, with the file it came from; None if not captured."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            tr = json.load(f)
    except Exception:
        return None
    rec = tr.get(workload_name, {})
    if kernel not in rec:
        return None
    return {"bytes": rec[kernel], "source": "ncu capture, %s" % rec.get("source", "profiles/traffic.json")}


def cpu_scenes_rate(scenes, parts, substeps: int, threads: int | None = None, inplace: bool = False):
    """The CPU restatement over a set of scenes: each scene stepped by one host thread (the
    reference's serial path below 50 000 particles; its rayon path above uses the same arithmetic),
    the scenes spread over every host core.  Returns (particle-updates/s, threads, description)."""
    import concurrent.futures as cf

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    threads = threads or os.cpu_count() or 1
    qs = parts if inplace else [p.copy() for p in parts]
    order = sorted(range(len(parts)), key=lambda i: -parts[i].n)  # largest first: even finish
    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(threads) as ex:
        list(ex.map(lambda i: O.run(scenes[i], qs[i], substeps, threads=1), order))
    dt = time.perf_counter() - t0
    n = sum(p.n for p in parts)
    return n * substeps / dt, threads, ("all %d scenes (%d particles), %d substeps each, scenes spread over %d "
                                        "threads, %.1f s" % (len(parts), n, substeps, threads, dt))


def active_nodes(scene, p) -> int:
    """Distinct grid nodes covered by particle stencils (3x3x3 from the base node)."""
    X = (p.pos.astype(np.float64) - np.asarray(scene.origin)) / scene.dx
    base = np.floor(X - 0.5).astype(np.int64)
    n = np.asarray(scene.n, np.int64)
    cells = np.unique((base[:, 2] * n[1] + base[:, 1]) * n[0] + base[:, 0])
    bz, r = np.divmod(cells, n[0] * n[1])
    by, bx = np.divmod(r, n[0])
    nodes = set()
    out = []
    for dz in range(3):
        for dy in range(3):
            for dxx in range(3):
                out.append(((bz + dz) * n[1] + (by + dy)) * n[0] + (bx + dxx))
    nodes = np.unique(np.concatenate(out))
    return int(nodes.size)


def cpu_rate(scene, p, substeps: int, threads: int) -> tuple[float, float]:
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    q = p.copy()
    t0 = time.perf_counter()
    O.run(scene, q, substeps, threads=threads)
    dt = time.perf_counter() - t0
    return p.n * substeps / dt, dt


def run_reference(args, rank, pg):
    """CPU restatement of the reference substep on this host's cores, same workload and metric."""
    if args.workload == "tick":
        return run_tick(args, rank, 0, 1, pg, reference=True)
    if args.workload == "ck":
        return run_ck(args, rank, 0, 1, pg, reference=True)
    if args.workload == "midfield":
        return run_midfield(args, rank, 0, 1, pg, reference=True)
    if args.workload == "near":
        return run_near(args, rank, 0, 1, pg, reference=True)
    if rank != 0:
        return
    scenes, parts, cfg = workload(args.workload, 0, args.scenes, args.gpus)
    base = {"impl": "reference", "metric": "MPM particle-updates/s", "unit": "particle-updates/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded SplitMix64)",
            "config": cfg}
    if args.workload == "batched":
        # the reference steps one scene per call (simulation.rs:570-607); here every step is one
        # substep of every scene, the scenes spread over all host threads, one scene per thread
        threads = os.cpu_count() or 1
        qs = [p.copy() for p in parts]
        dt = 0.0
        for k in range(args.warmup + args.steps):
            rate, _, _ = cpu_scenes_rate(scenes, qs, 1, threads, inplace=True)
            if k >= args.warmup:
                dt += sum(p.n for p in parts) / rate
        value = sum(p.n for p in parts) * args.steps / dt
        desc = "all %d scenes (%d particles), 1 substep of every scene per step, scenes spread over %d threads" % (
            len(parts), sum(p.n for p in parts), threads)
        print(json.dumps(dict(base, value=value, ms_per_step=1000.0 * dt / args.steps,
                              cpu_baseline={"value": value, "unit": "particle-updates/s", "cores": threads,
                                            "kind": "port", "sample": desc},
                              e2e={"value": value, "unit": "particle-updates/s", "h2d_bytes_per_step": 0,
                                   "d2h_bytes_per_step": 0})), flush=True)
        return
    scene, p = scenes[0], parts[0]
    threads = os.cpu_count() or 1
    # Each step is one substep of the whole scene when the K + W steps fit in about four minutes.
    # A substep also clears and updates the whole grid, whatever the particle count, so a subset of
    # the particles would understate the reference's throughput; only a run too long for the
    # budget falls back to a subset (the first particles in scene order), sized from the timing
    # of one whole-scene substep.
    _, t_whole = cpu_rate(scene, p, 1, threads)
    budget_s = 240.0 / max(1, args.steps + args.warmup)
    n_sample = p.n if t_whole <= budget_s else max(1, int(p.n * budget_s / t_whole))
    sample = p.subset(np.arange(n_sample)) if n_sample < p.n else p
    for _ in range(args.warmup):
        cpu_rate(scene, sample, 1, threads)
    # the substeps alone (each call's input copy stays outside its timer)
    dt = sum(cpu_rate(scene, sample, 1, threads)[1] for _ in range(args.steps))
    value = sample.n * args.steps / dt
    desc = ("the whole scene (%d particles), 1 substep per step" % p.n if sample.n == p.n else
            "%d of %d particles (first in scene order), 1 substep per step" % (sample.n, p.n))
    print(json.dumps(dict(base, value=value, ms_per_step=1000.0 * dt / args.steps,
                          cpu_baseline={"value": value, "unit": "particle-updates/s", "cores": threads,
                                        "kind": "port", "sample": desc},
                          e2e={"value": value, "unit": "particle-updates/s", "h2d_bytes_per_step": 0,
                               "d2h_bytes_per_step": 0})), flush=True)


# ---------------------------------------------------------------------------------------------
# "tick": the engine's particle passes around the substep on one frame that reclassifies: LOD
# classification, far-field update and coarse temperature field (simulation.rs:495-532, 612-679,
# 877-966), then the MpssBuffer housekeeping (ae_engine/src/lib.rs:347-358), over a 1M-particle
# MpssBuffer.  Synthetic: a 1.6 km cube around the player with 3% of the particles within 40 m
# (so the 10 000 near cap binds), 95% active, materials wood/water/concrete/iron.
# ---------------------------------------------------------------------------------------------
TICK_N = 1 << 20
TICK = dict(near=50.0, mid=200.0, max_near=10000, coarse_n=16, coarse_dx=50.0, far_dt=1.0, bounds=750.0,
            min_temp=10.0, max_temp=8000.0)


def tick_population(n, seed):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(-800, 800, (n, 3))
    k = n * 3 // 100
    pos[:k] = rng.uniform(-40, 40, (k, 3))
    pos = pos[rng.permutation(n)].astype(np.float32)
    return {"pos": pos, "vel": rng.normal(0, 3, (n, 3)).astype(np.float32),
            "temp": rng.uniform(250, 2500, n).astype(np.float32), "mass": rng.uniform(0.5, 2, n).astype(np.float32),
            "active": (rng.uniform(size=n) > 0.05).astype(np.uint8), "phase": np.zeros(n, np.uint8),
            "mat": rng.integers(0, 4, n).astype(np.uint16)}


def tick_cfg(n):
    return {"workload": "engine tick around the substep: LOD reclassify + far-field update + coarse field + "
                        "MpssBuffer housekeeping, %d particles, near cap %d, coarse field %d^3"
                        % (n, TICK["max_near"], TICK["coarse_n"]),
            "particles": n, "l2": "L2 flushed between ticks (256 MB write, outside the timed events): the tick's "
                                  "36 B/particle would otherwise stay L2-resident"}


def tick_oracle(d, player, origin):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    near, mid, far = O.lod_classify(d["pos"], d["active"], player, TICK["near"], TICK["mid"], TICK["max_near"])
    O.far_field_update(d["pos"], d["vel"], d["temp"], far, d["coarse"], TICK["coarse_dx"], origin, TICK["far_dt"])
    O.coarse_field_update(d["pos"], d["mass"], d["temp"], d["active"], np.sort(near), d["coarse"], TICK["coarse_dx"],
                          origin, TICK["far_dt"])
    b = TICK["bounds"]
    O.mpss_housekeeping(d["pos"], d["vel"], d["temp"], d["phase"], d["mat"], d["active"], [-b] * 3, [b] * 3,
                        TICK["min_temp"], TICK["max_temp"], 7)


# The mid-field call of the engine tick (simulation.rs:598-607 -> mpm_step_velocity_only_parallel): the
# reference's own measurement is 490 045 mid particles of a 1M-particle MpssBuffer on a 32^3 grid, one
# substep of mid_dt = 12 / 60 s, in 32-47 ms on its CPU (ARCHITECTURE_V7_CRITIQUE.md:542-549).
MID = dict(n_near=10000, n_mid=490045, n_far=500010, near=50.0, mid=200.0, far=400.0, grid=32, dx=12.5,
           origin=-200.0, total_dt=0.2)
MID_PUBLISHED = MID["n_mid"] / 0.032  # the best of the quoted 32-47 ms, as particle-updates/s


def midfield_setup(seed):
    """A 1 000 055-particle buffer: near, mid and far shells around the player at the origin, in shuffled
    buffer order; the mid indices ascending, as the LOD scan builds them."""
    import ae_mpm as M

    rng = np.random.default_rng(seed)

    def shell(n, r0, r1):
        d = rng.normal(size=(n, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        return d * (rng.uniform(r0 ** 3, r1 ** 3, n) ** (1.0 / 3.0))[:, None]

    pos = np.concatenate([shell(MID["n_near"], 0.0, MID["near"]), shell(MID["n_mid"], MID["near"], MID["mid"]),
                          shell(MID["n_far"], MID["mid"], MID["far"])])
    cls = np.repeat([0, 1, 2], [MID["n_near"], MID["n_mid"], MID["n_far"]])
    perm = rng.permutation(pos.shape[0])
    pos, cls = pos[perm], cls[perm]
    p = M.Particles.empty(pos.shape[0])
    p.pos[:] = pos.astype(np.float32)
    p.vel[:] = rng.normal(0.0, 3.0, p.pos.shape).astype(np.float32)
    p.mass[:] = 1.0
    idx = np.flatnonzero(cls == 1).astype(np.uint64)
    n = MID["grid"]
    grid = M.Grid(n, n, n, MID["dx"], (MID["origin"],) * 3)
    cfg = M.Config(grid_dx=MID["dx"], grid_size=(n, n, n), substeps=1, gravity=(0, -9.81, 0), damping=0.995)
    return p, idx, grid, cfg


def midfield_cfg():
    return {"workload": "mid-field velocity-only MPM call (mpm_step_velocity_only_parallel): %d mid particles of a "
                        "%d-particle buffer, %d^3 grid, dx %.1f m, 1 substep of %.1f s"
                        % (MID["n_mid"], MID["n_near"] + MID["n_mid"] + MID["n_far"], MID["grid"], MID["dx"],
                           MID["total_dt"]),
            "particles": MID["n_mid"], "grid": MID["grid"],
            "baseline": "reference's own CPU measurement of this call: 32-47 ms (vs_baseline uses 32 ms)"}


def run_midfield(args, rank, local, world_size, pg, reference=False):
    metric, unit = "mid-field MPM particle-updates/s", "particle-updates/s"
    p, idx, grid, mcfg = midfield_setup(0xAE06 + 1000 * rank)
    n = int(idx.size)
    cfg = midfield_cfg()
    steps = max(1, min(args.steps, 50))
    if reference:  # the CPU restatement of mpm_step_velocity_only_parallel on all host threads
        if rank != 0:
            return
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O

        threads = os.cpu_count() or 1
        for _ in range(max(1, min(args.warmup, 3))):
            O.step_velocity_only_parallel(p, grid, mcfg, MID["total_dt"], idx, threads=threads)
        t0 = time.perf_counter()
        for _ in range(steps):
            O.step_velocity_only_parallel(p, grid, mcfg, MID["total_dt"], idx, threads=threads)
        dt = time.perf_counter() - t0
        value = n * steps / dt
        print(json.dumps({"impl": "reference", "metric": metric, "value": value, "unit": unit, "n_gpus": args.gpus,
                          "steps": steps, "warmup": args.warmup, "ms_per_step": 1000.0 * dt / steps,
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": value / MID_PUBLISHED,
                          "dtype": "f32", "data": "synthetic (seeded numpy)", "config": cfg,
                          "cpu_baseline": {"value": value, "unit": unit, "cores": threads, "kind": "port",
                                           "sample": "the whole call, %d calls" % steps},
                          "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}),
              flush=True)
        return
    import torch

    import ae_mpm as M

    ctx = M.Context(local)
    # end to end: the drop-in call on the host buffer, as the engine makes it (host gather, upload, substep,
    # download, host scatter); timed on the host clock, since the host work is part of the call
    for _ in range(max(args.warmup, 3)):
        ctx.step_velocity_only_parallel(p, grid, mcfg, MID["total_dt"], idx)
    clocks = Clocks(local)
    barrier(pg)
    torch.cuda.synchronize(local)
    clocks.start()
    time.sleep(0.3)
    calls = []
    for _ in range(steps):
        t0 = time.perf_counter()
        ctx.step_velocity_only_parallel(p, grid, mcfg, MID["total_dt"], idx)
        calls.append(time.perf_counter() - t0)
    clk = clocks.stop()
    t_call = max_over_ranks(pg, statistics.median(calls))
    e2e_value = n * world_size / t_call
    # ascending indices selecting a quarter or more of the buffer: the call copies the buffer's position,
    # velocity and mass arrays whole plus the index list in, and position and velocity out
    cap = p.n
    h2d, d2h = 28 * cap + 8 * n, 24 * cap

    # device-resident: the same substep in a velocity-only world holding the mid particles
    sub = p.subset(idx.astype(np.int64))
    sc = M.Scene(n=(MID["grid"],) * 3, dx=MID["dx"], dt=MID["total_dt"], materials=[M.material()],
                 mode=M.MODE_VELOCITY_ONLY, origin=(MID["origin"],) * 3, gravity=(0.0, -9.81, 0.0), wall_margin=0,
                 damping=0.995, wall_origin=1, max_particles=n)
    world = M.World(ctx, [sc], M.exec_opts())
    world.upload(0, sub)
    world.step(max(args.warmup, 3))
    world.sync()
    stages = world.stage_times(STAGE_SUBSTEPS)
    graph_warm(world)
    stream = torch.cuda.ExternalStream(world.stream(), device=local)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(pg)
    torch.cuda.synchronize(local)
    hold_stream(torch, stream)
    timed_range(torch, True)
    e0.record(stream)
    world.step(args.steps)
    e1.record(stream)
    e1.synchronize()
    timed_range(torch, False)
    world.sync(raise_on_error=False)
    launches = world.launches()
    ms = max_over_ranks(pg, e0.elapsed_time(e1))
    value = n * world_size * args.steps / (ms / 1e3)
    world.close()

    cpu = None
    if rank == 0 and world_size == 1 and not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O

        threads = os.cpu_count() or 1
        q = p.copy()
        O.step_velocity_only_parallel(q, grid, mcfg, MID["total_dt"], idx, threads=threads)
        t0 = time.perf_counter()
        O.step_velocity_only_parallel(q, grid, mcfg, MID["total_dt"], idx, threads=threads)
        dt = time.perf_counter() - t0
        cpu = {"value": n / dt, "unit": unit, "cores": threads, "kind": "port",
               "sample": "one whole call (%d mid particles), %.2f s" % (n, dt)}
    if rank == 0:
        print(json.dumps({
            "metric": metric, "value": value, "unit": unit, "n_gpus": world_size, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": value / MID_PUBLISHED, "dtype": "f32", "data": "synthetic (seeded numpy)",
            "config": dict(cfg, parallelism="replicas" if world_size > 1 else "single GPU",
                           l2="the mid particles' state (%.0f MB) exceeds L2" % (224 * n / 1e6)),
            "stages_us": {k: round(v, 2) for k, v in stages.items()},
            "e2e": {"value": e2e_value, "unit": unit, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms_per_step": 1000.0 * t_call, "calls": steps, "timer": "host clock around each call",
                    "vs_baseline": e2e_value / MID_PUBLISHED},
            "cpu_baseline": cpu, "gpu_launches": launches, "clocks": clk}), flush=True)
    ctx.close()


# The engine's near-field call (simulation.rs:566-581 -> mpm_step_parallel_with_grid): the near set of the
# same buffer (10 000 particles within 50 m, the LOD cap), the engine's 4-material table
# (simulation.rs:251-294), a 64^3 grid of dx 1.6 m centred on the player (:218-226, :545-549), one
# substep of the frame's dt.
NEAR = dict(grid=64, dx=1.6, dt=1.0 / 60.0)


def near_setup(seed):
    import ae_mpm as M

    p, _, _, _ = midfield_setup(seed)
    r = np.linalg.norm(p.pos.astype(np.float64), axis=1)
    idx = np.flatnonzero(r < MID["near"]).astype(np.uint64)
    rng = np.random.default_rng(seed + 1)
    p.mat[:] = rng.integers(0, 4, p.n).astype(np.uint16)
    mats = [M.material(young_modulus=1.0e6, poisson_ratio=0.3, yield_stress=1.0e4, hardening=0.01, density=1000.0,
                       friction_angle=35.0, cohesion=0.0),
            M.material(young_modulus=2.0e6, poisson_ratio=0.45, yield_stress=0.0, hardening=0.0, density=1000.0,
                       friction_angle=0.0, cohesion=0.0),
            M.material(young_modulus=5.0e7, poisson_ratio=0.3, yield_stress=0.0, hardening=0.0, density=1600.0,
                       friction_angle=35.0, cohesion=0.0),
            M.material(young_modulus=2.0e11, poisson_ratio=0.3, yield_stress=2.5e8, hardening=0.01, density=7850.0,
                       friction_angle=0.0, cohesion=0.0)]
    models = [M.NEO_HOOKEAN, M.NEWTONIAN_FLUID, M.DRUCKER_PRAGER, M.VON_MISES]
    n = NEAR["grid"]
    half = n * NEAR["dx"] / 2
    grid = M.Grid(n, n, n, NEAR["dx"], (-half,) * 3)
    cfg = M.Config(grid_dx=NEAR["dx"], grid_size=(n, n, n), substeps=1, gravity=(0, -9.81, 0), damping=0.995)
    return p, idx, grid, cfg, mats, models


def run_near(args, rank, local, world_size, pg, reference=False):
    metric, unit = "near-field MPM particle-updates/s", "particle-updates/s"
    p, idx, grid, ncfg, mats, models = near_setup(0xAE07 + 1000 * rank)
    n = int(idx.size)
    cfg = {"workload": "near-field MPM call (mpm_step_parallel_with_grid): %d near particles of a %d-particle buffer, "
                       "the engine's 4-material table, %d^3 grid, dx %.1f m, 1 substep of 1/60 s"
                       % (n, p.n, NEAR["grid"], NEAR["dx"]),
           "particles": n, "grid": NEAR["grid"]}
    steps = max(1, min(args.steps, 100))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    if reference:  # the CPU restatement of the call (below 50 000 indices the reference's serial path)
        if rank != 0:
            return
        import oracle as O

        for _ in range(max(1, min(args.warmup, 3))):
            O.step_parallel_with_grid(p, grid, ncfg, mats, models, NEAR["dt"], idx)
        t0 = time.perf_counter()
        for _ in range(steps):
            O.step_parallel_with_grid(p, grid, ncfg, mats, models, NEAR["dt"], idx)
        dt = time.perf_counter() - t0
        value = n * steps / dt
        print(json.dumps({"impl": "reference", "metric": metric, "value": value, "unit": unit, "n_gpus": args.gpus,
                          "steps": steps, "warmup": args.warmup, "ms_per_step": 1000.0 * dt / steps,
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                          "data": "synthetic (seeded numpy)", "config": cfg,
                          "cpu_baseline": {"value": value, "unit": unit, "cores": 1, "kind": "port",
                                           "sample": "the whole call, %d calls" % steps},
                          "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}),
              flush=True)
        return
    import torch

    import ae_mpm as M

    ctx = M.Context(local)
    for _ in range(max(args.warmup, 3)):
        ctx.step_parallel_with_grid(p, grid, ncfg, mats, models, NEAR["dt"], idx)
    clocks = Clocks(local)
    barrier(pg)
    torch.cuda.synchronize(local)
    clocks.start()
    time.sleep(0.3)
    calls = []
    for _ in range(steps):
        t0 = time.perf_counter()
        ctx.step_parallel_with_grid(p, grid, ncfg, mats, models, NEAR["dt"], idx)
        calls.append(time.perf_counter() - t0)
    clk = clocks.stop()
    t_call = max_over_ranks(pg, statistics.median(calls))
    value = n * world_size / t_call
    staged = 106 * n  # a sparse index list: every field of the selected particles is gathered and staged
    cpu = None
    if rank == 0 and world_size == 1 and not args.no_cpu_baseline:
        import oracle as O

        q = p.copy()
        O.step_parallel_with_grid(q, grid, ncfg, mats, models, NEAR["dt"], idx)
        t0 = time.perf_counter()
        reps = 5
        for _ in range(reps):
            O.step_parallel_with_grid(q, grid, ncfg, mats, models, NEAR["dt"], idx)
        dt = (time.perf_counter() - t0) / reps
        cpu = {"value": n / dt, "unit": unit, "cores": 1, "kind": "port",
               "sample": "%d whole calls (%d near particles, the serial path), %.1f ms each" % (reps, n, 1e3 * dt)}
    if rank == 0:
        print(json.dumps({
            "metric": metric, "value": value, "unit": unit, "n_gpus": world_size, "steps": steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * t_call, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded numpy)",
            "config": dict(cfg, parallelism="replicas" if world_size > 1 else "single GPU",
                           timer="host clock around each call: the call is the unit the engine waits on"),
            "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": staged, "d2h_bytes_per_step": staged,
                    "ms_per_step": 1000.0 * t_call, "calls": steps},
            "cpu_baseline": cpu, "clocks": clk}), flush=True)
    ctx.close()


def run_tick(args, rank, local, world_size, pg, reference=False):
    import ctypes as C

    n = TICK_N
    d = tick_population(n, 0xAE05 + 1000 * rank)
    player = np.zeros(3, np.float32)
    origin = (player - np.float32(TICK["coarse_n"] * TICK["coarse_dx"] / 2)).astype(np.float32)
    d["coarse"] = np.full(TICK["coarse_n"] ** 3, 288.15, np.float32)
    cfg = tick_cfg(n)
    metric, unit = "engine-tick particles/s", "particles/s"
    if reference:  # the CPU restatement on this host (single thread, as the reference's serial passes)
        if rank != 0:
            return
        for _ in range(max(1, args.warmup)):
            tick_oracle({k: v.copy() for k, v in d.items()}, player, origin)
        steps = max(1, min(args.steps, 20))
        t0 = time.perf_counter()
        for _ in range(steps):
            tick_oracle(d, player, origin)
        dt = time.perf_counter() - t0
        value = n * steps / dt
        print(json.dumps({"impl": "reference", "metric": metric, "value": value, "unit": unit, "n_gpus": args.gpus,
                          "steps": steps, "warmup": args.warmup, "ms_per_step": 1000.0 * dt / steps,
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                          "data": "synthetic (seeded numpy)", "config": cfg,
                          "cpu_baseline": {"value": value, "unit": unit, "cores": 1, "kind": "port",
                                           "sample": "the whole %d-particle tick" % n},
                          "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}),
              flush=True)
        return
    import torch

    import ae_mpm as M

    ctx = M.Context(local)
    lib, h = ctx.lib, ctx.h
    dev = {k: torch.from_numpy(v.copy()).cuda(local) for k, v in d.items()}
    outs = [torch.empty(n, dtype=torch.int64, device="cuda:%d" % local) for _ in range(3)]
    cnt = [C.c_uint64(0) for _ in range(3)]
    pl, og = player.copy(), origin.copy()
    blo = np.full(3, -TICK["bounds"], np.float32)
    bhi = np.full(3, TICK["bounds"], np.float32)
    trans = C.c_uint32(0)

    def tick_device():
        ctx.check(lib.ae_mpm_lod_classify(h, dev["pos"].data_ptr(), dev["active"].data_ptr(), n, pl.ctypes.data,
                                          TICK["near"], TICK["mid"], TICK["max_near"], outs[0].data_ptr(),
                                          C.byref(cnt[0]), outs[1].data_ptr(), C.byref(cnt[1]), outs[2].data_ptr(),
                                          C.byref(cnt[2])))
        ctx.check(lib.ae_mpm_far_field_update(h, dev["pos"].data_ptr(), dev["vel"].data_ptr(), dev["temp"].data_ptr(),
                                              n, outs[2].data_ptr(), cnt[2].value, dev["coarse"].data_ptr(),
                                              TICK["coarse_n"], TICK["coarse_dx"], og.ctypes.data, TICK["far_dt"]))
        ctx.check(lib.ae_mpm_coarse_field_update(h, dev["pos"].data_ptr(), dev["mass"].data_ptr(),
                                                 dev["temp"].data_ptr(), dev["active"].data_ptr(), n,
                                                 outs[0].data_ptr(), cnt[0].value, dev["coarse"].data_ptr(),
                                                 TICK["coarse_n"], TICK["coarse_dx"], og.ctypes.data, TICK["far_dt"]))
        ctx.check(lib.ae_mpm_mpss_housekeeping(h, dev["pos"].data_ptr(), dev["vel"].data_ptr(), dev["temp"].data_ptr(),
                                               dev["phase"].data_ptr(), dev["mat"].data_ptr(), dev["active"].data_ptr(),
                                               n, blo.ctypes.data, bhi.ctypes.data, TICK["min_temp"],
                                               TICK["max_temp"], 7, C.byref(trans)))

    for _ in range(max(args.warmup, 3)):
        tick_device()
    flush = torch.empty(64 << 20, dtype=torch.float32, device="cuda:%d" % local)  # 256 MB > L2
    clocks = Clocks(local)
    barrier(pg)
    torch.cuda.synchronize(local)
    clocks.start()
    time.sleep(0.3)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    ms = 0.0
    for _ in range(args.steps):
        flush.zero_()
        e0.record()
        tick_device()
        e1.record()
        e1.synchronize()
        ms += e0.elapsed_time(e1)
    clk = clocks.stop()
    ms = max_over_ranks(pg, ms)
    value = n * world_size * args.steps / (ms / 1e3)
    n_near, n_far = cnt[0].value, cnt[2].value
    capped = n_near >= TICK["max_near"]
    # kernels per tick: classify 3 (7 with the cap: radix select, second partition), far 1, coarse 12
    # (cell keys, 2-pass sort, gather, runs, sums, relaxation, diffusion), housekeeping 1
    launches = args.steps * ((7 if capped else 3) + 1 + 12 + 1)
    # algorithmic bytes per tick: classify reads pos + active twice and writes one 8-byte index per
    # particle; far: index 8 + pos 12 read, pos.y, vel.y, temperature read and written; coarse: near
    # index 8, pos 12, mass 4, temperature 4, active 1; housekeeping: pos, vel, temperature and
    # phase read and written, material and active read (61 B)
    alg = 34 * n + 40 * n_far + 29 * n_near + 61 * n
    achieved = alg / (ms / args.steps * 1e-3) / 1e9
    peak, peak_kind = peaks()
    # end to end: the same tick through the C ABI on host (MpssBuffer) arrays in pinned memory; the
    # library stages them to the device and back inside every call
    torch_of = {np.float32: torch.float32, np.uint8: torch.uint8, np.uint16: torch.int16, np.uint64: torch.int64}
    pinned_keep = []

    def pinned(a):
        t = torch.empty(a.shape, dtype=torch_of[a.dtype.type], pin_memory=True)
        pinned_keep.append(t)
        v = t.numpy().view(a.dtype)
        v[...] = a
        return v

    hd = {k: pinned(v) for k, v in d.items()}
    houts = [pinned(np.zeros(n, np.uint64)) for _ in range(3)]
    hcnt = [C.c_uint64(0) for _ in range(3)]

    def tick_host():
        ctx.check(lib.ae_mpm_lod_classify(h, hd["pos"].ctypes.data, hd["active"].ctypes.data, n, pl.ctypes.data,
                                          TICK["near"], TICK["mid"], TICK["max_near"], houts[0].ctypes.data,
                                          C.byref(hcnt[0]), houts[1].ctypes.data, C.byref(hcnt[1]),
                                          houts[2].ctypes.data, C.byref(hcnt[2])))
        ctx.check(lib.ae_mpm_far_field_update(h, hd["pos"].ctypes.data, hd["vel"].ctypes.data, hd["temp"].ctypes.data,
                                              n, houts[2].ctypes.data, hcnt[2].value, hd["coarse"].ctypes.data,
                                              TICK["coarse_n"], TICK["coarse_dx"], og.ctypes.data, TICK["far_dt"]))
        ctx.check(lib.ae_mpm_coarse_field_update(h, hd["pos"].ctypes.data, hd["mass"].ctypes.data,
                                                 hd["temp"].ctypes.data, hd["active"].ctypes.data, n,
                                                 houts[0].ctypes.data, hcnt[0].value, hd["coarse"].ctypes.data,
                                                 TICK["coarse_n"], TICK["coarse_dx"], og.ctypes.data, TICK["far_dt"]))
        ctx.check(lib.ae_mpm_mpss_housekeeping(h, hd["pos"].ctypes.data, hd["vel"].ctypes.data, hd["temp"].ctypes.data,
                                               hd["phase"].ctypes.data, hd["mat"].ctypes.data,
                                               hd["active"].ctypes.data, n, blo.ctypes.data, bhi.ctypes.data,
                                               TICK["min_temp"], TICK["max_temp"], 7, C.byref(trans)))

    tick_host()  # warm: staging buffers
    e2e_steps = max(1, min(args.steps, 20))
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        tick_host()
    e2e_dt = time.perf_counter() - t0
    # bytes copied by the library's host paths: classify (pos, active in; the three lists out), far
    # field (whole pos, vel, temperature and the far list when at least a quarter of the particles
    # are far, else the gathered far particles), coarse field (the gathered near particles and the
    # field in, the field out), housekeeping (pos, vel, temperature, phase, material, active in;
    # pos, vel, temperature, phase out)
    cells = TICK["coarse_n"] ** 3
    far_in, far_out = (28 * n + 8 * n_far + 4 * cells, 28 * n) if 4 * n_far >= n else (28 * n_far + 4 * cells,
                                                                                        28 * n_far)
    h2d = 13 * n + far_in + 21 * n_near + 4 * cells + 32 * n
    d2h = 8 * n + far_out + 4 * cells + 29 * n
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        t0 = time.perf_counter()
        tick_oracle({k: v.copy() for k, v in d.items()}, player, origin)
        cdt = time.perf_counter() - t0
        cpu = {"value": n / cdt, "unit": unit, "cores": 1, "kind": "port", "sample": "one whole %d-particle tick" % n}
    if rank == 0:
        print(json.dumps({
            "metric": metric, "value": value, "unit": unit, "n_gpus": world_size, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded numpy)",
            "config": dict(cfg, parallelism="replicas" if world_size > 1 else "single GPU"),
            "roofline": {"bound": "hbm", "kernel": "tick (all passes)", "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "traffic": None, "peak_kind": peak_kind,
                         "algorithmic_bytes": alg},
            "tick_counts": {"near": n_near, "mid": cnt[1].value, "far": n_far, "phase_transitions": trans.value},
            "e2e": {"value": n * e2e_steps / e2e_dt, "unit": unit, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_per_step": 1000.0 * e2e_dt / e2e_steps,
                    "host_memory": "pinned"},
            "cpu_baseline": cpu, "gpu_launches": launches, "clocks": clk}), flush=True)


# "ck": CK-MPM (ae_compute/src/ck_mpm.rs, CkMpmSolver::step) on an elastic block: 128^3 particles
# on a jittered lattice at half the cell size (8 per cell, in lattice order as the reference's
# tests add them) in a 128^3 grid of h = 1 m, falling at 1 m/s; E 1e5, nu 0.3, density 1000,
# dt 5e-3 (0.05 of the elastic CFL limit).  At h = 1 the kernel's weights sum to ~1 over a node
# stencil, so the solver stays far below its 50 m/s speed cap; at the reference's default
# h = 0.05 the weights sum to ~6000 and every moving particle runs at the cap.
CK_SIDE = 128
CK_E2E_STEPS = 200  # steps per host call in the end-to-end leg (the reference's longest test runs 200-300)
# algorithmic bytes per particle-step of the particle kernel: the 104-byte record read, the 96
# bytes that change (position, velocity, affine matrix, deformation gradient) written
CK_BYTES_PER_PARTICLE = 104 + 96


def ck_scene(seed=0xC4, h=1.0):
    import ae_mpm as M

    grid_n = 128
    rng = np.random.default_rng(seed)
    g = np.stack(np.meshgrid(*[np.arange(CK_SIDE)] * 3, indexing="ij"), -1).reshape(-1, 3)
    spacing = 0.5 * h
    pos = np.array([32.0, 40.0, 32.0]) * h + (g + rng.uniform(0.25, 0.75, g.shape)) * spacing
    vel = np.zeros_like(pos)
    vel[:, 1] = -1.0
    vol = spacing ** 3
    p = M.ck_particles(pos, 1000.0 * vol, vol, velocity=vel + rng.normal(0, 0.05, pos.shape))
    cfg = M.ck_config(dt=5e-3, grid_n=grid_n, grid_h=h, bounds_min=(0, 0, 0), bounds_max=(128 * h,) * 3)
    n = p.shape[0]
    info = {"workload": "CK-MPM elastic block: %d particles (128^3 jittered lattice, 8 per cell), 128^3 grid "
                        "h=%g, dt 5e-3, E 1e5, nu 0.3, falling at 1 m/s" % (n, h),
            "particles": n, "grid_n": grid_n,
            "l2": "inputs larger than L2 (%.0f MB of particle records), no flush" % (104 * n / 1e6)}
    return p, cfg, info


def ck_oracle_rate(p, cfg, steps):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    q = p.copy()
    t0 = time.perf_counter()
    O.ck_step(q, cfg, steps)
    return p.shape[0] * steps / (time.perf_counter() - t0)


def run_ck(args, rank, local, world_size, pg, reference=False):
    import ctypes as C

    p, cfg, info = ck_scene(0xC4 + rank, args.ck_h)
    n = p.shape[0]
    metric, unit = "CK-MPM particle-updates/s", "particle-updates/s"
    if reference:  # the CPU restatement of CkMpmSolver::step (serial, as the reference's loops)
        if rank != 0:
            return
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O

        q = p.copy()
        O.ck_step(q, cfg, max(1, min(args.warmup, 1)))
        steps = max(1, min(args.steps, 5))
        t0 = time.perf_counter()
        O.ck_step(q, cfg, steps)
        dt = time.perf_counter() - t0
        value = n * steps / dt
        print(json.dumps({"impl": "reference", "metric": metric, "value": value, "unit": unit, "n_gpus": args.gpus,
                          "steps": steps, "warmup": args.warmup, "ms_per_step": 1000.0 * dt / steps,
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                          "data": "synthetic (seeded numpy)", "config": info,
                          "cpu_baseline": {"value": value, "unit": unit, "cores": 1, "kind": "port",
                                           "sample": "%d whole steps of the %d-particle scene" % (steps, n)},
                          "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}),
              flush=True)
        return
    import torch

    import ae_mpm as M

    ctx = M.Context(local)
    lib, h = ctx.lib, ctx.h
    dp = torch.from_numpy(p.ravel().copy()).cuda(local)
    steps = args.steps

    def run(k, timed=None):
        ctx.check(lib.ae_mpm_ck_step_timed(h, dp.data_ptr(), n, C.byref(cfg), k, timed))

    run(max(args.warmup, 3))
    clocks = Clocks(local)
    barrier(pg)
    torch.cuda.synchronize(local)
    clocks.start()
    time.sleep(0.3)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    run(steps)
    e1.record()
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    clk = clocks.stop()
    ms = max_over_ranks(pg, ms)
    value = n * world_size * steps / (ms / 1e3)
    # per-kernel durations from events around every launch, on a separate run of the same length
    km = (C.c_double * 2)()
    run(steps, km)
    part_us = 1000.0 * km[0] / (steps + 1)
    grid_us = 1000.0 * km[1] / steps  # block compaction + grid update
    achieved = CK_BYTES_PER_PARTICLE * n / (part_us * 1e-6) / 1e9
    peak, peak_kind = peaks()
    # end to end: host records through the drop-in call, CK_E2E_STEPS steps per call, pinned memory
    hp = torch.from_numpy(p.ravel().copy()).pin_memory()
    e2e_calls = max(1, args.e2e_reps)
    t0 = time.perf_counter()
    for _ in range(e2e_calls):
        ctx.check(lib.ae_mpm_ck_step(h, hp.data_ptr(), n, C.byref(cfg), CK_E2E_STEPS))
    e2e_dt = time.perf_counter() - t0
    e2e_value = n * CK_E2E_STEPS * e2e_calls / e2e_dt
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu = {"value": ck_oracle_rate(p, cfg, 2), "unit": unit, "cores": 1, "kind": "port",
               "sample": "2 whole steps of the %d-particle scene" % n}
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        t = json.load(open(tpath)).get("ck")
        if t:
            traffic = t["particles_bytes_per_particle"] * n
    if rank == 0:
        print(json.dumps({
            "metric": metric, "value": value, "unit": unit, "n_gpus": world_size, "steps": steps,
            "warmup": args.warmup, "ms_per_step": ms / steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded numpy)",
            "config": dict(info, parallelism="replicas" if world_size > 1 else "single GPU"),
            "roofline": {"bound": "hbm", "kernel": "ck_particles_kernel (G2P + next P2G + forces)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic, "peak_kind": peak_kind,
                         "algorithmic_bytes": CK_BYTES_PER_PARTICLE * n},
            "kernel_us": {"particles": part_us, "grid": grid_us},
            "e2e": {"value": e2e_value, "unit": unit, "h2d_bytes_per_step": 104 * n / CK_E2E_STEPS,
                    "d2h_bytes_per_step": 104 * n / CK_E2E_STEPS,
                    "ms_per_step": 1000.0 * e2e_dt / (CK_E2E_STEPS * e2e_calls),
                    "call": "ae_mpm_ck_step on pinned host records, %d steps per call" % CK_E2E_STEPS},
            "cpu_baseline": cpu, "gpu_launches": 1 + 3 * steps, "clocks": clk}), flush=True)


STAGE_SUBSTEPS = 20
# untimed substeps run just before each timed region: at least one full CUDA-graph period (at most
# 32 substeps: lcm(2, sort interval <= 32)), so the graph is captured and instantiated outside
# the timing; stage_times steps eagerly and builds none
GRAPH_WARM = 64


def graph_warm(world) -> None:
    world.step(GRAPH_WARM)
    world.sync(raise_on_error=False)


def run_ours(args, rank, local, world_size, pg):
    import torch

    import ae_mpm as M

    if args.workload == "tick":
        return run_tick(args, rank, local, world_size, pg)
    if args.workload == "ck":
        return run_ck(args, rank, local, world_size, pg)
    if args.workload == "midfield":
        return run_midfield(args, rank, local, world_size, pg)
    if args.workload == "near":
        return run_near(args, rank, local, world_size, pg)
    ctx = M.Context(local)
    scenes, parts, cfg = workload(args.workload, rank, args.scenes, world_size)
    if args.workload == "served":
        return run_served(args, rank, local, world_size, pg, ctx, scenes, parts, cfg)
    if args.workload == "batched":
        return run_batched(args, rank, local, world_size, pg, ctx, scenes, parts, cfg)
    fixed = fixed_options(args)
    opts = M.exec_opts(**fixed)
    world = M.World(ctx, scenes, opts)
    for i, p in enumerate(parts):
        world.upload(i, p)
    n_total = sum(p.n for p in parts)
    tune = {"fixed": {k: int(v) for k, v in fixed.items()}} if fixed else None
    tuned_kw = dict(fixed)
    if not args.no_autotune and not fixed:
        r = world.autotune(8)
        tuned_kw = {"p2g_variant": r.p2g_variant, "block_threads": r.block_threads, "sort_interval": r.sort_interval}
        tune = {"p2g_variant": {1: "tile", 2: "warp_agg", 3: "global", 4: "lanes"}.get(r.p2g_variant, r.p2g_variant),
                "block_threads": r.block_threads, "sort_interval": r.sort_interval,
                "us_per_substep": round(r.us_per_substep, 2)}
    world.step(max(args.warmup, 3))
    world.sync()
    # per-kernel event times over the next STAGE_SUBSTEPS substeps (eager, one event per stage)
    stages = world.stage_times(STAGE_SUBSTEPS)
    t0_sub = max(args.warmup, 3) + STAGE_SUBSTEPS + GRAPH_WARM  # the timed substeps start here, from the initial state
    # active grid nodes of the state the kernel times were taken on (for the roofline's node bytes)
    A = sum(active_nodes(s, world.download(i, p.n)) for i, (s, p) in enumerate(zip(scenes[:64], parts[:64])))
    if len(scenes) > 64:
        A = int(A * len(scenes) / 64)
    graph_warm(world)
    stream = torch.cuda.ExternalStream(world.stream(), device=local)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    clocks = Clocks(local)
    barrier(pg)
    torch.cuda.synchronize(local)
    clocks.start()
    time.sleep(0.3)
    hold_stream(torch, stream)
    timed_range(torch, True)
    e0.record(stream)
    world.step(args.steps)
    e1.record(stream)
    e1.synchronize()
    timed_range(torch, False)
    torch.cuda.synchronize(local)
    clk = clocks.stop()
    world.sync(raise_on_error=False)
    launches = world.launches()
    ms = e0.elapsed_time(e1)
    ms = max_over_ranks(pg, ms)
    value = n_total * world_size * args.steps / (ms / 1e3)
    # the same per-kernel times where the timed region ended (the state evolves: boxes collide, fluid spreads)
    stages_end = world.stage_times(STAGE_SUBSTEPS)

    # roofline of the dominant kernel (P2G or G2P), from its event-timed mean duration
    kern, kern_us = dominant_kernel(stages)
    per_p, per_n = KERNEL_BYTES[kern]
    alg_bytes = per_p * n_total + per_n * A
    achieved = alg_bytes / (kern_us * 1e-6) / 1e9
    peak, peak_kind = peaks()
    traffic = traffic_record(args.workload, kern)

    # end to end through the public API with pinned host buffers
    e2e = None
    if args.e2e_reps > 0 and len(scenes) == 1:
        def pinned_like(a):
            t = torch.empty(a.shape, dtype={np.float32: torch.float32, np.uint16: torch.int16}[a.dtype.type],
                            pin_memory=True)
            v = t.numpy().view(a.dtype)
            v[...] = a
            return t, v

        keep = []
        arrays = {}
        for f in ("pos", "vel", "F", "J", "C", "mass", "mat"):
            t, v = pinned_like(getattr(parts[0], f))
            keep.append(t)
            arrays[f] = v
        hin = M.Particles(**arrays)
        outs = {}
        for f in ("pos", "vel", "F", "J", "C", "mass", "mat"):
            t, v = pinned_like(getattr(parts[0], f))
            keep.append(t)
            outs[f] = v
        hout = M.Particles(**outs)
        h2d = sum(getattr(hin, f).nbytes for f in arrays)
        d2h = h2d
        world.upload(0, hin)
        world.step(args.e2e_substeps)
        world.download_into(0, hout)
        times, phases = [], []
        for _ in range(args.e2e_reps):
            barrier(pg)
            torch.cuda.synchronize(local)
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
            ev[0].record(stream)
            world.upload(0, hin)
            ev[1].record(stream)
            world.step(args.e2e_substeps)
            ev[2].record(stream)
            world.download_into(0, hout)
            ev[3].record(stream)
            ev[3].synchronize()
            times.append(max_over_ranks(pg, ev[0].elapsed_time(ev[3])))
            phases.append([ev[k].elapsed_time(ev[k + 1]) for k in range(3)])
        t = statistics.median(times)
        ph = [statistics.median(p[k] for p in phases) for k in range(3)]
        e2e = {"value": n_total * world_size * args.e2e_substeps / (t / 1e3), "unit": "particle-updates/s",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "substeps_per_step": args.e2e_substeps, "ms_per_step": t,
               "phases_ms": {"upload": round(ph[0], 3), "substeps": round(ph[1], 3), "download": round(ph[2], 3)}}

    # error of the end-to-end f32 run against the FP64 run of the same kernels, same substeps
    err = None
    if e2e is not None and not args.no_fp64:
        ref = fp64_run(ctx, scenes, parts, tuned_kw, args.e2e_substeps)
        err = dict(position_error(scenes, [hout], ref), substeps=args.e2e_substeps)

    cpu = None
    if rank == 0 and world_size == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        scene, p = scenes[0], parts[0]
        sub = 2
        rate, dt = cpu_rate(scene, p, sub, threads)
        cpu = {"value": rate, "unit": "particle-updates/s", "cores": threads, "kind": "port",
               "sample": "%d particles (whole scene), %d substeps, %.1f s" % (p.n, sub, dt)}

    if rank == 0:
        line = {
            "metric": "MPM particle-updates/s", "value": value, "unit": "particle-updates/s",
            "n_gpus": world_size, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded SplitMix64 scenes)",
            "config": cfg, "timed_substeps": [t0_sub, t0_sub + args.steps],
            "error_vs_fp64": err,
            "roofline": {"bound": "hbm", "kernel": kern, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic["bytes"] if traffic else None,
                         "traffic_source": traffic["source"] if traffic else None, "peak_kind": peak_kind,
                         "algorithmic_bytes": alg_bytes, "bytes_per_particle": per_p, "bytes_per_node": per_n,
                         "active_nodes": A, "kernel_us": kern_us,
                         "kernel_substeps": [t0_sub - STAGE_SUBSTEPS, t0_sub],
                         **substep_roofline(n_total, A, stages, peak)},
            "stages_us": {k: round(v, 2) for k, v in stages.items()},
            "stages_us_end": dict({k: round(v, 2) for k, v in stages_end.items()},
                                  substeps=[t0_sub + args.steps, t0_sub + args.steps + STAGE_SUBSTEPS]),
            "autotune": tune,
            "e2e": e2e, "cpu_baseline": cpu, "gpu_launches": launches, "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    world.close()


def percentile(xs, q):
    xs = sorted(xs)
    if not xs:
        return None
    k = (len(xs) - 1) * q / 100.0
    lo, hi = int(math.floor(k)), int(math.ceil(k))
    return xs[lo] + (xs[hi] - xs[lo]) * (k - lo)


def time_world(torch, world, local, steps, warmup):
    """CUDA-event time (ms) of `steps` substeps on the world's stream after `warmup` untimed ones
    and a graph warm-up."""
    world.step(warmup)
    graph_warm(world)
    stream = torch.cuda.ExternalStream(world.stream(), device=local)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    hold_stream(torch, stream, 2.0)
    e0.record(stream)
    world.step(steps)
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1)


def pinned_staging(torch, parts, fill=True):
    """Pinned host buffers, one per scene, carved from one page-locked allocation and laid out as
    the world's upload staging (pos, vel, F, J, C and mass back to back, then the material
    indices), so each scene crosses PCIe in one copy.  Returns (owner, [Particles views])."""
    import ae_mpm as M

    offs, total = [], 0
    for p in parts:
        offs.append(total)
        total += (106 * p.n + 255) // 256 * 256
    owner = torch.empty(max(total, 256), dtype=torch.uint8, pin_memory=True)
    raw = owner.numpy()
    views = []
    for p, o in zip(parts, offs):
        n = p.n
        f = raw[o:o + 104 * n].view(np.float32)
        v = M.Particles(pos=f[0:3 * n].reshape(n, 3), vel=f[3 * n:6 * n].reshape(n, 3), F=f[6 * n:15 * n].reshape(n, 9),
                        J=f[15 * n:16 * n], C=f[16 * n:25 * n].reshape(n, 9), mass=f[25 * n:26 * n],
                        mat=raw[o + 104 * n:o + 106 * n].view(np.uint16))
        if fill:
            for k in ("pos", "vel", "F", "J", "C", "mass", "mat"):
                getattr(v, k)[...] = getattr(p, k)
        views.append(v)
    return owner, views


def particle_bytes(p) -> int:
    return sum(getattr(p, k).nbytes for k in ("pos", "vel", "F", "J", "C", "mass", "mat"))


def position_error(scenes, got, ref) -> dict:
    """Per-particle position error of an f32 run against the FP64 run of the same kernels from the
    same initial state: |x32 - x64| relative to |x64| (max and 99th percentile over every particle)
    and in grid cells (|x32 - x64| / dx)."""
    rel, cells, worst = [], [], []
    for sc, a, b in zip(scenes, got, ref):
        d = np.linalg.norm(a.pos.astype(np.float64) - b.pos, axis=1)
        r = d / np.maximum(np.linalg.norm(b.pos, axis=1), 1e-30)
        rel.append(r)
        cells.append(d / sc.dx)
        worst.append(float(r.max()) if r.size else 0.0)
    rel = np.concatenate(rel)
    cells = np.concatenate(cells)
    return {"max_rel": float(rel.max()), "p99_rel": float(np.percentile(rel, 99)),
            "max_cells": float(cells.max()), "p99_cells": float(np.percentile(cells, 99)),
            "scenes_over_1e-4": int(sum(w > 1e-4 for w in worst)), "target_rel": 1e-4}


def fp64_run(ctx, scenes, parts, opts_kw, substeps):
    """The FP64 instantiation of the same kernels (precision 64), `substeps` from the initial state."""
    import ae_mpm as M

    w = M.World(ctx, scenes, M.exec_opts(precision=64, **opts_kw))
    for i, p in enumerate(parts):
        w.upload(i, p.astype(np.float64))
    w.step(substeps)
    w.sync(raise_on_error=False)
    out = [w.download(i, p.n) for i, p in enumerate(parts)]
    w.close()
    return out




def run_batched(args, rank, local, world_size, pg, ctx, scenes, parts, cfg):
    """The batched workload (512 scenes, grids 32^3-64^3, 2k-64k particles): every scene in one world
    (one launch per kernel per substep for all scenes) against the plain path, the same kernels
    stepping one world per scene, one scene at a time."""
    import torch

    import ae_mpm as M

    n_total = sum(p.n for p in parts)
    n_job = int(sum_over_ranks(pg, n_total))  # the ranks hold different scenes of one list
    tuned = fixed_options(args)
    world = M.World(ctx, scenes, M.exec_opts(**tuned))
    for i, p in enumerate(parts):
        world.upload(i, p)
    tune = {"fixed": {k: int(v) for k, v in tuned.items()}} if tuned else None
    if not args.no_autotune and not tuned:
        r = world.autotune(8)
        tuned = {"p2g_variant": r.p2g_variant, "block_threads": r.block_threads, "sort_interval": r.sort_interval}
        tune = dict(tuned, p2g_variant={1: "tile", 2: "warp_agg", 3: "global", 4: "lanes"}.get(r.p2g_variant),
                    us_per_substep=round(r.us_per_substep, 2))
    warm = max(args.warmup, 3)
    world.step(warm)
    world.sync()
    stages = world.stage_times(STAGE_SUBSTEPS)
    t0_sub = warm + STAGE_SUBSTEPS + GRAPH_WARM
    state = [world.download(i, p.n) for i, p in enumerate(parts)]
    A = sum(active_nodes(s, q) for s, q in zip(scenes, state))
    graph_warm(world)
    stream = torch.cuda.ExternalStream(world.stream(), device=local)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    clocks = Clocks(local)
    barrier(pg)
    torch.cuda.synchronize(local)
    clocks.start()
    time.sleep(0.3)
    hold_stream(torch, stream)
    timed_range(torch, True)
    e0.record(stream)
    world.step(args.steps)
    e1.record(stream)
    e1.synchronize()
    timed_range(torch, False)
    torch.cuda.synchronize(local)
    clk = clocks.stop()
    launches = world.launches()
    world.sync(raise_on_error=False)
    ms = max_over_ranks(pg, e0.elapsed_time(e1))
    value = n_job * args.steps / (ms / 1e3)

    # plain path: every scene in a world of its own (same kernels and options), stepped one scene
    # after another; the same K substeps per scene, each timed with events on that world's stream
    plain = [] if args.no_plain else [M.World(ctx, [sc], M.exec_opts(**tuned)) for sc in scenes]
    t_plain = 0.0
    for w1, p in zip(plain, parts):
        w1.upload(0, p)
        t_plain += time_world(torch, w1, local, args.steps, 3)
    t_plain = max_over_ranks(pg, t_plain)
    plain_value = n_job * args.steps / (t_plain / 1e3) if plain else None

    # end to end through the C ABI: every scene submitted at once from pinned host memory, the
    # config's run length of substeps, every scene downloaded; a scene completes when its results
    # are in the caller's buffer.  Batched: one world; plain: one world per scene, in turn.
    run = args.e2e_substeps
    own_in, hin = pinned_staging(torch, parts)
    own_out, hout = pinned_staging(torch, parts, fill=False)
    own_pl, hpl = pinned_staging(torch, parts, fill=False)
    h2d = sum(particle_bytes(p) for p in parts)
    e2e_b, e2e_p, lat_b, lat_p = [], [], [], []
    for rep in range(max(1, args.e2e_reps)):
        barrier(pg)
        torch.cuda.synchronize(local)
        ev0 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        ids = list(range(len(hin)))
        world.upload_many(ids, hin)  # every scene's copy back to back, one call
        world.step(run)
        world.download_many(ids, hout)  # returns when every scene's results are in place
        ev = torch.cuda.Event(enable_timing=True)
        ev.record(stream)
        ev.synchronize()
        lat = [ev0.elapsed_time(ev) / 1e3] * len(hout)  # lockstep: every scene completes together
        e2e_b.append(max_over_ranks(pg, lat[-1]))
        lat_b.append(lat)
        if plain and (rep == 0 or args.e2e_reps > 1):
            barrier(pg)
            torch.cuda.synchronize(local)
            s0 = torch.cuda.ExternalStream(plain[0].stream(), device=local)
            ev0 = torch.cuda.Event(enable_timing=True)
            ev0.record(s0)
            done = []
            for w1, q, o in zip(plain, hin, hpl):
                w1.upload(0, q)
                w1.step(run)
                w1.download_into(0, o)
                ev = torch.cuda.Event(enable_timing=True)
                ev.record(torch.cuda.ExternalStream(w1.stream(), device=local))
                done.append(ev)
            done[-1].synchronize()
            lat = [ev0.elapsed_time(ev) / 1e3 for ev in done]
            e2e_p.append(max_over_ranks(pg, lat[-1]))
            lat_p.append(lat)
    kb = int(np.argsort(e2e_b)[len(e2e_b) // 2])
    kp = int(np.argsort(e2e_p)[len(e2e_p) // 2]) if e2e_p else None
    e2e_world = {"value": n_job * run / e2e_b[kb], "unit": "particle-updates/s",
                 "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": h2d, "substeps_per_step": run,
                 "ms_per_step": 1e3 * e2e_b[kb],
                 "call": "ae_mpm_world_upload_many of every scene from pinned host memory, ae_mpm_world_step(%d), "
                         "ae_mpm_world_download_many of every scene" % run}

    # the same work through the pipelined batch call: the scenes in groups whose copies overlap
    # the other groups' substeps; one blocking call, timed on the host clock around it
    groups = max(1, args.e2e_groups)
    batch = M.Batch(ctx, scenes, M.exec_opts(**tuned), groups=groups)
    own_bt, hbt = pinned_staging(torch, parts, fill=False)
    vin, vbt = M.ViewArray(hin), M.ViewArray(hbt)  # the caller's view arrays, built once
    batch.run(vin, GRAPH_WARM, out=vbt, raise_on_error=False)  # first call: graphs, tables, staging
    e2e_t = []
    for rep in range(max(1, args.e2e_reps)):
        barrier(pg)
        torch.cuda.synchronize(local)
        t0 = time.perf_counter()
        batch.run(vin, run, out=vbt, raise_on_error=False)
        e2e_t.append(max_over_ranks(pg, time.perf_counter() - t0))
    tb = sorted(e2e_t)[len(e2e_t) // 2]
    e2e = {"value": n_job * run / tb, "unit": "particle-updates/s",
           "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": h2d, "substeps_per_step": run,
           "ms_per_step": 1e3 * tb, "timer": "host clock around the call", "groups": batch.groups(),
           "call": "ae_mpm_batch_run of every scene from pinned host memory to pinned host memory, %d substeps, "
                   "%d groups pipelined" % (run, groups),
           "one_world": e2e_world}
    batch.close()
    plain_e2e = n_job * run / e2e_p[kp] if e2e_p else None
    for w1 in plain:
        w1.close()

    # error of the batched f32 run against the FP64 run of the same kernels, same substeps
    err = None
    if not args.no_fp64:
        ref = fp64_run(ctx, scenes, parts, tuned, run)
        err = dict(position_error(scenes, hbt, ref), substeps=run, path="the pipelined batch call's results")

    kern, kern_us = dominant_kernel(stages)
    per_p, per_n = KERNEL_BYTES[kern]
    alg_bytes = per_p * n_total + per_n * A
    achieved = alg_bytes / (kern_us * 1e-6) / 1e9
    peak, peak_kind = peaks()
    traffic = traffic_record("batched", kern)

    cpu = None
    if rank == 0 and world_size == 1 and not args.no_cpu_baseline:
        rate, threads, desc = cpu_scenes_rate(scenes, parts, 2)
        cpu = {"value": rate, "unit": "particle-updates/s", "cores": threads, "kind": "port", "sample": desc}
    world.close()
    if rank == 0:
        line = {
            "metric": "MPM particle-updates/s", "value": value, "unit": "particle-updates/s", "n_gpus": world_size,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded SplitMix64 scenes)",
            "config": cfg, "timed_substeps": [t0_sub, t0_sub + args.steps],
            "batched_vs_plain": {"ratio": value / plain_value, "plain_value": plain_value,
                                 "e2e_ratio": e2e["value"] / plain_e2e, "plain_e2e_value": plain_e2e,
                                 "plain_scenes": len(scenes),
                                 "plain_kind": "one world per scene (same kernels and options), scenes in turn"}
            if plain else None,
            "scene_latency_s": {"substeps": run, "batched_p50": tb, "batched_p99": tb,
                                "one_world_p50": percentile(lat_b[kb], 50),
                                "one_world_p99": percentile(lat_b[kb], 99),
                                "plain_p50": percentile(lat_p[kp], 50) if plain else None,
                                "plain_p99": percentile(lat_p[kp], 99) if plain else None,
                                "definition": "every scene submitted at t=0; done when its results are in the "
                                              "caller's pinned buffer (batched: the pipelined batch call returns "
                                              "every scene at once; one_world: one world steps them in lockstep "
                                              "and returns them in one call)"},
            "error_vs_fp64": err,
            "roofline": {"bound": "hbm", "kernel": kern, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic["bytes"] if traffic else None,
                         "traffic_source": traffic["source"] if traffic else None, "peak_kind": peak_kind,
                         "algorithmic_bytes": alg_bytes, "bytes_per_particle": per_p, "bytes_per_node": per_n,
                         "active_nodes": A, "kernel_us": kern_us,
                         "kernel_substeps": [t0_sub - STAGE_SUBSTEPS, t0_sub],
                         **substep_roofline(n_total, A, stages, peak)},
            "stages_us": {a: round(b, 2) for a, b in stages.items()}, "autotune": tune,
            "e2e": e2e, "cpu_baseline": cpu, "gpu_launches": launches, "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    del own_in, own_out, own_pl


def run_served(args, rank, local, world_size, pg, ctx, scenes, parts, cfg):
    """Served: Poisson arrivals of batched-workload scenes plus 5% large 1M-particle snow scenes, each
    with 100..2000 substeps, into the continuous-batching server; per rate the throughput and the
    p50/p99 completion latency (submit -> results in the caller's buffers)."""
    import ae_mpm as M
    import ae_mpm_scenes as S

    rates = [float(r) for r in args.rates.split(",") if r]
    free = 0
    try:
        import torch

        free = torch.cuda.mem_get_info(local)[0]
    except Exception:
        pass
    budget = int(min(free * 0.6, 64 << 30)) if free else (32 << 30)
    # warm-up, untimed: a few requests through a server of their own, so that first-use costs
    # (module loading, the caching allocator's first blocks) do not land in the first rate's window
    wrng = S.Rng(0xAE05 - 1 - 1000 * rank)
    srv = M.Server(ctx, hbm_budget_bytes=budget, substeps_per_tick=20)
    for _ in range(24):
        sc, p, k = S.config5_request(wrng)
        srv.submit(sc, p, min(k, 100))
    srv.drain(600.0)
    srv.poll(4096)
    srv.close()
    out = []
    for ri, rate in enumerate(rates):
        rng = S.Rng(0xAE05 + 100 * ri + 1000 * rank)
        n_req = int(min(args.served_max, max(1, rate * args.served_seconds)))
        reqs = [S.config5_request(rng) for _ in range(n_req)]
        gaps = [-math.log(1.0 - rng.scalar()) / rate for _ in range(n_req)]
        outs = [M.Particles(*(np.empty_like(a) for a in (p.pos, p.vel, p.F, p.J, p.C, p.mass, p.mat)))
                for _, p, _ in reqs]  # result buffers, allocated before the arrivals start
        srv = M.Server(ctx, hbm_budget_bytes=budget, substeps_per_tick=20)
        lat, work = [], 0
        done, max_resident, t_submit = 0, 0, 0.0
        t0 = time.perf_counter()
        nxt = t0
        for (sc, p, k), o, gap in zip(reqs, outs, gaps):
            nxt += gap
            while time.perf_counter() < nxt:
                for rid, st, ts, ta, td, res in srv.poll():
                    done += 1
                    lat.append(td - ts)
                time.sleep(0.0005)
            ts0 = time.perf_counter()
            srv.submit(sc, p, k, o)
            t_submit += time.perf_counter() - ts0
            max_resident = max(max_resident, srv.stats()["resident_scenes"])
            work += p.n * k
        # the busy window: from the first arrival to the last one, the server's throughput while
        # requests keep arriving (the tail after it drains the last, longest requests alone)
        t_arr = time.perf_counter() - t0
        ps_arr = srv.stats()["particle_substeps"]
        srv.drain(900.0)
        for rid, st, ts, ta, td, res in srv.poll(1 << 16):
            done += 1
            lat.append(td - ts)
        wall = time.perf_counter() - t0
        stats = srv.stats()
        srv.close()
        out.append({"rate_per_s": rate, "requests": n_req, "completed": done,
                    "throughput": stats["particle_substeps"] / wall,
                    "throughput_while_arriving": ps_arr / t_arr if t_arr > 0 else None,
                    "p50_s": percentile(lat, 50), "p99_s": percentile(lat, 99), "ticks": stats["ticks"],
                    "max_resident_scenes": max_resident, "arrival_window_s": t_arr, "wall_s": wall,
                    "submit_ms_mean": 1e3 * t_submit / n_req})
    # the batched path on the same kind of scenes (the 512-scene batched workload, one world), for comparison
    bsc, bparts, _ = workload("batched", rank, 512, world_size)
    bw = M.World(ctx, bsc, M.exec_opts(p2g_variant=M.P2G_LANES, sort_interval=8, block_threads=128))
    for i, q in enumerate(bparts):
        bw.upload(i, q)
    import torch

    b_ms = time_world(torch, bw, local, 40, 5)
    bw.close()
    batched_value = sum(q.n for q in bparts) * 40 / (b_ms / 1e3)
    for r in out:
        r["throughput_vs_batched"] = r["throughput"] / batched_value
    if rank == 0:
        best = max(out, key=lambda r: r["throughput"])
        line = {"metric": "MPM particle-updates/s", "value": best["throughput"], "unit": "particle-updates/s",
                "n_gpus": world_size, "steps": None, "warmup": None, "ms_per_step": None, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded SplitMix64 scenes)",
                "config": {"workload": "served: Poisson arrivals of batched-workload scenes + 5% 128^3 1M-particle snow, "
                                       "100-2000 substeps each", "hbm_budget_bytes": budget},
                "batched_value": batched_value, "served": out}
        print(json.dumps(line), flush=True)


# substeps of one run of each configuration (the default number of timed steps)
RUN_LENGTH = {"snow": 500, "dam": 1000, "jelly": 200, "batched": 200}


def main():
    args = parse()
    if args.steps is None:
        args.steps = RUN_LENGTH.get(args.workload, 200)
    if args.e2e_substeps is None:
        args.e2e_substeps = RUN_LENGTH.get(args.workload, 500)
    rank, local, world_size, pg = dist_setup(args)
    try:
        if args.impl == "reference":
            run_reference(args, rank, pg)
        else:
            run_ours(args, rank, local, world_size, pg)
    finally:
        if pg is not None:
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
