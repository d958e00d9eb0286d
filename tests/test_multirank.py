"""Multi-rank host logic of bench.py on CPU (gloo, world_size 2): the max-over-ranks timing and the
round-robin scene sharding of the batched workload when --gpus N > 1 (bench.workload deals one
seeded list of N x scenes to the ranks).  The substep itself does not shard within a scene, so there
is no data-path collective to test."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import datetime
    import sys

    import torch.distributed as dist

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench

    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        got = bench.max_over_ranks(dist, 10.0 + 5.0 * rank)
        total = bench.sum_over_ranks(dist, 1.0 + rank)
        mine = bench.shard(list(range(11)), rank, world)
        scenes, parts, cfg = bench.workload("batched", rank, 3, world)
        out.put((rank, got, mine, [p.n for p in parts], cfg["scenes"], total))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_scene_sharding_with_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [15.0, 15.0]
    assert [r[5] for r in res] == [3.0, 3.0]  # job-wide particle counts: the sum over ranks
    assert res[0][2] == [0, 2, 4, 6, 8, 10] and res[1][2] == [1, 3, 5, 7, 9]
    assert sorted(res[0][2] + res[1][2]) == list(range(11))
    # the batched workload: each rank holds 3 scenes of one 6-scene population, dealt round-robin
    import sys

    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "ae-engine_b200"))
    import ae_mpm_scenes as S

    full = [p.n for _, p in S.config4_batched(6, 0xAE04)]
    assert res[0][4] == res[1][4] == 3
    assert res[0][3] == full[0::2] and res[1][3] == full[1::2]
