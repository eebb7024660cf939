"""The multi-GPU path's host logic with two gloo ranks on CPU: disjoint shards per rank,
the max-over-ranks step time and the whole-job rate every rank agrees on."""
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from ferrousalign_b200 import replicas


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    import datetime
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        ws, r, local = replicas.dist_env()
        from ferrousalign_b200 import synth
        b = synth.workload_ext_plain(500, seed=replicas.shard_seed(2, r))
        step_ms = 10.0 + 5.0 * r                     # rank 1 is the slower one
        dist.barrier()
        rate, slowest = replicas.whole_job_rate(len(b.jobs), step_ms)
        q.put((r, ws, local, rate, slowest, bytes(b.qseq[:200])))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    assert [r[0] for r in res] == [0, 1] and all(r[1] == 2 and r[2] == r[0] for r in res)
    # every rank reports the slowest rank's time and the same whole-job rate
    assert all(r[4] == 15.0 for r in res)
    assert all(np.isclose(r[3], 2 * 500 / 15.0e-3) for r in res)
    assert res[0][5] != res[1][5]                   # disjoint synthetic shards


def test_single_process_identity():
    assert replicas.max_over_ranks(3.5) == 3.5
    rate, ms = replicas.whole_job_rate(1000, 2.0)
    assert ms == 2.0 and rate == 1000 / 2.0e-3
