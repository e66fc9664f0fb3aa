"""The multi-GPU replica path on CPU: two gloo ranks (no GPU), checking the
work partition and the whole-job aggregation bench.py uses for N > 1."""
from __future__ import annotations

import os
import socket

import pytest

from hpvcd_b200 import replicas


def test_shard_units_partition():
    for n in (0, 1, 7, 48, 256, 1541):
        for world in (1, 2, 3, 8):
            seen = []
            for r in range(world):
                block = replicas.shard_units(n, r, world)
                assert len(block) in (n // world, n // world + 1)
                seen.extend(block)
            assert seen == list(range(n))
    with pytest.raises(ValueError):
        replicas.shard_units(4, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    from datetime import timedelta
    dist.init_process_group("gloo", timeout=timedelta(seconds=60))
    r, w, local = replicas.dist_info()
    units = len(replicas.shard_units(1541, r, w))       # the serving set's tiles
    seconds = 0.5 + 0.25 * r                            # rank 1 is slower
    dist.barrier()
    rate = replicas.whole_job_rate(units, seconds)
    mx = replicas.max_over_ranks(float(r))
    q.put((r, units, rate, mx))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_aggregate_like_bench():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, u0, rate0, mx0), (r1, u1, rate1, mx1) = res
    assert u0 + u1 == 1541
    expect = 1541 / 0.75                                 # all units / slowest rank
    assert abs(rate0 - expect) < 1e-6 and abs(rate1 - expect) < 1e-6
    assert mx0 == mx1 == 1.0
