"""The N>1 bench path on CPU: two gloo ranks (no GPU).

Multi-GPU runs of the single-domain step are replicas (no exchange between
GPUs); what crosses ranks is the timing reduction: every rank times its own
K cycles and the job's throughput uses the slowest rank.  Here two ranks
report different times and both must agree on the max and on the whole-job
rate.
"""
import os
import sys

import pytest
import torch.multiprocessing as mp

from conftest import REPO


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    sys.path.insert(0, REPO)
    import datetime

    import torch.distributed as dist

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    local_ms = [12.5, 17.0][rank]
    ms = bench.max_over_ranks(local_ms, dist, "cpu")
    rate = bench.aggregate_rate(1_000_000 * 10, ms / 1e3, world)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, ms, rate))


def test_two_rank_timing_reduction():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() % 2000)
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [17.0, 17.0]
    assert res[0][2] == pytest.approx(2 * 1e7 / 0.017)
    assert res[0][2] == res[1][2]
