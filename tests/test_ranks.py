"""CPU tests of the multi-GPU host logic with two gloo ranks (no GPU): the batched worlds split
over ranks covers every world exactly once and balances bodies, and timings reduce to the
maximum over ranks."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from beatbox import ranks, scenes


def test_balanced_share_partitions_the_batch():
    sizes = scenes.batch_sizes(4096, seed=0)
    shares = [ranks.balanced_share(sizes, r, 3) for r in range(3)]
    flat = sorted(k for s in shares for k in s)
    assert flat == list(range(len(sizes)))
    loads = [int(sizes[s].sum()) for s in map(np.asarray, shares)]
    assert max(loads) - min(loads) <= int(sizes.max())
    assert all(s == sorted(s) for s in shares)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world_size, port, out):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world_size, timeout=datetime.timedelta(seconds=60))
    sizes = scenes.batch_sizes(512, seed=1)
    mine = ranks.balanced_share(sizes, rank, world_size)
    local_ms = 10.0 + 5.0 * rank  # rank 1 is the slow one
    slowest = ranks.max_over_ranks(local_ms, dist)
    bodies = ranks.max_over_ranks(float(sizes[mine].sum()), dist)
    dist.barrier()
    dist.destroy_process_group()
    out[rank] = (slowest, len(mine), bodies)


@pytest.mark.timeout(120)
def test_two_gloo_ranks_reduce_to_the_slowest():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(90)
    assert all(p.exitcode == 0 for p in procs)
    assert out[0][0] == out[1][0] == 15.0
    assert out[0][1] + out[1][1] == 512
    assert out[0][2] == out[1][2]
    assert ranks.job_throughput([100, 100], 2.0) == 100.0
