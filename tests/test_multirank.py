"""N>1 path of bench.py on CPU: two gloo ranks, each with its own system
(weak scaling), timings combined as the max over ranks."""

from __future__ import annotations

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank: int, world: int, port: int, q):
    import sys
    import torch.distributed as dist
    sys.path.insert(0, os.path.abspath(os.path.join(os.path.dirname(__file__), "..")))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import bench
    m = bench.max_over_ranks(10.0 * (rank + 1), world, "cpu")
    seeds = bench.rank_seeds(rank)
    # each rank generates its own (small) system from its seeds
    from detnqs_b200 import synthetic as S
    sysm = S.make_system(8, 3, 3, 16, seeds[0])
    V = S.heat_bath_sample(sysm, 200, seeds[1])
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, m, seeds, V[:5].tolist()))


def test_two_rank_weak_scaling_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(2):
        r, m, seeds, head = q.get(timeout=120)
        out[r] = (m, seeds, head)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[0][0] == out[1][0] == 20.0            # max over ranks
    assert out[0][1] != out[1][1]                    # different systems per rank
    assert out[0][2] != out[1][2]
