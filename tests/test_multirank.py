"""The N > 1 path of bench.py on CPU: two gloo ranks.

Ensembles shard by box with no data-path collective; the only collective is
the max over ranks of each rank's device time (bench.max_over_ranks), and
every rank takes it in the same order.  Two processes with different
"device times" must both see the larger one.
"""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(ws), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    assert bench.dist() == (ws, rank, rank)
    mine = [3.5, 7.25][rank]
    out[rank] = bench.max_over_ranks(mine, ws, "cpu")
    out[2 + rank] = bench.max_over_ranks(1.0 + rank, ws, "cpu")   # a second reduction, same order
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    out = ctx.Array("d", 4)
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert list(out) == [7.25, 7.25, 2.0, 2.0]


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(4.0, 1, "cpu") == 4.0
