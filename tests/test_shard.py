"""Sharding of independent boxes across ranks (janus_treepm.shard), on CPU.

The partition is computed alike on every rank, covers each box once and
balances the cost model within Graham's bound; a sharded ensemble over two
gloo ranks steps each box exactly once per step (a host stand-in for the
batch: a per-box checksum), takes the max over ranks of the time and
gathers the per-rank metrics to rank 0 (the only collectives, in the same
order on every rank).
"""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "janus-sim_b200"))
sys.path.insert(0, ROOT)

from janus_treepm import shard  # noqa: E402


def _ensemble_costs(n=64):
    import bench
    boxes = bench.ensemble_boxes(n)
    return boxes, [shard.box_cost(2 * bx["n"] ** 3, bx["M"]) for bx in boxes]


@pytest.mark.parametrize("ws", [1, 2, 3, 4, 8])
def test_partition_covers_every_box_once_and_balances(ws):
    boxes, costs = _ensemble_costs()
    shares = shard.partition(costs, ws)
    assert len(shares) == ws
    flat = sorted(i for s in shares for i in s)
    assert flat == list(range(len(boxes)))
    ld = shard.loads(costs, shares)
    # LPT: the heaviest rank is within 4/3 of the optimum, itself at least
    # the mean load and the largest box
    opt_lb = max(sum(costs) / ws, max(costs))
    assert max(ld) <= 4.0 / 3.0 * opt_lb + 1e-6 * sum(costs)
    assert shard.partition(costs, ws) == shares   # deterministic


def test_partition_edge_cases():
    assert shard.partition([], 3) == [[], [], []]
    assert shard.partition([5.0], 2) == [[0], []]
    # equal costs go round-robin by index
    assert shard.partition([1.0] * 4, 2) == [[0, 2], [1, 3]]
    with pytest.raises(ValueError):
        shard.partition([1.0], 0)
    with pytest.raises(ValueError):
        shard.partition([-1.0], 1)


def test_box_cost_weights_grid_cells():
    assert shard.box_cost(1000, 0) == 1000.0
    assert shard.box_cost(0, 64) == pytest.approx(shard.GRID_WEIGHT * 64 ** 3)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, out, steps):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, os.path.join(ROOT, "janus-sim_b200"))
    sys.path.insert(0, ROOT)
    import bench
    from janus_treepm import shard as sh
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(ws), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    boxes = bench.ensemble_boxes(64)
    costs = [sh.box_cost(2 * bx["n"] ** 3, bx["M"]) for bx in boxes]
    mine = sh.partition(costs, ws)[rank]
    # host stand-in for a batched step: each box contributes its seed and its
    # particles once per step; the "time" is the share's cost
    seen, parts = 0, 0
    for _ in range(steps):
        for i in mine:
            seen += boxes[i]["seed"]
            parts += 2 * boxes[i]["n"] ** 3
    t = sum(costs[i] for i in mine)
    t_max = bench.max_over_ranks(t, ws, "cpu")
    metrics = sh.gather({"rank": rank, "boxes": mine, "seen": seen, "parts": parts, "t": t}, ws)
    if rank == 0:
        all_boxes = sorted(i for m in metrics for i in m["boxes"])
        out[0] = float(all_boxes == list(range(64)))
        out[1] = float(sum(m["seen"] for m in metrics))
        out[2] = float(sum(m["parts"] for m in metrics))
        out[3] = float(t_max == max(m["t"] for m in metrics))
        out[4] = float([m["rank"] for m in metrics] == list(range(ws)))
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_ensemble_two_gloo_ranks():
    import bench
    boxes = bench.ensemble_boxes(64)
    steps = 3
    ctx = mp.get_context("spawn")
    out = ctx.Array("d", 5)
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out, steps)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert out[0] == 1.0 and out[3] == 1.0 and out[4] == 1.0
    assert out[1] == steps * sum(bx["seed"] for bx in boxes)
    assert out[2] == steps * sum(2 * bx["n"] ** 3 for bx in boxes)


@pytest.mark.gpu
def test_sharded_ensemble_leg_on_one_rank():
    """bench.run_ensemble_sharded on one GPU as rank 0 of 1: every box in its
    share, the value and the gathered metrics consistent."""
    import bench
    import janus_treepm as J
    from janus_treepm import ics
    w = bench.workload()
    r = bench.run_ensemble_sharded(J, ics, 6, 1, 1, 0.07, w["dt"], 0, 1)
    boxes = bench.ensemble_boxes(6)
    n_part = sum(2 * bx["n"] ** 3 for bx in boxes)
    assert r["ranks"] == 1 and r["per_rank"][0]["boxes"] == 6
    assert r["per_rank"][0]["particles"] == n_part
    assert r["value"] > 0 and r["value"] == pytest.approx(n_part / (r["ms_per_step"] * 1e-3))
    assert r["cost_max_over_mean"] == 1.0


@pytest.mark.gpu
def test_sharded_serving_leg_on_one_rank():
    """bench.run_serving_sharded on one GPU as rank 0 of 1: every job served
    for every step."""
    import bench
    import janus_treepm as J
    from janus_treepm import ics
    w = bench.workload()
    r = bench.run_serving_sharded(J, ics, 4, 0, 2, 0.07, w["dt"], 0, 1, budget_gb=8.0)
    assert r["ranks"] == 1 and r["per_rank"][0]["jobs"] == 4 and r["per_rank"][0]["requests"] == 8
    assert r["saturated_value"] > 0 and r["makespan_s"] > 0
