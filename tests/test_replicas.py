"""Replica partitioning and the host-side collectives, with two gloo ranks on
the CPU (one process per rank, as torchrun launches the bench)."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from protomol_b200 import replicas, serve


def test_partition_covers_every_item_once():
    costs = [5.0, 1.0, 3.0, 3.0, 2.0, 8.0, 1.0]
    parts = replicas.partition(costs, 3)
    flat = sorted(k for p in parts for k in p)
    assert flat == list(range(len(costs)))
    loads = [sum(costs[k] for k in p) for p in parts]
    assert max(loads) <= 4.0 / 3.0 * (sum(costs) / 3) + max(costs)
    assert replicas.partition(costs, 3) == parts  # deterministic


def test_partition_rejects_empty_world():
    with pytest.raises(ValueError):
        replicas.partition([1.0], 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        reqs = serve.request_stream(20, 3)
        mine = replicas.my_share(reqs, world, rank)
        t = replicas.max_over_ranks(1.0 + rank, dist)
        got = replicas.gather_summaries({"rank": rank, "rids": [r.rid for r in mine]}, dist)
        out[rank] = {"max": t, "gathered": got}
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_split_a_stream():
    world = 2
    port = _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_rank_main, args=(world, port, out), nprocs=world, join=True)
    assert out[0]["max"] == out[1]["max"] == 2.0
    gathered = out[0]["gathered"]
    assert [g["rank"] for g in gathered] == [0, 1]
    rids = sorted(r for g in gathered for r in g["rids"])
    assert rids == list(range(20))
    assert out[1]["gathered"] == gathered
