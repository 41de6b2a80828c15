"""Host logic of multi-GPU runs (imcom_b200/replicas.py), on CPU.

* The cost-balanced shard gives every patch to exactly one rank, the same
  partition on every rank, and loads within one item of each other.
* Two gloo ranks (world size 2, spawned processes): each computes its shard
  of the batched-patch workload, the shards are disjoint and cover the batch,
  and the job time is the MAX of the ranks' times on both ranks.
"""
import os
import socket

import pytest

from imcom_b200 import replicas


def loads(costs, world):
    out = []
    for r in range(world):
        out.append(sum(costs[i] for i in replicas.shard_by_cost(costs, r, world)))
    return out


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_shard_partitions_and_balances(world):
    import numpy as np
    rng = np.random.default_rng(world)
    costs = list(rng.integers(900, 2300, 256).astype(float) ** 3)
    shards = [replicas.shard_by_cost(costs, r, world) for r in range(world)]
    flat = sorted(i for sh in shards for i in sh)
    assert flat == list(range(256))
    ld = loads(costs, world)
    assert max(ld) - min(ld) <= max(costs)
    assert shards == [replicas.shard_by_cost(costs, r, world) for r in range(world)]


def test_shard_rejects_bad_rank():
    with pytest.raises(ValueError):
        replicas.shard_by_cost([1.0], 2, 2)


def test_job_rate_and_single_process_max():
    assert replicas.job_rate(256, 4.0) == 64.0
    assert replicas.job_rate(1, 0.0) == 0.0
    assert replicas.max_over_ranks(3.5) == 3.5


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import json

    import torch.distributed as dist

    from imcom_b200 import batch
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        problems = batch.make_batch(24, seed0=1000)
        costs = [replicas.patch_cost(p) for p in problems]
        mine = replicas.shard_by_cost(costs, rank, world)
        shards = [None] * world
        dist.all_gather_object(shards, mine)
        t = replicas.max_over_ranks(1.5 + rank, dist)
        with open(os.path.join(out_dir, f"r{rank}.json"), "w") as f:
            json.dump({"mine": mine, "shards": shards, "t": t,
                       "rate": replicas.job_rate(len(problems), t)}, f)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_max(tmp_path):
    import json

    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    res = [json.load(open(tmp_path / f"r{r}.json")) for r in range(2)]
    assert res[0]["shards"] == res[1]["shards"]
    assert res[0]["shards"][0] == res[0]["mine"] and res[0]["shards"][1] == res[1]["mine"]
    assert sorted(res[0]["mine"] + res[1]["mine"]) == list(range(24))
    assert res[0]["t"] == res[1]["t"] == 2.5
    assert res[0]["rate"] == res[1]["rate"] == 24 / 2.5
