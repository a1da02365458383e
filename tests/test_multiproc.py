"""Multi-process host logic on CPU (gloo, world size 2): the batched workload
shards independent graphs over ranks with no collective on the data path;
the host gathers the per-rank results afterwards."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, weights, out_dir):
    import torch
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from gpuscc_code_b200.batch import shard_graphs
        shards = shard_graphs(weights, world)
        mine = shards[rank]
        # every rank derives the same plan on its own
        plan = torch.tensor([i for s in shards for i in s], dtype=torch.int64)
        gathered = [torch.zeros_like(plan) for _ in range(world)]
        dist.all_gather(gathered, plan)
        assert all(torch.equal(g, plan) for g in gathered)
        # per-rank "solve": a stand-in count per graph (the weight), summed over ranks
        local = torch.tensor([sum(int(weights[i]) for i in mine)], dtype=torch.int64)
        dist.all_reduce(local)
        np.save(os.path.join(out_dir, f"r{rank}.npy"), np.array([local.item()] + mine))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_sharded_batch_plan_over_gloo_ranks(tmp_path, world):
    weights = np.random.default_rng(3).integers(1, 10_000, size=37)
    mp.spawn(_worker, args=(world, _free_port(), weights, str(tmp_path)), nprocs=world, join=True)
    parts = [np.load(tmp_path / f"r{r}.npy") for r in range(world)]
    assert all(p[0] == weights.sum() for p in parts)
    ids = sorted(int(i) for p in parts for i in p[1:])
    assert ids == list(range(len(weights)))
