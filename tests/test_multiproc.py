"""Multi-process host logic on CPU (gloo ranks): the batched workload shards
independent graphs over ranks with no collective on the data path, each rank
solves its shard, and the labels gathered afterwards equal a single-rank
solve of the whole batch and the oracle's Tarjan.  Failure detection between
steps: a rank that announces leaving, a rank that goes silent, and the short
process-group timeout that ends a collective a dead peer never joins."""
import os
import socket
import time

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _graphs():
    import gpuscc_code_b200 as scc

    out = [scc.gen_rmat(s, 8 << s, seed=100 + s) for s in (7, 9, 10, 12)]
    out += [scc.gen_er(700 + 50 * i, 1400 + 90 * i, seed=200 + i) for i in range(5)]
    out += [scc.gen_grid(20 + 7 * i, 0.2, 0.002, seed=300 + i) for i in range(4)]
    return out


def _cpu_solve(graphs):
    """A rank's solve on a host without a GPU: the library's own CPU
    decomposition (the apps' -t path, tarjan.h:5) per graph."""
    import gpuscc_code_b200 as scc

    res = []
    for g in graphs:
        labels, cnt, _ = scc.tarjan(g)
        res.append((labels, cnt))
    return res


def _init(rank, world, port, timeout_s=30):
    import datetime

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=timeout_s))


def _shard_worker(rank, world, port, out_dir):
    _init(rank, world, port)
    try:
        from gpuscc_code_b200.batch import gather_results, shard_graphs, solve_shard, graph_weight

        graphs = _graphs()
        local = solve_shard(graphs, rank, world, _cpu_solve)
        # every rank derives the same plan on its own; check that it did
        plan = shard_graphs([graph_weight(g.n, g.m) for g in graphs], world)
        assert sorted(local) == plan[rank]
        merged = gather_results(local, world)
        np.save(os.path.join(out_dir, f"r{rank}_mine.npy"), np.array(sorted(local), dtype=np.int64))
        np.savez(os.path.join(out_dir, f"r{rank}.npz"), *[lab for lab, _ in merged],
                 counts=np.array([c for _, c in merged]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_batch_solved_and_gathered_over_gloo_ranks(tmp_path, world):
    import oracle

    mp.spawn(_shard_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    graphs = _graphs()
    single = _cpu_solve(graphs)
    mine = [set(np.load(tmp_path / f"r{r}_mine.npy").tolist()) for r in range(world)]
    assert set().union(*mine) == set(range(len(graphs)))
    assert sum(len(m) for m in mine) == len(graphs)  # no graph solved twice
    for r in range(world):
        d = np.load(tmp_path / f"r{r}.npz")
        assert list(d["counts"]) == [c for _, c in single]
        for i, (lab, _) in enumerate(single):
            assert np.array_equal(d[f"arr_{i}"], lab)
    for g, (lab, cnt) in zip(graphs, single):
        ref, rcnt = oracle.tarjan_labels(g.n, g.nodes, g.edges)
        assert cnt == rcnt and np.array_equal(lab, ref)


def _leave_worker(rank, world, port, out_dir, announce):
    _init(rank, world, port)
    from gpuscc_code_b200.batch import PeerLeft, PeerLost, RankWatch

    store = dist.distributed_c10d._get_default_store()
    watch = RankWatch(store, rank, world, timeout_s=2.0)
    status = "finished"
    try:
        for step in range(4):
            if rank == 1 and step == 2:  # leaves between steps, nothing in flight
                if announce:
                    watch.leave()
                os._exit(0)
            watch.step(step)
            import torch

            x = torch.ones(1)
            dist.all_reduce(x)
            assert x.item() == world
    except PeerLeft as e:
        status = f"left:{e}"
    except PeerLost as e:
        status = f"lost:{e}"
    with open(os.path.join(out_dir, f"r{rank}.txt"), "w") as f:
        f.write(status)
    os._exit(0)  # the group lost a member: no destroy_process_group barrier


@pytest.mark.parametrize("announce", [True, False])
def test_rank_leaving_between_steps_is_detected_on_the_host(tmp_path, announce):
    world = 3
    t0 = time.monotonic()
    ctx = mp.spawn(_leave_worker, args=(world, _free_port(), str(tmp_path), announce), nprocs=world, join=False)
    while not ctx.join(timeout=30):
        if time.monotonic() - t0 > 60:
            for p in ctx.processes:
                p.kill()
            pytest.fail("ranks did not finish")
    for r in (0, 2):
        status = (tmp_path / f"r{r}.txt").read_text()
        if announce:
            assert status.startswith("left:") and "rank 1" in status, status
        else:
            assert status.startswith("lost:") and "rank 1" in status, status
    assert not (tmp_path / "r1.txt").exists()
    assert time.monotonic() - t0 < 60


def _dead_peer_worker(rank, world, port, out_dir):
    _init(rank, world, port, timeout_s=3)
    import torch

    x = torch.ones(1)
    dist.all_reduce(x)
    if rank == 1:
        os._exit(0)  # dies between steps without telling anyone
    t0 = time.monotonic()
    try:
        dist.all_reduce(x)
        status = "completed"
    except Exception as e:  # gloo: the peer's connection closed, or the group timeout
        status = f"error:{type(e).__name__}"
    with open(os.path.join(out_dir, f"r{rank}.txt"), "w") as f:
        f.write(f"{status} {time.monotonic() - t0:.2f}")
    os._exit(0)


def test_collective_with_a_dead_peer_ends_with_an_error(tmp_path):
    world = 2
    ctx = mp.spawn(_dead_peer_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=False)
    t0 = time.monotonic()
    while not ctx.join(timeout=30):
        if time.monotonic() - t0 > 60:
            for p in ctx.processes:
                p.kill()
            pytest.fail("the surviving rank hung in its collective")
    status, secs = (tmp_path / "r0.txt").read_text().split()
    assert status.startswith("error:")
    assert float(secs) < 30
