"""Batched solve on the GPU: packed graphs, one persistent launch (plain and
replayed from a captured CUDA graph), device batch generator, autotuner."""
import numpy as np
import pytest

import gpuscc_code_b200 as scc
import oracle
from gpuscc_code_b200 import autotune, batch

pytestmark = pytest.mark.gpu


def mixed_graphs():
    return ([scc.gen_rmat(s, 8 << s, seed=60 + s) for s in (6, 9, 11)] +
            [scc.gen_er(500, 1500, seed=70), scc.gen_grid(25, 0.2, 0.002, seed=71)] +
            [scc.csr_from_edges(5, np.array([1, 2, 3], np.uint32), np.array([2, 3, 1], np.uint32))])


@pytest.mark.parametrize("capture", [True, False])
def test_batched_labels_equal_per_graph_oracle(capture):
    graphs = mixed_graphs()
    solver = batch.BatchSolver(0, scc.Options(alg="h", wcc=True, trim2=True), capture=capture)
    try:
        res = solver.solve(graphs)
        for g, (labels, cnt) in zip(graphs, res):
            ref, rcnt = oracle.tarjan_labels(g.n, g.nodes, g.edges)
            assert cnt == rcnt and np.array_equal(labels, ref)
        # replay again: same result
        again = solver.solve(graphs)
        for (a, ca), (b, cb) in zip(res, again):
            assert ca == cb and np.array_equal(a, b)
    finally:
        solver.close()


def test_batched_equals_solve_each():
    graphs = mixed_graphs()
    with scc.SCCContext(0, alg="q") as ctx:
        each, _ = batch.solve_each(graphs, ctx)
    solver = batch.BatchSolver(0, scc.Options(alg="q"))
    try:
        res = solver.solve(graphs)
    finally:
        solver.close()
    for (a, ca), (b, cb) in zip(each, res):
        assert ca == cb and np.array_equal(a, b)


def test_device_batch_matches_host_generator():
    host, seg_h = scc.gen_batch(48, 50, 3000, 2.0, 16.0, seed=4)
    with scc.SCCContext(0) as ctx:
        seg_d = ctx.gen_batch_device(48, 50, 3000, 2.0, 16.0, seed=4)
        dev = ctx.download()
    assert np.array_equal(seg_h, seg_d)
    assert dev.n == host.n and dev.m == host.m
    assert np.array_equal(dev.nodes[1:], host.nodes[1:]) and np.array_equal(dev.edges, host.edges)
    assert np.array_equal(dev.nodesT[1:], host.nodesT[1:]) and np.array_equal(dev.edgesT, host.edgesT)


@pytest.mark.parametrize("alg", ["h", "l", "q"])
def test_device_batch_solve_matches_oracle(alg):
    with scc.SCCContext(0, alg=alg, wcc=True, trim2=True) as ctx:
        ctx.gen_batch_device(96, 100, 8000, 2.0, 16.0, seed=11)
        g = ctx.download()
        ctx.capture()
        cnt, _ = ctx.replay()
        labels = ctx.read_labels()
    ref, rcnt = oracle.tarjan_labels(g.n, g.nodes, g.edges)
    assert cnt == rcnt and np.array_equal(labels, ref)


def test_autotuner_keeps_labels():
    with scc.SCCContext(0, alg="h", wcc=True, trim2=True) as ctx:
        ctx.gen_batch_device(64, 100, 20000, 2.0, 16.0, seed=12)
        ref = ctx.solve()[0]
        space = {"block_size": [256, 512], "heavy_degree": [4096, 1024], "pull_alpha": [14, -1]}
        best, trials = autotune.autotune(ctx, space=space, repeats=1)
        assert len(trials) >= 4 and all(t[2] > 0 for t in trials)
        labels, _, _ = ctx.solve()
        assert np.array_equal(labels, ref)
