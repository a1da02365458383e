"""The request loop on the GPU: each result is the same alone and in the mix
(and equal to the oracle), admission by memory, rejection, batching, and a
loaded strategy network."""
import numpy as np
import pytest

import gpuscc_code_b200 as scc
from gpuscc_code_b200 import learned
from gpuscc_code_b200.serve import Server, make_graph, poisson_arrivals, run_stream, stream_spec
from gpu_util import oracle_labels

pytestmark = pytest.mark.gpu

BASE = scc.Options(alg="h", wcc=True, trim2=True)


@pytest.fixture(scope="module")
def graphs():
    out = [make_graph(stream_spec(i, seed=41, rmat_scale=(10, 16), grid_side=(30, 200))) for i in range(24)]
    out += [scc.gen_er(3000, 3500, seed=5), scc.csr_from_edges(1, np.zeros(0, np.uint32), np.zeros(0, np.uint32))]
    return out


@pytest.fixture(scope="module")
def alone(graphs):
    ctx = scc.SCCContext(0, BASE)
    res = []
    for g in graphs:
        ctx.upload(g)
        labels, cnt, _ = ctx.solve()
        res.append((labels.copy(), cnt))
    ctx.close()
    for g, (labels, cnt) in zip(graphs, res):
        ref, rcnt = oracle_labels(g)
        assert cnt == rcnt and np.array_equal(labels, ref)
    return res


@pytest.mark.parametrize("batching", [True, False])
def test_results_same_alone_and_in_the_mix(graphs, alone, batching):
    with Server(0, BASE, batching=batching) as srv:
        ids = [srv.submit(g) for g in graphs]  # all at once: the loop batches what is ready
        out = [srv.wait(i) for i in ids]
        st = srv.stats()
    for (labels, info), (ref, cnt) in zip(out, alone):
        assert np.array_equal(labels, ref)
        assert info["nscc"] == cnt
    sizes = [info["batch_graphs"] for _, info in out]
    if batching:
        assert max(sizes) > 1
    else:
        assert max(sizes) == 1
    assert st["completed"] == len(graphs) and st["resident_bytes"] == 0


def test_poisson_stream_with_tight_memory_budget(graphs, alone):
    budget = 3 * max(8 * (g.n + 2) + 8 * g.m for g in graphs)
    with Server(0, BASE, mem_budget=budget) as srv:
        res = run_stream(srv, graphs, poisson_arrivals(len(graphs), rate=400.0, seed=2))
        st = srv.stats()
    for labels, (ref, _) in zip(res["labels"], alone):
        assert np.array_equal(labels, ref)
    assert st["peak_resident_bytes"] <= budget
    assert res["p99_ms"] >= res["p50_ms"] > 0


def test_graph_larger_than_the_budget_is_rejected(graphs):
    with Server(0, BASE, mem_budget=4096) as srv:
        with pytest.raises(scc.SCCError) as ei:
            srv.submit(graphs[0])
        assert ei.value.code == -10
        assert srv.stats()["rejected"] == 1


def test_small_batch_limits_split_batches(graphs, alone):
    with Server(0, BASE, max_batch_graphs=3, max_batch_vertices=1 << 16) as srv:
        ids = [srv.submit(g) for g in graphs]
        out = [srv.wait(i) for i in ids]
    for (labels, info), (ref, _) in zip(out, alone):
        assert np.array_equal(labels, ref)
        assert info["batch_graphs"] <= 3


def test_network_picks_options_and_labels_stay_exact(graphs, alone):
    net = learned.StrategyNet(0, seed=11)  # untrained: arbitrary picks must not change labels
    rng = np.random.default_rng(0)
    p = net.params
    net.params = p + rng.normal(0, 1.0, p.size).astype(np.float32)
    with Server(0, BASE, model=net) as srv:
        ids = [srv.submit(g) for g in graphs]
        out = [srv.wait(i) for i in ids]
    picks = {info["choice"] for _, info in out}
    for (labels, info), (ref, _) in zip(out, alone):
        assert np.array_equal(labels, ref)
    assert len(picks) >= 1


def test_stop_finishes_queued_requests(graphs, alone):
    srv = Server(0, BASE)
    ids = [srv.submit(g) for g in graphs[:8]]
    keep = dict(srv._keep)  # labels buffers stay alive through stop
    srv.stop()
    for rid, (ref, _) in zip(ids, alone[:8]):
        assert np.array_equal(keep[rid][1], ref)
