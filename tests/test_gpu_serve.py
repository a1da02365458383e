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


def _dev_bytes(g):
    """Device bytes of one uploaded graph: offsets and lists of both directions
    (4-entry padded) and the 16-byte flag of its upload check."""
    pad4 = lambda x: (x + 3) // 4 * 4
    return 2 * 4 * pad4(g.n + 2) + 2 * 4 * pad4(g.m) + 16


def test_malformed_graph_is_refused_at_registration():
    nodes = np.array([0, 0, 1, 2], np.uint32)
    bad = scc.HostCSR.from_arrays(nodes, np.array([2, 7], np.uint32), nodes, np.array([2, 1], np.uint32))
    with Server(0, BASE) as srv:
        with pytest.raises(scc.SCCError) as ei:
            srv.register(bad)
        assert ei.value.code == -1
        assert srv.stats()["resident_bytes"] == 0


@pytest.mark.parametrize("batching", [True, False])
def test_resident_graphs_same_alone_and_mixed_with_uploads(graphs, alone, batching):
    with Server(0, BASE, batching=batching) as srv:
        handles = [srv.register(g) for g in graphs[:12]]
        st0 = srv.stats()
        # each resident graph twice, interleaved with host graphs uploaded per request
        items = []
        for i, h in enumerate(handles):
            items += [(i, h), (12 + i % (len(graphs) - 12), graphs[12 + i % (len(graphs) - 12)]), (i, h)]
        ids = [srv.submit(x) for _, x in items]
        out = [srv.wait(i) for i in ids]
        st = srv.stats()
        for h in handles:
            srv.unregister(h)
        assert srv.stats()["resident_bytes"] == 0
    for (gi, _), (labels, info) in zip(items, out):
        assert np.array_equal(labels, alone[gi][0])
        assert info["nscc"] == alone[gi][1]
    assert st0["registered"] == 12 and st["evictions"] == 0 and st["reuploads"] == 0
    # the resident graphs stayed on the device: only the host graphs were uploaded per request
    assert st["resident_bytes"] == sum(_dev_bytes(g) for g in graphs[:12])


def test_resident_graphs_evicted_least_recently_used_and_uploaded_again(graphs, alone):
    big = sorted(range(len(graphs)), key=lambda i: -graphs[i].m)[:3]
    sizes = [_dev_bytes(graphs[i]) for i in big]
    budget = sizes[0] + sizes[1] + sizes[2] - 1  # two of the three fit, not all three
    with Server(0, BASE, mem_budget=budget) as srv:
        h0 = srv.register(graphs[big[0]])
        h1 = srv.register(graphs[big[1]])
        srv.wait(srv.submit(h0))                 # h0 used last: h1 is now the least recently used
        h2 = srv.register(graphs[big[2]])        # needs room: evicts h1
        st = srv.stats()
        assert st["evictions"] >= 1 and st["resident_bytes"] <= budget
        labels, info = srv.wait(srv.submit(h1))  # evicted: uploaded again, labels still exact
        st2 = srv.stats()
        l0, _ = srv.wait(srv.submit(h0))
        l2, _ = srv.wait(srv.submit(h2))
    assert st2["reuploads"] >= 1
    assert st2["peak_resident_bytes"] <= budget
    assert np.array_equal(labels, alone[big[1]][0])
    assert np.array_equal(l0, alone[big[0]][0]) and np.array_equal(l2, alone[big[2]][0])


def test_unknown_or_dropped_handle_is_refused(graphs):
    with Server(0, BASE) as srv:
        h = srv.register(graphs[0])
        srv.unregister(h)
        with pytest.raises(scc.SCCError):
            srv.unregister(h)
        with pytest.raises((scc.SCCError, KeyError)):
            srv.submit(h)
