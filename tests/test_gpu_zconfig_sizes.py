"""Label parity at the full sizes of the benchmark workloads.

Every SCC partition the engine produces on the graphs the benchmarks are
quoted on is compared bit-exactly (after canonicalising each component to its
minimum vertex id) with the oracle's restatement of the reference's Tarjan
(tarjan.cpp:110-190), and the SCC count with the reference's own
TR_Decomposition (tarjan.cpp:72) where oracle/_ref is built:

  * R-MAT 2^26 vertices, 2^30 samples, seed 2, scc_2_w -a h (the headline);
  * the 4096 x 4096 grid, 15 % bidirectional, 0.1 % long-range edges, seed 3;
  * all 4096 graphs of the mixed ER / R-MAT batch (seed 4), solved in one
    captured launch with the autotuner's kind of options, each graph checked
    on its own;
  * the two largest graph kinds of the served stream: R-MAT 2^22 at average
    degree 16 and a 2048-side grid at 30 % bidirectional.

These are the slowest tests of the suite (Tarjan over 10^9 edges on one host
thread), so the file sorts after the other GPU tests.
"""
from concurrent.futures import ThreadPoolExecutor
import os

import numpy as np
import pytest

import gpuscc_code_b200 as scc
import oracle

pytestmark = pytest.mark.gpu

ABC = (0.57, 0.19, 0.19)
SCC_2_W = dict(alg="h", wcc=True, trim2=True)


def _largest(labels):
    return int(np.bincount(labels[1:]).max()) if len(labels) > 1 else 0


def _check_against_tarjan(g, labels, cnt):
    ref, rcnt = oracle.tarjan_labels(g.n, g.nodes, g.edges)
    assert cnt == rcnt, (cnt, rcnt)
    assert np.array_equal(labels, ref), f"{int((labels != ref).sum())} labels differ from Tarjan"
    if oracle.ref_lib() is not None:
        own_cnt, _ = oracle.ref_tarjan(g.n, g.nodes, g.edges)
        assert own_cnt == cnt, (own_cnt, cnt)
    return ref


def test_rmat26_headline_bit_exact():
    with scc.SCCContext(0, **SCC_2_W) as ctx:
        d = ctx.gen_rmat_device(26, 1 << 30, ABC, seed=2)
        assert d.n == 1 << 26
        cnt, st = ctx.solve_device()
        labels = ctx.read_labels()
        g = ctx.download()
    ref = _check_against_tarjan(g, labels, cnt)
    assert st["largest_scc"] == _largest(ref)


def test_grid4096_bit_exact():
    g = scc.gen_grid(4096, 0.15, 0.001, seed=3)
    with scc.SCCContext(0, **SCC_2_W) as ctx:
        ctx.upload(g)
        labels, cnt, st = ctx.solve()
    ref = _check_against_tarjan(g, labels, cnt)
    assert st["largest_scc"] == _largest(ref)


def _local_graph(nodes, edges, nodesT, edgesT, lo, hi):
    """Graph on global ids lo .. hi-1 of a packed batch, in local ids."""
    e0, e1 = int(nodes[lo]), int(nodes[hi])
    t0, t1 = int(nodesT[lo]), int(nodesT[hi])
    k = hi - lo
    ln = np.zeros(k + 2, np.uint32)
    ln[1:] = nodes[lo:hi + 1] - e0
    lt = np.zeros(k + 2, np.uint32)
    lt[1:] = nodesT[lo:hi + 1] - t0
    return ln, edges[e0:e1] - np.uint32(lo - 1), lt, edgesT[t0:t1] - np.uint32(lo - 1)


def test_batch4096_every_graph_bit_exact():
    opts = scc.Options(block_size=512, heavy_degree=1024, pull_alpha=6, switch_permille=50, **SCC_2_W)
    with scc.SCCContext(0, opts) as ctx:
        seg = ctx.gen_batch_device(4096, 1000, 200_000, 2.0, 16.0, seed=4)
        ctx.capture()
        cnt, st = ctx.replay()
        labels = ctx.read_labels()
        full = ctx.download()
    nodes, edges = np.asarray(full.nodes), np.asarray(full.edges)
    nodesT, edgesT = np.asarray(full.nodesT), np.asarray(full.edgesT)

    def one(gi):
        lo, hi = int(seg[gi]), int(seg[gi + 1])
        ln, le, _, _ = _local_graph(nodes, edges, nodesT, edgesT, lo, hi)
        ref, rcnt = oracle.tarjan_labels(hi - lo, ln, le)
        mine = np.zeros(hi - lo + 1, np.uint32)
        mine[1:] = labels[lo:hi] - np.uint32(lo - 1)
        return gi, rcnt, bool(np.array_equal(mine, ref))

    # ctypes drops the GIL inside the oracle, so host threads check graphs side by side
    with ThreadPoolExecutor(max_workers=min(16, os.cpu_count() or 1)) as ex:
        res = list(ex.map(one, range(len(seg) - 1)))
    bad = [gi for gi, _, ok in res if not ok]
    assert not bad, f"{len(bad)} graphs differ from Tarjan, first {bad[:5]}"
    assert sum(r for _, r, _ in res) == cnt


@pytest.mark.parametrize("kind", ["rmat22_deg16", "grid2048_bidir30"])
def test_stream_sized_graphs_bit_exact(kind):
    with scc.SCCContext(0, **SCC_2_W) as ctx:
        if kind.startswith("rmat"):
            ctx.gen_rmat_device(22, 16 << 22, ABC, seed=5)
            g = ctx.download()
        else:
            g = scc.gen_grid(2048, 0.30, 0.001, seed=5)
            ctx.upload(g)
        labels, cnt, _ = ctx.solve()
    _check_against_tarjan(g, labels, cnt)
