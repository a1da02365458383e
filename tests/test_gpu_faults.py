"""Failure paths of the persistent kernel, made to happen without faulting or
hanging the GPU: a grid-barrier wait that runs out (one CTA delays its arrival
by a bounded spin longer than timeout_ms) and a worklist that would overflow
(its usable length capped below what the graph needs).  Both must come back as
SCC_ERR_TIMEOUT with the cause in the message, and the next solve on the same
context must be exact.  The reference has neither check: its barriers are
kernel boundaries and its worklist drops pushes past the end silently
(worklistc.h:79-81)."""
import numpy as np
import pytest

import gpuscc_code_b200 as scc
import oracle

pytestmark = pytest.mark.gpu

BASE = dict(alg="h", wcc=True, trim2=True)


@pytest.fixture(scope="module")
def graph():
    g = scc.gen_rmat(14, 16 << 14, seed=21)
    ref, cnt = oracle.tarjan_labels(g.n, g.nodes, g.edges)
    return g, ref, cnt


def test_barrier_wait_runs_out_and_context_recovers(graph):
    g, ref, cnt = graph
    with scc.SCCContext(0, **BASE) as ctx:
        ctx.upload(g)
        ctx.set_options(scc.Options(timeout_ms=1, test_stall_us=30_000, **BASE))
        with pytest.raises(scc.SCCError) as ei:
            ctx.solve()
        assert ei.value.code == -5
        assert "barrier wait timed out" in str(ei.value)
        ctx.set_options(scc.Options(**BASE))
        labels, got, _ = ctx.solve()
        assert got == cnt and np.array_equal(labels, ref)


def test_stall_shorter_than_the_timeout_changes_nothing(graph):
    g, ref, cnt = graph
    with scc.SCCContext(0, timeout_ms=2000, test_stall_us=2_000, **BASE) as ctx:
        ctx.upload(g)
        labels, got, _ = ctx.solve()
    assert got == cnt and np.array_equal(labels, ref)


@pytest.mark.parametrize("alg", ["h", "d", "l"])
def test_worklist_overflow_is_reported_not_dropped(graph, alg):
    g, ref, cnt = graph
    opts = dict(BASE, alg=alg)
    with scc.SCCContext(0, test_queue_cap=16, **opts) as ctx:
        ctx.upload(g)
        with pytest.raises(scc.SCCError) as ei:
            ctx.solve()
        assert ei.value.code == -5
        assert "queue overflow" in str(ei.value)
        ctx.set_options(scc.Options(**opts))
        labels, got, _ = ctx.solve()
        assert got == cnt and np.array_equal(labels, ref)


def test_queue_cap_above_need_changes_nothing(graph):
    g, ref, cnt = graph
    with scc.SCCContext(0, test_queue_cap=g.n + 1, **BASE) as ctx:
        ctx.upload(g)
        labels, got, _ = ctx.solve()
    assert got == cnt and np.array_equal(labels, ref)
