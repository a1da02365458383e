"""Asynchronous phases of the engine against the oracle: reaches that
continue without level barriers (the forward and backward reaches of a round
sharing one queue, claims kept by the warp that made them), asynchronous
HYBRID / COMBINE / BEST tails and asynchronous trim worklists on thin graphs.
Labels must equal the oracle's Tarjan whatever async_depth says, with the
reference's synchronous levels (async_depth = -1) as the control, for every
block size (the staging segments that hold kept claims differ in size), and
queues capped far below the graph's needs must report the overflow and leave
the context exact."""
import numpy as np
import pytest

import gpuscc_code_b200 as scc
from gpu_util import oracle_labels

pytestmark = pytest.mark.gpu


def thin_graphs():
    # grids: thousands of levels, cascading trims, deep tails
    return [("grid300_b15", scc.gen_grid(300, 0.15, 0.001, seed=11)),
            ("grid200_b30", scc.gen_grid(200, 0.30, 0.002, seed=12)),
            ("grid128_b05", scc.gen_grid(128, 0.05, 0.0, seed=13)),
            ("er_deg2", scc.gen_er(40_000, 90_000, seed=14))]


@pytest.fixture(scope="module")
def graphs():
    return [(name, g, *oracle_labels(g)) for name, g in thin_graphs()]


@pytest.mark.parametrize("async_depth", [-1, 0, 1, 16])
@pytest.mark.parametrize("alg", ["h", "t", "b", "c"])
def test_labels_equal_oracle_for_every_async_depth(graphs, alg, async_depth):
    with scc.SCCContext(0, alg=alg, wcc=True, trim2=True, async_depth=async_depth) as ctx:
        for name, g, ref, rcnt in graphs:
            ctx.upload(g)
            labels, cnt, _ = ctx.solve()
            assert cnt == rcnt, name
            assert np.array_equal(labels, ref), name


@pytest.mark.parametrize("block_size", [128, 256, 512, 1024])
def test_asynchronous_phases_at_every_block_size(graphs, block_size):
    with scc.SCCContext(0, alg="h", wcc=True, trim2=True, block_size=block_size) as ctx:
        for name, g, ref, rcnt in graphs:
            ctx.upload(g)
            labels, cnt, _ = ctx.solve()
            assert cnt == rcnt and np.array_equal(labels, ref), name


def test_repeated_solves_leave_the_queue_clean(graphs):
    # every asynchronous phase must hand back an all-empty queue: the same
    # context solves every graph three times over, interleaved
    with scc.SCCContext(0, alg="h", wcc=True, trim2=True) as ctx:
        for _ in range(3):
            for name, g, ref, rcnt in graphs:
                ctx.upload(g)
                labels, cnt, _ = ctx.solve()
                assert cnt == rcnt and np.array_equal(labels, ref), name


def test_async_queue_overflow_is_reported_and_context_recovers(graphs):
    name, g, ref, rcnt = graphs[0]
    with scc.SCCContext(0, alg="h", wcc=True, trim2=True, async_depth=1, test_queue_cap=64) as ctx:
        ctx.upload(g)
        with pytest.raises(scc.SCCError) as ei:
            ctx.solve()
        assert ei.value.code == -5
        assert "queue overflow" in str(ei.value)
        # a failed solve may leave queue slots and election slots filled:
        # the next solve on the context restores them and is exact
        ctx.set_options(scc.Options(alg="h", wcc=True, trim2=True))
        labels, cnt, _ = ctx.solve()
        assert cnt == rcnt and np.array_equal(labels, ref)


def test_phase_api_reach_is_asynchronous_alone(graphs):
    # the phase-level reach has no partner direction: it runs its
    # asynchronous part at once; states and partitions after the round equal
    # those of the reference's synchronous levels
    name, g, ref, rcnt = graphs[0]
    out = []
    for depth in (1, -1):
        with scc.SCCContext(0, alg="t", async_depth=depth) as ctx:
            ctx.upload(g)
            ctx.phase_begin()
            ctx.trim1()
            ctx.select_pivots()
            fd = ctx.fwd_reach("t", first_step=True)
            bd = ctx.bwd_reach("t", first_step=True)
            assert fd >= 1 and bd >= 1
            ctx.update()
            out.append((ctx.states().copy(), ctx.ranges().copy()))
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])
