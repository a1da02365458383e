"""Phase-level parity: each C-ABI phase (trim1, trim, trim2, reach, update,
unsetPivots, update_wcc) against the oracle's restatement of the reference
kernel semantics, on the same state."""
import numpy as np
import pytest

import gpuscc_code_b200 as scc
import oracle
from gpu_util import random_graphs

pytestmark = pytest.mark.gpu

E, T, P, F, B = 4, 8, 16, 2, 1


@pytest.fixture(scope="module")
def ctx():
    c = scc.SCCContext(0)
    yield c
    c.close()


def live_sets(states):
    live = (states & E) == 0
    return live, (states & F).astype(bool) & live, (states & B).astype(bool) & live


def compare(ctx, ref: oracle.PhaseState, what):
    st = ctx.states()
    live_g, f_g, b_g = live_sets(st)
    live_o, f_o, b_o = live_sets(ref.states)
    assert np.array_equal(live_g[1:], live_o[1:]), f"{what}: eliminated sets differ"
    assert np.array_equal((st[1:] & T) > 0, (ref.states[1:] & T) > 0), f"{what}: trimmed sets differ"
    assert np.array_equal(f_g[1:], f_o[1:]), f"{what}: F sets differ"
    assert np.array_equal(b_g[1:], b_o[1:]), f"{what}: B sets differ"
    rg = ctx.ranges()
    ro = np.where(live_o, ref.ranges, 0)
    assert np.array_equal(rg[1:], ro[1:]), f"{what}: partitions differ"


@pytest.mark.parametrize("variant", ["q", "t", "d", "l", "b"])
def test_phase_sequence(ctx, variant):
    for name, g in random_graphs()[:5]:
        ctx.set_options(scc.Options(alg="t"))
        ctx.upload(g)
        ctx.phase_begin()
        ref = oracle.PhaseState(g)
        ctx.trim1()
        ref.trim(ranged=False)
        compare(ctx, ref, f"{name} trim1")
        assert ctx.select_pivots() == (1 if ref.first_pivot() else 0)
        compare(ctx, ref, f"{name} first pivot")
        for step in range(1, 6):
            first = step == 1
            ctx.fwd_reach(variant, first_step=first)
            ctx.bwd_reach(variant, first_step=first)
            ref.reach(True, ranged=not first)
            ref.reach(False, ranged=not first)
            compare(ctx, ref, f"{name} step {step} reach")
            if first:
                ctx.trim1()
                ref.trim(ranged=False)
            else:
                ctx.trim()
                ref.trim(ranged=True)
            compare(ctx, ref, f"{name} step {step} trim")
            has = ctx.update()
            np_ref = ref.update()
            assert has == (np_ref > 0)
            compare(ctx, ref, f"{name} step {step} update")
            if step == 2:
                ctx.unset_pivots()
                ref.unset_pivots()
                compare(ctx, ref, f"{name} unset")
                ctx.trim2()
                ref.trim2()
                compare(ctx, ref, f"{name} trim2")
                _, has = ctx.update_wcc()
                assert has == (ref.wcc() > 0)
                compare(ctx, ref, f"{name} wcc")
            if not has:
                break
        assert ctx.count_elimmed() == int(((ref.states[1:] & 12) == 4).sum())


def test_phases_then_labels_match_oracle(ctx):
    for name, g in random_graphs()[:3]:
        ctx.upload(g)
        ctx.phase_begin()
        ctx.trim1()
        ctx.select_pivots()
        step, has = 0, True
        while has:
            step += 1
            ctx.fwd_reach("t", first_step=step == 1)
            ctx.bwd_reach("t", first_step=step == 1)
            ctx.trim1() if step == 1 else ctx.trim()
            has = ctx.update()
        labels, cnt = ctx.labels()
        ref, rcnt = oracle.tarjan_labels(g.n, g.nodes, g.edges)
        assert cnt == rcnt and np.array_equal(labels, ref), name
