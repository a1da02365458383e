"""Device-side timers of a solve (the engine's counterpart of the reference's
STOPWATCH timers, timing.h:14 / timing.cpp:5-19, which time each phase on the
host with a device sync): per-phase totals and counts (scc_get_profile), the
per-event trace (scc_get_trace) and the stats' phase times.  They must be
consistent with each other and with the kernel's own time, cover the phases
the solve ran, and start afresh with every solve."""
import numpy as np
import pytest

import gpuscc_code_b200 as scc

pytestmark = pytest.mark.gpu

SLOTS = set(scc.SCCContext.PROFILE_SLOTS)


def solve(g, **opts):
    with scc.SCCContext(0, alg="h", wcc=True, trim2=True, **opts) as ctx:
        ctx.upload(g)
        ctx.solve()  # the first launch of a context also pays for loading the kernel
        labels, cnt, st = ctx.solve()
        return st, ctx.profile(), ctx.trace()


def test_profile_covers_the_phases_and_fits_in_the_kernel():
    st, prof, trace = solve(scc.gen_rmat(16, 1 << 20, seed=1))
    for slot in ("trim_sweep", "update", "wcc", "finalize"):
        assert slot in prof, slot
    assert "pull" in prof or "worklist_level" in prof
    assert set(prof) <= SLOTS
    total = sum(ms for ms, _ in prof.values())
    assert all(ms >= 0 and n >= 1 for ms, n in prof.values())
    # phases run inside the persistent kernel: their sum is most of its time and never more
    assert 0.5 * st["ms_total"] <= total <= 1.05 * st["ms_total"]
    phases = st["ms_trim"] + st["ms_fwd"] + st["ms_bwd"] + st["ms_update"] + st["ms_wcc"]
    assert 0 < phases <= 1.05 * st["ms_total"]


def test_trace_agrees_with_profile():
    st, prof, trace = solve(scc.gen_rmat(14, 16 << 14, seed=3))
    assert 0 < len(trace) < 128  # not truncated: every event is in the trace
    per = {}
    for name, a, b, ms in trace:
        assert name in SLOTS
        assert ms >= 0
        t, n = per.get(name, (0.0, 0))
        per[name] = (t + ms, n + 1)
    assert set(per) == set(prof)
    for name, (ms, n) in prof.items():
        assert per[name][1] == n, name
        assert abs(per[name][0] - ms) <= 1e-3 * max(1, n), name
    # the solve starts with the first trim sweep and ends with finalize
    assert trace[0][0] == "trim_sweep" and trace[-1][0] == "finalize"


def test_asynchronous_and_wcc_sweep_events_on_a_grid():
    st, prof, trace = solve(scc.gen_grid(256, 0.15, 0.001, seed=3))
    assert "async" in prof and "wcc_sweep" in prof
    # an asynchronous event reports the vertices it created and the warp steps taken
    ev = [(a, b) for name, a, b, _ in trace if name == "async"]
    assert ev and all(a >= 1 and b >= 1 for a, b in ev)


def test_timers_start_afresh_with_every_solve():
    big, small = scc.gen_grid(256, 0.15, 0.001, seed=3), scc.gen_rmat(10, 8 << 10, seed=5)
    with scc.SCCContext(0, alg="h", wcc=True, trim2=True) as ctx:
        ctx.upload(big)
        ctx.solve()
        n_big = sum(n for _, n in ctx.profile().values())
        ctx.upload(small)
        ctx.solve()
        prof = ctx.profile()
        n_small = sum(n for _, n in prof.values())
        assert n_small < n_big
        assert np.isclose(sum(ms for ms, _ in prof.values()), sum(ms for *_, ms in ctx.trace()), atol=1e-2)
