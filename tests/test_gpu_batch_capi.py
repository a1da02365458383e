"""scc_batch_pack / scc_batch_solve through the C-ABI: the packed CSR equals
the Python packing, and every graph's labels and count from one batched
launch equal the oracle's for that graph alone."""
import ctypes as C

import numpy as np
import pytest

import gpuscc_code_b200 as scc
from gpuscc_code_b200 import _capi
from gpuscc_code_b200.batch import pack
from gpu_util import oracle_labels
import oracle


def graphs():
    return [scc.gen_rmat(10, 8 << 10, seed=61), scc.gen_er(900, 2000, seed=62), scc.gen_grid(24, 0.2, 0.0, seed=63),
            scc.csr_from_edges(1, np.zeros(0, np.uint32), np.zeros(0, np.uint32)),
            scc.gen_rmat(12, 16 << 12, seed=64)]


def test_batch_pack_matches_python_packing():
    gs = graphs()
    arr = (_capi.scc_host_csr * len(gs))(*[g.raw for g in gs])
    out = _capi.scc_host_csr()
    seg = np.zeros(len(gs) + 1, np.uint32)
    _capi.check(_capi.lib.scc_batch_pack(len(gs), arr, C.byref(out), seg.ctypes.data_as(_capi.u32p)))
    packed = scc.HostCSR(out)
    ref, rseg = pack(gs)
    assert np.array_equal(seg, rseg)
    for a in ("nodes", "edges", "nodesT", "edgesT"):
        assert np.array_equal(getattr(packed, a), getattr(ref, a)), a


def test_batch_pack_rejects_broken_offsets():
    g = scc.gen_er(50, 80, seed=1)
    bad = _capi.scc_host_csr.from_buffer_copy(g.raw)
    bad.m = g.m + 1
    out = _capi.scc_host_csr()
    seg = np.zeros(2, np.uint32)
    rc = _capi.lib.scc_batch_pack(1, C.byref(bad), C.byref(out), seg.ctypes.data_as(_capi.u32p))
    assert rc == _capi.SCC_ERR_INVALID


@pytest.mark.gpu
def test_batch_solve_equals_each_graph_alone():
    gs = graphs()
    arr = (_capi.scc_host_csr * len(gs))(*[g.raw for g in gs])
    outs = [np.zeros(g.n + 1, np.uint32) for g in gs]
    ptrs = (_capi.u32p * len(gs))(*[o.ctypes.data_as(_capi.u32p) for o in outs])
    counts = np.zeros(len(gs), np.uint32)
    with scc.SCCContext(0, alg="h", wcc=True, trim2=True) as ctx:
        for _ in range(2):
            _capi.check(_capi.lib.scc_batch_solve(ctx.handle, len(gs), arr, ptrs, counts.ctypes.data_as(_capi.u32p)))
            for g, o, c in zip(gs, outs, counts):
                ref, rcnt = oracle_labels(g)
                assert np.array_equal(o, ref) and c == rcnt


@pytest.mark.gpu
def test_segment_table_with_a_crossing_edge_is_refused():
    # two 3-vertex graphs packed side by side, plus one edge 2 -> 5 across them
    src = np.array([1, 2, 3, 4, 5, 6, 2], np.uint32)
    dst = np.array([2, 3, 1, 5, 6, 4, 5], np.uint32)
    g = scc.csr_from_edges(6, src, dst)
    with scc.SCCContext(0) as ctx:
        ctx.upload(g)
        with pytest.raises(scc.SCCError) as ei:
            ctx.set_segments(np.array([1, 4, 7], np.uint32))
        assert ei.value.code == -1 and "segment" in str(ei.value)
        labels, cnt, _ = ctx.solve()  # the table was dropped: one graph again
        ref, rcnt = oracle.tarjan_labels(g.n, g.nodes, g.edges)
        assert cnt == rcnt and np.array_equal(labels, ref)
        ok = scc.csr_from_edges(6, src[:6], dst[:6])
        ctx.upload(ok)
        ctx.set_segments(np.array([1, 4, 7], np.uint32))
        labels, cnt, _ = ctx.solve()
        assert cnt == 2 and list(labels) == [0, 1, 1, 1, 4, 4, 4]
