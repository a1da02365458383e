"""scc_solve_noalloc: the decomposition for callers that cannot allocate
device memory (plugins whose host framework owns the whole device-memory
budget, loops that must avoid the allocator's implicit synchronisation).  Its scratch is a static device array shared by all calls,
so the test calls it twice in a row — on two different graphs and then on the
first again — and compares each result, bit-exact, with scc_solve_device's
(the context-owned-scratch entry point) on the same graph.

Named test_zz_* so pytest collects it last; it also passes alone in a fresh
process."""
import ctypes as C

import numpy as np
import pytest

import gpuscc_code_b200 as scc
from gpuscc_code_b200._capi import SCC_ERR_CAPACITY, SCC_ERR_INVALID, check, lib, scc_dev_csr, scc_opts

pytestmark = pytest.mark.gpu


def _device_graph(g):
    import torch

    keep = [torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint32).view(np.int32)).cuda()
            for a in (g.nodes, g.edges if g.m else np.zeros(1, np.uint32), g.nodesT,
                      g.edgesT if g.m else np.zeros(1, np.uint32))]
    d = scc_dev_csr(n=g.n, m=g.m, sorted_unique=1, nodes=keep[0].data_ptr(), edges=keep[1].data_ptr(),
                    nodesT=keep[2].data_ptr(), edgesT=keep[3].data_ptr())
    return d, keep


def _reference_labels(g, **opts):
    """Labels from the existing entry point (context-owned scratch)."""
    import torch

    with scc.SCCContext(0, **opts) as ctx:
        ctx.upload(g)
        out = torch.zeros(g.n + 1, dtype=torch.int32, device="cuda")
        cnt, _ = ctx.solve_device(out.data_ptr())
        torch.cuda.synchronize()
        return out.cpu().numpy().view(np.uint32).copy(), cnt


def _noalloc(g, d, **opts):
    import torch

    o = scc.Options(**opts).to_c()
    out = torch.full((g.n + 1,), -1, dtype=torch.int32, device="cuda")
    cnt = C.c_uint32()
    check(lib.scc_solve_noalloc(C.byref(d), C.byref(o), C.c_void_p(out.data_ptr()), C.byref(cnt), None))
    torch.cuda.synchronize()
    return out.cpu().numpy().view(np.uint32).copy(), int(cnt.value)


def test_noalloc_matches_solve_device_on_consecutive_calls():
    opts = dict(alg="h", wcc=True, trim2=True)
    g1 = scc.gen_rmat(16, 1 << 20, seed=1)            # the 2^16-vertex R-MAT: the largest size allowed
    g2 = scc.gen_grid(90, 0.15, 0.001, seed=3)         # smaller, different structure
    d1, k1 = _device_graph(g1)
    d2, k2 = _device_graph(g2)
    ref1, c1 = _reference_labels(g1, **opts)
    ref2, c2 = _reference_labels(g2, **opts)
    for g, d, ref, cnt in ((g1, d1, ref1, c1), (g2, d2, ref2, c2), (g1, d1, ref1, c1)):
        labels, got = _noalloc(g, d, **opts)
        assert got == cnt
        assert np.array_equal(labels, ref)
    del k1, k2


def test_noalloc_rejects_graphs_beyond_its_limit():
    g = scc.gen_er(70000, 10, seed=4)
    d, keep = _device_graph(g)
    o = scc_opts()
    lib.scc_opts_default(C.byref(o))
    cnt = C.c_uint32()
    rc = lib.scc_solve_noalloc(C.byref(d), C.byref(o), None, C.byref(cnt), None)
    assert rc == SCC_ERR_CAPACITY
    assert b"65536" in lib.scc_last_error()
    del keep


def test_noalloc_rejects_the_options_the_context_rejects():
    g = scc.gen_rmat(8, 1 << 11, seed=2)
    d, keep = _device_graph(g)
    for bad in (dict(occupancy=9), dict(block_size=300), dict(heavy_degree=10), dict(pivot_rule=5)):
        o = scc.Options(**bad).to_c()
        cnt = C.c_uint32()
        rc = lib.scc_solve_noalloc(C.byref(d), C.byref(o), None, C.byref(cnt), None)
        assert rc == SCC_ERR_INVALID, bad
        with pytest.raises(scc.SCCError):
            scc.SCCContext(0, **bad)
    del keep
