"""Host-side checks that need no GPU: every symbol the C header declares is
exported and bound, host-only entry points (loader, generators, option
mapping) behave and fail as documented."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import gpuscc_code_b200 as scc
from gpuscc_code_b200 import _capi

HEADER = Path(__file__).resolve().parents[1] / "include" / "scc_capi.h"


def declared_functions():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"^[a-z_][\w \*]*?\b(scc_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_the_public_api():
    names = declared_functions()
    for must in ["scc_load", "scc_tarjan", "scc_solve", "scc_trim1", "scc_trim2", "scc_reach", "scc_update",
                 "scc_update_wcc", "scc_solve_noalloc", "scc_mlp_train", "scc_server_submit", "scc_graph_features"]:
        assert must in names
    assert len(names) >= 60


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(str(_capi.LIB_PATH))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_every_declared_symbol():
    bound = {name for name, _, _ in _capi.SIGNATURES}
    assert set(declared_functions()) == bound


def test_struct_sizes_match_the_header_layout():
    assert C.sizeof(_capi.scc_opts) == 21 * 4
    assert C.sizeof(_capi.scc_stats) == 16 * 4 + 6 * 8
    # the trailing scc_opts (4-byte aligned) is padded to the struct's 8-byte alignment
    assert C.sizeof(_capi.scc_server_cfg) == (6 * 4 + 8 + C.sizeof(_capi.scc_opts) + 7) // 8 * 8
    assert C.sizeof(_capi.scc_request_info) == 6 * 4 + 3 * 8


def test_load_missing_file_is_an_io_error(tmp_path):
    with pytest.raises(scc.SCCError) as ei:
        scc.load(str(tmp_path / "nope.graph"))
    assert ei.value.code == _capi.SCC_ERR_IO


def test_load_garbage_is_rejected(tmp_path):
    p = tmp_path / "bad.graph"
    p.write_text("this is not a graph\n")
    with pytest.raises(scc.SCCError):
        scc.load(str(p))


def test_csr_from_edges_rejects_out_of_range_ids():
    with pytest.raises(scc.SCCError) as ei:
        scc.csr_from_edges(3, np.array([1, 5], np.uint32), np.array([2, 1], np.uint32))
    assert ei.value.code == _capi.SCC_ERR_INVALID


def test_csr_from_edges_sorts_and_deduplicates():
    g = scc.csr_from_edges(4, np.array([2, 1, 2, 1, 4], np.uint32), np.array([3, 2, 3, 3, 4], np.uint32))
    assert g.m == 4
    assert g.nodes.tolist() == [0, 0, 2, 3, 3, 4]
    assert g.edges.tolist() == [2, 3, 3, 4]
    assert g.nodesT.tolist() == [0, 0, 0, 1, 3, 4]
    assert g.edgesT.tolist() == [1, 1, 2, 4]


@pytest.mark.parametrize("make", [
    lambda: scc.gen_rmat(11, 8 << 11, seed=3),
    lambda: scc.gen_er(1500, 4000, seed=4),
    lambda: scc.gen_grid(40, 0.2, 0.001, seed=5),
])
def test_generators_are_deterministic_and_well_formed(make):
    a, b = make(), make()
    assert np.array_equal(a.nodes, b.nodes) and np.array_equal(a.edges, b.edges)
    n, m = a.n, a.m
    assert a.nodes[1] == 0 and a.nodes[n + 1] == m and a.nodesT[n + 1] == m
    assert np.all(np.diff(a.nodes[1:].astype(np.int64)) >= 0)
    assert a.edges.min() >= 1 and a.edges.max() <= n
    # transpose holds the same edge multiset
    src = np.repeat(np.arange(1, n + 1), np.diff(a.nodes[1:].astype(np.int64)))
    srcT = np.repeat(np.arange(1, n + 1), np.diff(a.nodesT[1:].astype(np.int64)))
    fwd = sorted(zip(src.tolist(), a.edges.tolist()))
    bwd = sorted(zip(a.edgesT.tolist(), srcT.tolist()))
    assert fwd == bwd


def test_gen_batch_segments_partition_the_ids():
    g, seg = scc.gen_batch(12, 100, 2000, 2.0, 6.0, seed=9)
    assert seg[0] == 1 and seg[-1] == g.n + 1 and np.all(np.diff(seg.astype(np.int64)) > 0)
    src = np.repeat(np.arange(1, g.n + 1), np.diff(g.nodes[1:].astype(np.int64)))
    seg_of = np.searchsorted(seg, np.arange(1, g.n + 1), side="right")
    assert np.array_equal(seg_of[src - 1], seg_of[g.edges.astype(np.int64) - 1])  # no edge crosses graphs


@pytest.mark.parametrize("choice,expect", [
    ((0, 0, 0), dict(pivot_rule=0, trim_depth=0, alg=4, switch_permille=10)),
    ((1, 1, 1), dict(pivot_rule=1, trim_depth=1, alg=4, switch_permille=100)),
    ((0, 1, 2), dict(pivot_rule=0, trim_depth=1, alg=4, switch_permille=1000)),
    ((1, 0, 3), dict(pivot_rule=1, trim_depth=0, alg=5, switch_permille=10)),
])
def test_strategy_choice_maps_to_options(choice, expect):
    o = _capi.scc_opts()
    _capi.lib.scc_opts_default(C.byref(o))
    o.wcc = 1
    ch = np.array(choice, np.int32)
    _capi.check(_capi.lib.scc_mlp_apply(ch.ctypes.data_as(C.POINTER(C.c_int32)), C.byref(o)))
    for k, v in expect.items():
        assert getattr(o, k) == v
    assert o.wcc == 1  # untouched


def test_strategy_choice_out_of_range_is_rejected():
    o = _capi.scc_opts()
    ch = np.array([0, 0, 4], np.int32)
    assert _capi.lib.scc_mlp_apply(ch.ctypes.data_as(C.POINTER(C.c_int32)), C.byref(o)) == _capi.SCC_ERR_INVALID


def test_stream_spec_is_deterministic_and_in_range():
    from gpuscc_code_b200.serve import poisson_arrivals, stream_spec
    specs = [stream_spec(i, seed=5) for i in range(400)]
    assert specs == [stream_spec(i, seed=5) for i in range(400)]
    kinds = [s["type"] for s in specs]
    assert 150 < kinds.count("rmat") < 250
    for s in specs:
        if s["type"] == "rmat":
            assert 14 <= s["scale"] <= 22
            assert 8 <= s["samples"] / (1 << s["scale"]) <= 32
        else:
            assert 256 <= s["side"] <= 2048 and 0.10 <= s["bidir"] <= 0.30
    t = poisson_arrivals(20000, rate=50.0, seed=1)
    assert np.all(np.diff(t) > 0)
    assert abs(len(t) / t[-1] - 50.0) < 2.0


def test_shard_plan_partitions_and_balances():
    from gpuscc_code_b200.batch import shard_graphs
    rng = np.random.default_rng(0)
    w = rng.integers(1, 1000, size=101)
    for world in (1, 2, 3, 8):
        shards = shard_graphs(w, world)
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(101))
        loads = [w[s].sum() for s in shards]
        assert max(loads) - min(loads) <= w.max()


def test_no_cpu_fallback_without_a_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(scc.SCCError) as ei:
        scc.SCCContext(0)
    assert ei.value.code == _capi.SCC_ERR_NODEVICE
    with pytest.raises(scc.SCCError):
        from gpuscc_code_b200.serve import Server
        Server(0)


def test_trace_labels_and_pick_times():
    from gpuscc_code_b200 import learned
    assert len(learned.CHOICES) == 16 and learned.CHOICES[0] == learned.PLAIN
    T = np.full((3, 16), 10.0)
    T[0, 5] = 1.0
    T[1, 0] = 2.0
    T[2, 15] = 3.0
    y = learned.labels_from_times(T)
    assert [tuple(r) for r in y] == [learned.CHOICES[5], learned.CHOICES[0], learned.CHOICES[15]]
    assert learned.choice_times(T, y).tolist() == [1.0, 2.0, 3.0]


def test_apply_choice_keeps_base_options():
    from gpuscc_code_b200 import learned
    base = scc.Options(alg="h", wcc=True, trim2=True, heavy_degree=1024)
    o = learned.apply_choice((1, 1, 3), base)
    assert o.alg == "c" and o.pivot_rule == 1 and o.trim_depth == 1 and o.switch_permille == 10
    assert o.wcc is True and o.trim2 is True and o.heavy_degree == 1024
