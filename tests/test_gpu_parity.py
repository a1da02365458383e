"""End-to-end parity on the GPU: scc_solve labels == the oracle's canonical
Tarjan labels, bit-exact, for every reachability arm and app variant."""
import numpy as np
import pytest

import gpuscc_code_b200 as scc
import oracle
from gpu_util import EDGE_CASES, hand_graph, oracle_labels, random_graphs

pytestmark = pytest.mark.gpu

ARMS = ["q", "t", "d", "l", "h", "c", "b"]
VARIANTS = {"scc": dict(wcc=False, trim2=False), "scc_w": dict(wcc=True, trim2=False),
            "scc_2_w": dict(wcc=True, trim2=True)}


@pytest.fixture(scope="module")
def ctx():
    c = scc.SCCContext(0)
    yield c
    c.close()


def solve(ctx, g, **opts):
    ctx.set_options(scc.Options(**opts))
    ctx.upload(g)
    labels, cnt, st = ctx.solve()
    return labels, cnt, st


@pytest.mark.parametrize("variant", list(VARIANTS))
@pytest.mark.parametrize("alg", ARMS)
def test_golden_files(ctx, golden, golden_dir, alg, variant):
    for name, exp in golden.items():
        g = scc.load(str(golden_dir / name))
        labels, cnt, _ = solve(ctx, g, alg=alg, **VARIANTS[variant])
        assert cnt == exp["nscc_reference"], name
        assert labels.tolist() == exp["labels"], name


@pytest.mark.parametrize("case", list(EDGE_CASES))
@pytest.mark.parametrize("alg", ["q", "t", "d", "l", "h"])
def test_edge_cases(ctx, case, alg):
    n, edges = EDGE_CASES[case]
    g = hand_graph(n, edges)
    ref, rcnt = oracle_labels(g)
    for variant in VARIANTS.values():
        labels, cnt, _ = solve(ctx, g, alg=alg, **variant)
        assert cnt == rcnt
        assert np.array_equal(labels, ref)


def test_empty_graph(ctx):
    g = hand_graph(0, [])
    labels, cnt, _ = solve(ctx, g, alg="h", wcc=True, trim2=True)
    assert cnt == 0 and labels.tolist() == [0]


@pytest.mark.parametrize("alg", ARMS)
def test_random_graphs_all_arms(ctx, alg):
    for name, g in random_graphs():
        ref, rcnt = oracle_labels(g)
        for vname, variant in VARIANTS.items():
            labels, cnt, st = solve(ctx, g, alg=alg, **variant)
            assert cnt == rcnt, (name, vname)
            assert np.array_equal(labels, ref), (name, vname)


@pytest.mark.parametrize("opts", [
    dict(alg="h", wcc=True, trim2=True, pivot_rule=1),
    dict(alg="t", pivot_rule=1, pull_alpha=-1),
    dict(alg="b", heavy_degree=256),
    dict(alg="l", heavy_degree=256, block_size=128),
    dict(alg="q", block_size=512, trim_depth=1),
    dict(alg="d", block_size=1024, trim_depth=-1),
    dict(alg="h", trim_first=False, wcc=True),
    dict(alg="h", switch_permille=0, wcc=True, trim2=True),
    dict(alg="h", switch_permille=1000, wcc=True, trim2=True),
    dict(alg="t", grid_blocks=7),
    dict(alg="h", wcc=True, trim2=True, async_depth=-1),
    dict(alg="b", wcc=True, async_depth=1, block_size=1024),
])
def test_option_space(ctx, opts):
    for name, g in random_graphs()[:4]:
        ref, rcnt = oracle_labels(g)
        labels, cnt, _ = solve(ctx, g, **opts)
        assert cnt == rcnt, name
        assert np.array_equal(labels, ref), name


@pytest.mark.parametrize("alg", ARMS)
def test_graphs_needing_several_sweep_iterations_per_cta(ctx, alg):
    """More vertices than threads in the persistent grid (148 SMs x 1024),
    so every full-id sweep runs several grid-stride iterations per CTA."""
    for g in (scc.gen_rmat(18, 4 << 18, seed=3), scc.gen_er(300_000, 450_000, seed=8)):
        ref, rcnt = oracle_labels(g)
        labels, cnt, _ = solve(ctx, g, alg=alg, wcc=True, trim2=True)
        assert cnt == rcnt and np.array_equal(labels, ref)


def test_config1_rmat16(ctx):
    """R-MAT 2^16 vertices, 2^20 samples, (0.57, 0.19, 0.19, 0.05), seed 1."""
    g = scc.gen_rmat(16, 1 << 20, seed=1)
    ref, rcnt = oracle_labels(g)
    if oracle.ref_lib() is not None:
        assert oracle.ref_tarjan(g.n, g.nodes, g.edges)[0] == rcnt
    for alg in ["q", "d", "l", "h"]:
        for variant in VARIANTS.values():
            labels, cnt, st = solve(ctx, g, alg=alg, **variant)
            assert cnt == rcnt
            assert np.array_equal(labels, ref)


def test_solve_is_repeatable(ctx):
    g = scc.gen_rmat(13, 16 << 13, seed=5)
    first = solve(ctx, g, alg="h", wcc=True, trim2=True)[0]
    for _ in range(3):
        assert np.array_equal(ctx.solve()[0], first)


def test_segments_equal_independent_solves(ctx):
    graphs = [scc.gen_rmat(9, 4 << 9, seed=40 + i) for i in range(3)] + \
             [scc.gen_er(700, 1400, seed=50), scc.gen_grid(20, 0.2, 0.0, seed=51)]
    src_all, dst_all, seg, base = [], [], [1], 0
    expect = [np.zeros(1, np.uint32)]
    for g in graphs:
        s, d = g.edge_list()
        src_all.append(s + base)
        dst_all.append(d + base)
        ref, _ = oracle_labels(g)
        expect.append(ref[1:] + base)
        base += g.n
        seg.append(base + 1)
    packed = scc.csr_from_edges(base, np.concatenate(src_all), np.concatenate(dst_all))
    exp = np.concatenate(expect)
    for alg in ["h", "q", "l"]:
        ctx.set_options(scc.Options(alg=alg, wcc=True, trim2=True))
        ctx.upload(packed)
        ctx.set_segments(seg)
        labels, cnt, _ = ctx.solve()
        ctx.set_segments(None)
        assert np.array_equal(labels, exp)
        assert cnt == int((exp[1:] == np.arange(1, base + 1)).sum())


def test_device_generator_matches_host(ctx):
    d = ctx.gen_rmat_device(12, 16 << 12, seed=2)
    dev = ctx.download()
    host = scc.gen_rmat(12, 16 << 12, seed=2)
    assert dev.n == host.n and dev.m == host.m
    assert np.array_equal(dev.nodes[1:], host.nodes[1:])
    assert np.array_equal(dev.edges, host.edges)
    assert np.array_equal(dev.nodesT[1:], host.nodesT[1:])
    assert np.array_equal(dev.edgesT, host.edgesT)


def test_iteration_cap_reports_error_and_context_recovers(ctx):
    g = scc.gen_grid(40, 0.1, 0.0, seed=9)
    ctx.set_options(scc.Options(alg="q", max_iters=1))
    ctx.upload(g)
    with pytest.raises(scc.SCCError) as ei:
        ctx.solve()
    assert ei.value.code == -5
    ref, rcnt = oracle_labels(g)
    labels, cnt, _ = solve(ctx, g, alg="q")
    assert cnt == rcnt and np.array_equal(labels, ref)


def test_invalid_graph_rejected(ctx):
    nodes = np.array([0, 0, 1, 2], np.uint32)
    raw = scc.HostCSR.from_arrays(nodes, [2, 7], nodes, [2, 1])  # edge to vertex 7 of 2
    with pytest.raises(scc.SCCError) as ei:
        ctx.upload(raw)
    assert ei.value.code == -1
