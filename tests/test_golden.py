"""Oracle and loader pinned against the reference's own outputs (golden.json,
written by tests/golden/make_golden.py from the reference load() and
TR_Decomposition())."""
import numpy as np
import pytest

import gpuscc_code_b200 as scc
import oracle


def test_demo_graph_known_answer(golden):
    # hand trace of demo.graph: {1} {3} {4} {2,5,6} {8,13} {7,9,10,11,12}
    g = golden["demo.graph"]
    assert g["nscc_reference"] == 6
    comps = {}
    for v, l in enumerate(g["labels"][1:], start=1):
        comps.setdefault(l, []).append(v)
    assert sorted(comps.values()) == sorted([[1], [3], [4], [2, 5, 6], [8, 13], [7, 9, 10, 11, 12]])


@pytest.mark.parametrize("name", ["demo.graph", "rand_sparse.graph", "rand_dense.graph", "cycles.graph",
                                  "isolated.graph", "general.mtx", "pattern_sym.mtx"])
def test_loader_matches_reference_load(golden, golden_dir, name):
    exp = golden[name]
    g = scc.load(str(golden_dir / name))
    assert g.n == exp["n"]
    assert g.nnz_header == exp["nnz"]
    assert g.nodes[1:].tolist() == exp["nodes"][1:]
    assert g.edges.tolist() == exp["edges"]
    assert g.nodesT[1:].tolist() == exp["nodesT"][1:]
    assert g.edgesT.tolist() == exp["edgesT"]


@pytest.mark.parametrize("name", ["demo.graph", "rand_sparse.graph", "rand_dense.graph", "cycles.graph",
                                  "isolated.graph", "general.mtx", "pattern_sym.mtx"])
def test_oracle_tarjan_pinned(golden, name):
    exp = golden[name]
    nodes, edges = np.array(exp["nodes"], np.uint32), np.array(exp["edges"], np.uint32)
    labels, cnt = oracle.tarjan_labels(exp["n"], nodes, edges)
    assert cnt == exp["nscc_reference"]
    assert labels.tolist() == exp["labels"]


@pytest.mark.parametrize("name", ["demo.graph", "rand_dense.graph", "cycles.graph", "general.mtx"])
def test_product_tarjan_matches_golden(golden, golden_dir, name):
    g = scc.load(str(golden_dir / name))
    labels, cnt, _ = scc.tarjan(g)
    assert cnt == golden[name]["nscc_reference"]
    assert labels.tolist() == golden[name]["labels"]


def test_reference_objects_agree_when_present(golden, golden_dir):
    if oracle.ref_lib() is None:
        pytest.skip("oracle/_ref not built here")
    for name, exp in golden.items():
        r = oracle.ref_load(golden_dir / name)
        assert r["edges"].tolist() == exp["edges"]
        cnt, _ = oracle.ref_tarjan(r["n"], r["nodes"], r["edges"])
        assert cnt == exp["nscc_reference"]


def test_verify_partition_catches_planted_mistakes(golden):
    exp = golden["demo.graph"]
    n = exp["n"]
    arrs = [np.array(exp[k], np.uint32) for k in ("nodes", "edges", "nodesT", "edgesT")]
    good = np.array(exp["labels"], np.uint32)
    assert oracle.verify_partition(n, *arrs, good) == 0
    split = good.copy()
    split[5] = 5  # 5 leaves {2,5,6}
    assert oracle.verify_partition(n, *arrs, split) != 0
    merged = good.copy()
    merged[merged == 8] = 7  # {8,13} merged into {7,...}: 7 -> 8 -> 13 -> 8, no way back
    merged[7] = 7
    assert oracle.verify_partition(n, *arrs, merged) != 0
