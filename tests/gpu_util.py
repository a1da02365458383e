"""Shared helpers for the GPU tests (graphs and oracle comparisons)."""
import numpy as np

import gpuscc_code_b200 as scc
import oracle


def oracle_labels(g):
    labels, cnt = oracle.tarjan_labels(g.n, g.nodes, g.edges)
    return labels, cnt


def hand_graph(n, edges, drop_self=False):
    if edges:
        src = np.array([e[0] for e in edges], np.uint32)
        dst = np.array([e[1] for e in edges], np.uint32)
    else:
        src = dst = np.zeros(0, np.uint32)
    return scc.csr_from_edges(n, src, dst, drop_self_loops=drop_self)


EDGE_CASES = {
    "single": (1, []),
    "self_loop": (1, [(1, 1)]),
    "two_cycle": (2, [(1, 2), (2, 1)]),
    "chain": (50, [(i, i + 1) for i in range(1, 50)]),
    "ring": (64, [(i, i % 64 + 1) for i in range(1, 65)]),
    "ring_reverse_ids": (40, [(i + 1, i) for i in range(1, 40)] + [(1, 40)]),
    "isolated_plus_cycle": (10, [(3, 4), (4, 5), (5, 3)]),
    "pairs": (12, [(1, 2), (2, 1), (3, 4), (4, 3), (4, 5), (6, 7), (7, 6), (8, 9), (9, 8), (9, 10), (10, 9)]),
    "complete": (9, [(a, b) for a in range(1, 10) for b in range(1, 10) if a != b]),
    "dag_fan": (30, [(1, i) for i in range(2, 31)] + [(i, 30) for i in range(2, 30)]),
    "self_loops_everywhere": (6, [(i, i) for i in range(1, 7)] + [(1, 2), (2, 3), (3, 1)]),
}


def random_graphs():
    """(name, HostCSR) small-to-medium graphs of every family."""
    out = [
        ("rmat10", scc.gen_rmat(10, 8 << 10, seed=11)),
        ("rmat12_dense", scc.gen_rmat(12, 64 << 12, seed=12)),
        ("rmat14_noperm", scc.gen_rmat(14, 8 << 14, seed=13, permute=False)),
        ("er_sparse", scc.gen_er(3000, 3300, seed=14)),
        ("er_mid", scc.gen_er(2000, 4000, seed=15)),
        ("grid64", scc.gen_grid(64, 0.15, 0.001, seed=16)),
        ("grid100_bidir", scc.gen_grid(100, 0.30, 0.002, seed=17)),
    ]
    return out
