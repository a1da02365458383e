"""The CPU oracle of the strategy network and of the graph features, checked
against finite differences and hand-computed values (no GPU)."""
import numpy as np
import pytest

from oracle import mlp_oracle as mo


def rand_problem(B=7, seed=0):
    rng = np.random.default_rng(seed)
    p = rng.normal(0, 0.3, mo.N_PARAMS)
    x = rng.normal(0, 1, (B, mo.N_IN))
    y = np.stack([rng.integers(0, k, B) for _, k in mo.HEADS], axis=1)
    mean = rng.normal(0, 0.1, mo.N_IN)
    scale = rng.uniform(0.5, 2.0, mo.N_IN)
    return p, x, y, mean, scale


def test_param_count():
    assert mo.N_PARAMS == 16 * 64 + 64 + 64 * 64 + 64 + 64 * 8 + 8


def test_gradient_matches_finite_differences():
    p, x, y, mean, scale = rand_problem()
    loss, g = mo.loss_grad(p, x, y, mean, scale)
    rng = np.random.default_rng(1)
    idx = rng.choice(mo.N_PARAMS, 60, replace=False)
    eps = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += eps
        pm[i] -= eps
        fd = (mo.loss_grad(pp, x, y, mean, scale)[0] - mo.loss_grad(pm, x, y, mean, scale)[0]) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, g[i])


def test_loss_of_uniform_logits():
    p = np.zeros(mo.N_PARAMS)
    x = np.ones((3, mo.N_IN))
    y = np.zeros((3, 3), int)
    loss, g = mo.loss_grad(p, x, y)
    assert loss == pytest.approx(np.log(2) + np.log(2) + np.log(4))


def test_predict_is_argmax_per_head():
    p, x, _, mean, scale = rand_problem(B=5)
    logits, _ = mo.forward(p, x, mean, scale)
    pr = mo.predict(p, x, mean, scale)
    assert pr.shape == (5, 3)
    assert np.array_equal(pr[:, 2], logits[:, 4:8].argmax(1))


def csr(n, edges):
    nodes = np.zeros(n + 2, np.int64)
    nodesT = np.zeros(n + 2, np.int64)
    out = [[] for _ in range(n + 1)]
    inn = [[] for _ in range(n + 1)]
    for a, b in edges:
        out[a].append(b)
        inn[b].append(a)
    adj, adjT = [], []
    for v in range(1, n + 1):
        nodes[v + 1] = nodes[v] + len(out[v])
        nodesT[v + 1] = nodesT[v] + len(inn[v])
        adj += sorted(out[v])
        adjT += sorted(inn[v])
    return nodes, np.array(adj, np.int64), nodesT


def test_features_of_a_small_graph_by_hand():
    # 1->2->3->1 cycle, 3->4, 4->5, 5->4 (reciprocal pair), 6 isolated
    nodes, adj, nodesT = csr(6, [(1, 2), (2, 3), (3, 1), (3, 4), (4, 5), (5, 4)])
    f = mo.features(nodes, adj, nodesT)
    n, m = 6, 6
    assert f[0] == pytest.approx(np.log2(n)) and f[1] == pytest.approx(np.log2(m + 1))
    assert f[2] == pytest.approx(1.0)
    od = np.array([1, 1, 2, 1, 1, 0])
    assert f[3] == pytest.approx(np.log2(1 + (od ** 2).mean() - 1.0))
    assert f[4] == pytest.approx(np.log2(3)) and f[5] == pytest.approx(np.log2(3))  # max in-degree 2 (vertex 4)
    assert f[6] == pytest.approx(1 / 6) and f[7] == pytest.approx(1 / 6) and f[8] == pytest.approx(1 / 6)
    assert f[9] == pytest.approx(4 / 6) and f[10] == pytest.approx(4 / 6)
    assert f[11] == pytest.approx(1.0)
    assert f[12] == pytest.approx(2 / 6)  # 4->5 and 5->4 of the 6 sampled edges
    # hub = largest in+out degree: vertex 3 (1 in, 2 out) and 4 (2 in, 1 out) tie -> 3
    # levels from 3: {1, 4}, {2, 5}, {}
    ln = np.log2(7.0)
    assert f[13] == pytest.approx(np.log2(3) / ln) and f[14] == pytest.approx(np.log2(3) / ln)
    assert f[15] == 0.0


def test_shipped_network_on_recorded_traces():
    """The shipped parameters (trained on the device from the recorded traces
    of plain-method runs on a B200) read back through the CPU oracle pick
    choices that cost less than the plain hybrid on those traces."""
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    net = np.load(root / "gpuscc_code_b200" / "strategy_net.npz")
    tr = np.load(root / "tests" / "golden" / "strategy_traces.npz")
    X, T = tr["X"], tr["T"]
    assert net["params"].size == mo.N_PARAMS and X.shape[1] == 16 and T.shape[1] == 16
    picks = mo.predict(net["params"].astype(np.float64), X, net["mean"], net["scale"])
    import itertools
    choices = list(itertools.product(range(2), range(2), range(4)))
    idx = np.array([choices.index(tuple(int(v) for v in p)) for p in picks])
    learned = T[np.arange(len(T)), idx].sum()
    plain = T[:, 0].sum()
    assert learned < plain
    assert learned <= 1.1 * T.min(axis=1).sum()
