"""Strategy network on the GPU: forward and gradients of the CUDA kernels
against the CPU oracle (oracle/mlp_oracle.py), training on the device,
features against the oracle, and the A/B test of what the trained network
gains over the plain hybrid — with labels exact under every choice."""
import numpy as np
import pytest

import gpuscc_code_b200 as scc
from gpuscc_code_b200 import learned
from gpu_util import oracle_labels
from oracle import mlp_oracle as mo

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = scc.SCCContext(0)
    yield c
    c.close()


def rand_batch(B, seed):
    rng = np.random.default_rng(seed)
    x = rng.normal(0, 2, (B, 16)).astype(np.float32)
    y = np.stack([rng.integers(0, k, B) for k in learned.HEADS], axis=1).astype(np.int32)
    return x, y


def test_forward_matches_oracle():
    net = learned.StrategyNet(0, seed=3)
    x, _ = rand_batch(33, 0)
    mean = np.linspace(-1, 1, 16).astype(np.float32)
    scale = np.linspace(0.5, 2, 16).astype(np.float32)
    net.set_norm(mean, scale)
    got = net.forward(x)
    ref, _ = mo.forward(net.params.astype(np.float64), x, mean, scale)
    np.testing.assert_allclose(got, ref, rtol=1e-4, atol=1e-4)  # fp32 kernels vs fp64 oracle
    assert np.array_equal(net.predict(x), mo.predict(net.params.astype(np.float64), x, mean, scale))


@pytest.mark.parametrize("B", [1, 17, 300])
def test_gradient_matches_oracle(B):
    net = learned.StrategyNet(0, seed=B)
    x, y = rand_batch(B, B)
    net.fit_norm(x)
    mean, scale = net.norm
    loss, g = net.loss_grad(x, y)
    rloss, rg = mo.loss_grad(net.params.astype(np.float64), x, y, mean, scale)
    assert loss == pytest.approx(rloss, rel=1e-4, abs=1e-5)
    # fp32 accumulation vs fp64: relative error of the whole gradient vector
    assert np.linalg.norm(g - rg) <= 1e-4 * np.linalg.norm(rg) + 1e-6


def test_training_on_the_device_fits_a_learnable_rule():
    rng = np.random.default_rng(7)
    x = rng.normal(0, 1, (2000, 16)).astype(np.float32)
    y = np.stack([(x[:, 0] > 0), (x[:, 1] + x[:, 2] > 0), np.digitize(x[:, 3], [-0.7, 0, 0.7])], 1).astype(np.int32)
    net = learned.StrategyNet(0, seed=1)
    net.fit_norm(x)
    before = net.loss_grad(x, y)[0]
    net.train(x, y, epochs=60, batch=64, lr=3e-3, seed=2)
    after = net.loss_grad(x, y)[0]
    assert after < 0.3 * before
    acc = (net.predict(x) == y).mean(axis=0)
    assert acc.min() > 0.9


def test_save_and_load_roundtrip(tmp_path):
    net = learned.StrategyNet(0, seed=5)
    x, _ = rand_batch(10, 1)
    net.fit_norm(x)
    path = tmp_path / "net.npz"
    net.save(path)
    other = learned.StrategyNet.load(path)
    assert np.array_equal(other.params, net.params)
    assert np.array_equal(other.forward(x), net.forward(x))


@pytest.mark.parametrize("make", [
    lambda: scc.gen_rmat(12, 16 << 12, seed=4),
    lambda: scc.gen_grid(50, 0.2, 0.001, seed=6),
    lambda: scc.gen_er(5000, 9000, seed=8),
    lambda: scc.csr_from_edges(6, np.array([1, 2, 3, 3, 4, 5], np.uint32), np.array([2, 3, 1, 4, 5, 4], np.uint32)),
])
def test_features_match_oracle(ctx, make):
    g = make()
    ctx.upload(g)
    got = learned.graph_features(ctx)
    ref = mo.features(g.nodes, g.edges, g.nodesT)
    np.testing.assert_allclose(got, ref, rtol=1e-5, atol=1e-6)


def small_stream(count, seed):
    """Graphs of the served families at sizes a test can time quickly."""
    from gpuscc_code_b200.serve import make_graph, stream_spec
    return [make_graph(stream_spec(i, seed=seed, rmat_scale=(10, 15), grid_side=(40, 160))) for i in range(count)]


def test_labels_are_exact_under_every_choice(ctx):
    base = scc.Options(alg="h", wcc=True, trim2=True)
    for g in small_stream(6, seed=21):
        ref, rcnt = oracle_labels(g)
        ctx.upload(g)
        learned.time_choices(ctx, base, repeats=1, check_labels=ref)


def test_trained_network_gain_over_plain(ctx):
    """A/B: train on traces of the plain method under every choice, then on
    held-out graphs compare the time of the network's picks with the plain
    hybrid's (choice (0,0,0)) and with the best choice per graph."""
    base = scc.Options(alg="h", wcc=True, trim2=True)
    train = small_stream(64, seed=31)
    test = small_stream(24, seed=32)
    X, T = learned.collect_traces(ctx, train, base, repeats=2)
    net = learned.train_net(X, T, epochs=300, batch=32, lr=3e-3, seed=0)
    Xt, Tt = learned.collect_traces(ctx, test, base, repeats=2)
    picks = net.predict(Xt)
    plain = Tt[:, learned.CHOICES.index(learned.PLAIN)].sum()
    mine = learned.choice_times(Tt, picks).sum()
    best = Tt.min(axis=1).sum()
    print(f"\nheld-out device ms: plain {plain:.2f}  learned {mine:.2f}  best-per-graph {best:.2f}  "
          f"gain {plain / mine:.3f}x")
    assert mine <= plain * 1.02
    # labels stay exact with the picked options
    for g, ch in zip(test[:6], picks[:6]):
        ref, _ = oracle_labels(g)
        ctx.set_options(learned.apply_choice(ch, base))
        ctx.upload(g)
        assert np.array_equal(ctx.solve()[0], ref)
