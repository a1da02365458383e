"""Learned strategy selection: a small MLP picks, per graph, the options of the
decomposition that never change its labels (pivot rule, trim depth, reach arm
/ switch point) from 16 graph statistics computed on the device.

The network's training, inference and gradients run in the library's own
CUDA kernels (scc_mlp_* in include/scc_capi.h); this module holds the host
side: the trace collection that labels graphs by timing the plain method
under every choice, the normalisation, and saving/loading the parameters.
The plain hybrid (choice (0, 0, 0)) stays the fallback: without a network,
or for a choice the caller rejects, the options are the base options.
"""
from __future__ import annotations

import ctypes as C
import itertools
from pathlib import Path

import numpy as np

from ._capi import check, lib, scc_opts
from .scc import Options, SCCContext, HostCSR

HEADS = (2, 2, 4)
N_FEATURES = 16
FEATURE_NAMES = [
    "log2_n", "log2_m", "mean_out_degree", "log2_var_out_degree", "log2_max_out_degree", "log2_max_in_degree",
    "frac_out0", "frac_in0", "frac_trim_first_sweep", "frac_out1", "frac_in1", "frac_low_degree",
    "reciprocity", "bfs_level1", "bfs_level2", "bfs_level3",
]
CHOICES = [tuple(c) for c in itertools.product(range(HEADS[0]), range(HEADS[1]), range(HEADS[2]))]
PLAIN = (0, 0, 0)
DEFAULT_MODEL = Path(__file__).resolve().parent / "strategy_net.npz"


def graph_features(ctx: SCCContext) -> np.ndarray:
    """16 statistics of the graph bound to ctx (device pass, see scc_features.h)."""
    f = np.zeros(N_FEATURES, np.float32)
    check(lib.scc_graph_features(ctx.handle, f.ctypes.data_as(C.POINTER(C.c_float))))
    return f


def apply_choice(choice, base: Options) -> Options:
    """Options for a choice (scc_mlp_apply), all other fields from base."""
    o = base.to_c()
    ch = np.ascontiguousarray(choice, np.int32)
    check(lib.scc_mlp_apply(ch.ctypes.data_as(C.POINTER(C.c_int32)), C.byref(o)))
    from ._capi import ALG_NAMES
    kw = {k: getattr(o, k) for k, _ in scc_opts._fields_}
    kw["alg"] = ALG_NAMES[kw["alg"]]
    return Options(**{k: (bool(v) if isinstance(getattr(base, k), bool) else v) for k, v in kw.items()})


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, np.float32)


def _fp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class StrategyNet:
    """Handle on the device-resident network (scc_mlp)."""

    def __init__(self, device: int = 0, seed: int = 0):
        h = C.c_void_p()
        check(lib.scc_mlp_create(device, seed, C.byref(h)))
        self._h = h
        self.device = device

    def close(self):
        if getattr(self, "_h", None):
            lib.scc_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    @staticmethod
    def param_count() -> int:
        return int(lib.scc_mlp_param_count())

    @property
    def params(self) -> np.ndarray:
        p = np.zeros(self.param_count(), np.float32)
        check(lib.scc_mlp_params(self._h, _fp(p), 1))
        return p

    @params.setter
    def params(self, p) -> None:
        p = _f32(p)
        if p.size != self.param_count():
            raise ValueError(f"expected {self.param_count()} parameters, got {p.size}")
        check(lib.scc_mlp_params(self._h, _fp(p), 0))

    @property
    def norm(self):
        mean = np.zeros(N_FEATURES, np.float32)
        scale = np.zeros(N_FEATURES, np.float32)
        check(lib.scc_mlp_norm(self._h, _fp(mean), _fp(scale), 1))
        return mean, scale

    def set_norm(self, mean, scale) -> None:
        mean, scale = _f32(mean), _f32(scale)
        check(lib.scc_mlp_norm(self._h, _fp(mean), _fp(scale), 0))

    def fit_norm(self, x) -> None:
        """Standardise with the training set's mean and spread."""
        x = np.asarray(x, np.float64)
        sd = x.std(axis=0)
        self.set_norm(x.mean(axis=0), 1.0 / np.where(sd > 1e-6, sd, 1.0))

    def forward(self, x) -> np.ndarray:
        x = _f32(np.atleast_2d(x))
        out = np.zeros((x.shape[0], 8), np.float32)
        check(lib.scc_mlp_forward(self._h, _fp(x), x.shape[0], _fp(out)))
        return out

    def loss_grad(self, x, y):
        x = _f32(np.atleast_2d(x))
        y = np.ascontiguousarray(np.atleast_2d(y), np.int32)
        loss = np.zeros(1, np.float32)
        g = np.zeros(self.param_count(), np.float32)
        check(lib.scc_mlp_loss_grad(self._h, _fp(x), y.ctypes.data_as(C.POINTER(C.c_int32)), x.shape[0],
                                    _fp(loss), _fp(g)))
        return float(loss[0]), g

    def train(self, x, y, epochs: int = 200, batch: int = 64, lr: float = 3e-3, seed: int = 0) -> float:
        x = _f32(np.atleast_2d(x))
        y = np.ascontiguousarray(np.atleast_2d(y), np.int32)
        loss = np.zeros(1, np.float32)
        check(lib.scc_mlp_train(self._h, _fp(x), y.ctypes.data_as(C.POINTER(C.c_int32)), x.shape[0], epochs,
                                batch, lr, seed, _fp(loss)))
        return float(loss[0])

    def predict(self, x) -> np.ndarray:
        x = _f32(np.atleast_2d(x))
        out = np.zeros((x.shape[0], 3), np.int32)
        check(lib.scc_mlp_predict(self._h, _fp(x), x.shape[0], out.ctypes.data_as(C.POINTER(C.c_int32))))
        return out

    def save(self, path) -> None:
        mean, scale = self.norm
        np.savez(path, params=self.params, mean=mean, scale=scale)

    @classmethod
    def load(cls, path=DEFAULT_MODEL, device: int = 0) -> "StrategyNet":
        d = np.load(path)
        net = cls(device)
        net.params = d["params"]
        net.set_norm(d["mean"], d["scale"])
        return net


def time_choices(ctx: SCCContext, base: Options, repeats: int = 2, choices=CHOICES,
                 check_labels: np.ndarray | None = None) -> np.ndarray:
    """Device time (ms, min over repeats) of the bound graph's solve under every
    choice.  With check_labels, every solve's labels are compared with it."""
    out = np.zeros(len(choices))
    for i, ch in enumerate(choices):
        ctx.set_options(apply_choice(ch, base))
        best = float("inf")
        for _ in range(repeats):
            labels, cnt, st = ctx.solve(want_labels=check_labels is not None)
            if check_labels is not None and not np.array_equal(labels, check_labels):
                raise AssertionError(f"labels changed under choice {ch}")
            best = min(best, st["ms_total"])
        out[i] = best
    return out


def labels_from_times(times: np.ndarray, choices=CHOICES) -> np.ndarray:
    """Training target per graph: the choice with the smallest time, split
    into its three heads (B x 3)."""
    idx = np.argmin(times, axis=1)
    return np.array([choices[i] for i in idx], np.int32)


def collect_traces(ctx: SCCContext, graphs, base: Options, repeats: int = 2):
    """Runs the plain method under every choice on each graph (a HostCSR, or
    a callable that binds a graph to ctx) and returns (features B x 16,
    times B x 16 choices)."""
    X, T = [], []
    for g in graphs:
        if isinstance(g, HostCSR):
            ctx.upload(g)
        else:
            g(ctx)
        X.append(graph_features(ctx))
        T.append(time_choices(ctx, base, repeats))
    return np.array(X, np.float32), np.array(T)


def train_net(X, T, device: int = 0, epochs: int = 300, batch: int = 64, lr: float = 3e-3,
              seed: int = 0) -> StrategyNet:
    net = StrategyNet(device, seed)
    net.fit_norm(X)
    net.train(X, labels_from_times(T), epochs=epochs, batch=batch, lr=lr, seed=seed)
    return net


def choice_times(T: np.ndarray, picks: np.ndarray, choices=CHOICES) -> np.ndarray:
    """Time of each graph under the picked choice (T: B x len(choices))."""
    index = {c: i for i, c in enumerate(choices)}
    return np.array([T[b, index[tuple(int(v) for v in picks[b])]] for b in range(len(picks))])
