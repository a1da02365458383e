"""CPU oracle for the strategy network and its graph features — TEST INFRASTRUCTURE ONLY.

Plain numpy (float64) restatement of the math the CUDA kernels in
gpuscc_code_b200/csrc/scc_mlp.cu and scc_features.cu implement, used by the
tests as the checker.  The reference has no learned component (its strategy
is the fixed -a flag, scc.cu:80-96), so this oracle is pinned by finite
differences of its own loss, not by reference vectors.

Parameter layout (flat, float32 on the device): W1[16][64], b1[64],
W2[64][64], b2[64], W3[64][8], b3[8]; row index = input unit.  Heads:
logits[0:2] pivot rule, [2:4] trim depth, [4:8] reach arm / switch point.
"""
from __future__ import annotations

import numpy as np

N_IN, N_H, N_OUT = 16, 64, 8
HEADS = ((0, 2), (2, 2), (4, 4))  # (first logit, classes)
SHAPES = [("W1", (N_IN, N_H)), ("b1", (N_H,)), ("W2", (N_H, N_H)), ("b2", (N_H,)), ("W3", (N_H, N_OUT)),
          ("b3", (N_OUT,))]
N_PARAMS = sum(int(np.prod(s)) for _, s in SHAPES)


def unflatten(p: np.ndarray) -> dict:
    out, o = {}, 0
    for name, shape in SHAPES:
        k = int(np.prod(shape))
        out[name] = np.asarray(p[o:o + k], np.float64).reshape(shape)
        o += k
    return out


def forward(p: np.ndarray, x: np.ndarray, mean=None, scale=None):
    """Returns (logits, cache).  x: (B, 16) raw features; normalised as
    (x - mean) * scale before the first layer."""
    w = unflatten(p)
    x = np.asarray(x, np.float64)
    mean = np.zeros(N_IN) if mean is None else np.asarray(mean, np.float64)
    scale = np.ones(N_IN) if scale is None else np.asarray(scale, np.float64)
    xn = (x - mean) * scale
    h1 = np.maximum(xn @ w["W1"] + w["b1"], 0.0)
    h2 = np.maximum(h1 @ w["W2"] + w["b2"], 0.0)
    logits = h2 @ w["W3"] + w["b3"]
    return logits, (w, xn, h1, h2)


def loss_grad(p: np.ndarray, x: np.ndarray, y: np.ndarray, mean=None, scale=None):
    """Mean over samples of the summed per-head softmax cross-entropy, and its
    gradient w.r.t. the flat parameter vector."""
    logits, (w, xn, h1, h2) = forward(p, x, mean, scale)
    B = logits.shape[0]
    y = np.asarray(y, np.int64)
    dlog = np.zeros_like(logits)
    loss = 0.0
    for h, (lo, k) in enumerate(HEADS):
        z = logits[:, lo:lo + k]
        z = z - z.max(axis=1, keepdims=True)
        lse = np.log(np.exp(z).sum(axis=1))
        pr = np.exp(z - lse[:, None])
        loss += float((lse - z[np.arange(B), y[:, h]]).sum())
        g = pr.copy()
        g[np.arange(B), y[:, h]] -= 1.0
        dlog[:, lo:lo + k] = g
    loss /= B
    dlog /= B
    d2 = (dlog @ w["W3"].T) * (h2 > 0)
    d1 = (d2 @ w["W2"].T) * (h1 > 0)
    grads = {"W3": h2.T @ dlog, "b3": dlog.sum(0), "W2": h1.T @ d2, "b2": d2.sum(0), "W1": xn.T @ d1,
             "b1": d1.sum(0)}
    flat = np.concatenate([grads[name].reshape(-1) for name, _ in SHAPES])
    return loss, flat


def predict(p: np.ndarray, x: np.ndarray, mean=None, scale=None) -> np.ndarray:
    logits, _ = forward(p, x, mean, scale)
    return np.stack([logits[:, lo:lo + k].argmax(axis=1) for lo, k in HEADS], axis=1).astype(np.int32)


def features(nodes: np.ndarray, edges: np.ndarray, nodesT: np.ndarray, samples: int = 1 << 16) -> np.ndarray:
    """The 16 graph statistics of scc_features.cu, restated on the host
    (1-based CSR in the reference layout)."""
    nodes = np.asarray(nodes, np.int64)
    nodesT = np.asarray(nodesT, np.int64)
    edges = np.asarray(edges, np.int64)
    n = len(nodes) - 2
    m = int(nodes[n + 1])
    f = np.zeros(16, np.float64)
    if n == 0:
        return f
    od = nodes[2:n + 2] - nodes[1:n + 1]
    idg = nodesT[2:n + 2] - nodesT[1:n + 1]
    mean = od.sum() / n
    var = max((od.astype(np.float64) ** 2).sum() / n - mean * mean, 0.0)
    ln = np.log2(n + 1.0)
    f[0] = np.log2(n)
    f[1] = np.log2(m + 1.0)
    f[2] = mean
    f[3] = np.log2(1 + var)
    f[4] = np.log2(1 + od.max())
    f[5] = np.log2(1 + idg.max())
    f[6] = (od == 0).sum() / n
    f[7] = (idg == 0).sum() / n
    f[8] = ((od == 0) | (idg == 0)).sum() / n
    f[9] = (od == 1).sum() / n
    f[10] = (idg == 1).sum() / n
    f[11] = ((od <= 2) & (idg <= 2)).sum() / n
    # sampled reciprocity: edge k*m//S, self-loops skipped
    S = min(m, samples)
    hit = cnt = 0
    for k in range(S):
        e = (k * m) // S
        u = int(np.searchsorted(nodes[1:n + 2], e, side="right"))  # largest v with nodes[v] <= e
        w = int(edges[e])
        if w == u:
            continue
        cnt += 1
        lst = edges[nodes[w]:nodes[w + 1]]
        hit += int(u in set(lst.tolist())) if len(lst) else 0
    f[12] = hit / cnt if cnt else 0.0
    # BFS levels 1..3 from the vertex of largest total degree (ties: smaller id)
    tot = od + idg
    hub = int(np.argmax(tot)) + 1
    seen = np.zeros(n + 2, bool)
    seen[hub] = True
    cur = [hub]
    for lvl in range(3):
        nxt = []
        for v in cur:
            for w in edges[nodes[v]:nodes[v + 1]]:
                if not seen[w]:
                    seen[w] = True
                    nxt.append(int(w))
        f[13 + lvl] = np.log2(1.0 + len(nxt)) / ln
        cur = nxt
    return f
