"""Numpy restatement of the project's R-MAT generator — BENCH/TEST INFRASTRUCTURE.

bench.py's reference leg times the reference's own Tarjan (oracle/_ref) on a
sample of the headline workload.  That process must not load the product
library, so it builds the sample here, with numpy alone, drawing exactly the
graph the product's generator draws (gpuscc_code_b200/csrc/scc_gen.h:
splitmix64 finaliser, Rmat::draw, the 4-round Feistel Perm with cycle
walking; self-loops dropped and duplicates merged as scc_gen_rmat does).
tests/test_rmat_sample.py checks it array for array against the product's
scc_gen_rmat.

Returns the reference CSR layout (load.cpp:144-191): 1-based ids,
nodes[n+2] with nodes[1] = 0 and the out-list of v in
edges[nodes[v] .. nodes[v+1]), lists sorted.
"""
from __future__ import annotations

import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np

_U = np.uint64
_GOLD = _U(0x9E3779B97F4A7C15)
_M1 = _U(0xBF58476D1CE4E5B9)
_M2 = _U(0x94D049BB133111EB)
_LO32 = _U(0xFFFFFFFF)


def mix64(z):
    """splitmix64 finaliser on uint64 arrays (wrapping arithmetic)."""
    z = z + _GOLD
    z = (z ^ (z >> _U(30))) * _M1
    z = (z ^ (z >> _U(27))) * _M2
    return z ^ (z >> _U(31))


def _threshold(ppm: int) -> np.uint64:
    return _U((ppm << 32) // 1_000_000)


def permutation(bits: int, seed: int) -> np.ndarray:
    """Table of the seeded bijection of [0, 2^bits) (Feistel over 2*ceil(bits/2)
    bits, cycle-walked back into range)."""
    if bits == 0:
        return np.zeros(1, np.uint32)
    half = max(1, (bits + 1) // 2)
    mask = _U((1 << half) - 1)
    key = mix64(np.array([seed ^ 0x7065726D75746174], dtype=np.uint64))[0]
    lim = _U(1 << bits)

    def once(x):
        l, r = x >> _U(half), x & mask
        for i in range(4):
            t = l ^ (mix64(key ^ _U(i << 40) ^ r) & mask)
            l, r = r, t
        return (l << _U(half)) | r

    x = np.arange(1 << bits, dtype=np.uint64)
    x = once(x)
    todo = np.nonzero(x >= lim)[0]
    while len(todo):
        y = once(x[todo])
        x[todo] = y
        todo = todo[y >= lim]
    return x.astype(np.uint32)


def _draw(scale, seed, ta, tb, tc, i0, i1):
    i = np.arange(i0, i1, dtype=np.uint64)
    base = mix64(_U(seed) ^ mix64(i ^ _U(0x524D4154)))
    s = np.zeros(len(i), np.uint32)
    d = np.zeros(len(i), np.uint32)
    h = None
    for lvl in range(scale):
        if lvl % 2 == 0:
            h = mix64(base + _U(((lvl >> 1) * 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF))
            r = h & _LO32
        else:
            r = h >> _U(32)
        sb = r >= tb                       # quadrants c, d
        db = ((r >= ta) & (r < tb)) | (r >= tc)  # quadrants b, d
        s = (s << np.uint32(1)) | sb.astype(np.uint32)
        d = (d << np.uint32(1)) | db.astype(np.uint32)
    return s, d


def rmat_csr(scale: int, samples: int, abc=(0.57, 0.19, 0.19), seed: int = 2, permute: bool = True,
             threads: int | None = None):
    """(n, nodes, edges): the graph scc_gen_rmat(scale, samples, abc, seed, permute) builds."""
    a, b, c = (int(round(x * 1_000_000)) for x in abc)
    ta, tb, tc = _threshold(a), _threshold(a + b), _threshold(a + b + c)
    n = 1 << scale
    perm = permutation(scale, seed) if permute else None
    chunk = 1 << 22
    spans = [(i, min(samples, i + chunk)) for i in range(0, samples, chunk)]

    def keys(span):
        s, d = _draw(scale, seed, ta, tb, tc, *span)
        if perm is not None:
            s, d = perm[s], perm[d]
        keep = s != d
        return (s[keep].astype(np.uint64) << _U(32)) | d[keep].astype(np.uint64)

    # numpy releases the GIL inside its loops: chunks are drawn side by side
    with ThreadPoolExecutor(max_workers=threads or min(16, os.cpu_count() or 1)) as ex:
        parts = list(ex.map(keys, spans))
    k = np.concatenate(parts) if parts else np.zeros(0, np.uint64)
    del parts
    k.sort()  # sort + neighbour test: np.unique is far slower on 10^8 keys
    if len(k):
        keep = np.empty(len(k), bool)
        keep[0] = True
        np.not_equal(k[1:], k[:-1], out=keep[1:])
        k = k[keep]
    src = (k >> _U(32)).astype(np.uint32)
    edges = (k & _LO32).astype(np.uint32) + np.uint32(1)
    del k
    nodes = np.zeros(n + 2, np.uint32)
    np.cumsum(np.bincount(src, minlength=n), out=nodes[2:])
    return n, nodes, edges
