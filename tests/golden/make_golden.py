"""Regenerates the golden fixtures in this directory from the reference itself.

Run in a container that has the reference tree (oracle/_ref built by
`make -C oracle`):  python tests/golden/make_golden.py

* demo.graph is copied verbatim from the reference (its only shipped input).
* A few small graphs are written in the reference's input formats (plain
  "n nnz" + "dst src" lines, and MatrixMarket general / symmetric / pattern)
  from a seeded numpy generator.
* For every file, golden.json records what the reference's own load()
  (load.cpp:18) produced (n, header nnz, CSR and transpose arrays) and the SCC
  count its own TR_Decomposition (tarjan.cpp:72) reports, plus canonical
  labels from the C restatement (oracle/scc_oracle.c), which must agree with
  that count and pass the independent partition check.
"""
from __future__ import annotations

import json
import os
import shutil
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))
import oracle  # noqa: E402

REF = Path(os.environ.get("SCC_REFERENCE_DIR", "/root/reference"))  # the reference checkout (read only)


def write_plain(path: Path, n: int, pairs):
    with open(path, "w") as f:
        f.write(f"{n}\t{len(pairs)}\n")
        for d, s in pairs:
            f.write(f"{d}\t{s}\n")


def write_mtx(path: Path, n: int, pairs, kind: str, weighted: bool):
    with open(path, "w") as f:
        f.write(f"%%MatrixMarket matrix coordinate {'real' if weighted else 'pattern'} {kind}\n")
        f.write("% generated fixture\n")
        f.write(f"{n} {n} {len(pairs)}\n")
        for i, (d, s) in enumerate(pairs):
            f.write(f"{d} {s} {0.5 + i % 3}\n" if weighted else f"{d} {s}\n")


def random_pairs(rng, n, m, self_loops=True, dup=True):
    d = rng.integers(1, n + 1, size=m)
    s = rng.integers(1, n + 1, size=m)
    pairs = list(zip(d.tolist(), s.tolist()))
    if not self_loops:
        pairs = [(a, b) for a, b in pairs if a != b]
    if dup and pairs:
        pairs += pairs[: max(1, len(pairs) // 10)]
    return pairs


def cycles_and_tails(n):
    # several cycles of different lengths chained by one-way edges, plus 2-cycles and tails
    pairs, v = [], 1
    for length in (5, 3, 2, 2, 1, 4):
        ids = list(range(v, v + length))
        for i, a in enumerate(ids):
            b = ids[(i + 1) % length]
            if length > 1:
                pairs.append((b, a))  # "dst src" -> edge a->b
        if v > 1:
            pairs.append((v, v - 1))
        v += length
    while v <= n:
        pairs.append((v, v - 1))
        v += 1
    pairs.append((1, 1))
    return pairs


def main():
    if oracle.ref_lib() is None:
        oracle.build()
    if oracle.ref_lib() is None:
        raise SystemExit("reference objects unavailable (need the reference tree)")
    shutil.copyfile(REF / "demo.graph", HERE / "demo.graph")
    rng = np.random.default_rng(20261203)
    write_plain(HERE / "rand_sparse.graph", 60, random_pairs(rng, 60, 90))
    write_plain(HERE / "rand_dense.graph", 40, random_pairs(rng, 40, 400))
    write_plain(HERE / "cycles.graph", 30, cycles_and_tails(30))
    write_plain(HERE / "isolated.graph", 7, [(2, 1), (1, 2)])
    write_mtx(HERE / "general.mtx", 50, random_pairs(rng, 50, 120), "general", weighted=True)
    write_mtx(HERE / "pattern_sym.mtx", 35, random_pairs(rng, 35, 30, self_loops=True), "symmetric", weighted=False)
    files = ["demo.graph", "rand_sparse.graph", "rand_dense.graph", "cycles.graph", "isolated.graph", "general.mtx",
             "pattern_sym.mtx"]
    out = {}
    for name in files:
        r = oracle.ref_load(HERE / name)
        n = r["n"]
        cnt, _ = oracle.ref_tarjan(n, r["nodes"], r["edges"])
        labels, cnt2 = oracle.tarjan_labels(n, r["nodes"], r["edges"])
        assert cnt == cnt2, (name, cnt, cnt2)
        assert oracle.verify_partition(n, r["nodes"], r["edges"], r["nodesT"], r["edgesT"], labels) == 0, name
        out[name] = dict(n=n, nnz=r["nnz"], nodes=r["nodes"].tolist(), edges=r["edges"].tolist(),
                         nodesT=r["nodesT"].tolist(), edgesT=r["edgesT"].tolist(), nscc_reference=cnt,
                         labels=labels.tolist())
    with open(HERE / "golden.json", "w") as f:
        json.dump(out, f, indent=0)
    print("wrote", len(out), "fixtures")


if __name__ == "__main__":
    main()
