"""Trains the strategy network on traces of the plain method.

Each trace graph is drawn from the served stream's families (R-MAT scale
14-22 with average degree 8-32, grids of side 256-2048 with 10-30 %
bidirectional edges; a different seed than the stream a server is measured
on), solved under every one of the 16 choices, and labelled with the fastest
one.  The network is trained on the device by the library's own kernels and
saved as an .npz (params, mean, scale) that Server / StrategyNet.load read.

    python gpuscc_code_b200/train_strategy.py --runs 20000 --out gpuscc_code_b200/strategy_net.npz
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

import numpy as np

if __package__ in (None, ""):
    sys.path.insert(0, str(Path(__file__).resolve().parents[1]))

from gpuscc_code_b200 import learned  # noqa: E402
from gpuscc_code_b200.scc import Options, SCCContext  # noqa: E402
from gpuscc_code_b200.serve import make_graph, stream_spec  # noqa: E402


def collect(runs: int, seed: int, repeats: int, budget_s: float, device: int = 0, log=print):
    """Trace graphs until `runs` solves (graphs x 16 choices x repeats) or the time budget."""
    base = Options(alg="h", wcc=True, trim2=True)
    ctx = SCCContext(device, base)
    per_graph = len(learned.CHOICES) * repeats
    want = max(1, runs // per_graph)
    X, T, specs = [], [], []
    t0 = time.time()
    with ThreadPoolExecutor(max_workers=2) as pool:
        # grids are built on the host (prefetched while the device times the previous graph);
        # R-MAT graphs are built on the device
        def host_graph(i):
            s = stream_spec(i, seed=seed)
            return s, (make_graph(s) if s["type"] == "grid" else None)
        fut = pool.submit(host_graph, 0)
        for i in range(want):
            spec, g = fut.result()
            if i + 1 < want:
                fut = pool.submit(host_graph, i + 1)
            if g is None:
                ctx.gen_rmat_device(spec["scale"], spec["samples"], seed=spec["seed"])
            else:
                ctx.upload(g)
            X.append(learned.graph_features(ctx))
            T.append(learned.time_choices(ctx, base, repeats))
            specs.append(spec)
            if (i + 1) % 50 == 0:
                log(f"  {i + 1}/{want} graphs, {time.time() - t0:.0f} s")
            if time.time() - t0 > budget_s:
                log(f"  time budget reached after {i + 1} graphs")
                break
    ctx.close()
    return np.array(X, np.float32), np.array(T), specs


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--runs", type=int, default=20000, help="plain-method solves to trace")
    ap.add_argument("--repeats", type=int, default=1)
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--budget-s", type=float, default=1500.0)
    ap.add_argument("--epochs", type=int, default=400)
    ap.add_argument("--holdout", type=float, default=0.2)
    ap.add_argument("--out", default=str(learned.DEFAULT_MODEL))
    ap.add_argument("--traces", default="", help="save the raw traces (.npz) here")
    args = ap.parse_args()

    X, T, specs = collect(args.runs, args.seed, args.repeats, args.budget_s)
    if args.traces:
        np.savez(args.traces, X=X, T=T)
    n = len(X)
    cut = max(1, int(n * (1 - args.holdout)))
    net = learned.train_net(X[:cut], T[:cut], epochs=args.epochs, batch=64, lr=3e-3, seed=0)
    summary = {"graphs": n, "runs": int(n * len(learned.CHOICES) * args.repeats), "train": cut, "holdout": n - cut}
    if n - cut > 0:
        Xh, Th = X[cut:], T[cut:]
        picks = net.predict(Xh)
        plain = float(Th[:, learned.CHOICES.index(learned.PLAIN)].sum())
        mine = float(learned.choice_times(Th, picks).sum())
        best = float(Th.min(axis=1).sum())
        summary.update(holdout_ms_plain=plain, holdout_ms_learned=mine, holdout_ms_best=best,
                       gain=plain / mine if mine > 0 else None)
    # final network on every trace
    net = learned.train_net(X, T, epochs=args.epochs, batch=64, lr=3e-3, seed=0)
    net.save(args.out)
    best_idx = np.argmin(T, axis=1)
    summary["label_histogram"] = {str(learned.CHOICES[k]): int((best_idx == k).sum())
                                  for k in range(len(learned.CHOICES)) if (best_idx == k).any()}
    print(json.dumps(summary))


if __name__ == "__main__":
    main()
