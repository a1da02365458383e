"""Autotuner for the engine's launch and load-balance parameters.

Tunes, on the graph (or packed batch) bound to a context, the knobs that
change speed but never results: threads per CTA (block_size), the
register budget (occupancy), the adjacency length split across the grid
(heavy_degree), the push/pull switch points (pull_alpha, pull_beta) and the
topology/data-driven switch point (switch_permille).  Coordinate descent from
the engine defaults: one parameter at a time over its candidate values, the
others fixed, keeping the fastest; the time of a candidate is the minimum
device time (CUDA events) of `repeats` solves after one warm-up.
"""
from __future__ import annotations

import json
from dataclasses import asdict, replace
from pathlib import Path

from .scc import Options, SCCContext, SCCError

SPACE = {
    "block_size": [256, 512, 128],
    "occupancy": [4, 5, 3],
    "heavy_degree": [4096, 1024, 16384],
    "pull_alpha": [14, 6, 32, -1],
    "pull_beta": [24, 8, 64],
    "switch_permille": [10, 50, 2],
}


def _time(ctx: SCCContext, opts: Options, repeats: int) -> float:
    ctx.set_options(opts)
    ctx.solve_device()  # warm-up
    best = float("inf")
    for _ in range(repeats):
        _, st = ctx.solve_device()
        best = min(best, st["ms_total"])
    return best


def autotune(ctx: SCCContext, base: Options | None = None, space: dict | None = None, repeats: int = 2,
             passes: int = 1):
    """Returns (best Options, trials [(changed field, value, ms)])."""
    space = space or SPACE
    best = base or ctx.options
    best_ms = _time(ctx, best, repeats)
    trials = [("base", None, best_ms)]
    for _ in range(passes):
        for field, values in space.items():
            for v in values:
                if getattr(best, field) == v:
                    continue
                cand = replace(best, **{field: v})
                try:
                    ms = _time(ctx, cand, repeats)
                except SCCError:
                    continue  # e.g. a register budget the device cannot co-schedule
                trials.append((field, v, ms))
                if ms < best_ms:
                    best, best_ms = cand, ms
    ctx.set_options(best)
    return best, trials


def save(opts: Options, path: str | Path, key: str) -> None:
    """Store tuned options under `key` (e.g. a workload signature) in a JSON file."""
    p = Path(path)
    data = json.loads(p.read_text()) if p.exists() else {}
    data[key] = asdict(opts)
    p.write_text(json.dumps(data, indent=1, sort_keys=True))


def load(path: str | Path, key: str) -> Options | None:
    p = Path(path)
    if not p.exists():
        return None
    d = json.loads(p.read_text()).get(key)
    return Options(**d) if d else None
