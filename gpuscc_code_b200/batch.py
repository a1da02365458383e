"""Batched decomposition: many independent graphs in one persistent launch.

The graphs are packed into one CSR with disjoint id ranges (a segment per
graph).  Each segment starts as its own partition, so the first FB round
already elects one pivot per graph and every later phase processes all
graphs at once; SCCs never cross segments, so the packed labels are the
per-graph labels shifted by the segment base.  The solve sequence is
captured once into a CUDA graph and replayed.
"""
from __future__ import annotations

import numpy as np

from .scc import HostCSR, Options, SCCContext


def pack(graphs: list[HostCSR]):
    """Concatenate graphs (reference layout each) into one CSR.
    Returns (HostCSR, seg_first[count+1]) with graph g on ids
    seg_first[g] .. seg_first[g+1]-1."""
    nodes = [np.zeros(2, dtype=np.uint64)]  # placeholder for ids 0 and 1 (nodes[1] = 0)
    nodesT = [np.zeros(2, dtype=np.uint64)]
    edges, edgesT = [], []
    seg = np.zeros(len(graphs) + 1, dtype=np.uint32)
    seg[0] = 1
    vbase, ebase = 0, 0
    sorted_unique = True
    for i, g in enumerate(graphs):
        n, m = g.n, g.m
        nodes.append(g.nodes[2:n + 2].astype(np.uint64) + ebase)
        nodesT.append(g.nodesT[2:n + 2].astype(np.uint64) + ebase)
        edges.append(g.edges.astype(np.uint64) + vbase)
        edgesT.append(g.edgesT.astype(np.uint64) + vbase)
        sorted_unique &= bool(g.raw.sorted_unique)
        vbase += n
        ebase += m
        seg[i + 1] = vbase + 1
    if ebase >= 2 ** 32 or vbase >= 2 ** 30:
        raise ValueError("packed batch exceeds the 32-bit CSR limits")
    cat = lambda parts: np.concatenate(parts).astype(np.uint32) if parts else np.zeros(0, np.uint32)
    packed = HostCSR.from_arrays(cat(nodes), cat(edges), cat(nodesT), cat(edgesT), sorted_unique=sorted_unique)
    return packed, seg


def split(labels: np.ndarray, seg_first: np.ndarray) -> list[np.ndarray]:
    """Packed labels -> per-graph labels in local ids (index 0 = 0)."""
    out = []
    for g in range(len(seg_first) - 1):
        lo, hi = int(seg_first[g]), int(seg_first[g + 1])
        local = np.zeros(hi - lo + 1, dtype=np.uint32)
        local[1:] = labels[lo:hi] - (lo - 1)
        out.append(local)
    return out


class BatchSolver:
    """Solves a list of graphs in one launch (optionally a replayed CUDA graph)."""

    def __init__(self, device: int = 0, options: Options | None = None, capture: bool = True):
        self.ctx = SCCContext(device, options or Options(alg="h", wcc=True, trim2=True))
        self.capture = capture
        self.seg = None

    def close(self):
        self.ctx.close()

    def load(self, graphs: list[HostCSR]):
        packed, seg = pack(graphs)
        self.ctx.upload(packed)
        self.ctx.set_segments(seg)
        self.seg = seg
        self._packed = packed  # keeps the host arrays alive
        if self.capture:
            self.ctx.capture()
        return seg

    def run(self):
        """Solve the loaded batch -> (packed labels, total count, stats)."""
        if self.capture:
            cnt, st = self.ctx.replay()
            labels = self.ctx.read_labels()
        else:
            labels, cnt, st = self.ctx.solve()
        return labels, cnt, st

    def solve(self, graphs: list[HostCSR]):
        """Per-graph (labels, count) for a list of graphs."""
        self.load(graphs)
        labels, _, _ = self.run()
        res = []
        for g, local in enumerate(split(labels, self.seg)):
            idx = np.arange(len(local), dtype=np.uint32)
            res.append((local, int((local[1:] == idx[1:]).sum())))
        return res


def solve_each(graphs: list[HostCSR], ctx: SCCContext):
    """Plain per-graph processing: one upload + one solve launch per graph.
    Returns [(labels, count)] and the summed device solve time in ms."""
    out, ms = [], 0.0
    for g in graphs:
        ctx.upload(g)
        labels, cnt, st = ctx.solve()
        out.append((labels, cnt))
        ms += st["ms_total"]
    return out, ms


def shard_graphs(weights, world: int) -> list[list[int]]:
    """Independent graphs over `world` ranks (one GPU each): longest-processing-
    time greedy on the weights (edge bytes), heaviest first, each to the
    least-loaded rank (ties to the lower rank).  Deterministic, so every rank
    computes the same plan without exchanging it; graph order is kept inside
    a shard.  No graph crosses ranks, so the solves need no collective."""
    if world < 1:
        raise ValueError("world must be >= 1")
    w = np.asarray(weights, dtype=np.float64)
    order = sorted(range(len(w)), key=lambda i: (-w[i], i))
    load = [0.0] * world
    shards: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        shards[r].append(i)
        load[r] += w[i]
    return [sorted(s) for s in shards]


def graph_weight(n: int, m: int) -> int:
    """Bytes the solve of one graph must touch (CSR + transpose + labels)."""
    return 8 * (n + 1) + 8 * m + 4 * n


def solve_shard(graphs, rank: int, world: int, solve_fn):
    """This rank's part of a batch spread over `world` ranks: the graphs of
    shard_graphs' plan for `rank`, solved by solve_fn(list of graphs) ->
    [(labels, count)].  Returns {graph index: (labels, count)}; no graph
    crosses ranks, so the solve itself needs no collective."""
    plan = shard_graphs([graph_weight(g.n, g.m) for g in graphs], world)
    mine = plan[rank]
    res = solve_fn([graphs[i] for i in mine]) if mine else []
    return dict(zip(mine, res))


def gather_results(local: dict, world: int, group=None):
    """All ranks' {graph index: (labels, count)} merged on every rank (one
    object all-gather over the process group, after the solves)."""
    import torch.distributed as dist

    parts = [None] * world
    dist.all_gather_object(parts, local, group=group)
    merged = {}
    for p in parts:
        merged.update(p)
    return [merged[i] for i in sorted(merged)]


class PeerLeft(RuntimeError):
    """A rank announced that it left between steps."""


class PeerLost(RuntimeError):
    """A rank neither reached the step nor announced leaving in time."""


class RankWatch:
    """Host-side failure detection between steps of a multi-rank run.

    Each rank records the step it is about to start in the process group's
    store; before its next launch (and so before any collective of that
    step) a rank waits, for at most `timeout_s`, until every peer has reached
    the same step.  A peer that announced leaving raises PeerLeft at once; a
    peer that went silent raises PeerLost when the wait runs out.  Ranks leave
    only between steps, with none of their kernels or collectives in flight,
    so the others learn of it on the host and never launch work that would
    wait for the missing rank."""

    def __init__(self, store, rank: int, world: int, timeout_s: float = 5.0, poll_s: float = 0.01):
        self.store, self.rank, self.world = store, rank, world
        self.timeout_s, self.poll_s = timeout_s, poll_s

    def leave(self) -> None:
        self.store.set(f"scc_watch/left/{self.rank}", "1")

    def _get(self, key):
        try:
            if self.store.check([key]):
                return self.store.get(key).decode()
        except Exception:
            return None
        return None

    def step(self, i: int) -> None:
        import time

        self.store.set(f"scc_watch/step/{self.rank}", str(i))
        deadline = time.monotonic() + self.timeout_s
        for peer in range(self.world):
            if peer == self.rank:
                continue
            while True:
                if self._get(f"scc_watch/left/{peer}") is not None:
                    raise PeerLeft(f"rank {peer} left before step {i}")
                s = self._get(f"scc_watch/step/{peer}")
                if s is not None and int(s) >= i:
                    break
                if time.monotonic() > deadline:
                    raise PeerLost(f"rank {peer} did not reach step {i} within {self.timeout_s} s")
                time.sleep(self.poll_s)
