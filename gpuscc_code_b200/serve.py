"""Serving: the request loop of scc_server_* (include/scc_capi.h) and a
Poisson-arrival driver that measures per-request latency and throughput.

The server admits graphs by device memory, keeps registered graphs' CSR
resident (evicting idle ones, least recently used first, when an upload needs
room), and batches the requests that are ready whenever the device frees up
(continuous batching); with a strategy network loaded, each request's options
are picked by the network and only requests with equal options share a
launch.  The labels of a request are the same whichever batch it lands in.
"""
from __future__ import annotations

import ctypes as C
import math
import threading
import time

import numpy as np

from ._capi import (SCC_ERR_BUSY, SCCError, check, lib, scc_host_csr, scc_request_info, scc_server_cfg,
                    scc_server_stats)
from .scc import HostCSR, Options, SCCContext


class Server:
    """One device's request loop."""

    def __init__(self, device: int = 0, options: Options | None = None, batching: bool = True,
                 max_batch_graphs: int = 256, max_batch_vertices: int = 1 << 24, max_batch_edges: int = 1 << 27,
                 solo_vertices: int = 1 << 18, mem_budget: int = 0, model=None):
        cfg = scc_server_cfg()
        lib.scc_server_cfg_default(C.byref(cfg))
        cfg.device = device
        cfg.batching = 1 if batching else 0
        cfg.max_batch_graphs = max_batch_graphs
        cfg.max_batch_vertices = max_batch_vertices
        cfg.max_batch_edges = max_batch_edges
        cfg.solo_vertices = solo_vertices
        cfg.mem_budget = mem_budget
        if options is not None:
            cfg.opts = options.to_c()
        h = C.c_void_p()
        check(lib.scc_server_start(C.byref(cfg), C.byref(h)))
        self._h = h
        self._keep = {}  # request id -> (graph, labels) kept alive until retired
        self._resident = {}  # handle -> registered graph (its host arrays back re-uploads)
        self._lock = threading.Lock()
        if model is not None:
            self.set_model(model)

    def set_model(self, model) -> None:
        """model: a StrategyNet, a path to its .npz, or None to unload."""
        if model is None:
            check(lib.scc_server_set_model(self._h, None, None, None))
            return
        if isinstance(model, (str, bytes)) or hasattr(model, "__fspath__"):
            d = np.load(model)
            params, mean, scale = d["params"], d["mean"], d["scale"]
        else:
            params = model.params
            mean, scale = model.norm
        fp = C.POINTER(C.c_float)
        params, mean, scale = (np.ascontiguousarray(a, np.float32) for a in (params, mean, scale))
        check(lib.scc_server_set_model(self._h, params.ctypes.data_as(fp), mean.ctypes.data_as(fp),
                                       scale.ctypes.data_as(fp)))

    def register(self, g: HostCSR) -> int:
        """Upload g once and keep its CSR resident; returns the handle that
        submit() accepts in place of a graph."""
        h = C.c_uint64()
        check(lib.scc_server_register(self._h, C.byref(g.raw), C.byref(h)))
        with self._lock:
            self._resident[h.value] = g
        return h.value

    def unregister(self, handle: int) -> None:
        check(lib.scc_server_unregister(self._h, handle))
        with self._lock:
            self._resident.pop(handle, None)

    def submit(self, g, out: np.ndarray | None = None) -> int:
        """Queue g (a HostCSR, uploaded for this request, or a handle from
        register()); its labels land in `out` (uint32, n+1; e.g. pinned) or a
        new array."""
        resident = isinstance(g, (int, np.integer))
        if resident:
            with self._lock:
                graph = self._resident[int(g)]
        else:
            graph = g
        labels = np.zeros(graph.n + 1, np.uint32) if out is None else out
        if labels.dtype != np.uint32 or labels.size < graph.n + 1 or not labels.flags.c_contiguous:
            raise ValueError("out must be a contiguous uint32 array of n+1 entries")
        rid = C.c_uint64()
        lp = labels.ctypes.data_as(C.POINTER(C.c_uint32))
        if resident:
            check(lib.scc_server_submit_resident(self._h, int(g), lp, C.byref(rid)))
        else:
            check(lib.scc_server_submit(self._h, C.byref(g.raw), lp, C.byref(rid)))
        with self._lock:
            self._keep[rid.value] = (g, labels)
        return rid.value

    def _retire(self, rid: int, rc: int, info: scc_request_info):
        with self._lock:
            g, labels = self._keep.pop(rid)
        check(rc)
        return labels, {"nscc": info.nscc, "batch_graphs": info.batch_graphs, "choice": tuple(info.choice),
                        "queue_ms": info.queue_ms, "latency_ms": info.latency_ms, "solve_ms": info.solve_ms}

    def poll(self, rid: int):
        """(labels, info) when done, else None."""
        info = scc_request_info()
        rc = lib.scc_server_poll(self._h, rid, C.byref(info))
        if rc == SCC_ERR_BUSY:
            return None
        return self._retire(rid, rc, info)

    def wait(self, rid: int, timeout_ms: int = 0):
        info = scc_request_info()
        rc = lib.scc_server_wait(self._h, rid, timeout_ms, C.byref(info))
        if rc == SCC_ERR_BUSY:
            raise TimeoutError(f"request {rid} not done after {timeout_ms} ms")
        return self._retire(rid, rc, info)

    def stats(self) -> dict:
        st = scc_server_stats()
        check(lib.scc_server_get_stats(self._h, C.byref(st)))
        return st.as_dict()

    def stop(self) -> None:
        if getattr(self, "_h", None):
            lib.scc_server_stop(self._h)
            self._h = None

    __del__ = stop

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.stop()


# ------------------------------------------------------------- the stream
def _mix64(x: int) -> int:
    x = (x + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
    return x ^ (x >> 31)


def _unit(seed: int, i: int, k: int) -> float:
    return (_mix64(seed * 0x100000001B3 ^ _mix64(i * 8 + k)) >> 11) / float(1 << 53)


def stream_spec(i: int, seed: int = 5, rmat_scale=(14, 22), grid_side=(256, 2048), deg=(8.0, 32.0),
                bidir=(0.10, 0.30)) -> dict:
    """Parameters of graph i of the served stream: R-MAT or grid (50/50);
    R-MAT scale uniform in rmat_scale (n = 2^scale, 2^14 >= 1e4 .. 2^22),
    average degree uniform in deg; grid side log-uniform in grid_side,
    bidirectional fraction uniform in bidir, 0.1% long-range edges."""
    if _unit(seed, i, 0) < 0.5:
        lo, hi = rmat_scale
        scale = lo + min(int(_unit(seed, i, 1) * (hi - lo + 1)), hi - lo)
        d = deg[0] + _unit(seed, i, 2) * (deg[1] - deg[0])
        return {"type": "rmat", "scale": scale, "samples": int(round(d * (1 << scale))),
                "seed": _mix64(seed ^ i) & 0x7FFFFFFF}
    lo, hi = math.log(grid_side[0]), math.log(grid_side[1])
    side = int(round(math.exp(lo + _unit(seed, i, 1) * (hi - lo))))
    b = bidir[0] + _unit(seed, i, 2) * (bidir[1] - bidir[0])
    return {"type": "grid", "side": side, "bidir": b, "seed": _mix64(seed ^ i) & 0x7FFFFFFF}


def make_graph(spec: dict, ctx: SCCContext | None = None) -> HostCSR:
    """Host graph of a stream spec (R-MAT built on ctx's device when given)."""
    from .scc import gen_grid, gen_rmat
    if spec["type"] == "rmat":
        if ctx is not None:
            ctx.gen_rmat_device(spec["scale"], spec["samples"], seed=spec["seed"])
            return ctx.download()
        return gen_rmat(spec["scale"], spec["samples"], seed=spec["seed"])
    return gen_grid(spec["side"], spec["bidir"], 0.001, seed=spec["seed"])


def poisson_arrivals(count: int, rate: float, seed: int = 5) -> np.ndarray:
    """Arrival times (s from the start) of a Poisson process of `rate` per second."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, size=count))


def run_stream(server: Server, graphs, arrivals, outs=None) -> dict:
    """Submits graphs[i] at arrivals[i] seconds (labels into outs[i] when
    given) and waits for all of them.  Returns per-request latency, labels
    and the span of the run."""
    ids = [None] * len(graphs)
    results = [None] * len(graphs)
    t0 = time.perf_counter()

    def waiter(i):
        try:
            results[i] = server.wait(ids[i])
        except Exception as e:  # surfaced after the join
            results[i] = e

    threads = []
    for i, (g, at) in enumerate(zip(graphs, arrivals)):
        delay = t0 + at - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        ids[i] = server.submit(g, None if outs is None else outs[i])
        th = threading.Thread(target=waiter, args=(i,))
        th.start()
        threads.append(th)
    for th in threads:
        th.join()
    t1 = time.perf_counter()
    for r in results:
        if isinstance(r, Exception):
            raise r
    lat = np.array([r[1]["latency_ms"] for r in results])
    return {"labels": [r[0] for r in results], "info": [r[1] for r in results], "latency_ms": lat,
            "span_s": t1 - t0, "graphs_per_s": len(graphs) / (t1 - t0),
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99))}


__all__ = ["Server", "stream_spec", "make_graph", "poisson_arrivals", "run_stream", "SCCError"]
