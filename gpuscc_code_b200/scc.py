"""Host-side mirror of the reference's SCC interface on top of the C ABI.

Reference interface (chenxuhao/gpuscc_code)      here
  load.h:5       load(file, header, ...)        load(path, header)
  tarjan.h:5     TR_Decomposition(m, n, Fc, Fr) tarjan(graph)            (the apps' -t)
  scc.cu:150     computeSCC(n, m, ..., alg_opt) computeSCC(graph, ...)  / SCCContext.solve
  scc_routines.h trim1 / trim / trim2 / update / unsetPivots           SCCContext.<same>
  reach_*.h      fwd_reach[1]_x / bwd_reach[1]_x                        SCCContext.fwd_reach / bwd_reach
  wcc.h:23       update_wcc                                             SCCContext.update_wcc
Graphs keep the reference layout: ids 1..n, nodes[n+2], 1-based edges.
Errors raise SCCError (the reference calls exit()).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, fields

import numpy as np

from ._capi import (ALG, SCCError, check, lib, scc_dev_csr, scc_host_csr, scc_opts, scc_stats, u32p)

__all__ = [
    "HostCSR", "load", "save", "csr_from_edges", "gen_rmat", "gen_er", "gen_grid", "tarjan", "Options",
    "SCCContext", "computeSCC", "SCCError",
]

RMAT_ABC = (0.57, 0.19, 0.19)


def _u32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.uint32)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(u32p)


class HostCSR:
    """Host graph in the reference layout (load.cpp:125-197)."""

    def __init__(self, raw: scc_host_csr, keep=None):
        self._raw = raw
        self._keep = keep  # numpy arrays backing a non-owned struct

    def __del__(self):
        raw = getattr(self, "_raw", None)
        if raw is not None and raw.owned:
            lib.scc_host_csr_free(C.byref(raw))

    @property
    def raw(self) -> scc_host_csr:
        return self._raw

    n = property(lambda self: int(self._raw.n))
    m = property(lambda self: int(self._raw.m))
    nnz_header = property(lambda self: int(self._raw.nnz_header))
    symmetric = property(lambda self: bool(self._raw.symmetric))

    def _view(self, p, count):
        if count == 0:
            return np.zeros(0, dtype=np.uint32)
        return np.ctypeslib.as_array(p, shape=(count,))

    @property
    def nodes(self) -> np.ndarray:
        return self._view(self._raw.nodes, self.n + 2)

    @property
    def edges(self) -> np.ndarray:
        return self._view(self._raw.edges, self.m)

    @property
    def nodesT(self) -> np.ndarray:
        return self._view(self._raw.nodesT, self.n + 2)

    @property
    def edgesT(self) -> np.ndarray:
        return self._view(self._raw.edgesT, self.m)

    @classmethod
    def from_arrays(cls, nodes, edges, nodesT, edgesT, sorted_unique: bool = False) -> "HostCSR":
        """Wraps caller arrays without copying when they already are contiguous
        uint32 (e.g. pinned buffers); edges/edgesT need at least m entries."""
        nodes, nodesT = _u32(nodes), _u32(nodesT)
        edges, edgesT = _u32(edges), _u32(edgesT)
        if len(edges) == 0:
            edges = np.zeros(1, np.uint32)
        if len(edgesT) == 0:
            edgesT = np.zeros(1, np.uint32)
        n = len(nodes) - 2
        raw = scc_host_csr(n=n, m=int(nodes[n + 1]), nnz_header=int(nodes[n + 1]), symmetric=0,
                           sorted_unique=int(sorted_unique), owned=0, nodes=_ptr(nodes), edges=_ptr(edges),
                           nodesT=_ptr(nodesT), edgesT=_ptr(edgesT))
        return cls(raw, keep=(nodes, edges, nodesT, edgesT))

    def edge_list(self):
        """(src, dst) 1-based arrays of the stored edges."""
        deg = np.diff(self.nodes[1:].astype(np.int64))
        src = np.repeat(np.arange(1, self.n + 1, dtype=np.uint32), deg)
        return src, self.edges.copy()


def load(path: str, header: bool = False) -> HostCSR:
    """load.h:5 — text or MatrixMarket file -> CSR + transpose."""
    raw = scc_host_csr()
    check(lib.scc_load(str(path).encode(), int(header), C.byref(raw)))
    return HostCSR(raw)


def save(g: HostCSR, path: str) -> None:
    """Binary CSR cache: load() reads it back without parsing."""
    check(lib.scc_save(str(path).encode(), C.byref(g.raw)))


def csr_from_edges(n: int, src, dst, drop_self_loops: bool = False) -> HostCSR:
    src, dst = _u32(src), _u32(dst)
    raw = scc_host_csr()
    check(lib.scc_csr_from_edges(n, len(src), _ptr(src), _ptr(dst), int(drop_self_loops), C.byref(raw)))
    return HostCSR(raw)


def _ppm(x: float) -> int:
    return int(round(x * 1_000_000))


def gen_rmat(scale: int, samples: int, abc=RMAT_ABC, seed: int = 1, permute: bool = True) -> HostCSR:
    raw = scc_host_csr()
    a, b, c = abc
    check(lib.scc_gen_rmat(scale, samples, _ppm(a), _ppm(b), _ppm(c), seed, int(permute), C.byref(raw)))
    return HostCSR(raw)


def gen_er(n: int, samples: int, seed: int = 1) -> HostCSR:
    raw = scc_host_csr()
    check(lib.scc_gen_er(n, samples, seed, C.byref(raw)))
    return HostCSR(raw)


def gen_grid(side: int, bidir: float = 0.15, longrange: float = 0.001, seed: int = 3) -> HostCSR:
    raw = scc_host_csr()
    check(lib.scc_gen_grid(side, _ppm(bidir), _ppm(longrange), seed, C.byref(raw)))
    return HostCSR(raw)


BATCH_DEFAULTS = dict(n_lo=1000, n_hi=200_000, deg_lo=2.0, deg_hi=16.0)


def gen_batch(count: int, n_lo: int = 1000, n_hi: int = 200_000, deg_lo: float = 2.0, deg_hi: float = 16.0,
              seed: int = 4):
    """`count` independent ER / R-MAT graphs packed into one CSR.
    Returns (HostCSR, seg_first[count+1])."""
    raw = scc_host_csr()
    seg = np.zeros(count + 1, dtype=np.uint32)
    check(lib.scc_gen_batch(count, n_lo, n_hi, int(round(deg_lo * 1000)), int(round(deg_hi * 1000)), seed,
                            C.byref(raw), _ptr(seg)))
    return HostCSR(raw), seg


def tarjan(g: HostCSR):
    """tarjan.h:5 — the sequential CPU decomposition behind the apps' -t flag.
    Returns (labels[n+1], count, seconds)."""
    labels = np.zeros(g.n + 1, dtype=np.uint32)
    cnt = C.c_uint32()
    secs = C.c_double()
    check(lib.scc_tarjan(C.byref(g.raw), _ptr(labels), C.byref(cnt), C.byref(secs)))
    return labels, int(cnt.value), float(secs.value)


@dataclass
class Options:
    """scc.h:19-27 alg_opt plus the engine's knobs (see scc_opts in scc_capi.h)."""
    alg: str = "t"
    wcc: bool = False
    trim2: bool = False
    trim_first: bool = True
    block_size: int = 256
    warp_size: int = 32
    pivot_rule: int = 0
    switch_permille: int = 10
    trim_depth: int = 0
    pull_alpha: int = 0
    pull_beta: int = 0
    warp_degree: int = 0
    heavy_degree: int = 0
    max_iters: int = 0
    grid_blocks: int = 0
    timeout_ms: int = 0
    trim_first_depth: int = 1
    occupancy: int = 0
    async_depth: int = 0
    test_stall_us: int = 0
    test_queue_cap: int = 0

    def to_c(self) -> scc_opts:
        o = scc_opts()
        lib.scc_opts_default(C.byref(o))
        for f in fields(self):
            v = getattr(self, f.name)
            if f.name == "alg":
                v = ALG[v] if isinstance(v, str) else int(v)
            setattr(o, f.name, int(v))
        return o


class SCCContext:
    """One device context (own CUDA stream, resident graph, per-vertex state)."""

    def __init__(self, device: int = 0, options: Options | None = None, **kw):
        self.options = options or Options(**kw)
        h = C.c_void_p()
        o = self.options.to_c()
        check(lib.scc_ctx_create(device, C.byref(o), C.byref(h)))
        self._h = h
        self.n = 0

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib.scc_ctx_destroy(self._h)
            self._h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    @property
    def stream(self) -> int:
        return int(lib.scc_ctx_stream(self._h) or 0)

    def set_options(self, options: Options | None = None, **kw):
        if options is None:
            options = Options(**{**self.options.__dict__, **kw})
        o = options.to_c()
        check(lib.scc_ctx_set_opts(self._h, C.byref(o)))
        self.options = options

    # --------------------------------------------------------- residency
    def upload(self, g: HostCSR):
        check(lib.scc_ctx_upload(self._h, C.byref(g.raw)))
        self.n = g.n

    def bind_device(self, n: int, m: int, nodes: int, edges: int, nodesT: int, edgesT: int,
                    sorted_unique: bool = False):
        d = scc_dev_csr(n=n, m=m, sorted_unique=int(sorted_unique), nodes=nodes, edges=edges, nodesT=nodesT,
                        edgesT=edgesT)
        check(lib.scc_ctx_bind_device(self._h, C.byref(d)))
        self.n = n

    def gen_rmat_device(self, scale: int, samples: int, abc=RMAT_ABC, seed: int = 2, permute: bool = True):
        d = scc_dev_csr()
        a, b, c = abc
        check(lib.scc_gen_rmat_device(self._h, scale, samples, _ppm(a), _ppm(b), _ppm(c), seed, int(permute),
                                      C.byref(d)))
        self.n = int(d.n)
        return d

    def gen_batch_device(self, count: int, n_lo: int = 1000, n_hi: int = 200_000, deg_lo: float = 2.0,
                         deg_hi: float = 16.0, seed: int = 4):
        """Same batch as gen_batch, built on the device, bound with its segments.
        Returns seg_first[count+1]."""
        d = scc_dev_csr()
        seg = np.zeros(count + 1, dtype=np.uint32)
        check(lib.scc_gen_batch_device(self._h, count, n_lo, n_hi, int(round(deg_lo * 1000)),
                                       int(round(deg_hi * 1000)), seed, C.byref(d), _ptr(seg)))
        self.n = int(d.n)
        self.m = int(d.m)
        return seg

    def capture(self, d_labels: int = 0):
        """Capture the solve sequence into a CUDA graph (scc_solve_capture)."""
        check(lib.scc_solve_capture(self._h, C.c_void_p(d_labels or None)))

    def replay(self):
        """Launch the captured solve -> (count, stats)."""
        cnt = C.c_uint32()
        st = scc_stats()
        check(lib.scc_solve_replay(self._h, C.byref(cnt), C.byref(st)))
        return int(cnt.value), st.as_dict()

    def read_labels(self) -> np.ndarray:
        """Labels of the last solve into the context's own buffer (host copy)."""
        out = np.zeros(self.n + 1, dtype=np.uint32)
        check(lib.scc_read_labels(self._h, _ptr(out)))
        return out

    def download(self) -> HostCSR:
        raw = scc_host_csr()
        check(lib.scc_ctx_download(self._h, C.byref(raw)))
        return HostCSR(raw)

    def set_segments(self, seg_first):
        if seg_first is None or len(seg_first) == 0:
            check(lib.scc_ctx_set_segments(self._h, 0, None))
            return
        s = _u32(seg_first)
        check(lib.scc_ctx_set_segments(self._h, len(s) - 1, _ptr(s)))

    # -------------------------------------------------------------- solve
    def download_into(self, nodes: np.ndarray, edges: np.ndarray, nodesT: np.ndarray, edgesT: np.ndarray):
        """Copy the bound graph into caller-owned uint32 host arrays (n+2 / m)."""
        check(lib.scc_ctx_download_into(self._h, _ptr(nodes), _ptr(edges), _ptr(nodesT), _ptr(edgesT)))

    def solve(self, want_labels: bool = True, out: np.ndarray | None = None):
        """scc.cu:150 computeSCC -> (labels[n+1] or None, count, stats dict).
        `out`: optional caller-owned uint32 array of n+1 entries for the labels."""
        if out is not None:
            labels = out
        else:
            labels = np.zeros(self.n + 1, dtype=np.uint32) if want_labels else None
        want_labels = labels is not None
        cnt = C.c_uint32()
        st = scc_stats()
        check(lib.scc_solve(self._h, _ptr(labels) if want_labels else None, C.byref(cnt), C.byref(st)))
        return labels, int(cnt.value), st.as_dict()

    def solve_device(self, d_labels: int = 0):
        cnt = C.c_uint32()
        st = scc_stats()
        check(lib.scc_solve_device(self._h, C.c_void_p(d_labels or None), C.byref(cnt), C.byref(st)))
        return int(cnt.value), st.as_dict()

    def solve_enqueue(self, d_labels: int = 0):
        check(lib.scc_solve_enqueue(self._h, C.c_void_p(d_labels or None)))

    def solve_collect(self):
        cnt = C.c_uint32()
        st = scc_stats()
        check(lib.scc_solve_collect(self._h, C.byref(cnt), C.byref(st)))
        return int(cnt.value), st.as_dict()

    PROFILE_SLOTS = ["trim_sweep", "trim_worklist", "push", "pull", "heavy", "worklist_level", "quadratic",
                     "update", "wcc", "trim2", "compact", "finalize", "first_pivot", "async", "wcc_sweep"]

    def profile(self) -> dict:
        """Device-side phase timers of the last call: {slot: (ms, count)}."""
        ms = (C.c_double * 16)()
        cnt = (C.c_uint32 * 16)()
        check(lib.scc_get_profile(self._h, ms, cnt))
        return {name: (round(ms[i], 4), int(cnt[i])) for i, name in enumerate(self.PROFILE_SLOTS) if cnt[i]}

    def trace(self) -> list:
        """Per-event device trace of the last call: [(slot name, a, b, ms)]."""
        n = C.c_uint32()
        sl, a, b = (C.c_uint32 * 128)(), (C.c_uint32 * 128)(), (C.c_uint32 * 128)()
        ms = (C.c_double * 128)()
        check(lib.scc_get_trace(self._h, C.byref(n), sl, a, b, ms))
        names = self.PROFILE_SLOTS
        return [(names[sl[i]] if sl[i] < len(names) else str(sl[i]), int(a[i]), int(b[i]), round(ms[i], 4))
                for i in range(n.value)]

    # -------------------------------------------------------- phase level
    def phase_begin(self):
        check(lib.scc_phase_begin(self._h))

    def _u32_out(self, fn, *args) -> int:
        out = C.c_uint32()
        check(fn(self._h, *args, C.byref(out)))
        return int(out.value)

    def trim1(self) -> int:
        """scc_routines.h:47 trim1 -> iterations."""
        return self._u32_out(lib.scc_trim1)

    def trim(self) -> int:
        """scc_routines.h:41 trim (partition-aware) -> iterations."""
        return self._u32_out(lib.scc_trim)

    def trim2(self) -> int:
        """scc_routines.h:50 trim2 -> vertices removed."""
        return self._u32_out(lib.scc_trim2)

    def select_pivots(self) -> int:
        return self._u32_out(lib.scc_select_pivots)

    def fwd_reach(self, variant: str = "q", first_step: bool = False) -> int:
        """reach_x.h fwd_reach[1]_x -> sweeps."""
        return self._u32_out(lib.scc_reach, 0, ALG[variant], int(first_step))

    def bwd_reach(self, variant: str = "q", first_step: bool = False) -> int:
        return self._u32_out(lib.scc_reach, 1, ALG[variant], int(first_step))

    def update(self) -> bool:
        """scc_routines.h:33 update -> hasPivot."""
        hp = C.c_int32()
        check(lib.scc_update(self._h, C.byref(hp)))
        return bool(hp.value)

    def count_elimmed(self) -> int:
        return self._u32_out(lib.scc_count_elimmed)

    def unset_pivots(self):
        check(lib.scc_unset_pivots(self._h))

    def update_wcc(self):
        """wcc.h:23 update_wcc -> (iterations, hasPivot)."""
        d = C.c_uint32()
        hp = C.c_int32()
        check(lib.scc_update_wcc(self._h, C.byref(d), C.byref(hp)))
        return int(d.value), bool(hp.value)

    def states(self) -> np.ndarray:
        out = np.zeros(self.n + 1, dtype=np.uint8)
        check(lib.scc_get_states(self._h, out.ctypes.data_as(C.POINTER(C.c_uint8))))
        return out

    def ranges(self) -> np.ndarray:
        out = np.zeros(self.n + 1, dtype=np.uint32)
        check(lib.scc_get_ranges(self._h, _ptr(out)))
        return out

    def labels(self):
        out = np.zeros(self.n + 1, dtype=np.uint32)
        cnt = C.c_uint32()
        check(lib.scc_get_labels(self._h, _ptr(out), C.byref(cnt)))
        return out, int(cnt.value)


def computeSCC(g: HostCSR, alg: str = "t", wcc: bool = False, trim2: bool = False, block_size: int = 256,
               device: int = 0):
    """scc.cu:150 computeSCC -> (count of SCC, seconds), the reference's return pair."""
    with SCCContext(device, Options(alg=alg, wcc=wcc, trim2=trim2, block_size=block_size)) as ctx:
        ctx.upload(g)
        _, cnt, st = ctx.solve(want_labels=False)
    return cnt, st["ms_total"] / 1000.0
