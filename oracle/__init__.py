"""CPU oracle for the SCC path — TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
legs use this package, as the checker.  The product never imports it.

  _build/liboracle.so  C restatement of the reference algorithms (scc_oracle.c)
  _ref/libscc_ref.so   the reference's own load.cpp / tarjan.cpp / timing.cpp
                       (built by oracle/Makefile where the reference tree exists;
                       None when it is absent)
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "_build" / "liboracle.so"
REF_SO = HERE / "_ref" / "libscc_ref.so"

u32p = C.POINTER(C.c_uint32)
u8p = C.POINTER(C.c_uint8)


def build() -> None:
    """make -C oracle (the C restatement; the reference objects where the reference
    checkout named by SCC_REFERENCE_DIR exists)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True, capture_output=True)


def _lib() -> C.CDLL:
    if not ORACLE_SO.exists():
        build()
    lib = C.CDLL(str(ORACLE_SO))
    lib.oracle_tarjan.restype = C.c_long
    lib.oracle_tarjan.argtypes = [C.c_uint32, u32p, u32p, u32p]
    lib.oracle_canonicalize.restype = C.c_long
    lib.oracle_canonicalize.argtypes = [C.c_uint32, u32p]
    lib.oracle_verify_partition.restype = C.c_int
    lib.oracle_verify_partition.argtypes = [C.c_uint32, u32p, u32p, u32p, u32p, u32p]
    lib.oracle_trim.restype = C.c_long
    lib.oracle_trim.argtypes = [C.c_uint32, u32p, u32p, u32p, u32p, u32p, u8p, u32p]
    lib.oracle_reach.restype = C.c_long
    lib.oracle_reach.argtypes = [C.c_uint32, u32p, u32p, u32p, u8p, C.c_uint32]
    lib.oracle_update.restype = C.c_long
    lib.oracle_update.argtypes = [C.c_uint32, u32p, u8p, u32p, u32p]
    lib.oracle_trim2.restype = C.c_long
    lib.oracle_trim2.argtypes = [C.c_uint32, u32p, u32p, u32p, u32p, u32p, u8p, u32p]
    lib.oracle_wcc.restype = C.c_long
    lib.oracle_wcc.argtypes = [C.c_uint32, u32p, u32p, u32p, u8p, u32p]
    return lib


_L = None


def lib() -> C.CDLL:
    global _L
    if _L is None:
        _L = _lib()
    return _L


def _p(a):
    if a is None:
        return None
    return a.ctypes.data_as(u8p if a.dtype == np.uint8 else u32p)


def _u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


def tarjan_labels(n, nodes, edges):
    """tarjan.cpp restated: canonical (min-id) labels[n+1] and the SCC count."""
    nodes, edges = _u32(nodes), _u32(edges if len(edges) else np.zeros(1, np.uint32))
    labels = np.zeros(n + 1, dtype=np.uint32)
    cnt = lib().oracle_tarjan(n, _p(nodes), _p(edges), _p(labels))
    if cnt < 0:
        raise MemoryError("oracle_tarjan")
    lib().oracle_canonicalize(n, _p(labels))
    return labels, int(cnt)


def canonicalize(labels):
    labels = _u32(labels).copy()
    cnt = lib().oracle_canonicalize(len(labels) - 1, _p(labels))
    return labels, int(cnt)


def verify_partition(n, nodes, edges, nodesT, edgesT, labels) -> int:
    """0 when `labels` is exactly the SCC partition (see scc_oracle.c)."""
    z = np.zeros(1, np.uint32)
    return int(lib().oracle_verify_partition(n, _p(_u32(nodes)), _p(_u32(edges) if len(edges) else z),
                                             _p(_u32(nodesT)), _p(_u32(edgesT) if len(edgesT) else z),
                                             _p(_u32(labels))))


class PhaseState:
    """Reference-encoded per-vertex state (u8 states, u32 ranges, labels, rpivot)."""

    def __init__(self, g):
        self.g = g
        n = g.n
        self.n = n
        self.nodes, self.nodesT = _u32(g.nodes), _u32(g.nodesT)
        z = np.zeros(1, np.uint32)
        self.edges = _u32(g.edges) if g.m else z
        self.edgesT = _u32(g.edgesT) if g.m else z
        self.states = np.zeros(n + 1, dtype=np.uint8)
        self.states[0] = 4
        self.ranges = np.zeros(n + 1, dtype=np.uint32)
        self.labels = np.zeros(n + 1, dtype=np.uint32)
        self.rpivot = np.zeros(n + 1, dtype=np.uint32)

    def trim(self, ranged: bool) -> int:
        return int(lib().oracle_trim(self.n, _p(self.nodes), _p(self.edges), _p(self.nodesT), _p(self.edgesT),
                                     _p(self.ranges) if ranged else None, _p(self.states), _p(self.labels)))

    def first_pivot(self) -> int:
        live = np.nonzero((self.states[1:] & 4) == 0)[0]
        if len(live) == 0:
            return 0
        p = int(live[0]) + 1
        self.states[p] = 19
        self.rpivot[0] = p
        return p

    def reach(self, forward: bool, ranged: bool) -> int:
        off, adj = (self.nodes, self.edges) if forward else (self.nodesT, self.edgesT)
        return int(lib().oracle_reach(self.n, _p(off), _p(adj), _p(self.ranges) if ranged else None,
                                      _p(self.states), 2 if forward else 1))

    def update(self) -> int:
        return int(lib().oracle_update(self.n, _p(self.ranges), _p(self.states), _p(self.labels), _p(self.rpivot)))

    def unset_pivots(self):
        live = (self.states & 4) == 0
        self.states[live] = 0

    def trim2(self) -> int:
        return int(lib().oracle_trim2(self.n, _p(self.nodes), _p(self.edges), _p(self.nodesT), _p(self.edgesT),
                                      _p(self.ranges), _p(self.states), _p(self.labels)))

    def wcc(self) -> int:
        return int(lib().oracle_wcc(self.n, _p(self.nodes), _p(self.edges), _p(self.ranges), _p(self.states),
                                    _p(self.rpivot)))


# ------------------------------------------------------------ reference
_R = None


def ref_lib():
    """The reference's own tarjan.cpp / load.cpp (oracle/_ref), or None."""
    global _R
    if _R is None:
        if not REF_SO.exists():
            return None
        r = C.CDLL(str(REF_SO))
        r.ref_tarjan.restype = C.c_int
        r.ref_tarjan.argtypes = [C.c_uint, C.c_uint, u32p, u32p, u32p, C.POINTER(C.c_float)]
        r.ref_load.restype = C.c_int
        r.ref_load.argtypes = [C.c_char_p, u32p, u32p, C.POINTER(u32p), C.POINTER(u32p), C.POINTER(u32p),
                               C.POINTER(u32p)]
        r.ref_free.restype = None
        r.ref_free.argtypes = [C.c_void_p]
        _R = r
    return _R


def ref_tarjan(n, nodes, edges):
    """Reference TR_Decomposition (tarjan.cpp:72) -> (count, seconds by its own timer)."""
    r = ref_lib()
    if r is None:
        raise FileNotFoundError("oracle/_ref/libscc_ref.so not built")
    nodes = _u32(nodes)
    edges = _u32(np.append(_u32(edges), np.uint32(0)))
    cnt = C.c_uint32()
    secs = C.c_float()
    r.ref_tarjan(int(nodes[n + 1]), n, _p(edges), _p(nodes), C.byref(cnt), C.byref(secs))
    return int(cnt.value), float(secs.value)


def ref_load(path):
    """Reference load() (load.cpp:18) -> dict(n, nnz, nodes, edges, nodesT, edgesT) as numpy copies."""
    r = ref_lib()
    if r is None:
        raise FileNotFoundError("oracle/_ref/libscc_ref.so not built")
    n = C.c_uint32()
    nnz = C.c_uint32()
    ptrs = [u32p() for _ in range(4)]
    rc = r.ref_load(str(path).encode(), C.byref(n), C.byref(nnz), *[C.byref(p) for p in ptrs])
    if rc != 0:
        raise IOError(path)
    nv = n.value
    nodes = np.ctypeslib.as_array(ptrs[0], shape=(nv + 2,)).copy()
    m = int(nodes[nv + 1])
    edges = np.ctypeslib.as_array(ptrs[1], shape=(max(m, 1),))[:m].copy()
    same = C.cast(ptrs[2], C.c_void_p).value == C.cast(ptrs[0], C.c_void_p).value
    nodesT = np.ctypeslib.as_array(ptrs[2], shape=(nv + 2,)).copy()
    edgesT = np.ctypeslib.as_array(ptrs[3], shape=(max(m, 1),))[:m].copy()
    for i, p in enumerate(ptrs):
        if i >= 2 and same:
            break
        r.ref_free(C.cast(p, C.c_void_p))
    nodes[0] = 0
    nodesT[0] = 0
    return dict(n=nv, nnz=int(nnz.value), nodes=nodes, edges=edges, nodesT=nodesT, edgesT=edgesT)
