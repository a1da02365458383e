"""The reference's own GPU FB decomposition, timed — TEST / BENCH INFRASTRUCTURE ONLY.

Loads oracle/_ref/libscc_ref_gpu.so (the reference's scc.cu and kernels,
built by oracle/Makefile with -DWCC -DTRIM_2 for sm_100a) and runs its
computeSCC on one graph.  The reference prints progress to stdout and calls
exit() on CUDA errors, so callers run this module in a child process:

    python -m oracle.ref_gpu --rmat 16 --samples-log2 20 --seed 1 --alg h

prints one JSON line: SCC count, the reference's own timer (seconds; device
work from resident CSR to the count, scc.cu:217-1011) and the call's wall time.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import sys
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB = HERE / "_ref" / "libscc_ref_gpu.so"
ALGS = {"q": 0, "t": 1, "d": 2, "l": 3, "h": 4, "c": 5, "b": 6}  # reach_strategy, scc.h:7-16


def available() -> bool:
    return LIB.exists()


def run(g, alg: str = "h", block_size: int = 256):
    lib = C.CDLL(str(LIB))
    u32p = C.POINTER(C.c_uint32)
    lib.ref_gpu_scc.argtypes = [C.c_uint, C.c_uint, u32p, u32p, u32p, u32p, C.c_int, C.c_int, u32p,
                                C.POINTER(C.c_float)]
    import numpy as np
    # the reference copies m + 1 adjacency entries (scc.cu:205-208)
    arrs = [np.ascontiguousarray(g.nodes, np.uint32), np.append(np.asarray(g.edges, np.uint32), np.uint32(0)),
            np.ascontiguousarray(g.nodesT, np.uint32), np.append(np.asarray(g.edgesT, np.uint32), np.uint32(0))]
    p = [a.ctypes.data_as(u32p) for a in arrs]
    cnt = C.c_uint32()
    secs = C.c_float()
    sys.stdout.flush()
    saved = os.dup(1)
    dn = os.open(os.devnull, os.O_WRONLY)
    os.dup2(dn, 1)  # the reference's per-step printf
    try:
        t0 = time.perf_counter()
        lib.ref_gpu_scc(g.n, g.m, p[0], p[1], p[2], p[3], ALGS[alg], block_size, C.byref(cnt), C.byref(secs))
        wall = time.perf_counter() - t0
    finally:
        os.dup2(saved, 1)
        os.close(saved)
        os.close(dn)
    return int(cnt.value), float(secs.value), wall


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--rmat", type=int, help="R-MAT scale (0.57, 0.19, 0.19, 0.05), ids permuted")
    ap.add_argument("--samples-log2", type=int, default=20)
    ap.add_argument("--grid", type=int, help="grid side (15%% bidirectional, 0.1%% long-range)")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--alg", default="h", choices=list(ALGS))
    ap.add_argument("--repeats", type=int, default=2)
    ap.add_argument("--batch", type=int, default=0,
                    help="solve the first N graphs of the 4096-graph batch (ER / R-MAT, n in [1e3, 2e5], "
                         "degree 2-16, seed 4) one by one")
    args = ap.parse_args()
    sys.path.insert(0, str(HERE.parent))
    import gpuscc_code_b200 as scc
    if args.batch:
        import numpy as np
        with scc.SCCContext(0) as ctx:
            seg = ctx.gen_batch_device(4096, 1000, 200_000, 2.0, 16.0, seed=4)
            full = ctx.download()
        nodes, edges, nodesT, edgesT = (np.asarray(a) for a in (full.nodes, full.edges, full.nodesT, full.edgesT))
        tot_secs = tot_wall = 0.0
        tot_cnt = 0
        for gi in range(args.batch):
            lo, hi = int(seg[gi]), int(seg[gi + 1])
            e0, e1, t0, t1 = int(nodes[lo]), int(nodes[hi]), int(nodesT[lo]), int(nodesT[hi])
            k = hi - lo
            ln = np.zeros(k + 2, np.uint32)
            ln[1:] = nodes[lo:hi + 1] - e0
            lt = np.zeros(k + 2, np.uint32)
            lt[1:] = nodesT[lo:hi + 1] - t0
            g = scc.HostCSR.from_arrays(ln, edges[e0:e1] - (lo - 1), lt, edgesT[t0:t1] - (lo - 1), sorted_unique=True)
            cnt, secs, wall = run(g, args.alg)
            tot_secs += secs
            tot_wall += wall
            tot_cnt += cnt
        print(json.dumps({"graphs": args.batch, "nscc_total": tot_cnt, "alg": args.alg, "secs": tot_secs,
                          "wall_s": tot_wall, "graphs_per_s_timer": args.batch / tot_secs,
                          "graphs_per_s_wall": args.batch / tot_wall}), flush=True)
        return
    if args.grid:
        g = scc.gen_grid(args.grid, 0.15, 0.001, seed=args.seed)
    else:
        with scc.SCCContext(0) as ctx:
            ctx.gen_rmat_device(args.rmat, 1 << args.samples_log2, seed=args.seed)
            g = ctx.download()
    runs = [run(g, args.alg) for _ in range(args.repeats)]
    cnt = runs[-1][0]
    print(json.dumps({"n": g.n, "m": g.m, "nscc": cnt, "alg": args.alg,
                      "secs": min(r[1] for r in runs), "wall_s": min(r[2] for r in runs)}), flush=True)


if __name__ == "__main__":
    main()
