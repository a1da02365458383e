#!/usr/bin/env python
"""SCC throughput on B200: edges/s and HBM-roofline fraction of the scc_2_w path.

Workload (one step = one complete decomposition): R-MAT, 2^26 vertices,
2^30 edge samples, (a,b,c,d) = (0.57, 0.19, 0.19, 0.05), vertex ids permuted,
self-loops dropped, duplicates merged, seed 2, u32 CSR + transpose resident in
HBM; path = scc_2_w -a h (global trim-1, hybrid reach, WCC colouring and
trim-2 once, then partition rounds), labels written to device memory.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

value   = m / device time per step (CUDA events on the engine's stream), summed
          over replicas for N > 1 (a single graph does not shard: N independent
          replicas, no collective; scaling "weak").
e2e     = the same metric through the public API from pinned host buffers:
          each step uploads the CSR (+ device validation), solves and copies
          the labels back.
roofline: bytes the decomposition must touch, 2*4(n+1) + 2*4m + 4n (offsets
          and adjacency of the graph and its transpose once, one u32 label per
          vertex), divided by the step's device time, against the measured HBM
          copy bandwidth in MEASURED_PEAKS.json.
--impl reference: the reference's own CPU decomposition (tarjan.cpp
          TR_Decomposition, compiled from the reference sources into
          oracle/_ref) on a bounded sample of the workload, rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

ABC = (0.57, 0.19, 0.19)
METRIC = "SCC edges/s (R-MAT 2^26 / 2^30 samples, scc_2_w -a h, 1 B200)"
UNIT = "edges/s"


def workload_config(scale: int, samples_log2: int, seed: int, extra: dict | None = None) -> dict:
    cfg = {
        "workload": f"rmat{scale}_e{samples_log2}_scc_2_w_hybrid",
        "graph": f"R-MAT scale {scale}, 2^{samples_log2} samples, (a,b,c,d)=(0.57,0.19,0.19,0.05), "
                 f"ids permuted, self-loops dropped, duplicates merged, seed {seed}",
        "path": "scc_2_w -a h: trim-1, hybrid reach (pull-capable topology sweeps, then quadratic), "
                "WCC + trim-2 once, partition rounds",
        "index_dtype": "u32",
        "l2": "inputs larger than L2 (CSR + transpose ~8.6 GB vs 126 MB L2); no flush",
    }
    if extra:
        cfg.update(extra)
    return cfg


def b_alg(n: int, m: int) -> int:
    return 2 * 4 * (n + 1) + 2 * 4 * m + 4 * n


def load_peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


class ClockSampler:
    """Polls NVML (read-only) every few ms while the timed region runs."""

    def __init__(self, device_index: int, period_s: float = 0.01):
        self.dev = device_index
        self.period = period_s
        self.samples: list[tuple[float, int, int]] = []
        self.max_mhz = None
        self._stop = threading.Event()
        self._t = None
        self.ok = False

    def start(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self.dev)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
            self._nv, self._h = pynvml, h
            self.ok = True
        except Exception:
            return self
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def _run(self):
        nv, h = self._nv, self._h
        while not self._stop.is_set():
            try:
                mhz = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                reasons = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.samples.append((time.perf_counter(), mhz, reasons))
            except Exception:
                pass
            time.sleep(self.period)

    def stop(self):
        self._stop.set()
        if self._t:
            self._t.join()

    def summary(self, t0: float, t1: float) -> dict:
        if not self.ok:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvml unavailable"]}
        win = [s for s in self.samples if t0 <= s[0] <= t1] or self.samples[-3:]
        names = {
            0x0000000000000001: "gpu_idle", 0x0000000000000002: "applications_clocks_setting",
            0x0000000000000004: "sw_power_cap", 0x0000000000000008: "hw_slowdown",
            0x0000000000000010: "sync_boost", 0x0000000000000020: "sw_thermal_slowdown",
            0x0000000000000040: "hw_thermal_slowdown", 0x0000000000000080: "hw_power_brake_slowdown",
            0x0000000000000100: "display_clock_setting",
        }
        seen = set()
        for _, _, r in win:
            for bit, nm in names.items():
                if r & bit:
                    seen.add(nm)
        return {"sm_mhz": statistics.median([s[1] for s in win]) if win else None, "sm_max_mhz": self.max_mhz,
                "reasons": sorted(seen), "samples": len(win)}


def quiet_stdout():
    """Redirect fd 1 (the reference's printf) to /dev/null; returns a restore function."""
    sys.stdout.flush()
    saved = os.dup(1)
    dn = os.open(os.devnull, os.O_WRONLY)
    os.dup2(dn, 1)
    os.close(dn)

    def restore():
        sys.stdout.flush()
        os.dup2(saved, 1)
        os.close(saved)
    return restore


def cpu_tarjan_rate(scale: int, seed: int, device: int):
    """Reference Tarjan (oracle/_ref, else the oracle's port) on a R-MAT sample
    built on the device -> (edges/s, kind, sample description, seconds)."""
    import numpy as np

    import gpuscc_code_b200 as scc
    import oracle

    with scc.SCCContext(device) as ctx:
        ctx.gen_rmat_device(scale, 16 << scale, ABC, seed)
        g = ctx.download()
    kind = "reference" if oracle.ref_lib() is not None else "port"
    restore = quiet_stdout()
    try:
        t0 = time.perf_counter()
        if kind == "reference":
            cnt, own = oracle.ref_tarjan(g.n, g.nodes, g.edges)
        else:
            _, cnt = oracle.tarjan_labels(g.n, g.nodes, g.edges)
        wall = time.perf_counter() - t0
    finally:
        restore()
    secs = wall
    sample = (f"R-MAT scale {scale}, 2^{scale + 4} samples, same (a,b,c,d), permuted, seed {seed}: n={g.n}, "
              f"m={g.m}, {cnt} SCCs; {'tarjan.cpp TR_Decomposition' if kind == 'reference' else 'oracle port'} "
              f"on 1 host thread, wall {secs:.2f} s")
    del np
    return g.m / secs, kind, sample, secs


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle  # noqa: F401
    import gpuscc_code_b200 as scc

    scale = args.ref_scale
    grid = args.workload == "grid"
    if grid:
        g = scc.gen_grid(args.grid_side, 0.15, 0.001, seed=3)
    else:
        with scc.SCCContext(0) as ctx:
            ctx.gen_rmat_device(scale, 16 << scale, ABC, args.seed)
            g = ctx.download()
    kind = "reference" if oracle.ref_lib() is not None else "port"
    times = []
    restore = quiet_stdout()
    try:
        for i in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            if kind == "reference":
                oracle.ref_tarjan(g.n, g.nodes, g.edges)
            else:
                oracle.tarjan_labels(g.n, g.nodes, g.edges)
            if i >= args.warmup:
                times.append(time.perf_counter() - t0)
    finally:
        restore()
    per = sum(times) / len(times)
    value = g.m / per
    sample = (f"R-MAT scale {scale}, 2^{scale + 4} samples (same generator, (a,b,c,d), permutation, seed "
              f"{args.seed}): n={g.n}, m={g.m}; one decomposition per step")
    metric = METRIC
    if grid:
        sample = f"the whole {args.grid_side}^2 grid graph (n={g.n}, m={g.m}); one decomposition per step"
        metric = f"SCC edges/s ({args.grid_side}x{args.grid_side} grid, 15% bidirectional, scc_2_w -a h, 1 B200)"
    line = {
        "impl": "reference", "metric": metric, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": per * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": workload_config(args.scale, args.samples_log2, args.seed,
                                  {"reference_sample_scale": scale}),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args) -> None:
    import numpy as np
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    import gpuscc_code_b200 as scc

    scale, samples = args.scale, 1 << args.samples_log2
    overrides = {}
    for kv in args.opt:
        k, v = kv.split("=", 1)
        overrides[k] = v if k == "alg" else int(v)
    opts = scc.Options(**{"alg": "h", "wcc": True, "trim2": True, **overrides})
    ctx = scc.SCCContext(local, opts)
    grid = args.workload == "grid"
    if grid:
        # 4096 x 4096 grid, every grid edge oriented by a coin flip, 15 % kept in
        # both directions, plus random long-range edges numbering 0.1 % of the
        # grid edges, seed 3 (host generator, then uploaded)
        gh = scc.gen_grid(args.grid_side, 0.15, 0.001, seed=3)
        ctx.upload(gh)
        n, m = int(gh.n), int(gh.m)
    else:
        d = ctx.gen_rmat_device(scale, samples, ABC, args.seed)
        n, m = int(d.n), int(d.m)
    stream = torch.cuda.ExternalStream(ctx.stream)
    d_labels = torch.zeros(n + 1, dtype=torch.int32, device=f"cuda:{local}")

    for _ in range(args.warmup):
        cnt, st = ctx.solve_device(d_labels.data_ptr())
    nscc_check = cnt

    sampler = ClockSampler(local).start()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t_wall0 = time.perf_counter()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    step_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(args.steps)]
    ev0.record(stream)
    for i in range(args.steps):
        step_ev[i][0].record(stream)
        ctx.solve_enqueue(d_labels.data_ptr())
        step_ev[i][1].record(stream)
    ev1.record(stream)
    cnt, st = ctx.solve_collect()
    prof_last = ctx.profile()  # device phase timers of the last timed step
    trace_last = ctx.trace()
    torch.cuda.synchronize()
    t_wall1 = time.perf_counter()
    if dist:
        dist.barrier()
    sampler.stop()
    ms = ev0.elapsed_time(ev1)
    step_ms = [a.elapsed_time(b) for a, b in step_ev]
    if dist:
        t = torch.tensor([ms], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    if cnt != nscc_check:
        raise SystemExit(f"SCC count changed between runs: {nscc_check} vs {cnt}")
    ms_per_step = ms / args.steps
    value = world * m / (ms_per_step / 1e3)
    launches = args.steps * 2  # per step: state init + the persistent solve kernel

    # roofline of the dominant kernel (the persistent solve; its init pass is counted with it)
    peak, peak_kind = load_peaks()
    kern_ms = statistics.mean(step_ms)
    achieved = b_alg(n, m) / (kern_ms / 1e3) / 1e9
    traffic = None
    prof = ROOT / "profiles" / "traffic_rmat_scc_2_w.json"
    if prof.exists() and not grid:
        try:
            t = json.loads(prof.read_text())
            traffic = float(t["bytes_per_edge"]) * m + float(t.get("bytes_per_vertex", 0.0)) * n
        except Exception:
            traffic = None
    clocks = sampler.summary(t_wall0, t_wall1)

    # e2e through the public API from pinned host buffers
    e2e = None
    if not args.no_e2e:
        pin = lambda cnt_: torch.empty(int(cnt_), dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
        h_nodes, h_edges, h_nodesT, h_edgesT = pin(n + 2), pin(max(m, 1)), pin(n + 2), pin(max(m, 1))
        ctx.download_into(h_nodes, h_edges, h_nodesT, h_edgesT)
        hg = scc.HostCSR.from_arrays(h_nodes, h_edges, h_nodesT, h_edgesT, sorted_unique=True)
        h_labels = pin(n + 1)
        ctx.upload(hg)  # warm
        ctx.solve(out=h_labels)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e2e_steps = max(1, min(args.steps, args.e2e_steps))
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            ctx.upload(hg)
            _, c2, _ = ctx.solve(out=h_labels)
        torch.cuda.synchronize()
        e2e_s = (time.perf_counter() - t0) / e2e_steps
        if dist:
            t = torch.tensor([e2e_s], dtype=torch.float64, device=f"cuda:{local}")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_s = float(t.item())
        if c2 != cnt:
            raise SystemExit("e2e SCC count differs from the device-resident run")
        e2e = {"value": world * m / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 2 * 4 * (n + 2) + 2 * 4 * m,
               "d2h_bytes_per_step": 4 * (n + 1), "ms_per_step": e2e_s * 1e3, "steps": e2e_steps}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu and grid:
        import oracle
        kind = "reference" if oracle.ref_lib() is not None else "port"
        restore = quiet_stdout()
        try:
            t0 = time.perf_counter()
            if kind == "reference":
                oracle.ref_tarjan(gh.n, gh.nodes, gh.edges)
            else:
                oracle.tarjan_labels(gh.n, gh.nodes, gh.edges)
            secs = time.perf_counter() - t0
        finally:
            restore()
        cpu = {"value": m / secs, "unit": UNIT, "cores": 1, "kind": kind, "host_cores_available": os.cpu_count(),
               "sample": f"the whole grid graph (n={n}, m={m}); "
                         f"{'tarjan.cpp TR_Decomposition' if kind == 'reference' else 'oracle port'} on 1 host "
                         f"thread, wall {secs:.2f} s"}
    elif rank == 0 and world == 1 and not args.no_cpu:
        rate, kind, sample, _ = cpu_tarjan_rate(args.cpu_scale, args.seed, local)
        cpu = {"value": rate, "unit": UNIT, "cores": 1, "kind": kind, "sample": sample,
               "host_cores_available": os.cpu_count()}

    if dist:
        dist.destroy_process_group()
    if rank != 0:
        ctx.close()
        return
    if grid:
        metric = f"SCC edges/s ({args.grid_side}x{args.grid_side} grid, 15% bidirectional, scc_2_w -a {opts.alg}, 1 B200)"
        data = "synthetic (grid generated on the host, seed 3)"
        config = {"workload": f"grid{args.grid_side}_bidir15_lr0.1_scc_2_w", "n": n, "m": m, "nscc": cnt,
                  "graph": f"{args.grid_side}^2 grid, edges oriented at random, 15% bidirectional, long-range "
                           "edges = 0.1% of grid edges, seed 3",
                  "index_dtype": "u32", "l2": "inputs larger than L2 (CSR + transpose ~0.4 GB); no flush",
                  "parallelism": f"replicas{world}", "engine_overrides": overrides,
                  "rounds": st.get("steps")}
    else:
        metric, data = METRIC, "synthetic (R-MAT generated on the device, seed 2)"
        config = workload_config(scale, args.samples_log2, args.seed,
                                 {"n": n, "m": m, "nscc": cnt, "parallelism": f"replicas{world}",
                                  "engine_overrides": overrides})
    line = {
        "metric": metric, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": data,
        "config": config,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                     "kernel": "scc_persistent<256> (+ per-step init pass)", "kernel_ms": kern_ms,
                     "algorithmic_bytes": b_alg(n, m)},
        "clocks": clocks,
        "gpu_launches": launches,
        "e2e": e2e,
        "cpu_baseline": cpu,
        "stats": {k: (round(v, 4) if isinstance(v, float) else v) for k, v in st.items()},
        "profile_ms": {k: v for k, v in prof_last.items()},
        "trace": trace_last if args.trace else None,
    }
    print(json.dumps(line), flush=True)
    ctx.close()


def run_batch(args) -> None:
    """4096 independent graphs (ER / R-MAT 50/50, n log-uniform in [1e3, 2e5],
    average out-degree U[2, 16], seed 4) packed into one segmented CSR and
    solved by one persistent launch replayed from a captured CUDA graph, with
    parameters from the autotuner; against the same graphs solved one launch
    per graph (upload + solve each, the plain way)."""
    import numpy as np
    import torch

    import gpuscc_code_b200 as scc
    from gpuscc_code_b200 import autotune

    count = args.batch_count
    # under torchrun every rank solves a batch of its own (seed 4 + rank) on
    # its GPU: independent graphs, no collective on the data path (weak scaling)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    ctx = scc.SCCContext(local, scc.Options(alg="h", wcc=True, trim2=True))
    seg = ctx.gen_batch_device(count, 1000, 200_000, 2.0, 16.0, seed=4 + rank)
    n, m = ctx.n, ctx.m
    tuned, trials = ctx.options, []
    if not args.no_tune:
        space = {"block_size": [256, 512], "heavy_degree": [4096, 1024, 16384], "pull_alpha": [14, 6, -1],
                 "switch_permille": [10, 50]}
        tuned, trials = autotune.autotune(ctx, space=space, repeats=2)
    ctx.capture()
    for _ in range(args.warmup):
        ctx.replay()
    stream = torch.cuda.ExternalStream(ctx.stream)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ms_dev = []
    if dist:
        dist.barrier()
    for _ in range(args.steps):
        ev0.record(stream)
        cnt, st = ctx.replay()
        ev1.record(stream)
        ev1.synchronize()
        ms_dev.append(ev0.elapsed_time(ev1))
    batched_ms = statistics.median(ms_dev)
    batch_profile = ctx.profile()  # device phase timers of the last replay
    batch_stats = st
    if dist:
        t = torch.tensor([batched_ms], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        batched_ms = float(t.item())
        dist.destroy_process_group()
        if rank != 0:
            ctx.close()
            return
        line = {
            "metric": "batched SCC graphs/s (4096 mixed ER/R-MAT graphs per GPU, one launch each)",
            "value": world * count / (batched_ms / 1e3), "unit": "graphs/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": batched_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32", "data": "synthetic (one batch per rank, seed 4 + rank)",
            "config": {"workload": f"batch{count}_er_rmat_n1e3-2e5_deg2-16", "graphs_per_gpu": count,
                       "parallelism": f"independent batches x{world}", "l2": "inputs larger than L2"},
            "gpu_launches": 2 * args.steps, "profile_ms": batch_profile,
        }
        print(json.dumps(line), flush=True)
        ctx.close()
        return
    # the same graphs, one launch each (local ids, uploaded and solved one by one)
    full = ctx.download()
    nodes, edges, nodesT, edgesT = (np.asarray(a) for a in (full.nodes, full.edges, full.nodesT, full.edgesT))
    per = scc.SCCContext(0, scc.Options(alg="h", wcc=True, trim2=True))
    locals_ = []
    for g in range(count):
        lo, hi = int(seg[g]), int(seg[g + 1])  # global ids lo .. hi-1
        e0, e1 = int(nodes[lo]), int(nodes[hi])
        t0_, t1_ = int(nodesT[lo]), int(nodesT[hi])
        k = hi - lo
        ln = np.zeros(k + 2, np.uint32)
        ln[1:] = nodes[lo:hi + 1] - e0
        lt = np.zeros(k + 2, np.uint32)
        lt[1:] = nodesT[lo:hi + 1] - t0_
        locals_.append(scc.HostCSR.from_arrays(ln, edges[e0:e1] - (lo - 1), lt, edgesT[t0_:t1_] - (lo - 1),
                                               sorted_unique=True))
    per.upload(locals_[0])
    per.solve()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    dev_sum = 0.0
    total_cnt = 0
    for hg in locals_:
        per.upload(hg)
        _, c, s2 = per.solve(want_labels=False)
        dev_sum += s2["ms_total"]
        total_cnt += c
    wall = time.perf_counter() - t0
    if total_cnt != cnt:
        raise SystemExit(f"per-graph SCC total {total_cnt} differs from the batched count {cnt}")
    line = {
        "metric": "batched SCC graphs/s (4096 mixed ER/R-MAT graphs, one launch)", "value": count / (batched_ms / 1e3),
        "unit": "graphs/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": batched_ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic (batch generated on the device, seed 4)",
        "config": {"workload": f"batch{count}_er_rmat_n1e3-2e5_deg2-16", "n": n, "m": m, "nscc": cnt,
                   "graphs": count, "launch": "captured CUDA graph: reset + init + one cooperative persistent kernel",
                   "l2": "inputs larger than L2"},
        "tuned": {k: getattr(tuned, k) for k in ("block_size", "occupancy", "heavy_degree", "pull_alpha",
                                                 "pull_beta", "switch_permille")},
        "tuning_trials": [[f, v, round(ms, 3)] for f, v, ms in trials],
        "per_graph_baseline": {"graphs_per_s_wall": count / wall, "graphs_per_s_device": count / (dev_sum / 1e3),
                               "ms_device_sum": dev_sum, "s_wall": wall,
                               "how": "one upload + one scc_solve per graph, same options, local ids"},
        "speedup_vs_per_graph": {"wall": (count / (batched_ms / 1e3)) / (count / wall),
                                 "device": dev_sum / batched_ms},
        "gpu_launches": 2 * args.steps,
        "profile_ms": batch_profile,
        "stats": {k: (round(v, 4) if isinstance(v, float) else v) for k, v in batch_stats.items()},
    }
    print(json.dumps(line), flush=True)
    per.close()
    ctx.close()


def run_serve(args) -> None:
    """Served stream: Poisson arrivals of R-MAT (scale 14-22, average degree
    8-32) and grid graphs (side 256-2048, 10-30 % bidirectional), seed 5.
    A pool of distinct graphs is generated first and the stream cycles
    through it.  Three arms serve the same arrival sequence: the plain
    hybrid one graph per launch, continuous batching, and continuous batching
    with the trained strategy network.  Every request's labels are compared
    with the same graph solved alone by the plain method."""
    import numpy as np
    import torch

    import gpuscc_code_b200 as scc
    from gpuscc_code_b200 import learned
    from gpuscc_code_b200.serve import Server, make_graph, poisson_arrivals, run_stream, stream_spec

    torch.cuda.set_device(0)
    base = scc.Options(alg="h", wcc=True, trim2=True)
    ctx = scc.SCCContext(0, base)

    def pinned(count):
        return torch.empty(int(count), dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)

    # clients hand over page-locked buffers (graph arrays and label outputs)
    pool = []
    for i in range(args.serve_pool):
        g = make_graph(stream_spec(i, seed=5), ctx)
        a = [pinned(g.n + 2), pinned(max(g.m, 1)), pinned(g.n + 2), pinned(max(g.m, 1))]
        a[0][:] = g.nodes
        a[1][:g.m] = g.edges
        a[2][:] = g.nodesT
        a[3][:g.m] = g.edgesT
        pool.append(scc.HostCSR.from_arrays(a[0], a[1][:g.m], a[2], a[3][:g.m], sorted_unique=True))
        del g
    # alone: plain method, one graph at a time, upload + solve + labels back (the
    # labels every arm must reproduce, and the service time that sets the rate)
    alone, svc_ms = [], []
    for g in pool:
        out = pinned(g.n + 1)
        t0 = time.perf_counter()
        ctx.upload(g)
        ctx.solve(out=out)
        svc_ms.append((time.perf_counter() - t0) * 1e3)
        alone.append(out.copy())
    ctx.close()
    reqs = [pool[i % len(pool)] for i in range(args.serve_requests)]
    ref = [alone[i % len(pool)] for i in range(args.serve_requests)]
    outs = [pinned(g.n + 1) for g in reqs]
    rate = args.serve_rate
    if rate <= 0:  # load the plain server close to its end-to-end capacity
        rate = 0.9 * 1e3 / float(np.mean(svc_ms))
    arrivals = poisson_arrivals(len(reqs), rate, seed=5)
    model = learned.DEFAULT_MODEL if learned.DEFAULT_MODEL.exists() else None
    arms = [("plain", dict(batching=False), None), ("batched", dict(batching=True), None)]
    if model is not None:
        arms.append(("batched_learned", dict(batching=True), model))
    out = {}
    for name, kw, mdl in arms:
        with Server(0, base, model=mdl, **kw) as srv:
            # capacity: every request at once (the server is never idle), after
            # one unmeasured burst that grows the server's memory pool
            run_stream(srv, reqs, np.zeros(len(reqs)), outs)
            burst = run_stream(srv, reqs, np.zeros(len(reqs)), outs)
            exact_burst = all(np.array_equal(a[:len(b)], b) for a, b in zip(burst["labels"], ref))
            st0 = srv.stats()
            res = run_stream(srv, reqs, arrivals, outs)
            st = srv.stats()
            st["batches"] -= st0["batches"]
        exact = all(np.array_equal(a[:len(b)], b) for a, b in zip(res["labels"], ref)) and exact_burst
        if not exact:
            raise SystemExit(f"serve arm {name}: labels differ from the graph solved alone")
        picks = {}
        for info in res["info"]:
            picks[str(info["choice"])] = picks.get(str(info["choice"]), 0) + 1
        out[name] = {"graphs_per_s": res["graphs_per_s"], "p50_ms": res["p50_ms"], "p99_ms": res["p99_ms"],
                     "capacity_graphs_per_s": burst["graphs_per_s"],
                     "mean_batch": float(np.mean([i["batch_graphs"] for i in res["info"]])),
                     "batches": st["batches"], "labels_exact": exact,
                     "peak_resident_bytes": st["peak_resident_bytes"], "choices": picks}
        del res
    best = max(out.values(), key=lambda a: a["capacity_graphs_per_s"])
    n_tot = sum(int(g.n) for g in reqs)
    m_tot = sum(int(g.m) for g in reqs)
    line = {
        "metric": "served SCC graphs/s (Poisson stream of R-MAT + grid graphs, p50/p99 latency)",
        "value": best["capacity_graphs_per_s"], "unit": "graphs/s", "n_gpus": 1, "steps": 1, "warmup": 1,
        "ms_per_step": 1e3 * len(reqs) / best["capacity_graphs_per_s"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic (stream generated in-process, seed 5)",
        "config": {"workload": f"serve{len(reqs)}_pool{len(pool)}_rmat14-22_grid256-2048",
                   "requests": len(reqs), "distinct_graphs": len(pool), "rate_per_s": rate,
                   "vertices": n_tot, "edges": m_tot, "model": str(model.name) if model else None},
        "arms": out,
        "capacity_vs_plain": {k: v["capacity_graphs_per_s"] / out["plain"]["capacity_graphs_per_s"]
                              for k, v in out.items()},
        "p99_vs_plain": {k: out["plain"]["p99_ms"] / v["p99_ms"] for k, v in out.items()},
        "plain_mean_service_ms": float(np.mean(svc_ms)),
        "note": "graphs and label buffers in page-locked host memory; service time = upload + solve + labels "
                "back, one graph alone; rate = 0.9 / mean service time unless given; p50/p99 at that rate; "
                "capacity = the same requests submitted at once, after one unmeasured such burst that grows the "
                "server's memory pool; value = the best arm's capacity",
    }
    print(json.dumps(line), flush=True)


def run_refgpu(args) -> None:
    """The reference's own GPU FB (scc_2_w build, compiled from its sources for
    sm_100a into oracle/_ref) against this engine on the same graphs and the
    same device: R-MAT scale 16 / 2^20 samples (seed 1, config 1), R-MAT at
    larger scales (seed 2) and a grid.  The reference runs in a child process
    (it prints and exit()s on errors) under a time limit; both sides report the
    solve time from a resident CSR (the reference's own timer, scc.cu:217-1011;
    CUDA events here) and the SCC count, which must agree."""
    import subprocess

    import torch

    import gpuscc_code_b200 as scc
    from oracle import ref_gpu

    if not ref_gpu.available():
        print(json.dumps({"metric": "reference GPU FB comparison", "unavailable": "oracle/_ref/libscc_ref_gpu.so "
                          "not built (the reference sources were absent at build time)"}))
        return
    torch.cuda.set_device(0)
    cases = [("rmat16_e20_seed1", ["--rmat", "16", "--samples-log2", "20", "--seed", "1"],
              lambda c: c.gen_rmat_device(16, 1 << 20, seed=1))]
    for sc in args.refgpu_scales:
        cases.append((f"rmat{sc}_e{sc + 4}_seed2", ["--rmat", str(sc), "--samples-log2", str(sc + 4), "--seed", "2"],
                      lambda c, sc=sc: c.gen_rmat_device(sc, 1 << (sc + 4), seed=2)))
    cases.append((f"grid{args.refgpu_grid}_seed3", ["--grid", str(args.refgpu_grid), "--seed", "3"], None))
    rows = []
    for name, cli, gen in cases:
        row = {"graph": name}
        for alg in args.refgpu_algs:
            try:
                r = subprocess.run([sys.executable, "-m", "oracle.ref_gpu", *cli, "--alg", alg], cwd=ROOT,
                                   capture_output=True, text=True, timeout=args.refgpu_timeout)
                ref = json.loads(r.stdout.strip().splitlines()[-1]) if r.returncode == 0 else {
                    "error": f"exit {r.returncode}: {(r.stderr or r.stdout).strip()[-200:]}"}
            except subprocess.TimeoutExpired:
                ref = {"error": f"no result within {args.refgpu_timeout} s"}
            row[f"reference_{alg}"] = ref
        ctx = scc.SCCContext(0, scc.Options(alg="h", wcc=True, trim2=True))
        if gen is None:
            ctx.upload(scc.gen_grid(args.refgpu_grid, 0.15, 0.001, seed=3))
        else:
            gen(ctx)
        for _ in range(3):
            cnt, st = ctx.solve_device()
        ms = []
        for _ in range(5):
            cnt, st = ctx.solve_device()
            ms.append(st["ms_total"])
        ctx.close()
        row["ours_h"] = {"n": ctx.n, "nscc": cnt, "secs": statistics.median(ms) / 1e3}
        for alg in args.refgpu_algs:
            ref = row[f"reference_{alg}"]
            if "secs" in ref:
                ref["count_matches"] = ref["nscc"] == cnt
                ref["speedup_of_ours"] = ref["secs"] / row["ours_h"]["secs"]
        rows.append(row)
    # the mixed batch: the reference solves graphs one at a time (a sample of
    # them), the engine all 4096 in one captured launch
    batch = {"graphs": 4096, "reference_sample": args.refgpu_batch}
    try:
        r = subprocess.run([sys.executable, "-m", "oracle.ref_gpu", "--batch", str(args.refgpu_batch), "--alg", "h"],
                           cwd=ROOT, capture_output=True, text=True, timeout=args.refgpu_timeout)
        batch["reference_h"] = json.loads(r.stdout.strip().splitlines()[-1]) if r.returncode == 0 else {
            "error": f"exit {r.returncode}: {(r.stderr or r.stdout).strip()[-200:]}"}
    except subprocess.TimeoutExpired:
        batch["reference_h"] = {"error": f"no result within {args.refgpu_timeout} s"}
    ctx = scc.SCCContext(0, scc.Options(alg="h", wcc=True, trim2=True))
    ctx.gen_batch_device(4096, 1000, 200_000, 2.0, 16.0, seed=4)
    ctx.capture()
    for _ in range(3):
        ctx.replay()
    ms = []
    for _ in range(5):
        _, st = ctx.replay()
        ms.append(st["ms_total"])
    ctx.close()
    batch["ours_batched_graphs_per_s"] = 4096 / (statistics.median(ms) / 1e3)
    ref = batch["reference_h"]
    if "graphs_per_s_timer" in ref:
        batch["speedup_vs_reference_timer"] = batch["ours_batched_graphs_per_s"] / ref["graphs_per_s_timer"]
        batch["speedup_vs_reference_wall"] = batch["ours_batched_graphs_per_s"] / ref["graphs_per_s_wall"]
    print(json.dumps({"metric": "SCC solve time vs the reference's GPU FB (same B200, same graphs)",
                      "unit": "s", "rows": rows, "batch": batch,
                      "note": "reference: scc.cu computeSCC of the scc_2_w build (-DWCC -DTRIM_2), its own timer; "
                              "ours: scc_2_w -a h, CUDA events, median of 5"}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--scale", type=int, default=26)
    ap.add_argument("--samples-log2", type=int, default=30)
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--cpu-scale", type=int, default=24, help="R-MAT scale of the cpu_baseline sample")
    ap.add_argument("--ref-scale", type=int, default=23, help="R-MAT scale of each --impl reference step")
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--trace", action="store_true", help="include the per-sweep device trace in the line")
    ap.add_argument("--opt", action="append", default=[], metavar="KEY=VALUE",
                    help="override an engine option (scc_opts field), e.g. --opt occupancy=3")
    ap.add_argument("--grid-side", type=int, default=4096, help="grid: side of the grid graph")
    ap.add_argument("--refgpu-scales", type=int, nargs="*", default=[20, 22],
                    help="refgpu: further R-MAT scales (2^(scale+4) samples, seed 2)")
    ap.add_argument("--refgpu-grid", type=int, default=1024, help="refgpu: grid side")
    ap.add_argument("--refgpu-algs", nargs="*", default=["h", "t"], help="refgpu: reference -a arms")
    ap.add_argument("--refgpu-timeout", type=int, default=300)
    ap.add_argument("--refgpu-batch", type=int, default=256, help="refgpu: batch graphs the reference solves")
    ap.add_argument("--workload", choices=["rmat26", "grid", "batch", "serve", "refgpu"], default="rmat26",
                    help="rmat26: the headline line; batch: 4096 packed graphs in one launch vs one launch each; "
                         "serve: Poisson stream through the request loop (plain / batched / batched + network); "
                         "grid: the 4096^2 high-diameter grid graph")
    ap.add_argument("--serve-pool", type=int, default=48, help="serve: distinct graphs in the stream")
    ap.add_argument("--serve-requests", type=int, default=240, help="serve: requests in the stream")
    ap.add_argument("--serve-rate", type=float, default=0.0,
                    help="serve: arrivals per second (0 = 0.9 x the plain method's device throughput)")
    ap.add_argument("--batch-count", type=int, default=4096)
    ap.add_argument("--no-tune", action="store_true", help="batch: skip the autotuner")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.workload == "refgpu":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the refgpu workload is itself a comparison"}))
            return
        run_refgpu(args)
        return
    if args.workload in ("batch", "serve"):
        if args.impl == "reference":
            if int(os.environ.get("RANK", "0")) == 0:
                print(json.dumps({"impl": "reference",
                                  "unavailable": f"the {args.workload} workload has no reference path"}))
            return
        run_batch(args) if args.workload == "batch" else run_serve(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
