#!/usr/bin/env python
"""SCC throughput on B200: edges/s and HBM-roofline fraction of the scc_2_w path.

Headline workload (one step = one complete decomposition): R-MAT, 2^26
vertices, 2^30 edge samples, (a,b,c,d) = (0.57, 0.19, 0.19, 0.05), vertex ids
permuted, self-loops dropped, duplicates merged, seed 2, u32 CSR + transpose
resident in HBM; path = scc_2_w -a h (global trim-1, hybrid reach, WCC
colouring and trim-2 once, then partition rounds), labels written to device
memory.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

value    = m / device time per step (CUDA events on the engine's stream), summed
           over replicas for N > 1 (a single graph does not shard: N independent
           replicas, no collective; scaling "weak").
e2e      = the same metric through the public API from pinned host buffers:
           each step uploads the CSR (+ device validation), solves and copies
           the labels back.
roofline : bytes the decomposition must touch, 2*4(n+1) + 2*4m + 4n (offsets
           and adjacency of the graph and its transpose once, one u32 label per
           vertex), divided by the step's device time, against the measured HBM
           copy bandwidth in MEASURED_PEAKS.json.
parity   : after the timed region, the labels of the e2e solve are compared
           bit-exactly with the oracle's restatement of the reference's Tarjan
           on the same graph.
workloads: (1 GPU) the other benchmark workloads, each with its own parity,
           clocks and baseline: the 4096^2 grid, the 4096-graph batch (against
           one launch per graph and the reference's own GPU FB) and the served
           stream (plain / batched / batched + network, three repeats).
--impl reference: the reference's own CPU decomposition (tarjan.cpp
           TR_Decomposition, compiled from the reference sources into
           oracle/_ref) on a bounded sample of the headline workload, rank 0
           only; the sample is drawn by a numpy restatement of the generator
           (oracle/rmat_sample.py), so that process loads no product library.
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


def headline_config(scale: int, samples_log2: int, seed: int, world: int) -> dict:
    """Workload description shared by both arms (graph statistics go elsewhere)."""
    return {
        "workload": f"rmat{scale}_e{samples_log2}_scc_2_w_hybrid",
        "graph": f"R-MAT scale {scale}, 2^{samples_log2} samples, (a,b,c,d)=(0.57,0.19,0.19,0.05), "
                 f"ids permuted, self-loops dropped, duplicates merged, seed {seed}",
        "path": "scc_2_w -a h: trim-1, hybrid reach (pull-capable topology sweeps, then quadratic), "
                "WCC + trim-2 once, partition rounds",
        "index_dtype": "u32",
        "l2": "inputs larger than L2 (CSR + transpose ~8.6 GB vs 126 MB L2); no flush",
        "parallelism": f"replicas{world}",
    }


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
    """Polls NVML (read-only) every few ms while a timed region runs."""

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
        return self

    def summary(self, t0: float | None = None, t1: float | None = None) -> dict:
        if not self.ok:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvml unavailable"]}
        win = self.samples if t0 is None else [s for s in self.samples if t0 <= s[0] <= t1]
        win = win or self.samples[-3:]
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


def cpu_tarjan(n, nodes, edges):
    """The reference's TR_Decomposition (oracle/_ref) or, without it, the
    oracle's restatement, on one host thread -> (seconds wall, SCC count, kind)."""
    import oracle

    kind = "reference" if oracle.ref_lib() is not None else "port"
    restore = quiet_stdout()
    try:
        t0 = time.perf_counter()
        if kind == "reference":
            cnt, _ = oracle.ref_tarjan(n, nodes, edges)
        else:
            _, cnt = oracle.tarjan_labels(n, nodes, edges)
        secs = time.perf_counter() - t0
    finally:
        restore()
    return secs, cnt, kind


def tarjan_parity(graph: str, n: int, nodes, edges, labels, nscc: int, largest: int | None = None) -> dict:
    """Labels of one solve against the oracle's Tarjan (tarjan.cpp:110-190
    restated), bit-exact after canonicalisation to minimum ids."""
    import numpy as np

    import oracle

    t0 = time.perf_counter()
    ref, rcnt = oracle.tarjan_labels(n, nodes, edges)
    eq = bool(np.array_equal(np.asarray(labels)[:n + 1], ref))
    out = {"checked": True, "graph": graph, "oracle": "Tarjan (tarjan.cpp:110-190 restated, oracle/scc_oracle.c)",
           "labels_equal": eq, "tarjan_count": rcnt, "engine_count": nscc, "counts_equal": rcnt == nscc,
           "tarjan_largest_scc": int(np.bincount(ref[1:]).max()) if n else 0}
    if largest is not None:
        out["engine_largest_scc"] = largest
    if not eq:
        out["labels_differing"] = int((np.asarray(labels)[:n + 1] != ref).sum())
    out["check_s"] = round(time.perf_counter() - t0, 2)
    return out


# ---------------------------------------------------------------- reference
def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    if args.workload != "rmat26":
        print(json.dumps({"impl": "reference", "unavailable": f"the reference arm covers the headline workload; "
                          f"the {args.workload} workload reports its CPU baseline in its own line"}), flush=True)
        return
    import oracle
    from oracle import rmat_sample

    scale = args.ref_scale
    t0 = time.perf_counter()
    n, nodes, edges = rmat_sample.rmat_csr(scale, 16 << scale, ABC, args.seed)
    gen_s = time.perf_counter() - t0
    m = len(edges)
    kind = "reference" if oracle.ref_lib() is not None else "port"
    times = []
    cnt = None
    for i in range(args.warmup + args.steps):
        secs, cnt, _ = cpu_tarjan(n, nodes, edges)
        if i >= args.warmup:
            times.append(secs)
    per = sum(times) / len(times)
    value = m / per
    sample = (f"R-MAT scale {scale}, 2^{scale + 4} samples (same generator, (a,b,c,d), permutation and seed "
              f"{args.seed} as the headline graph, drawn by oracle/rmat_sample.py): n={n}, m={m}, {cnt} SCCs; "
              f"one {'tarjan.cpp TR_Decomposition' if kind == 'reference' else 'oracle Tarjan'} per step on 1 "
              f"host thread (the algorithm is sequential); sample built in {gen_s:.1f} s")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": per * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": headline_config(args.scale, args.samples_log2, args.seed, world),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": kind, "sample": sample,
                         "host_cores_available": os.cpu_count()},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ ours
def pinned_u32(count):
    import numpy as np
    import torch

    return torch.empty(int(max(count, 1)), dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)


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
    if prof.exists():
        try:
            t = json.loads(prof.read_text())
            traffic = float(t["bytes_per_edge"]) * m + float(t.get("bytes_per_vertex", 0.0)) * n
        except Exception:
            traffic = None
    clocks = sampler.summary(t_wall0, t_wall1)

    # e2e through the public API from pinned host buffers
    h_nodes, h_edges, h_nodesT, h_edgesT = pinned_u32(n + 2), pinned_u32(m), pinned_u32(n + 2), pinned_u32(m)
    ctx.download_into(h_nodes, h_edges, h_nodesT, h_edgesT)
    hg = scc.HostCSR.from_arrays(h_nodes, h_edges[:m], h_nodesT, h_edgesT[:m], sorted_unique=True)
    h_labels = pinned_u32(n + 1)
    e2e = None
    ctx.upload(hg)  # warm
    _, c2, st2 = ctx.solve(out=h_labels)
    if not args.no_e2e:
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e2e_steps = max(1, min(args.steps, args.e2e_steps))
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            ctx.upload(hg)
            _, c2, st2 = ctx.solve(out=h_labels)
        torch.cuda.synchronize()
        e2e_s = (time.perf_counter() - t0) / e2e_steps
        if dist:
            t = torch.tensor([e2e_s], dtype=torch.float64, device=f"cuda:{local}")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_s = float(t.item())
        e2e = {"value": world * m / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 2 * 4 * (n + 2) + 2 * 4 * m,
               "d2h_bytes_per_step": 4 * (n + 1), "ms_per_step": e2e_s * 1e3, "steps": e2e_steps}
    if c2 != cnt:
        raise SystemExit("e2e SCC count differs from the device-resident run")
    ctx.close()
    if dist:
        dist.destroy_process_group()
    if rank != 0:
        return

    parity = None
    if not args.no_parity:
        parity = tarjan_parity(f"R-MAT 2^{scale}, 2^{args.samples_log2} samples, seed {args.seed} (the timed graph)",
                               n, h_nodes, h_edges[:m], h_labels, c2, st2.get("largest_scc"))
    cpu = None
    if world == 1 and not args.no_cpu:
        cpu = cpu_baseline_rmat(args.cpu_scale, args.seed, local)
    workloads = None
    if world == 1 and not args.no_workloads:
        workloads = {}
        for name, fn in (("small", measure_small), ("grid", measure_grid), ("batch", measure_batch),
                         ("serve", measure_serve)):
            t0 = time.perf_counter()
            try:
                workloads[name] = fn(args)
            except Exception as e:  # recorded, the headline line still prints
                workloads[name] = {"error": f"{type(e).__name__}: {e}"}
            workloads[name]["wall_s"] = round(time.perf_counter() - t0, 1)

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic (R-MAT generated on the device, seed 2)",
        "config": headline_config(scale, args.samples_log2, args.seed, world),
        "graph_stats": {"n": n, "m": m, "nscc": cnt, "largest_scc": st2.get("largest_scc"),
                        "rounds": st.get("steps")},
        "engine_overrides": overrides,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                     "kernel": f"scc_persistent<{opts.block_size}> (+ per-step init pass)", "kernel_ms": kern_ms,
                     "algorithmic_bytes": b_alg(n, m)},
        "clocks": clocks,
        "gpu_launches": launches,
        "e2e": e2e,
        "cpu_baseline": cpu,
        "parity": parity,
        "workloads": workloads,
        "stats": {k: (round(v, 4) if isinstance(v, float) else v) for k, v in st.items()},
        "profile_ms": {k: v for k, v in prof_last.items()},
        "trace": trace_last if args.trace else None,
    }
    print(json.dumps(line), flush=True)


def cpu_baseline_rmat(scale: int, seed: int, device: int) -> dict:
    """Reference Tarjan on a R-MAT sample of the headline workload (built on the device)."""
    import gpuscc_code_b200 as scc

    with scc.SCCContext(device) as ctx:
        ctx.gen_rmat_device(scale, 16 << scale, ABC, seed)
        g = ctx.download()
    secs, cnt, kind = cpu_tarjan(g.n, g.nodes, g.edges)
    return {"value": g.m / secs, "unit": UNIT, "cores": 1, "kind": kind, "host_cores_available": os.cpu_count(),
            "sample": f"R-MAT scale {scale}, 2^{scale + 4} samples, same (a,b,c,d), permuted, seed {seed}: "
                      f"n={g.n}, m={g.m}, {cnt} SCCs; "
                      f"{'tarjan.cpp TR_Decomposition' if kind == 'reference' else 'oracle port'} on 1 host "
                      f"thread, wall {secs:.2f} s"}


# ------------------------------------------------------------- workloads
def _events_ms(stream, fn, steps: int):
    """Device ms of each of `steps` calls of fn() (CUDA events on `stream`)."""
    import torch

    out = []
    for _ in range(steps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        b.synchronize()
        out.append(a.elapsed_time(b))
    return out


def _ref_gpu_leg(cli: list, count: int, ours_ms: float, timeout: int) -> dict:
    """The reference's own GPU FB (scc_2_w build, -a h) on the same graph in a
    child process: its own timer, against this engine's device time."""
    import subprocess

    from oracle import ref_gpu

    if not ref_gpu.available():
        return {"unavailable": "oracle/_ref/libscc_ref_gpu.so not built"}
    try:
        r = subprocess.run([sys.executable, "-m", "oracle.ref_gpu", *cli, "--alg", "h"], cwd=ROOT,
                           capture_output=True, text=True, timeout=timeout)
        ref = json.loads(r.stdout.strip().splitlines()[-1]) if r.returncode == 0 else {
            "error": f"exit {r.returncode}: {(r.stderr or r.stdout).strip()[-200:]}"}
    except subprocess.TimeoutExpired:
        ref = {"error": f"no result within {timeout} s"}
    if "secs" in ref:
        ref["count_matches"] = ref["nscc"] == count
        ref["speedup_of_ours"] = ref["secs"] * 1e3 / ours_ms
    return ref


def measure_small(args) -> dict:
    """R-MAT 2^16 vertices, 2^20 samples, seed 1 (config 1): the small-graph
    latency of one solve (scc_2_w -a h) on the device, end to end through
    scc_solve from pinned buffers, the reference's Tarjan on one host thread,
    the reference's GPU FB on the same graph, parity."""
    import torch

    import gpuscc_code_b200 as scc

    gh = scc.gen_rmat(16, 1 << 20, seed=1)
    n, m = gh.n, gh.m
    ctx = scc.SCCContext(0, scc.Options(alg="h", wcc=True, trim2=True))
    ctx.upload(gh)
    stream = torch.cuda.ExternalStream(ctx.stream)
    for _ in range(5):
        cnt, st = ctx.solve_device()
    sampler = ClockSampler(0).start()
    ms = _events_ms(stream, lambda: ctx.solve_enqueue(), max(50, args.workload_steps))
    cnt, st = ctx.solve_collect()
    clocks = sampler.stop().summary()
    prof = ctx.profile()
    dev_ms = statistics.median(ms)
    arrs = [pinned_u32(n + 2), pinned_u32(m), pinned_u32(n + 2), pinned_u32(m)]
    for a, src in zip(arrs, (gh.nodes, gh.edges, gh.nodesT, gh.edgesT)):
        a[:len(src)] = src
    hp = scc.HostCSR.from_arrays(arrs[0], arrs[1][:m], arrs[2], arrs[3][:m], sorted_unique=True)
    out = pinned_u32(n + 1)
    for _ in range(3):
        ctx.upload(hp)
        ctx.solve(out=out)
    reps = 20
    t0 = time.perf_counter()
    for _ in range(reps):
        ctx.upload(hp)
        _, c2, st2 = ctx.solve(out=out)
    e2e_s = (time.perf_counter() - t0) / reps
    ctx.close()
    peak, peak_kind = load_peaks()
    achieved = b_alg(n, m) / (dev_ms / 1e3) / 1e9
    secs, rcnt, kind = cpu_tarjan(n, gh.nodes, gh.edges)
    return {
        "metric": "SCC solve latency (R-MAT 2^16, 2^20 samples, seed 1, scc_2_w -a h)",
        "value": dev_ms, "unit": "ms", "higher_is_better": False, "edges_per_s": m / (dev_ms / 1e3),
        "steps": len(ms), "ms_all": [round(x, 4) for x in ms],
        "config": {"workload": "rmat16_e20_seed1_scc_2_w", "n": n, "m": m, "nscc": cnt, "rounds": st.get("steps"),
                   "grid_blocks": st.get("grid_blocks"), "l2": "graph fits in L2 (8.5 MB); no flush: the "
                   "latency of back-to-back solves of a resident graph"},
        "roofline": {"bound": "latency", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind, "algorithmic_bytes": b_alg(n, m)},
        "e2e": {"value": e2e_s * 1e3, "unit": "ms", "h2d_bytes_per_step": 8 * (n + 2) + 8 * m,
                "d2h_bytes_per_step": 4 * (n + 1)},
        "cpu_baseline": {"value": secs * 1e3, "unit": "ms", "cores": 1, "kind": kind, "count": rcnt,
                         "sample": "the whole graph, one Tarjan on 1 host thread"},
        "reference_gpu_fb": _ref_gpu_leg(["--rmat", "16", "--samples-log2", "20", "--seed", "1"], cnt, dev_ms,
                                         args.refgpu_timeout),
        "parity": tarjan_parity("R-MAT 2^16, 2^20 samples, seed 1", n, gh.nodes, gh.edges, out, c2,
                                st2.get("largest_scc")),
        "clocks": clocks, "profile_ms": prof, "gpu_launches": 2 * len(ms),
    }


def measure_grid(args) -> dict:
    """4096^2 grid (config 3): every grid edge oriented by a coin flip, 15 %
    kept in both directions, long-range edges numbering 0.1 % of the grid
    edges, seed 3; scc_2_w -a h; device time per solve, end to end through
    scc_solve from pinned buffers, the reference Tarjan, parity."""
    import torch

    import gpuscc_code_b200 as scc

    side = args.grid_side
    gh = scc.gen_grid(side, 0.15, 0.001, seed=3)
    n, m = gh.n, gh.m
    ctx = scc.SCCContext(0, scc.Options(alg="h", wcc=True, trim2=True))
    ctx.upload(gh)
    stream = torch.cuda.ExternalStream(ctx.stream)
    for _ in range(3):
        cnt, st = ctx.solve_device()
    sampler = ClockSampler(0).start()
    ms = _events_ms(stream, lambda: ctx.solve_enqueue(), args.workload_steps)
    cnt, st = ctx.solve_collect()
    clocks = sampler.stop().summary()
    prof = ctx.profile()
    dev_ms = statistics.median(ms)
    # end to end: pinned graph up, solve, labels down
    arrs = [pinned_u32(n + 2), pinned_u32(m), pinned_u32(n + 2), pinned_u32(m)]
    for a, src in zip(arrs, (gh.nodes, gh.edges, gh.nodesT, gh.edgesT)):
        a[:len(src)] = src
    hp = scc.HostCSR.from_arrays(arrs[0], arrs[1][:m], arrs[2], arrs[3][:m], sorted_unique=True)
    out = pinned_u32(n + 1)
    ctx.upload(hp)
    ctx.solve(out=out)
    t0 = time.perf_counter()
    reps = 3
    for _ in range(reps):
        ctx.upload(hp)
        _, c2, st2 = ctx.solve(out=out)
    e2e_s = (time.perf_counter() - t0) / reps
    ctx.close()
    peak, peak_kind = load_peaks()
    achieved = b_alg(n, m) / (dev_ms / 1e3) / 1e9
    secs, rcnt, kind = cpu_tarjan(n, gh.nodes, gh.edges)
    return {
        "metric": f"SCC edges/s ({side}x{side} grid, 15% bidirectional, scc_2_w -a h)",
        "value": m / (dev_ms / 1e3), "unit": UNIT, "ms_per_step": dev_ms, "steps": len(ms),
        "ms_all": [round(x, 3) for x in ms],
        "config": {"workload": f"grid{side}_bidir15_lr0.1_scc_2_w", "n": n, "m": m, "nscc": cnt,
                   "rounds": st.get("steps"), "l2": "inputs larger than L2 (CSR + transpose 0.44 GB); no flush"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind, "algorithmic_bytes": b_alg(n, m)},
        "e2e": {"value": m / e2e_s, "unit": UNIT, "ms_per_step": e2e_s * 1e3,
                "h2d_bytes_per_step": 8 * (n + 2) + 8 * m, "d2h_bytes_per_step": 4 * (n + 1)},
        "cpu_baseline": {"value": m / secs, "unit": UNIT, "cores": 1, "kind": kind, "count": rcnt,
                         "sample": "the whole grid graph, one Tarjan on 1 host thread"},
        "reference_gpu_fb": _ref_gpu_leg(["--grid", str(side), "--seed", "3"], cnt, dev_ms, args.refgpu_timeout),
        "parity": tarjan_parity(f"grid {side}^2, seed 3", n, gh.nodes, gh.edges, out, c2, st2.get("largest_scc")),
        "clocks": clocks, "profile_ms": prof, "gpu_launches": 2 * len(ms),
    }


def _local_graph(nodes, edges, nodesT, edgesT, lo, hi):
    """Graph on global ids lo .. hi-1 of a packed batch, in local ids (reference layout)."""
    import numpy as np

    e0, e1 = int(nodes[lo]), int(nodes[hi])
    t0, t1 = int(nodesT[lo]), int(nodesT[hi])
    k = hi - lo
    ln = np.zeros(k + 2, np.uint32)
    ln[1:] = nodes[lo:hi + 1] - e0
    lt = np.zeros(k + 2, np.uint32)
    lt[1:] = nodesT[lo:hi + 1] - t0
    return ln, edges[e0:e1] - np.uint32(lo - 1), lt, edgesT[t0:t1] - np.uint32(lo - 1)


def _batch_parity(labels, seg, nodes, edges, nodesT, edgesT) -> dict:
    """Every graph of a packed batch against the oracle's Tarjan, host threads side by side."""
    from concurrent.futures import ThreadPoolExecutor

    import numpy as np

    import oracle

    t0 = time.perf_counter()

    def one(gi):
        lo, hi = int(seg[gi]), int(seg[gi + 1])
        ln, le, _, _ = _local_graph(nodes, edges, nodesT, edgesT, lo, hi)
        ref, rcnt = oracle.tarjan_labels(hi - lo, ln, le)
        mine = np.zeros(hi - lo + 1, np.uint32)
        mine[1:] = labels[lo:hi] - np.uint32(lo - 1)
        return rcnt, bool(np.array_equal(mine, ref))

    with ThreadPoolExecutor(max_workers=min(32, os.cpu_count() or 1)) as ex:
        res = list(ex.map(one, range(len(seg) - 1)))
    bad = [i for i, (_, ok) in enumerate(res) if not ok]
    return {"checked": True, "graphs": len(res), "graphs_equal": len(res) - len(bad), "labels_equal": not bad,
            "first_differing": bad[:5], "tarjan_count": sum(c for c, _ in res),
            "oracle": "Tarjan (tarjan.cpp:110-190 restated) per graph", "check_s": round(time.perf_counter() - t0, 1)}


def measure_batch(args, rank: int = 0) -> dict:
    """4096 independent graphs (ER / R-MAT 50/50, n log-uniform in [1e3, 2e5],
    average out-degree U[2, 16], seed 4) packed into one segmented CSR and
    solved by one persistent launch replayed from a captured CUDA graph, with
    parameters from the autotuner; against the same graphs solved one launch
    per graph (upload + solve each) and the reference's own GPU FB."""
    import subprocess

    import numpy as np
    import torch

    import gpuscc_code_b200 as scc
    from gpuscc_code_b200 import autotune
    from oracle import ref_gpu

    count = args.batch_count
    ctx = scc.SCCContext(0, scc.Options(alg="h", wcc=True, trim2=True))
    seg = ctx.gen_batch_device(count, 1000, 200_000, 2.0, 16.0, seed=4 + rank)
    n, m = ctx.n, ctx.m
    tuned, trials = ctx.options, []
    if not args.no_tune:
        space = {"block_size": [256, 512], "heavy_degree": [4096, 1024, 16384], "pull_alpha": [14, 6, -1],
                 "switch_permille": [10, 50]}
        tuned, trials = autotune.autotune(ctx, space=space, repeats=2)
    ctx.capture()
    for _ in range(3):
        ctx.replay()
    stream = torch.cuda.ExternalStream(ctx.stream)
    sampler = ClockSampler(0).start()
    res = {}
    ms = _events_ms(stream, lambda: res.update(r=ctx.replay()), args.workload_steps)
    clocks = sampler.stop().summary()
    cnt, st = res["r"]
    prof = ctx.profile()
    labels = ctx.read_labels()
    batched_ms = statistics.median(ms)
    full = ctx.download()
    ctx.close()
    nodes, edges, nodesT, edgesT = (np.asarray(a) for a in (full.nodes, full.edges, full.nodesT, full.edgesT))
    # the same graphs, one launch each (local ids, uploaded and solved one by one)
    graphs = [scc.HostCSR.from_arrays(*_local_graph(nodes, edges, nodesT, edgesT, int(seg[g]), int(seg[g + 1])),
                                      sorted_unique=True) for g in range(count)]
    per = scc.SCCContext(0, scc.Options(alg="h", wcc=True, trim2=True))
    per.upload(graphs[0])
    per.solve()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    dev_sum, total_cnt = 0.0, 0
    for hg in graphs:
        per.upload(hg)
        _, c, s2 = per.solve(want_labels=False)
        dev_sum += s2["ms_total"]
        total_cnt += c
    wall = time.perf_counter() - t0
    per.close()
    del graphs
    gps = count / (batched_ms / 1e3)
    out = {
        "metric": f"batched SCC graphs/s ({count} mixed ER/R-MAT graphs, one captured launch)",
        "value": gps, "unit": "graphs/s", "ms_per_step": batched_ms, "steps": len(ms),
        "ms_all": [round(x, 3) for x in ms],
        "config": {"workload": f"batch{count}_er_rmat_n1e3-2e5_deg2-16", "n": n, "m": m, "nscc": cnt, "graphs": count,
                   "launch": "captured CUDA graph: reset + init + one cooperative persistent kernel",
                   "l2": "inputs larger than L2 (packed CSR + transpose ~11 GB); no flush"},
        "tuned": {k: getattr(tuned, k) for k in ("block_size", "occupancy", "heavy_degree", "pull_alpha",
                                                 "pull_beta", "switch_permille")},
        "tuning_trials": [[f, v, round(t, 3)] for f, v, t in trials],
        "per_graph_plain": {"graphs_per_s_wall": count / wall, "graphs_per_s_device": count / (dev_sum / 1e3),
                            "count_equal": total_cnt == cnt,
                            "how": "this engine, one upload + one scc_solve per graph, same options, local ids"},
        "speedup_vs_per_graph": {"wall": gps / (count / wall), "device": dev_sum / batched_ms},
        "clocks": clocks, "profile_ms": prof, "gpu_launches": 2 * len(ms),
        "stats": {k: (round(v, 4) if isinstance(v, float) else v) for k, v in st.items()},
    }
    # the reference's own GPU FB on the first graphs of the same batch, one at a time (child process)
    if ref_gpu.available() and args.refgpu_batch > 0:
        try:
            r = subprocess.run([sys.executable, "-m", "oracle.ref_gpu", "--batch", str(args.refgpu_batch), "--alg",
                                "h"], cwd=ROOT, capture_output=True, text=True, timeout=args.refgpu_timeout)
            ref = json.loads(r.stdout.strip().splitlines()[-1]) if r.returncode == 0 else {
                "error": f"exit {r.returncode}: {(r.stderr or r.stdout).strip()[-200:]}"}
        except subprocess.TimeoutExpired:
            ref = {"error": f"no result within {args.refgpu_timeout} s"}
        if "graphs_per_s_timer" in ref:
            ref["speedup_of_batched"] = {"vs_timer": gps / ref["graphs_per_s_timer"],
                                         "vs_wall": gps / ref["graphs_per_s_wall"]}
        out["reference_gpu_fb"] = ref
    else:
        out["reference_gpu_fb"] = {"unavailable": "oracle/_ref/libscc_ref_gpu.so not built"}
    if not args.no_parity:
        out["parity"] = _batch_parity(labels, seg, nodes, edges, nodesT, edgesT)
        out["parity"]["counts_equal"] = out["parity"]["tarjan_count"] == cnt
    return out


def measure_serve(args) -> dict:
    """Served stream (config 5): Poisson arrivals of R-MAT (scale 14-22,
    average degree 8-32) and grid graphs (side 256-2048, 10-30 %
    bidirectional), seed 5.  The graphs are registered with the server first
    (their CSR stays resident on the device); each request names a graph.
    Three arms serve the same arrival sequence: the plain hybrid one graph per
    launch, continuous batching, and continuous batching with the trained
    strategy network; each is run `serve_repeats` times.  Every request's
    labels are compared with the same graph solved alone by the plain method,
    and those with the oracle's Tarjan."""
    import numpy as np
    import torch

    import gpuscc_code_b200 as scc
    from gpuscc_code_b200 import learned
    from gpuscc_code_b200.serve import Server, make_graph, poisson_arrivals, run_stream, stream_spec

    base = scc.Options(alg="h", wcc=True, trim2=True)
    ctx = scc.SCCContext(0, base)
    pool = [make_graph(stream_spec(i, seed=5), ctx) for i in range(args.serve_pool)]
    # alone: plain method, one graph at a time (the labels every arm must reproduce)
    alone, svc_ms = [], []
    for g in pool:
        ctx.upload(g)
        labels, _, st = ctx.solve()
        svc_ms.append(st["ms_total"])
        alone.append(labels)
    ctx.close()
    oracle_ok = all(np.array_equal(a, __import__("oracle").tarjan_labels(g.n, g.nodes, g.edges)[0])
                    for g, a in zip(pool, alone))
    reqs = [i % len(pool) for i in range(args.serve_requests)]
    outs = [pinned_u32(pool[i].n + 1) for i in reqs]
    rate = args.serve_rate
    if rate <= 0:  # load the plain server close to its device capacity
        rate = 0.9 * 1e3 / float(np.mean(svc_ms))
    arrivals = poisson_arrivals(len(reqs), rate, seed=5)
    model = learned.DEFAULT_MODEL if learned.DEFAULT_MODEL.exists() else None
    arms = [("plain", dict(batching=False), None), ("batched", dict(batching=True), None)]
    if model is not None:
        arms.append(("batched_learned", dict(batching=True), model))
    out = {}
    exact_all = True
    for name, kw, mdl in arms:
        reps = []
        for rep in range(args.serve_repeats):
            with Server(0, base, model=mdl, **kw) as srv:
                handles = [srv.register(g) for g in pool]
                items = [handles[i] for i in reqs]
                run_stream(srv, items[:len(pool)], np.zeros(len(pool)), outs[:len(pool)])  # warm the pools
                burst = run_stream(srv, items, np.zeros(len(items)), outs)
                exact = all(np.array_equal(a[:len(alone[i])], alone[i]) for a, i in zip(burst["labels"], reqs))
                st0 = srv.stats()
                res = run_stream(srv, items, arrivals, outs)
                st = srv.stats()
            exact = exact and all(np.array_equal(a[:len(alone[i])], alone[i]) for a, i in zip(res["labels"], reqs))
            exact_all &= exact
            picks = {}
            for info in res["info"]:
                picks[str(info["choice"])] = picks.get(str(info["choice"]), 0) + 1
            reps.append({"capacity_graphs_per_s": burst["graphs_per_s"], "graphs_per_s": res["graphs_per_s"],
                         "p50_ms": res["p50_ms"], "p99_ms": res["p99_ms"],
                         "mean_batch": float(np.mean([i["batch_graphs"] for i in res["info"]])),
                         "batches": st["batches"] - st0["batches"], "labels_exact": exact, "choices": picks})
        agg = {}
        for key in ("capacity_graphs_per_s", "graphs_per_s", "p50_ms", "p99_ms"):
            v = [r[key] for r in reps]
            agg[key] = {"min": min(v), "median": statistics.median(v), "max": max(v)}
        out[name] = {"summary": agg, "repeats": reps}
    med = lambda arm, key: out[arm]["summary"][key]["median"]
    return {
        "metric": "served SCC graphs/s (Poisson stream of R-MAT + grid graphs, resident CSR, p50/p99 latency)",
        "value": max(med(a, "capacity_graphs_per_s") for a in out), "unit": "graphs/s",
        "config": {"workload": f"serve{len(reqs)}_pool{len(pool)}_rmat14-22_grid256-2048", "requests": len(reqs),
                   "distinct_graphs": len(pool), "rate_per_s": rate, "repeats": args.serve_repeats,
                   "vertices": int(sum(pool[i].n for i in reqs)), "edges": int(sum(pool[i].m for i in reqs)),
                   "model": str(model.name) if model else None},
        "arms": out,
        "capacity_vs_plain": {a: med(a, "capacity_graphs_per_s") / med("plain", "capacity_graphs_per_s") for a in out},
        "p99_vs_plain": {a: med("plain", "p99_ms") / med(a, "p99_ms") for a in out},
        "plain_mean_device_ms": float(np.mean(svc_ms)),
        "parity": {"checked": True, "labels_equal": bool(exact_all and oracle_ok),
                   "how": "every request's labels equal the graph solved alone by the plain method, and those "
                          "equal the oracle's Tarjan"},
        "note": "graphs registered with the server before the stream (CSR resident on the device); each request "
                "names a graph and receives its labels in page-locked host memory; rate = 0.9 / mean plain device "
                "time unless given; capacity = all requests submitted at once; value = best arm's median capacity",
    }


def run_workload(args) -> None:
    import torch

    torch.cuda.set_device(0)
    fn = {"small": measure_small, "grid": measure_grid, "batch": measure_batch, "serve": measure_serve}[args.workload]
    res = fn(args)
    res.setdefault("n_gpus", 1)
    print(json.dumps(res), flush=True)


def run_batch_multi(args) -> None:
    """--workload batch under torchrun: every rank solves a batch of its own
    (seed 4 + rank) on its GPU (independent graphs, no collective on the data
    path); the line reports N x graphs / the slowest rank's time."""
    import datetime

    import torch
    import torch.distributed as dist

    world = int(os.environ["WORLD_SIZE"])
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    import gpuscc_code_b200 as scc

    ctx = scc.SCCContext(local, scc.Options(alg="h", wcc=True, trim2=True, block_size=512, heavy_degree=1024,
                                            pull_alpha=6, switch_permille=50))
    ctx.gen_batch_device(args.batch_count, 1000, 200_000, 2.0, 16.0, seed=4 + rank)
    ctx.capture()
    for _ in range(args.warmup):
        ctx.replay()
    stream = torch.cuda.ExternalStream(ctx.stream)
    dist.barrier()
    ms = statistics.median(_events_ms(stream, ctx.replay, args.steps))
    t = torch.tensor([ms], dtype=torch.float64, device=f"cuda:{local}")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ctx.close()
    dist.destroy_process_group()
    if rank == 0:
        ms = float(t.item())
        print(json.dumps({
            "metric": "batched SCC graphs/s (mixed ER/R-MAT graphs per GPU, one launch each)",
            "value": world * args.batch_count / (ms / 1e3), "unit": "graphs/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32", "data": "synthetic (one batch per rank, seed 4 + rank)",
            "config": {"workload": f"batch{args.batch_count}_er_rmat_n1e3-2e5_deg2-16",
                       "parallelism": f"independent batches x{world}", "l2": "inputs larger than L2"},
            "gpu_launches": 2 * args.steps}), flush=True)


def run_refgpu(args) -> None:
    """The reference's own GPU FB (scc_2_w build, compiled from its sources for
    sm_100a into oracle/_ref) against this engine on the same graphs and the
    same device: R-MAT scale 16 / 2^20 samples (seed 1, config 1), R-MAT at
    larger scales (seed 2) and grids.  The reference runs in a child process
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
    for side in args.refgpu_grids:
        cases.append((f"grid{side}_seed3", ["--grid", str(side), "--seed", "3"],
                      lambda c, side=side: c.upload(scc.gen_grid(side, 0.15, 0.001, seed=3))))
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
    print(json.dumps({"metric": "SCC solve time vs the reference's GPU FB (same B200, same graphs)",
                      "unit": "s", "rows": rows,
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
    ap.add_argument("--no-parity", action="store_true", help="skip the Tarjan label checks")
    ap.add_argument("--no-workloads", action="store_true", help="headline line only")
    ap.add_argument("--workload-steps", type=int, default=10, help="timed steps of each workload")
    ap.add_argument("--trace", action="store_true", help="include the per-sweep device trace in the line")
    ap.add_argument("--opt", action="append", default=[], metavar="KEY=VALUE",
                    help="override an engine option (scc_opts field), e.g. --opt occupancy=3")
    ap.add_argument("--grid-side", type=int, default=4096, help="grid: side of the grid graph")
    ap.add_argument("--refgpu-scales", type=int, nargs="*", default=[20, 22],
                    help="refgpu: further R-MAT scales (2^(scale+4) samples, seed 2)")
    ap.add_argument("--refgpu-grids", type=int, nargs="*", default=[1024, 4096], help="refgpu: grid sides")
    ap.add_argument("--refgpu-algs", nargs="*", default=["h", "t"], help="refgpu: reference -a arms")
    ap.add_argument("--refgpu-timeout", type=int, default=300)
    ap.add_argument("--refgpu-batch", type=int, default=256, help="batch: graphs the reference GPU FB solves")
    ap.add_argument("--workload", choices=["rmat26", "small", "grid", "batch", "serve", "refgpu"], default="rmat26",
                    help="rmat26: the headline line (with the other workloads inside it); grid / batch / serve: "
                         "one workload alone; refgpu: the reference's GPU FB on the same graphs")
    ap.add_argument("--serve-pool", type=int, default=24, help="serve: distinct graphs in the stream")
    ap.add_argument("--serve-requests", type=int, default=96, help="serve: requests in the stream")
    ap.add_argument("--serve-repeats", type=int, default=3)
    ap.add_argument("--serve-rate", type=float, default=0.0,
                    help="serve: arrivals per second (0 = 0.9 x the plain method's device throughput)")
    ap.add_argument("--batch-count", type=int, default=4096)
    ap.add_argument("--no-tune", action="store_true", help="batch: skip the autotuner")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "refgpu":
        run_refgpu(args)
    elif args.workload == "batch" and world > 1:
        run_batch_multi(args)
    elif args.workload in ("grid", "batch", "serve"):
        if int(os.environ.get("RANK", "0")) == 0:
            run_workload(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
