"""Builds the engine in-tree: libgpuscc_b200.so plus the scc / scc_w / scc_2_w apps.

CUDA sources are compiled for sm_100a only (`-gencode arch=compute_100a,code=sm_100a`),
host sources with g++; objects go to gpuscc_code_b200/_build, the shared
library next to this file and the apps to gpuscc_code_b200/bin.
Run `python gpuscc_code_b200/build.py [--force]` (by path: importing the package loads the library).
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
BIN = PKG / "bin"
LIB = PKG / "libgpuscc_b200.so"
INCLUDE = ROOT / "include"
CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CU_SOURCES = ["scc_engine.cu", "scc_gen_device.cu", "scc_noalloc.cu", "scc_features.cu", "scc_mlp.cu", "scc_server.cu"]
CPP_SOURCES = ["scc_capi.cpp", "scc_host.cpp"]
HEADERS = ["scc_device.cuh", "scc_engine.h", "scc_gen.h", "scc_internal.h", "scc_features.h"]
APPS = {"scc": [], "scc_w": ["-DSCC_APP_WCC"], "scc_2_w": ["-DSCC_APP_WCC", "-DSCC_APP_TRIM2"]}


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} {cmd[-1]}")


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose_ptxas: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    BIN.mkdir(exist_ok=True)
    hdrs = [CSRC / h for h in HEADERS] + [INCLUDE / "scc_capi.h"]
    objs, jobs = [], []
    for src in CU_SOURCES:
        s = CSRC / src
        o = BUILD / (s.stem + ".o")
        if force or _stale(o, [s] + hdrs):
            cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", str(INCLUDE),
                   "-I", str(CSRC), "-c", str(s), "-o", str(o)]
            if verbose_ptxas:
                cmd.insert(-4, "-Xptxas=-v")
            jobs.append(cmd)
        objs.append(o)
    for src in CPP_SOURCES:
        s = CSRC / src
        o = BUILD / (s.stem + ".o")
        if force or _stale(o, [s] + hdrs):
            jobs.append(["g++", "-O2", "-std=c++17", "-fPIC", "-pthread", "-I", str(INCLUDE), "-I", str(CSRC),
                         "-I", str(CUDA_HOME / "include"), "-c", str(s), "-o", str(o)])
        objs.append(o)
    # independent translation units compile side by side
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        list(ex.map(_run, jobs))
    if force or _stale(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-Xcompiler", "-pthread"])
    main = CSRC / "apps" / "scc_main.cpp"
    for app, defs in APPS.items():
        exe = BIN / app
        if force or _stale(exe, [main, LIB, INCLUDE / "scc_capi.h"]):
            _run(["g++", "-O2", "-std=c++17", *defs, "-I", str(INCLUDE), str(main), "-o", str(exe),
                  "-L", str(PKG), "-lgpuscc_b200", "-Wl,-rpath,$ORIGIN/.."])
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose_ptxas="--ptxas" in sys.argv)
    print(LIB)
