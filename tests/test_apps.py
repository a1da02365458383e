"""The scc / scc_w / scc_2_w apps (the reference's command line, scc.cu:57-148):
the CPU -t path and argument handling here; the GPU arms against the golden
counts and labels on a GPU."""
import json
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
BIN = ROOT / "gpuscc_code_b200" / "bin"
GOLDEN = ROOT / "tests" / "golden"


def run(app, *args):
    return subprocess.run([str(BIN / app), *args], capture_output=True, text=True, timeout=300)


def counts(out):
    return [int(l.split(":")[1]) for l in out.splitlines() if "->count of SCC:" in l]


def test_apps_are_built():
    for app in ("scc", "scc_w", "scc_2_w"):
        assert (BIN / app).exists(), app


def test_usage_without_a_graph():
    r = run("scc")
    assert r.returncode == 1 and "usage" in r.stderr


def test_missing_file_is_reported():
    r = run("scc_2_w", "-f", str(GOLDEN / "no_such.graph"))
    assert r.returncode == 1 and "error" in r.stderr


def test_tarjan_count_then_no_cpu_fallback():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    r = run("scc", "-t", "-f", str(GOLDEN / "demo.graph"))
    assert counts(r.stdout) == [6]          # -t: the CPU decomposition
    assert r.returncode == 1 and "no CUDA device" in r.stderr  # and no CPU stand-in for the GPU arms


@pytest.mark.gpu
@pytest.mark.parametrize("app", ["scc", "scc_w", "scc_2_w"])
def test_gpu_arms_match_golden(app, tmp_path):
    golden = json.load(open(GOLDEN / "golden.json"))
    for name, exp in golden.items():
        out = tmp_path / "labels.txt"
        r = run(app, "-t", "-a", "h", "-f", str(GOLDEN / name), "-o", str(out))
        assert r.returncode == 0, r.stderr
        assert counts(r.stdout) == [exp["nscc_reference"]] * 2, name  # -t, then the GPU
        labels = [int(l.split()[1]) for l in out.read_text().splitlines()]
        assert labels == exp["labels"][1:], name


@pytest.mark.gpu
def test_all_arms_in_one_run():
    r = run("scc_2_w", "-a", "a", "-f", str(GOLDEN / "demo.graph"))
    assert r.returncode == 0, r.stderr
    assert counts(r.stdout) == [6] * 7


@pytest.mark.gpu
def test_verify_files_follow_the_labels(tmp_path):
    golden = json.load(open(GOLDEN / "golden.json"))
    for name in ("demo.graph", "cycles.graph", "general.mtx"):
        labels = golden[name]["labels"]
        d = tmp_path / name.replace(".", "_")
        d.mkdir()
        r = run("scc_2_w", "-a", "h", "-f", str(GOLDEN / name), "-v", str(d))
        assert r.returncode == 0, r.stderr
        groups = {}
        for v in range(1, len(labels)):
            groups.setdefault(labels[v], []).append(v)
        sccs = [list(map(int, l.split())) for l in (d / "parallel_scc.txt").read_text().splitlines()]
        assert sccs == [groups[k] for k in sorted(groups)]
        trivial = [int(l) for l in (d / "trivial.txt").read_text().splitlines()]
        assert trivial == sorted(k for k, m in groups.items() if len(m) == 1)
        dist = dict(tuple(map(int, l.split())) for l in (d / "scc_dist.txt").read_text().splitlines())
        sizes = {}
        for m in groups.values():
            sizes[len(m)] = sizes.get(len(m), 0) + 1
        assert dist == sizes
