"""The reference's own GPU FB (its scc_2_w build, compiled from its sources
into oracle/_ref) agrees with the engine's SCC count on the same graphs.
The reference prints and exit()s on errors, so it runs in a child process."""
import json
import subprocess
import sys
from pathlib import Path

import pytest

import gpuscc_code_b200 as scc
from oracle import ref_gpu

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]


@pytest.mark.skipif(not ref_gpu.available(), reason="oracle/_ref/libscc_ref_gpu.so not built")
@pytest.mark.parametrize("cli,make", [
    (["--rmat", "16", "--samples-log2", "20", "--seed", "1"], lambda: scc.gen_rmat(16, 1 << 20, seed=1)),
    (["--rmat", "14", "--samples-log2", "18", "--seed", "4"], lambda: scc.gen_rmat(14, 1 << 18, seed=4)),
    (["--grid", "128", "--seed", "3"], lambda: scc.gen_grid(128, 0.15, 0.001, seed=3)),
])
@pytest.mark.parametrize("alg", ["h", "t"])
def test_reference_gpu_count_matches(cli, make, alg):
    r = subprocess.run([sys.executable, "-m", "oracle.ref_gpu", *cli, "--alg", alg, "--repeats", "1"], cwd=ROOT,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-500:]
    ref = json.loads(r.stdout.strip().splitlines()[-1])
    g = make()
    with scc.SCCContext(0, alg="h", wcc=True, trim2=True) as ctx:
        ctx.upload(g)
        _, cnt, _ = ctx.solve(want_labels=False)
    assert ref["n"] == g.n and ref["m"] == g.m
    assert ref["nscc"] == cnt
