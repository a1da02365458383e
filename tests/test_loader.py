"""Loader extras (no GPU): the binary CSR cache round trip, and the
multi-threaded parse of large text files against an independent build of
the same edge list, including the reference reader's line rules."""
import numpy as np
import pytest

import gpuscc_code_b200 as scc
from gpuscc_code_b200 import _capi

ARRAYS = ("nodes", "edges", "nodesT", "edgesT")


def same(a, b):
    return a.n == b.n and a.m == b.m and all(np.array_equal(getattr(a, k), getattr(b, k)) for k in ARRAYS)


@pytest.mark.parametrize("name", ["demo.graph", "general.mtx", "pattern_sym.mtx", "isolated.graph"])
def test_binary_cache_round_trip(golden_dir, tmp_path, name):
    g = scc.load(str(golden_dir / name))
    scc.save(g, tmp_path / "g.bin")
    h = scc.load(str(tmp_path / "g.bin"))
    assert same(g, h)
    assert (h.raw.symmetric, h.raw.sorted_unique, h.raw.nnz_header) == (g.raw.symmetric, g.raw.sorted_unique,
                                                                      g.raw.nnz_header)


def test_truncated_binary_cache_is_rejected(tmp_path):
    g = scc.gen_er(100, 300, seed=2)
    scc.save(g, tmp_path / "g.bin")
    data = (tmp_path / "g.bin").read_bytes()
    (tmp_path / "t.bin").write_bytes(data[:-8])
    with pytest.raises(scc.SCCError) as ei:
        scc.load(str(tmp_path / "t.bin"))
    assert ei.value.code == _capi.SCC_ERR_IO


def big_text(tmp_path, n=200_000, lines=1_200_000, seed=5, extra=""):
    rng = np.random.default_rng(seed)
    d = rng.integers(1, n + 1, lines)
    s = rng.integers(1, n + 1, lines)
    body = "\n".join(f"{a} {b} 1" for a, b in zip(d, s))
    # blank lines in the middle, as the reader allows
    cut = len(body) // 2
    cut = body.index("\n", cut)
    body = body[:cut] + "\n\n\n" + body[cut:]
    path = tmp_path / "big.graph"
    path.write_text(f"{n} {lines}\n" + body + "\n" + extra)
    assert path.stat().st_size > 8 << 20  # the multi-threaded parse
    return path, n, s.astype(np.uint32), d.astype(np.uint32)


def test_parallel_parse_matches_edge_list(tmp_path):
    path, n, src, dst = big_text(tmp_path, extra="this line is past the edge count and is never read\n")
    g = scc.load(str(path))
    ref = scc.csr_from_edges(n, src, dst)
    assert same(g, ref)


def test_parallel_parse_reports_bad_line(tmp_path):
    path, n, _, _ = big_text(tmp_path)
    text = path.read_text().splitlines()
    text[700_000] = "12 x"
    path.write_text("\n".join(text) + "\n")
    with pytest.raises(scc.SCCError) as ei:
        scc.load(str(path))
    assert ei.value.code == _capi.SCC_ERR_IO and "bad edge line" in str(ei.value)


def test_parallel_parse_reports_short_file(tmp_path):
    path, n, _, _ = big_text(tmp_path)
    text = path.read_text().splitlines()
    text[0] = f"{n} {len(text) + 5}"
    path.write_text("\n".join(text) + "\n")
    with pytest.raises(scc.SCCError) as ei:
        scc.load(str(path))
    assert "edge lines expected" in str(ei.value)
