"""The numpy R-MAT restatement that bench.py's reference leg uses (so that
process loads no product library) draws exactly the product's graph."""
import numpy as np
import pytest

import gpuscc_code_b200 as scc
from oracle import rmat_sample


@pytest.mark.parametrize("scale,samples,seed,permute", [(10, 16 << 10, 2, True), (11, 8 << 11, 7, True),
                                                        (9, 16 << 9, 3, False), (1, 64, 1, True)])
def test_numpy_rmat_equals_product_generator(scale, samples, seed, permute):
    g = scc.gen_rmat(scale, samples, seed=seed, permute=permute)
    n, nodes, edges = rmat_sample.rmat_csr(scale, samples, seed=seed, permute=permute)
    assert n == g.n
    assert np.array_equal(nodes[1:], np.asarray(g.nodes)[1:])
    assert np.array_equal(edges, np.asarray(g.edges))


def test_permutation_is_a_bijection():
    for bits in (1, 5, 8, 13):
        p = rmat_sample.permutation(bits, 99)
        assert np.array_equal(np.sort(p), np.arange(1 << bits, dtype=np.uint32))
