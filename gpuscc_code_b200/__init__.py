"""B200-native strongly-connected-components engine (drop-in for chenxuhao/gpuscc_code).

The compute path is hand-written sm_100a CUDA behind the C ABI in
include/scc_capi.h (libgpuscc_b200.so, built in-tree); this package is the
Python host binding.  Importing it fails if the library is not built.
"""
from ._capi import ALG, SCCError, lib  # noqa: F401  (raises ImportError when the .so is missing)
from .scc import (HostCSR, Options, SCCContext, computeSCC, csr_from_edges, gen_batch, gen_er, gen_grid,  # noqa: F401
                  gen_rmat, load, save, tarjan)

__version__ = lib.scc_version().decode()
