"""ctypes binding of include/scc_capi.h (libgpuscc_b200.so, built in-tree).

There is no fallback: if the shared library is missing or fails to load,
importing this module raises.  Build it with `python gpuscc_code_b200/build.py`.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libgpuscc_b200.so"

SCC_OK = 0
SCC_ERR_INVALID = -1
SCC_ERR_IO = -2
SCC_ERR_NOMEM = -3
SCC_ERR_CUDA = -4
SCC_ERR_TIMEOUT = -5
SCC_ERR_NODEVICE = -6
SCC_ERR_STATE = -7
SCC_ERR_CAPACITY = -8
SCC_ERR_BUSY = -9
SCC_ERR_REJECTED = -10

ALG = {"q": 0, "t": 1, "d": 2, "l": 3, "h": 4, "c": 5, "b": 6}
ALG_NAMES = {v: k for k, v in ALG.items()}

u32p = C.POINTER(C.c_uint32)


class scc_opts(C.Structure):
    _fields_ = [
        ("alg", C.c_int32), ("wcc", C.c_int32), ("trim2", C.c_int32), ("trim_first", C.c_int32),
        ("block_size", C.c_int32), ("warp_size", C.c_int32), ("pivot_rule", C.c_int32),
        ("switch_permille", C.c_int32), ("trim_depth", C.c_int32), ("pull_alpha", C.c_int32),
        ("pull_beta", C.c_int32), ("warp_degree", C.c_uint32), ("heavy_degree", C.c_uint32),
        ("max_iters", C.c_uint32), ("grid_blocks", C.c_uint32), ("timeout_ms", C.c_uint32),
        ("trim_first_depth", C.c_int32), ("occupancy", C.c_int32), ("async_depth", C.c_int32),
        ("test_stall_us", C.c_uint32), ("test_queue_cap", C.c_uint32),
    ]


class scc_host_csr(C.Structure):
    _fields_ = [
        ("n", C.c_uint32), ("m", C.c_uint32), ("nnz_header", C.c_uint32), ("symmetric", C.c_int32),
        ("sorted_unique", C.c_int32), ("owned", C.c_int32),
        ("nodes", u32p), ("edges", u32p), ("nodesT", u32p), ("edgesT", u32p),
    ]


class scc_dev_csr(C.Structure):
    _fields_ = [
        ("n", C.c_uint32), ("m", C.c_uint32), ("sorted_unique", C.c_int32),
        ("nodes", C.c_void_p), ("edges", C.c_void_p), ("nodesT", C.c_void_p), ("edgesT", C.c_void_p),
    ]


class scc_stats(C.Structure):
    _fields_ = [
        ("steps", C.c_uint32), ("fwd_depth", C.c_uint32), ("bwd_depth", C.c_uint32), ("trim_iters", C.c_uint32),
        ("wcc_iters", C.c_uint32), ("wcc_step", C.c_uint32), ("n_trimmed", C.c_uint32), ("n_trim2", C.c_uint32),
        ("n_fb_elim", C.c_uint32), ("nscc", C.c_uint32), ("largest_scc", C.c_uint32),
        ("pull_sweeps", C.c_uint32), ("grid_blocks", C.c_uint32), ("block_size", C.c_uint32),
        ("kernel_launches", C.c_uint32), ("reserved", C.c_uint32),
        ("ms_total", C.c_double), ("ms_trim", C.c_double), ("ms_fwd", C.c_double), ("ms_bwd", C.c_double),
        ("ms_update", C.c_double), ("ms_wcc", C.c_double),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_ if name != "reserved"}


class scc_server_cfg(C.Structure):
    _fields_ = [
        ("device", C.c_int32), ("batching", C.c_int32), ("max_batch_graphs", C.c_uint32),
        ("max_batch_vertices", C.c_uint32), ("max_batch_edges", C.c_uint32), ("solo_vertices", C.c_uint32),
        ("mem_budget", C.c_uint64), ("opts", scc_opts),
    ]


class scc_request_info(C.Structure):
    _fields_ = [
        ("nscc", C.c_uint32), ("batch_graphs", C.c_uint32), ("choice", C.c_int32 * 3), ("status", C.c_int32),
        ("queue_ms", C.c_double), ("latency_ms", C.c_double), ("solve_ms", C.c_double),
    ]


class scc_server_stats(C.Structure):
    _fields_ = [(k, C.c_uint64) for k in ("submitted", "completed", "rejected", "batches", "graphs_batched",
                                           "resident_bytes", "peak_resident_bytes", "budget_bytes",
                                           "registered", "evictions", "reuploads")]

    def as_dict(self) -> dict:
        return {name: int(getattr(self, name)) for name, _ in self._fields_}


f32p = C.POINTER(C.c_float)
i32p = C.POINTER(C.c_int32)

# (name, restype, argtypes) for every symbol include/scc_capi.h declares
SIGNATURES = [
    ("scc_last_error", C.c_char_p, []),
    ("scc_version", C.c_char_p, []),
    ("scc_opts_default", None, [C.POINTER(scc_opts)]),
    ("scc_load", C.c_int, [C.c_char_p, C.c_int, C.POINTER(scc_host_csr)]),
    ("scc_host_csr_free", None, [C.POINTER(scc_host_csr)]),
    ("scc_save", C.c_int, [C.c_char_p, C.POINTER(scc_host_csr)]),
    ("scc_csr_from_edges", C.c_int, [C.c_uint32, C.c_uint64, u32p, u32p, C.c_int, C.POINTER(scc_host_csr)]),
    ("scc_tarjan", C.c_int, [C.POINTER(scc_host_csr), u32p, u32p, C.POINTER(C.c_double)]),
    ("scc_gen_rmat", C.c_int, [C.c_uint32, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64, C.c_int,
                               C.POINTER(scc_host_csr)]),
    ("scc_gen_er", C.c_int, [C.c_uint32, C.c_uint64, C.c_uint64, C.POINTER(scc_host_csr)]),
    ("scc_gen_grid", C.c_int, [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64, C.POINTER(scc_host_csr)]),
    ("scc_gen_rmat_device", C.c_int, [C.c_void_p, C.c_uint32, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32,
                                      C.c_uint64, C.c_int, C.POINTER(scc_dev_csr)]),
    ("scc_ctx_create", C.c_int, [C.c_int, C.POINTER(scc_opts), C.POINTER(C.c_void_p)]),
    ("scc_ctx_destroy", C.c_int, [C.c_void_p]),
    ("scc_ctx_set_opts", C.c_int, [C.c_void_p, C.POINTER(scc_opts)]),
    ("scc_ctx_get_opts", C.c_int, [C.c_void_p, C.POINTER(scc_opts)]),
    ("scc_ctx_stream", C.c_void_p, [C.c_void_p]),
    ("scc_ctx_upload", C.c_int, [C.c_void_p, C.POINTER(scc_host_csr)]),
    ("scc_ctx_bind_device", C.c_int, [C.c_void_p, C.POINTER(scc_dev_csr)]),
    ("scc_ctx_download", C.c_int, [C.c_void_p, C.POINTER(scc_host_csr)]),
    ("scc_ctx_download_into", C.c_int, [C.c_void_p, u32p, u32p, u32p, u32p]),
    ("scc_ctx_set_segments", C.c_int, [C.c_void_p, C.c_uint32, u32p]),
    ("scc_solve", C.c_int, [C.c_void_p, u32p, u32p, C.POINTER(scc_stats)]),
    ("scc_solve_device", C.c_int, [C.c_void_p, C.c_void_p, u32p, C.POINTER(scc_stats)]),
    ("scc_solve_noalloc", C.c_int, [C.POINTER(scc_dev_csr), C.POINTER(scc_opts), C.c_void_p, u32p, C.c_void_p]),
    ("scc_solve_enqueue", C.c_int, [C.c_void_p, C.c_void_p]),
    ("scc_solve_capture", C.c_int, [C.c_void_p, C.c_void_p]),
    ("scc_solve_replay", C.c_int, [C.c_void_p, u32p, C.POINTER(scc_stats)]),
    ("scc_read_labels", C.c_int, [C.c_void_p, u32p]),
    ("scc_gen_batch", C.c_int, [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64,
                                C.POINTER(scc_host_csr), u32p]),
    ("scc_gen_batch_device", C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                       C.c_uint64, C.POINTER(scc_dev_csr), u32p]),
    ("scc_solve_collect", C.c_int, [C.c_void_p, u32p, C.POINTER(scc_stats)]),
    ("scc_get_profile", C.c_int, [C.c_void_p, C.POINTER(C.c_double), u32p]),
    ("scc_get_trace", C.c_int, [C.c_void_p, u32p, u32p, u32p, u32p, C.POINTER(C.c_double)]),
    ("scc_phase_begin", C.c_int, [C.c_void_p]),
    ("scc_trim1", C.c_int, [C.c_void_p, u32p]),
    ("scc_trim", C.c_int, [C.c_void_p, u32p]),
    ("scc_trim2", C.c_int, [C.c_void_p, u32p]),
    ("scc_select_pivots", C.c_int, [C.c_void_p, u32p]),
    ("scc_reach", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, u32p]),
    ("scc_update", C.c_int, [C.c_void_p, C.POINTER(C.c_int32)]),
    ("scc_count_elimmed", C.c_int, [C.c_void_p, u32p]),
    ("scc_unset_pivots", C.c_int, [C.c_void_p]),
    ("scc_update_wcc", C.c_int, [C.c_void_p, u32p, C.POINTER(C.c_int32)]),
    ("scc_get_states", C.c_int, [C.c_void_p, C.POINTER(C.c_uint8)]),
    ("scc_get_ranges", C.c_int, [C.c_void_p, u32p]),
    ("scc_get_labels", C.c_int, [C.c_void_p, u32p, u32p]),
    ("scc_batch_pack", C.c_int, [C.c_uint32, C.POINTER(scc_host_csr), C.POINTER(scc_host_csr), u32p]),
    ("scc_batch_solve", C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(scc_host_csr), C.POINTER(u32p), u32p]),
    ("scc_graph_features", C.c_int, [C.c_void_p, f32p]),
    ("scc_mlp_create", C.c_int, [C.c_int, C.c_uint64, C.POINTER(C.c_void_p)]),
    ("scc_mlp_destroy", C.c_int, [C.c_void_p]),
    ("scc_mlp_param_count", C.c_uint32, []),
    ("scc_mlp_params", C.c_int, [C.c_void_p, f32p, C.c_int]),
    ("scc_mlp_norm", C.c_int, [C.c_void_p, f32p, f32p, C.c_int]),
    ("scc_mlp_forward", C.c_int, [C.c_void_p, f32p, C.c_uint32, f32p]),
    ("scc_mlp_loss_grad", C.c_int, [C.c_void_p, f32p, i32p, C.c_uint32, f32p, f32p]),
    ("scc_mlp_train", C.c_int, [C.c_void_p, f32p, i32p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_float,
                                C.c_uint64, f32p]),
    ("scc_mlp_predict", C.c_int, [C.c_void_p, f32p, C.c_uint32, i32p]),
    ("scc_mlp_apply", C.c_int, [i32p, C.POINTER(scc_opts)]),
    ("scc_server_cfg_default", None, [C.POINTER(scc_server_cfg)]),
    ("scc_server_start", C.c_int, [C.POINTER(scc_server_cfg), C.POINTER(C.c_void_p)]),
    ("scc_server_set_model", C.c_int, [C.c_void_p, f32p, f32p, f32p]),
    ("scc_server_submit", C.c_int, [C.c_void_p, C.POINTER(scc_host_csr), u32p, C.POINTER(C.c_uint64)]),
    ("scc_server_register", C.c_int, [C.c_void_p, C.POINTER(scc_host_csr), C.POINTER(C.c_uint64)]),
    ("scc_server_submit_resident", C.c_int, [C.c_void_p, C.c_uint64, u32p, C.POINTER(C.c_uint64)]),
    ("scc_server_unregister", C.c_int, [C.c_void_p, C.c_uint64]),
    ("scc_server_poll", C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(scc_request_info)]),
    ("scc_server_wait", C.c_int, [C.c_void_p, C.c_uint64, C.c_uint32, C.POINTER(scc_request_info)]),
    ("scc_server_get_stats", C.c_int, [C.c_void_p, C.POINTER(scc_server_stats)]),
    ("scc_server_stop", C.c_int, [C.c_void_p]),
]


class SCCError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def _load() -> C.CDLL:
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is not built; run `python gpuscc_code_b200/build.py`")
    lib = C.CDLL(str(LIB_PATH))
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def check(rc: int) -> None:
    if rc != SCC_OK:
        raise SCCError(rc, lib.scc_last_error().decode(errors="replace"))
