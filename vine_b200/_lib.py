"""ctypes binding of libvine.so (the C ABI declared in include/vine.h and
include/vine_workloads.h).

The library is the product: there is no Python or CPU fallback.  Importing
this module fails loudly when libvine.so is missing or stale.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

_HERE = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("VINE_LIB", _HERE / "libvine.so"))

VINE_OK = 0
VINE_ERR_INVALID = -1
VINE_ERR_CAPACITY = -2
VINE_ERR_CUDA = -3
VINE_ERR_TIMEOUT = -4
VINE_ERR_NO_DEVICE = -5
VINE_ERR_IO = -6
VINE_ERR_INTERNAL = -7

STATUS_NAMES = {
    VINE_OK: "VINE_OK", VINE_ERR_INVALID: "VINE_ERR_INVALID", VINE_ERR_CAPACITY: "VINE_ERR_CAPACITY",
    VINE_ERR_CUDA: "VINE_ERR_CUDA", VINE_ERR_TIMEOUT: "VINE_ERR_TIMEOUT",
    VINE_ERR_NO_DEVICE: "VINE_ERR_NO_DEVICE", VINE_ERR_IO: "VINE_ERR_IO",
    VINE_ERR_INTERNAL: "VINE_ERR_INTERNAL",
}

ENGINE_BATCH, ENGINE_PLAIN = 0, 1
LABEL_CSP, LABEL_HOP, LABEL_MAXCOST, LABEL_QOS = 1, 2, 3, 6
MODE_OPTIMAL, MODE_PARETO = 0, 1
POLICY_FIXED, POLICY_AR, POLICY_MLP = 0, 1, 2
STAT_NAMES = ["expanded", "relaxed", "inserted", "dominated", "buckets", "rounds", "spills",
              "cycles", "abort_site", "bound_rounds", "bound_cycles", "chain_steps",
              "split_cycles", "split_items", "policy_cycles", "load_cycles", "relax_cycles",
              "start_ns", "time_ns", "rest_items", "idle_cycles", "publish_cycles"]
STAT_COUNT = 22
STAT_CYCLES, STAT_START_NS, STAT_TIME_NS = 7, 17, 18
STAT_ABORT_SITE = 8
SITE_LOCK, SITE_ASYNC, SITE_TIME, SITE_RING = 7, 12, 13, 14
MLP_IN, MLP_HIDDEN, MLP_OUT = 16, 64, 2
MLP_PARAMS = 64 * 16 + 64 + 64 * 64 + 64 + 2 * 64 + 2
TRACE_COLS = 20


class vine_config(C.Structure):
    _fields_ = [
        ("engine", C.c_int32), ("mode", C.c_int32), ("policy", C.c_int32),
        ("use_bounds", C.c_int32), ("block_threads", C.c_int32), ("ctas_per_sm", C.c_int32),
        ("table_log2", C.c_int32), ("spill_log2", C.c_int32), ("bucket_width", C.c_float),
        ("split_threshold", C.c_int32), ("pool_labels", C.c_int64), ("far_capacity", C.c_int64),
        ("use_cuda_graph", C.c_int32), ("order_queries", C.c_int32), ("mlp", C.c_void_p),
        ("trace", C.c_int32), ("max_workers", C.c_int32), ("sync_rounds", C.c_int32), ("band_mult", C.c_int32), ("ar_scale", C.c_float),
        ("wait_limit", C.c_int32), ("time_limit_ms", C.c_int32), ("split_staging", C.c_int32),
    ]


class vine_results(C.Structure):
    _fields_ = [
        ("cost", C.c_void_p), ("delay", C.c_void_p), ("found", C.c_void_p), ("status", C.c_void_p),
        ("path_offsets", C.c_void_p), ("path", C.c_void_p), ("path_capacity", C.c_int64),
        ("pareto_d", C.c_void_p), ("pareto_delay", C.c_void_p), ("pareto_n", C.c_void_p),
        ("pareto_stride", C.c_int32), ("stats", C.c_void_p), ("retried", C.c_int32),
    ]


class vine_workload_params(C.Structure):
    _fields_ = [
        ("kind", C.c_int32), ("seed", C.c_uint64), ("rows", C.c_int32), ("cols", C.c_int32),
        ("n", C.c_int64), ("m_target", C.c_int64), ("exponent", C.c_double),
        ("n_pairs", C.c_int32), ("n_alpha", C.c_int32), ("alpha", C.c_float * 4),
        ("alpha_lo", C.c_float), ("alpha_hi", C.c_float), ("hop_lo", C.c_int32),
        ("hop_hi", C.c_int32), ("hop_log_uniform", C.c_int32), ("nthreads", C.c_int32),
        ("query_seed", C.c_uint64),
    ]


# exported symbol -> (restype, argtypes)
SIGNATURES = {
    "vine_last_error": (C.c_char_p, []),
    "vine_version": (C.c_char_p, []),
    "vine_graph_create": (C.c_int, [C.c_int32, C.c_int32, C.c_int64, C.c_void_p, C.c_void_p,
                                    C.c_void_p, C.c_void_p, C.POINTER(C.c_void_p)]),
    "vine_graph_destroy": (None, [C.c_void_p]),
    "vine_graph_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int64),
                                  C.POINTER(C.c_int32)]),
    "vine_config_default": (None, [C.POINTER(vine_config)]),
    "vine_solve": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                             C.POINTER(vine_config), C.POINTER(vine_results)]),
    "vine_solve_device": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.POINTER(vine_config), C.POINTER(vine_results), C.c_void_p]),
    "vine_solve_multi": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.POINTER(vine_config), C.POINTER(vine_results)]),
    "vine_solve_labels": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p,
                                    C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(vine_config),
                                    C.POINTER(vine_results), C.c_void_p]),
    "vine_solve_host": (C.c_int, [C.c_int32, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                                  C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                  C.c_int32, C.c_int32, C.POINTER(vine_results)]),
    "vine_mlp_create": (C.c_int, [C.c_int32, C.c_uint64, C.c_void_p, C.POINTER(C.c_void_p)]),
    "vine_mlp_destroy": (None, [C.c_void_p]),
    "vine_mlp_get_params": (C.c_int, [C.c_void_p, C.c_void_p]),
    "vine_mlp_set_params": (C.c_int, [C.c_void_p, C.c_void_p]),
    "vine_mlp_forward": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]),
    "vine_mlp_loss_grad": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p]),
    "vine_mlp_loss_grad_noalloc": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p,
                                             C.c_void_p, C.c_void_p, C.c_void_p]),
    "vine_mlp_train": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_int32,
                                 C.c_int32, C.c_float, C.c_uint64, C.POINTER(C.c_float)]),
    "vine_trace_fetch": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64), C.c_void_p, C.c_int64]),
    "vine_autotune": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                C.POINTER(vine_config), C.c_char_p, C.POINTER(vine_config)]),
    "vine_workload_default_params": (C.c_int, [C.c_int32, C.POINTER(vine_workload_params)]),
    "vine_workload_generate": (C.c_int, [C.POINTER(vine_workload_params), C.POINTER(C.c_void_p)]),
    "vine_workload_load_mtx": (C.c_int, [C.c_char_p, C.POINTER(C.c_void_p)]),
    "vine_workload_load_cola": (C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(C.c_void_p)]),
    "vine_workload_add_random_queries": (C.c_int, [C.c_void_p, C.c_uint64, C.c_int32, C.c_int32,
                                                   C.c_void_p]),
    "vine_workload_graph": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int64),
                                      C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                      C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]),
    "vine_workload_queries": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_void_p),
                                        C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                        C.POINTER(C.c_void_p)]),
    "vine_workload_destroy": (None, [C.c_void_p]),
}


class VineError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def _load():
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} not found: build the CUDA engine first (python -m vine_b200.build)")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def check(status: int) -> None:
    if status != VINE_OK:
        raise VineError(status, lib.vine_last_error().decode(errors="replace"))
