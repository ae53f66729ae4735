"""vine_b200: exact constrained-shortest-path queries on one B200.

The compute path is libvine.so (CUDA for sm_100a behind a C ABI,
include/vine.h).  This package is its Python host binding and mirrors the
reference's query interface (Graph, c_label, c_constraint, cspp)."""
from .api import (MLP, Config, Graph, Results, Workload, autotune, c_constraint, c_edge,
                  c_label, config_dict, cspp, fetch_trace, solve, solve_device, solve_host, solve_labels, solve_multi)
from ._lib import VineError, lib

__all__ = ["MLP", "Config", "Graph", "Results", "Workload", "autotune", "c_constraint", "c_edge",
           "c_label", "config_dict", "cspp", "fetch_trace", "solve", "solve_device", "solve_host", "solve_labels", "solve_multi", "VineError",
           "lib"]
