"""Python mirror of the reference's CSP query interface over the C ABI.

The reference exposes the path as C++ templates: the problem types
``c_label`` / ``c_constraint`` / ``c_edge`` (include/label.hpp:170-247,
include/constraint.hpp:81-105, include/edge.hpp:16-26), the graph
``Graph<c_edge>`` with ``adj_to_csr`` / ``make_gpu_graph``
(include/graph.hpp:90-195) and the query class
``cspp<Label_t, Edge_t>(g, ntask, src_labels, sinks, C_l).solve()``
(algorithm/cspp.hpp:11-69).  This module keeps those names and argument
meanings, and fills the results the reference left empty (``path_l``,
``size_of_result_l``) plus cost, delay and a feasibility flag per query.
Everything runs in libvine.so on the GPU; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import check, lib


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


# --------------------------------------------------------------------- problem


@dataclass
class c_edge:
    """Arc weights (include/edge.hpp:16-26)."""
    len: float
    delay: float


@dataclass
class c_label:
    """Partial path (vid, d, delay) (include/label.hpp:170-247).

    ``c_label(vid)`` is a source label with d = delay = 0, like the
    reference's host constructor (include/label.hpp:184-189)."""
    vid: int
    d: float = 0.0
    delay: float = 0.0

    def expand(self, next_v: int, e: c_edge) -> "c_label":
        # include/label.hpp:214-222 (device expand: additive)
        return c_label(next_v, np.float32(self.d) + np.float32(e.len),
                       np.float32(self.delay) + np.float32(e.delay))

    @staticmethod
    def dominate(a: "c_label", b: "c_label") -> bool:
        # include/label.hpp:234-236
        return a.d <= b.d and a.delay <= b.delay


@dataclass
class c_constraint:
    """Delay budget (include/constraint.hpp:81-105)."""
    delay_L: float

    def pass_constraints_check(self, l: c_label) -> bool:
        return not (l.delay > self.delay_L)


# ----------------------------------------------------------------------- graph


class Graph:
    """Directed graph in CSR form (row_ptr[n+1], col[m], len[m], delay[m]).

    Mirrors Graph<c_edge> (include/graph.hpp:90-134): ``N``, ``M`` and
    ``make_gpu_graph()`` (include/graph.hpp:169-195), which uploads it."""

    def __init__(self, row_ptr, col, length, delay, device: int = 0):
        self.row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int64)
        self.col = np.ascontiguousarray(col, dtype=np.int32)
        self.len = np.ascontiguousarray(length, dtype=np.float32)
        self.delay = np.ascontiguousarray(delay, dtype=np.float32)
        self.N = int(self.row_ptr.shape[0] - 1)
        self.M = int(self.col.shape[0])
        self.device = device
        self._h = None

    def adj_to_csr(self) -> int:  # include/graph.hpp:136-167 (already CSR)
        return 0

    def make_gpu_graph(self) -> int:
        if self._h is None:
            h = C.c_void_p()
            check(lib.vine_graph_create(self.device, self.N, self.M, _ptr(self.row_ptr),
                                        _ptr(self.col), _ptr(self.len), _ptr(self.delay),
                                        C.byref(h)))
            self._h = h
        return 0

    @property
    def handle(self):
        self.make_gpu_graph()
        return self._h

    def info(self):
        n, m, integral = C.c_int32(), C.c_int64(), C.c_int32()
        check(lib.vine_graph_info(self.handle, C.byref(n), C.byref(m), C.byref(integral)))
        return n.value, m.value, bool(integral.value)

    def out_edges(self, u: int):
        a, b = self.row_ptr[u], self.row_ptr[u + 1]
        return self.col[a:b], self.len[a:b], self.delay[a:b]

    def close(self):
        if self._h is not None:
            lib.vine_graph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------- config


def Config(**kw) -> _lib.vine_config:
    """vine_config with defaults (vine_config_default) and keyword overrides.

    engine: "batch" | "plain"; mode: "optimal" | "pareto";
    policy: "fixed" | "ar" | "mlp" (pass mlp=MLP)."""
    c = _lib.vine_config()
    lib.vine_config_default(C.byref(c))
    names = {"engine": {"batch": _lib.ENGINE_BATCH, "plain": _lib.ENGINE_PLAIN},
             "mode": {"optimal": _lib.MODE_OPTIMAL, "pareto": _lib.MODE_PARETO},
             "policy": {"fixed": _lib.POLICY_FIXED, "ar": _lib.POLICY_AR, "mlp": _lib.POLICY_MLP}}
    for k, v in kw.items():
        if k in names and isinstance(v, str):
            v = names[k][v]
        if k == "mlp":
            c.mlp = v.handle if v is not None else None
            c._mlp_ref = v  # keep the model alive with the config
            continue
        if not hasattr(c, k):
            raise TypeError(f"unknown config field {k}")
        setattr(c, k, v)
    return c


def config_dict(c: _lib.vine_config) -> dict:
    return {k: getattr(c, k) for k, _ in _lib.vine_config._fields_ if k != "mlp"}


# --------------------------------------------------------------------- results


@dataclass
class Results:
    cost: np.ndarray
    delay: np.ndarray
    found: np.ndarray
    status: np.ndarray
    path_offsets: Optional[np.ndarray] = None
    path_vertices: Optional[np.ndarray] = None
    pareto_d: Optional[np.ndarray] = None
    pareto_delay: Optional[np.ndarray] = None
    pareto_n: Optional[np.ndarray] = None
    stats: Optional[np.ndarray] = None
    rc: int = 0
    retried: int = 0
    extra: Optional[np.ndarray] = None  # label variants: [nq, 2] hop count, maxcost

    def path(self, q: int) -> np.ndarray:
        a, b = self.path_offsets[q], self.path_offsets[q + 1]
        return self.path_vertices[a:b]

    def pareto(self, q: int) -> np.ndarray:
        k = int(self.pareto_n[q])
        k = min(k, self.pareto_d.shape[1])
        return np.stack([self.pareto_d[q, :k], self.pareto_delay[q, :k]], axis=1)


def solve(graph: Graph, src, dst, budget, config=None, paths: bool = True,
          pareto_stride: int = 0, stats: bool = False, path_capacity: Optional[int] = None,
          raise_on_error: bool = True) -> Results:
    """Solves queries (src[q] -> dst[q] within budget[q]) from host arrays."""
    src = np.ascontiguousarray(src, dtype=np.int32)
    dst = np.ascontiguousarray(dst, dtype=np.int32)
    budget = np.ascontiguousarray(budget, dtype=np.float32)
    nq = int(src.shape[0])
    if dst.shape[0] != nq or budget.shape[0] != nq:
        raise ValueError("src, dst and budget must have the same length")
    cfg = config if config is not None else Config()
    r = Results(cost=np.empty(nq, np.float32), delay=np.empty(nq, np.float32),
                found=np.empty(nq, np.int32), status=np.empty(nq, np.int32))
    res = _lib.vine_results()
    res.cost, res.delay = _ptr(r.cost), _ptr(r.delay)
    res.found, res.status = _ptr(r.found), _ptr(r.status)
    if paths:
        cap = path_capacity if path_capacity is not None else max(1024, nq * 64)
        r.path_offsets = np.zeros(nq + 1, np.int64)
        r.path_vertices = np.zeros(cap, np.int32)
        res.path_offsets, res.path = _ptr(r.path_offsets), _ptr(r.path_vertices)
        res.path_capacity = cap
    if pareto_stride > 0:
        r.pareto_d = np.zeros((nq, pareto_stride), np.float32)
        r.pareto_delay = np.zeros((nq, pareto_stride), np.float32)
        r.pareto_n = np.zeros(nq, np.int32)
        res.pareto_d, res.pareto_delay = _ptr(r.pareto_d), _ptr(r.pareto_delay)
        res.pareto_n, res.pareto_stride = _ptr(r.pareto_n), pareto_stride
    if stats:
        r.stats = np.zeros((nq, _lib.STAT_COUNT), np.int64)
        res.stats = _ptr(r.stats)
    rc = lib.vine_solve(graph.handle, nq, _ptr(src), _ptr(dst), _ptr(budget), C.byref(cfg),
                        C.byref(res))
    if rc == _lib.VINE_ERR_CAPACITY and paths and r.path_offsets[nq] > res.path_capacity:
        # path buffer too small: grow it to the size the library reported, retry once
        return solve(graph, src, dst, budget, config, paths, pareto_stride, stats,
                     path_capacity=int(r.path_offsets[nq]), raise_on_error=raise_on_error)
    r.rc = rc
    r.retried = int(res.retried)
    if raise_on_error:
        check(rc)
    return r


def solve_multi(graphs: Sequence[Graph], src, dst, budget, config=None, paths: bool = True,
                stats: bool = False, raise_on_error: bool = True) -> Results:
    """One batch split over several graph handles (one per device) by
    vine_solve_multi; results in query order."""
    src = np.ascontiguousarray(src, dtype=np.int32)
    dst = np.ascontiguousarray(dst, dtype=np.int32)
    budget = np.ascontiguousarray(budget, dtype=np.float32)
    nq = int(src.shape[0])
    r = Results(cost=np.empty(nq, np.float32), delay=np.empty(nq, np.float32),
                found=np.empty(nq, np.int32), status=np.zeros(nq, np.int32))
    res = _lib.vine_results()
    res.cost, res.delay = _ptr(r.cost), _ptr(r.delay)
    res.found, res.status = _ptr(r.found), _ptr(r.status)
    if paths:
        cap = max(1024, nq * 4096)
        r.path_offsets = np.zeros(nq + 1, np.int64)
        r.path_vertices = np.zeros(cap, np.int32)
        res.path_offsets, res.path, res.path_capacity = _ptr(r.path_offsets), _ptr(r.path_vertices), cap
    if stats:
        r.stats = np.zeros((nq, _lib.STAT_COUNT), np.int64)
        res.stats = _ptr(r.stats)
    handles = (C.c_void_p * len(graphs))(*[gr.handle.value for gr in graphs])
    cfg = config if config is not None else Config()
    rc = lib.vine_solve_multi(handles, len(graphs), nq, _ptr(src), _ptr(dst), _ptr(budget),
                              C.byref(cfg), C.byref(res))
    r.rc = rc
    r.retried = int(res.retried)
    if raise_on_error:
        check(rc)
    return r


LABEL_KINDS = {"csp": _lib.LABEL_CSP, "hop": _lib.LABEL_HOP, "maxcost": _lib.LABEL_MAXCOST,
               "qos": _lib.LABEL_QOS}


def solve_labels(graph: Graph, kind, src, dst, delay_limit, hop_limit=None, maxcost_limit=None,
                 config=None, paths: bool = True, stats: bool = False,
                 raise_on_error: bool = True) -> Results:
    """Label-variant queries on the GPU (vine_solve_labels): kind "csp",
    "hop", "maxcost" or "qos" (the reference's CSP=1/4, 2, 3 and QoS labels).
    Results carry cost (d), delay (QoS: bandwidth) and `extra` [nq, 2] (hop
    count, maxcost) of the best feasible sink label."""
    k = LABEL_KINDS[kind] if isinstance(kind, str) else int(kind)
    src = np.ascontiguousarray(src, dtype=np.int32)
    dst = np.ascontiguousarray(dst, dtype=np.int32)
    nq = int(src.shape[0])
    dL = np.ascontiguousarray(delay_limit, dtype=np.float32)
    hL = None if hop_limit is None else np.ascontiguousarray(hop_limit, dtype=np.float32)
    mL = None if maxcost_limit is None else np.ascontiguousarray(maxcost_limit, dtype=np.float32)
    r = Results(cost=np.empty(nq, np.float32), delay=np.empty(nq, np.float32),
                found=np.empty(nq, np.int32), status=np.zeros(nq, np.int32))
    r.extra = np.zeros((nq, 2), np.float32)
    res = _lib.vine_results()
    res.cost, res.delay = _ptr(r.cost), _ptr(r.delay)
    res.found, res.status = _ptr(r.found), _ptr(r.status)
    if paths:
        cap = max(1024, nq * 4096)
        r.path_offsets = np.zeros(nq + 1, np.int64)
        r.path_vertices = np.zeros(cap, np.int32)
        res.path_offsets, res.path, res.path_capacity = _ptr(r.path_offsets), _ptr(r.path_vertices), cap
    if stats:
        r.stats = np.zeros((nq, _lib.STAT_COUNT), np.int64)
        res.stats = _ptr(r.stats)
    cfg = config if config is not None else Config()
    rc = lib.vine_solve_labels(graph.handle, k, nq, _ptr(src), _ptr(dst), _ptr(dL), _ptr(hL),
                               _ptr(mL), C.byref(cfg), C.byref(res), _ptr(r.extra))
    r.rc = rc
    if raise_on_error:
        check(rc)
    return r


def solve_host(graph: Graph, src, dst, budget, nthreads: int = 0, across_queries: bool = False,
               paths: bool = True, pareto_stride: int = 0, raise_on_error: bool = True) -> Results:
    """The race-free multi-core CPU engine (vine_solve_host) on the graph's
    host arrays: an explicitly chosen CPU solver, never a fallback of the GPU
    entry points."""
    src = np.ascontiguousarray(src, dtype=np.int32)
    dst = np.ascontiguousarray(dst, dtype=np.int32)
    budget = np.ascontiguousarray(budget, dtype=np.float32)
    nq = int(src.shape[0])
    r = Results(cost=np.empty(nq, np.float32), delay=np.empty(nq, np.float32),
                found=np.empty(nq, np.int32), status=np.zeros(nq, np.int32))
    res = _lib.vine_results()
    res.cost, res.delay = _ptr(r.cost), _ptr(r.delay)
    res.found, res.status = _ptr(r.found), _ptr(r.status)
    cap = max(1024, nq * 4096)
    if paths:
        r.path_offsets = np.zeros(nq + 1, np.int64)
        r.path_vertices = np.zeros(cap, np.int32)
        res.path_offsets, res.path, res.path_capacity = _ptr(r.path_offsets), _ptr(r.path_vertices), cap
    if pareto_stride > 0:
        r.pareto_d = np.zeros((nq, pareto_stride), np.float32)
        r.pareto_delay = np.zeros((nq, pareto_stride), np.float32)
        r.pareto_n = np.zeros(nq, np.int32)
        res.pareto_d, res.pareto_delay = _ptr(r.pareto_d), _ptr(r.pareto_delay)
        res.pareto_n, res.pareto_stride = _ptr(r.pareto_n), pareto_stride
    rc = lib.vine_solve_host(graph.N, graph.M, _ptr(graph.row_ptr), _ptr(graph.col),
                             _ptr(graph.len), _ptr(graph.delay), nq, _ptr(src), _ptr(dst),
                             _ptr(budget), nthreads, int(across_queries), C.byref(res))
    r.rc = rc
    if raise_on_error:
        check(rc)
    return r


def solve_device(graph: Graph, src, dst, budget, out: dict, config=None, stream=None) -> None:
    """Device-resident solve: src/dst/budget and out[...] are CUDA tensors
    (torch) already in HBM; enqueues on `stream` and returns immediately."""
    cfg = config if config is not None else Config()
    res = _lib.vine_results()
    res.cost = out["cost"].data_ptr()
    res.delay = out["delay"].data_ptr()
    res.found = out["found"].data_ptr()
    res.status = out["status"].data_ptr()
    if "stats" in out:
        res.stats = out["stats"].data_ptr()
    if "path_offsets" in out:
        res.path_offsets = out["path_offsets"].data_ptr()
        res.path = out["path"].data_ptr()
        res.path_capacity = out["path"].numel()
    check(lib.vine_solve_device(graph.handle, int(src.numel()), src.data_ptr(), dst.data_ptr(),
                                budget.data_ptr(), C.byref(cfg), C.byref(res),
                                C.c_void_p(stream) if stream else None))


class cspp:
    """Query class with the reference's constructor and method names
    (algorithm/cspp.hpp:11-69).  solve() runs the B200 engine and fills
    path_l / size_of_result_l (per task) plus cost_l / delay_l / found_l."""

    def __init__(self, g: Graph, ntask: int, source_state: Sequence[c_label],
                 sink_l: Sequence[int], C_l: Sequence[c_constraint], config=None):
        if not (len(source_state) >= ntask and len(sink_l) >= ntask and len(C_l) >= ntask):
            raise ValueError("need ntask source labels, sinks and constraints")
        self.g = g
        self.ntask = ntask
        self.init_state = list(source_state[:ntask])
        self.sink_l = list(sink_l[:ntask])
        self.C_l = list(C_l[:ntask])
        self.config = config
        self.path_l: list = []
        self.size_of_result_l: list = []
        self.cost_l = None
        self.delay_l = None
        self.found_l = None
        self.status_l = None

    def solve(self) -> int:
        for l in self.init_state:
            if l.d != 0 or l.delay != 0:
                raise ValueError("source labels must start at d = delay = 0")
        src = np.array([l.vid for l in self.init_state], np.int32)
        dst = np.array(self.sink_l, np.int32)
        bud = np.array([c.delay_L for c in self.C_l], np.float32)
        r = solve(self.g, src, dst, bud, self.config)
        self.cost_l, self.delay_l, self.found_l, self.status_l = r.cost, r.delay, r.found, r.status
        self.path_l = [r.path(q).copy() for q in range(self.ntask)]
        self.size_of_result_l = [len(p) for p in self.path_l]
        return 0

    def _solve_host(self, nthreads: int) -> int:
        src = np.array([l.vid for l in self.init_state], np.int32)
        dst = np.array(self.sink_l, np.int32)
        bud = np.array([c.delay_L for c in self.C_l], np.float32)
        r = solve_host(self.g, src, dst, bud, nthreads=nthreads)
        self.cost_l, self.delay_l, self.found_l, self.status_l = r.cost, r.delay, r.found, r.status
        self.path_l = [r.path(q).copy() for q in range(self.ntask)]
        self.size_of_result_l = [len(p) for p in self.path_l]
        return 0

    def solve_cpu(self) -> int:
        """algorithm/cspp.hpp:55-57: the host engine on one thread."""
        return self._solve_host(1)

    def solve_omp(self) -> int:
        """algorithm/cspp.hpp:59-61: the race-free multi-core host engine."""
        return self._solve_host(0)


# ------------------------------------------------------------------------ MLP


class MLP:
    """The 16-64-64-2 FP32 bucket scheduler, trained by libvine's kernels."""

    def __init__(self, device: int = 0, seed: int = 0, params: Optional[np.ndarray] = None):
        h = C.c_void_p()
        p = None if params is None else np.ascontiguousarray(params, np.float32)
        if p is not None and p.size != _lib.MLP_PARAMS:
            raise ValueError("wrong parameter count")
        check(lib.vine_mlp_create(device, seed, _ptr(p), C.byref(h)))
        self.handle = h

    @property
    def params(self) -> np.ndarray:
        out = np.empty(_lib.MLP_PARAMS, np.float32)
        check(lib.vine_mlp_get_params(self.handle, _ptr(out)))
        return out

    @params.setter
    def params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        check(lib.vine_mlp_set_params(self.handle, _ptr(p)))

    def forward(self, x) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float32).reshape(-1, _lib.MLP_IN)
        y = np.empty((x.shape[0], _lib.MLP_OUT), np.float32)
        check(lib.vine_mlp_forward(self.handle, x.shape[0], _ptr(x), _ptr(y)))
        return y

    def loss_grad(self, x, y):
        x = np.ascontiguousarray(x, np.float32).reshape(-1, _lib.MLP_IN)
        y = np.ascontiguousarray(y, np.float32).reshape(-1, _lib.MLP_OUT)
        loss = np.zeros(1, np.float32)
        grad = np.empty(_lib.MLP_PARAMS, np.float32)
        check(lib.vine_mlp_loss_grad(self.handle, x.shape[0], _ptr(x), _ptr(y), _ptr(loss),
                                     _ptr(grad)))
        return float(loss[0]), grad

    def train(self, x, y, epochs=50, batch=256, lr=1e-3, seed=0) -> float:
        x = np.ascontiguousarray(x, np.float32).reshape(-1, _lib.MLP_IN)
        y = np.ascontiguousarray(y, np.float32).reshape(-1, _lib.MLP_OUT)
        fl = C.c_float()
        check(lib.vine_mlp_train(self.handle, x.shape[0], _ptr(x), _ptr(y), epochs, batch, lr,
                                 seed, C.byref(fl)))
        return fl.value

    def close(self):
        if self.handle is not None:
            lib.vine_mlp_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def fetch_trace(graph: Graph) -> np.ndarray:
    rows = C.c_int64()
    check(lib.vine_trace_fetch(graph.handle, C.byref(rows), None, 0))
    buf = np.empty((rows.value, _lib.TRACE_COLS), np.float32)
    if rows.value:
        check(lib.vine_trace_fetch(graph.handle, C.byref(rows), _ptr(buf), rows.value))
    return buf


def autotune(graph: Graph, src, dst, budget, base=None, cache_path: Optional[str] = None):
    src = np.ascontiguousarray(src, np.int32)
    dst = np.ascontiguousarray(dst, np.int32)
    budget = np.ascontiguousarray(budget, np.float32)
    best = _lib.vine_config()
    b = base if base is not None else Config()
    check(lib.vine_autotune(graph.handle, src.shape[0], _ptr(src), _ptr(dst), _ptr(budget),
                            C.byref(b), cache_path.encode() if cache_path else None,
                            C.byref(best)))
    if getattr(b, "_mlp_ref", None) is not None:
        best._mlp_ref = b._mlp_ref
    return best


# ------------------------------------------------------------------- workloads


class Workload:
    """Seeded synthetic workloads (configs 1..5) and file loaders."""

    def __init__(self, handle):
        self._h = handle
        n, m = C.c_int32(), C.c_int64()
        rp, cp, lp, dp = C.c_void_p(), C.c_void_p(), C.c_void_p(), C.c_void_p()
        check(lib.vine_workload_graph(handle, C.byref(n), C.byref(m), C.byref(rp), C.byref(cp),
                                      C.byref(lp), C.byref(dp)))
        self.n, self.m = n.value, m.value

        def view(p, count, ct, dt):
            if count == 0 or not p.value:
                return np.zeros(0, dt)
            arr = np.ctypeslib.as_array(C.cast(p, C.POINTER(ct)), shape=(count,))
            return arr.astype(dt, copy=True)

        self.row_ptr = view(rp, self.n + 1, C.c_int64, np.int64)
        self.col = view(cp, self.m, C.c_int32, np.int32)
        self.len = view(lp, self.m, C.c_float, np.float32)
        self.delay = view(dp, self.m, C.c_float, np.float32)
        nq = C.c_int32()
        sp, tp, bp, ap = C.c_void_p(), C.c_void_p(), C.c_void_p(), C.c_void_p()
        check(lib.vine_workload_queries(handle, C.byref(nq), C.byref(sp), C.byref(tp),
                                        C.byref(bp), C.byref(ap)))
        self.nq = nq.value
        self.src = view(sp, self.nq, C.c_int32, np.int32)
        self.dst = view(tp, self.nq, C.c_int32, np.int32)
        self.budget = view(bp, self.nq, C.c_float, np.float32)
        self.alpha = view(ap, self.nq, C.c_float, np.float32)
        lib.vine_workload_destroy(handle)
        self._h = None

    @staticmethod
    def params(config_id: int) -> _lib.vine_workload_params:
        p = _lib.vine_workload_params()
        check(lib.vine_workload_default_params(config_id, C.byref(p)))
        return p

    @classmethod
    def generate(cls, config_id: int = 1, **overrides) -> "Workload":
        p = cls.params(config_id)
        for k, v in overrides.items():
            if k == "alpha":
                for i, a in enumerate(v):
                    p.alpha[i] = a
                p.n_alpha = len(v)
                continue
            setattr(p, k, v)
        h = C.c_void_p()
        check(lib.vine_workload_generate(C.byref(p), C.byref(h)))
        return cls(h)

    @classmethod
    def load_mtx(cls, path: str, n_pairs: int = 0, alpha=(0.5,), seed: int = 1) -> "Workload":
        """5-column edge list; optionally adds n_pairs random queries."""
        h = C.c_void_p()
        check(lib.vine_workload_load_mtx(path.encode(), C.byref(h)))
        if n_pairs > 0:
            a = np.ascontiguousarray(alpha, np.float32)
            rc = lib.vine_workload_add_random_queries(h, seed, n_pairs, a.size, _ptr(a))
            if rc != 0:
                lib.vine_workload_destroy(h)
                check(rc)
        return cls(h)

    @classmethod
    def load_cola(cls, graph_path: str, query_path: Optional[str] = None) -> "Workload":
        h = C.c_void_p()
        check(lib.vine_workload_load_cola(graph_path.encode(),
                                          query_path.encode() if query_path else None,
                                          C.byref(h)))
        return cls(h)

    def graph(self, device: int = 0) -> Graph:
        return Graph(self.row_ptr, self.col, self.len, self.delay, device)
