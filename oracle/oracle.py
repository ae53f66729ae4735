"""CPU oracle bindings -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
reference legs may import this module.  It is the checker, never the product:
nothing in vine_b200 imports it.

* liboracle.so (oracle/cspp_oracle.cpp): restatement of the reference CPU
  solver RUN_CSPP_CPU (algorithm/cspp_cpu.hpp:44-125) that returns the sink
  Pareto set, cost, delay, path and work counters; a label-setting search
  under the GPU engine's pruning rules; lexicographic Dijkstra.
* libvine_ref.so (oracle/ref_oracle.cpp): the reference's own
  RUN_CSPP_CPU template compiled from the reference sources, with an
  additive label type (the shipped host expand multiplies).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "_build" / "liboracle.so"
REF_SO = HERE / "_ref" / "libvine_ref.so"


# Where the reference sources are read from when building libvine_ref.so
# (VINE_REF_TREE overrides); machines without the tree use the prebuilt file.
REF_TREE = os.environ.get("VINE_REF_TREE", "/root/reference")


def build(ref_tree: str | None = None) -> None:
    """Builds liboracle.so, and libvine_ref.so when the reference tree exists."""
    tree = ref_tree or REF_TREE
    subprocess.run(["make", "-s", "-C", str(HERE), f"REF={tree}"], check=True)


class Result(C.Structure):
    _fields_ = [("cost", C.c_float), ("delay", C.c_float), ("found", C.c_int32),
                ("path_len", C.c_int32), ("pareto_n", C.c_int32), ("pad", C.c_int32),
                ("P", C.c_int64), ("R", C.c_int64), ("S", C.c_int64), ("I", C.c_int64),
                ("dom_calls", C.c_int64), ("rounds", C.c_int64)]


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


_oracle = None
_ref = None


def _lib_oracle():
    global _oracle
    if _oracle is None:
        if not ORACLE_SO.exists():
            build()
        lib = C.CDLL(str(ORACLE_SO))
        vp = C.c_void_p
        lib.oracle_solve_reference_rules.argtypes = [C.c_int32, vp, vp, vp, vp, C.c_int32,
                                                     C.c_int32, C.c_float, vp, C.c_int32, vp, vp,
                                                     C.c_int32, C.POINTER(Result)]
        lib.oracle_solve_label_setting.argtypes = [C.c_int32, vp, vp, vp, vp, C.c_int32,
                                                   C.c_int32, C.c_float, vp, vp, C.c_int32, vp,
                                                   C.c_int32, vp, vp, C.c_int32, C.POINTER(Result)]
        lib.oracle_dijkstra.argtypes = [C.c_int32, vp, vp, vp, vp, C.c_int32, vp, vp, vp]
        lib.oracle_set_time_limit.argtypes = [C.c_double]
        lib.oracle_set_time_limit.restype = None
        _oracle = lib
    return _oracle


def ref_available() -> bool:
    return REF_SO.exists()


def _lib_ref():
    global _ref
    if _ref is None:
        if not REF_SO.exists():
            raise FileNotFoundError(f"{REF_SO} missing: build it with `make -C oracle`")
        lib = C.CDLL(str(REF_SO))
        vp = C.c_void_p
        lib.ref_graph_create.restype = vp
        lib.ref_graph_create.argtypes = [C.c_int32, vp, vp, vp, vp]
        lib.ref_graph_destroy.argtypes = [vp]
        lib.ref_solve.argtypes = [vp, C.c_int32, vp, vp, vp, C.c_int32, C.c_int32, vp, vp, vp,
                                  vp, C.c_int32, vp, vp]
        lib.ref_solve_capped.argtypes = [vp, C.c_int32, vp, vp, vp, C.c_int32, C.c_double, vp,
                                         vp, vp, vp, vp]
        lib.ref_last_error.restype = C.c_char_p
        lib.ref_solve_variant.argtypes = [vp, C.c_int32, C.c_int32, vp, vp, vp, vp, vp, C.c_int32,
                                          C.c_double, vp, vp, vp, vp, C.c_int32, vp, vp]
        lib.vine_workload_default_params.argtypes = [C.c_int32, vp]
        lib.vine_workload_generate.argtypes = [vp, C.POINTER(vp)]
        lib.vine_workload_graph.argtypes = [vp] + [vp] * 6
        lib.vine_workload_queries.argtypes = [vp] + [vp] * 5
        lib.vine_workload_destroy.argtypes = [vp]
        lib.vine_workload_destroy.restype = None
        _ref = lib
    return _ref


class CsrGraph:
    """Host CSR arrays (int64 row_ptr, int32 col, float32 len / delay)."""

    def __init__(self, row_ptr, col, length, delay):
        self.row_ptr = np.ascontiguousarray(row_ptr, np.int64)
        self.col = np.ascontiguousarray(col, np.int32)
        self.len = np.ascontiguousarray(length, np.float32)
        self.delay = np.ascontiguousarray(delay, np.float32)
        self.n = int(self.row_ptr.shape[0] - 1)

    def reverse(self) -> "CsrGraph":
        n = self.n
        src = np.repeat(np.arange(n, dtype=np.int32), np.diff(self.row_ptr))
        order = np.argsort(self.col, kind="stable")
        counts = np.bincount(self.col, minlength=n)
        rp = np.zeros(n + 1, np.int64)
        np.cumsum(counts, out=rp[1:])
        return CsrGraph(rp, src[order], self.len[order], self.delay[order])


def solve_reference_rules(g: CsrGraph, src: int, dst: int, budget: float, path_cap=None,
                          pareto_cap: int = 4096):
    """Restated RUN_CSPP_CPU: returns dict(cost, delay, found, path, pareto, counters)."""
    lib = _lib_oracle()
    cap = path_cap or g.n + 1
    path = np.zeros(cap, np.int32)
    pd = np.zeros(pareto_cap, np.float32)
    pl = np.zeros(pareto_cap, np.float32)
    r = Result()
    rc = lib.oracle_solve_reference_rules(g.n, _p(g.row_ptr), _p(g.col), _p(g.len), _p(g.delay),
                                          src, dst, budget, _p(path), cap, _p(pd), _p(pl),
                                          pareto_cap, C.byref(r))
    if rc != 0:
        raise RuntimeError("oracle buffer too small")
    return _pack(r, path, pd, pl)


def solve_label_setting(g: CsrGraph, src: int, dst: int, budget: float, h_len=None, h_del=None,
                        use_incumbent: bool = True, path_cap=None, pareto_cap: int = 4096,
                        time_limit: float = 0.0):
    """Label setting under the engine's pruning rules (minimal work counts).
    With time_limit > 0 a search that runs longer returns None."""
    lib = _lib_oracle()
    lib.oracle_set_time_limit(float(time_limit))
    cap = path_cap or g.n + 1
    path = np.zeros(cap, np.int32)
    pd = np.zeros(pareto_cap, np.float32)
    pl = np.zeros(pareto_cap, np.float32)
    hl = None if h_len is None else np.ascontiguousarray(h_len, np.float32)
    hd = None if h_del is None else np.ascontiguousarray(h_del, np.float32)
    r = Result()
    rc = lib.oracle_solve_label_setting(g.n, _p(g.row_ptr), _p(g.col), _p(g.len), _p(g.delay),
                                        src, dst, budget, _p(hl), _p(hd), int(use_incumbent),
                                        _p(path), cap, _p(pd), _p(pl), pareto_cap, C.byref(r))
    lib.oracle_set_time_limit(0.0)
    if rc == 2:
        return None
    if rc != 0:
        raise RuntimeError("oracle buffer too small")
    return _pack(r, path, pd, pl)


def _pack(r: Result, path, pd, pl):
    n = min(r.pareto_n, pd.shape[0])
    return {
        "cost": np.float32(r.cost), "delay": np.float32(r.delay), "found": bool(r.found),
        "path": path[: r.path_len].copy(),
        "pareto": np.stack([pd[:n], pl[:n]], axis=1),
        "P": r.P, "R": r.R, "S": r.S, "I": r.I, "dom_calls": r.dom_calls, "rounds": r.rounds,
    }


def dijkstra(g: CsrGraph, src: int, primary: str = "len"):
    """Lexicographic Dijkstra; returns (dist_primary, dist_secondary, parent)."""
    lib = _lib_oracle()
    w1, w2 = (g.len, g.delay) if primary == "len" else (g.delay, g.len)
    d1 = np.empty(g.n, np.float32)
    d2 = np.empty(g.n, np.float32)
    par = np.empty(g.n, np.int32)
    lib.oracle_dijkstra(g.n, _p(g.row_ptr), _p(g.col), _p(w1), _p(w2), src, _p(d1), _p(d2),
                        _p(par))
    return d1, d2, par


def lower_bounds(g: CsrGraph, dst: int):
    """Exact lower bounds on the remaining cost and delay to dst (reverse SSSP)."""
    rg = g.reverse()
    h_len, _, _ = dijkstra(rg, dst, "len")
    h_del, _, _ = dijkstra(rg, dst, "delay")
    return h_len, h_del


class RefSolver:
    """The reference's own RUN_CSPP_CPU (compiled from its sources)."""

    def __init__(self, g: CsrGraph):
        self.lib = _lib_ref()
        self.g = g
        self.h = self.lib.ref_graph_create(g.n, _p(g.row_ptr), _p(g.col), _p(g.len), _p(g.delay))

    def solve(self, src, dst, budget, nthreads: int = 1, record_paths: bool = False,
              path_stride: int = 0):
        src = np.ascontiguousarray(src, np.int32)
        dst = np.ascontiguousarray(dst, np.int32)
        budget = np.ascontiguousarray(budget, np.float32)
        nq = src.shape[0]
        cost = np.empty(nq, np.float32)
        delay = np.empty(nq, np.float32)
        found = np.empty(nq, np.int32)
        calls = np.zeros((nq, 2), np.int64)
        stride = path_stride or (self.g.n + 1 if record_paths else 0)
        paths = np.zeros((nq, stride), np.int32) if record_paths else None
        plen = np.zeros(nq, np.int32) if record_paths else None
        self.lib.ref_solve(self.h, nq, _p(src), _p(dst), _p(budget), nthreads, int(record_paths),
                           _p(cost), _p(delay), _p(found), _p(paths), stride, _p(plen),
                           _p(calls))
        out = {"cost": cost, "delay": delay, "found": found.astype(bool), "calls": calls}
        if record_paths:
            out["paths"] = [paths[q, : plen[q]].copy() for q in range(nq)]
        return out

    def solve_capped(self, src, dst, budget, nthreads: int, cap_seconds: float):
        """Per-query wall times with a cap: returns seconds[q] (<= ~cap),
        finished[q], and cost / delay / found of the finished queries."""
        src = np.ascontiguousarray(src, np.int32)
        dst = np.ascontiguousarray(dst, np.int32)
        budget = np.ascontiguousarray(budget, np.float32)
        nq = src.shape[0]
        cost = np.empty(nq, np.float32)
        delay = np.empty(nq, np.float32)
        found = np.zeros(nq, np.int32)
        secs = np.zeros(nq, np.float64)
        fin = np.zeros(nq, np.int32)
        rc = self.lib.ref_solve_capped(self.h, nq, _p(src), _p(dst), _p(budget), nthreads,
                                       float(cap_seconds), _p(cost), _p(delay), _p(found),
                                       _p(secs), _p(fin))
        if rc != 0:
            raise RuntimeError("ref_solve_capped failed")
        return {"seconds": secs, "finished": fin.astype(bool), "cost": cost, "delay": delay,
                "found": found.astype(bool)}

    def solve_variant(self, kind: int, src, dst, delay_L, hop_L=None, max_L=None,
                      nthreads: int = 1, cap_seconds: float = 0.0, record_paths: bool = False):
        """A label variant through the reference's RUN_CSPP_CPU: kind 2
        hop-constrained, 3 max-cost, 6 QoS bottleneck.  Returns best[q] =
        (d, delay, hop, maxcost) (QoS: (d, bandwidth, 0, 0)), found,
        finished (False when stopped at cap_seconds), paths."""
        src = np.ascontiguousarray(src, np.int32)
        dst = np.ascontiguousarray(dst, np.int32)
        nq = src.shape[0]
        dL = np.ascontiguousarray(delay_L, np.float32)
        hL = np.ascontiguousarray(hop_L if hop_L is not None else np.full(nq, 100), np.int32)
        mL = np.ascontiguousarray(max_L if max_L is not None else np.full(nq, 10000), np.float32)
        best = np.zeros((nq, 4), np.float32)
        found = np.zeros(nq, np.int32)
        fin = np.zeros(nq, np.int32)
        stride = self.g.n + 1 if record_paths else 0
        paths = np.zeros((nq, stride), np.int32) if record_paths else None
        plen = np.zeros(nq, np.int32) if record_paths else None
        calls = np.zeros(nq, np.int64)
        rc = self.lib.ref_solve_variant(self.h, kind, nq, _p(src), _p(dst), _p(dL), _p(hL), _p(mL),
                                        nthreads, float(cap_seconds), _p(best), _p(found), _p(fin),
                                        _p(paths), stride, _p(plen), _p(calls))
        if rc != 0:
            raise ValueError("ref_solve_variant failed")
        out = {"best": best, "found": found.astype(bool), "finished": fin.astype(bool),
               "calls": calls}
        if record_paths:
            out["paths"] = [paths[q, : plen[q]].copy() for q in range(nq)]
        return out

    def close(self):
        if self.h:
            self.lib.ref_graph_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _WorkloadParams(C.Structure):
    """Layout of vine_workload_params (include/vine_workloads.h)."""
    _fields_ = [
        ("kind", C.c_int32), ("seed", C.c_uint64), ("rows", C.c_int32), ("cols", C.c_int32),
        ("n", C.c_int64), ("m_target", C.c_int64), ("exponent", C.c_double),
        ("n_pairs", C.c_int32), ("n_alpha", C.c_int32), ("alpha", C.c_float * 4),
        ("alpha_lo", C.c_float), ("alpha_hi", C.c_float), ("hop_lo", C.c_int32),
        ("hop_hi", C.c_int32), ("hop_log_uniform", C.c_int32), ("nthreads", C.c_int32),
        ("query_seed", C.c_uint64),
    ]


class HostWorkload:
    """A seeded workload built by the generator copy inside libvine_ref.so, so
    that CPU-only timing of the reference never loads the GPU engine's
    library.  Same fields as vine_b200.Workload (row_ptr, col, len, delay,
    src, dst, budget, alpha, n, m, nq); identical arrays for the same
    parameters (checked by the tests)."""

    def __init__(self, config_id: int = 1, **overrides):
        lib = _lib_ref()
        vp = C.c_void_p
        p = _WorkloadParams()
        if lib.vine_workload_default_params(config_id, C.byref(p)) != 0:
            raise ValueError(f"bad config_id {config_id}")
        for k, v in overrides.items():
            if k == "alpha":
                for i, a in enumerate(v):
                    p.alpha[i] = a
                p.n_alpha = len(v)
            else:
                setattr(p, k, v)
        h = vp()
        rc = lib.vine_workload_generate(C.byref(p), C.byref(h))
        if rc != 0:
            raise RuntimeError(f"generator failed ({rc}): {lib.ref_last_error().decode()}")
        try:
            n, m = C.c_int32(), C.c_int64()
            rp, cp, lp, dp = vp(), vp(), vp(), vp()
            lib.vine_workload_graph(h, C.byref(n), C.byref(m), C.byref(rp), C.byref(cp),
                                    C.byref(lp), C.byref(dp))
            self.n, self.m = n.value, m.value

            def view(ptr, count, ct, dt):
                if count == 0 or not ptr.value:
                    return np.zeros(0, dt)
                return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(ct)), shape=(count,)).astype(dt)

            self.row_ptr = view(rp, self.n + 1, C.c_int64, np.int64)
            self.col = view(cp, self.m, C.c_int32, np.int32)
            self.len = view(lp, self.m, C.c_float, np.float32)
            self.delay = view(dp, self.m, C.c_float, np.float32)
            nq = C.c_int32()
            sp, tp, bp, ap = vp(), vp(), vp(), vp()
            lib.vine_workload_queries(h, C.byref(nq), C.byref(sp), C.byref(tp), C.byref(bp),
                                      C.byref(ap))
            self.nq = nq.value
            self.src = view(sp, self.nq, C.c_int32, np.int32)
            self.dst = view(tp, self.nq, C.c_int32, np.int32)
            self.budget = view(bp, self.nq, C.c_float, np.float32)
            self.alpha = view(ap, self.nq, C.c_float, np.float32)
        finally:
            lib.vine_workload_destroy(h)


def bytes_per_query(counters: dict) -> int:
    """Algorithmic bytes of one query: 20 P + 12 R + 8 S + 24 I.

    P labels expanded (12-byte label + 8-byte row pointers), R arcs relaxed
    (4-byte head + 8-byte weights), S stored labels read by dominance tests
    (8 bytes), I labels inserted (12 bytes to the store + 12 to the frontier)."""
    return 20 * counters["P"] + 12 * counters["R"] + 8 * counters["S"] + 24 * counters["I"]


def cpu_count() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1
