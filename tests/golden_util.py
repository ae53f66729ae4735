"""Helpers shared by the tests: golden fixtures, path checks."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"
FIXTURES = ["kat3", "diamond", "line", "cycle", "grid", "road_small", "road_anticorr_small",
            "chunglu_small", "road_batch_small"]


def load_fixture(name: str) -> dict:
    """Fixture dict plus CSR arrays (rebuilt from the generator when needed)."""
    fx = json.loads((GOLDEN / f"{name}.json").read_text())
    if fx.get("graph") is not None:
        g = fx["graph"]
        fx["row_ptr"] = np.array(g["row_ptr"], np.int64)
        fx["col"] = np.array(g["col"], np.int32)
        fx["len"] = np.array(g["len"], np.float32)
        fx["delay"] = np.array(g["delay"], np.float32)
    else:
        import vine_b200 as v
        gen = fx["generator"]
        w = v.Workload.generate(gen["config_id"], **gen["overrides"])
        fx["row_ptr"], fx["col"], fx["len"], fx["delay"] = w.row_ptr, w.col, w.len, w.delay
    q = fx["queries"]
    fx["src"] = np.array([x["src"] for x in q], np.int32)
    fx["dst"] = np.array([x["dst"] for x in q], np.int32)
    fx["budget"] = np.array([x["budget"] for x in q], np.float32)
    return fx


def csr_digest(row_ptr, col, length, delay) -> str:
    import hashlib
    h = hashlib.sha256()
    for a, dt in ((row_ptr, np.int64), (col, np.int32), (length, np.float32), (delay, np.float32)):
        h.update(np.ascontiguousarray(a, dt).tobytes())
    return h.hexdigest()


def path_sums(row_ptr, col, length, delay, path):
    """Left-to-right FP32 sums of (len, delay) along a vertex path; the arc
    between consecutive vertices must exist (graphs here have no parallel
    arcs).  Returns None when an arc is missing."""
    d = np.float32(0.0)
    dl = np.float32(0.0)
    for u, v in zip(path[:-1], path[1:]):
        a, b = row_ptr[u], row_ptr[u + 1]
        hits = np.nonzero(col[a:b] == v)[0]
        if hits.size == 0:
            return None
        j = a + hits[0]
        d = np.float32(d + length[j])
        dl = np.float32(dl + delay[j])
    return float(d), float(dl)


def check_result(fx, res, q, expect, mode="optimal"):
    """Asserts one query's engine result against an expected record."""
    assert res.status[q] == 0, f"q{q}: status {res.status[q]}"
    if not expect["found"]:
        assert res.found[q] == 0, f"q{q}: found a path where the reference has none"
        return
    assert res.found[q] == 1, f"q{q}: no path, reference has cost {expect['cost']}"
    assert float(res.cost[q]) == expect["cost"], f"q{q}: cost {res.cost[q]} != {expect['cost']}"
    assert float(res.delay[q]) == expect["delay"], f"q{q}: delay {res.delay[q]} != {expect['delay']}"
    if res.path_offsets is not None:
        p = res.path(q)
        assert p[0] == fx["src"][q] and p[-1] == fx["dst"][q], f"q{q}: path endpoints"
        sums = path_sums(fx["row_ptr"], fx["col"], fx["len"], fx["delay"], p)
        assert sums is not None, f"q{q}: path uses a missing arc"
        assert sums == (expect["cost"], expect["delay"]), f"q{q}: path sums {sums}"
        assert sums[1] <= fx["budget"][q], f"q{q}: path violates the budget"


SCALE_CASES = ["tech_routers_rf", "tech_internet_as", "c4_chunglu100k", "c5_sample256",
               "c2_road264k", "c3_road1500k"]


def scale_fixture_path(name: str) -> Path:
    return GOLDEN / f"scale_{name}.json"


def load_scale(name: str, with_graph: bool = True) -> dict:
    """A full-size fixture (tests/golden/make_scale_golden.py) plus its CSR
    arrays and query arrays."""
    fx = json.loads(scale_fixture_path(name).read_text())
    if with_graph:
        if "graph_file" in fx:
            z = np.load(GOLDEN / fx["graph_file"])
            fx["row_ptr"] = z["row_ptr"].astype(np.int64)
            fx["col"] = z["col"].astype(np.int32)
            fx["len"] = z["len"].astype(np.float32)
            fx["delay"] = z["delay"].astype(np.float32)
        else:
            import vine_b200 as v
            gen = fx["generator"]
            w = v.Workload.generate(gen["config_id"], **gen["overrides"])
            fx["row_ptr"], fx["col"], fx["len"], fx["delay"] = w.row_ptr, w.col, w.len, w.delay
    q = fx["queries"]
    fx["src"] = np.array([x["src"] for x in q], np.int32)
    fx["dst"] = np.array([x["dst"] for x in q], np.int32)
    fx["budget"] = np.array([x["budget"] for x in q], np.float32)
    return fx

