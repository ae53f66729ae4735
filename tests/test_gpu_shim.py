"""GPU tests of the C++ drop-in header (include/vine/cspp.hpp): callers
written the way the reference drives its query path, compiled against the
header and run on the device."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

import cpp_callers as cc
from golden_util import check_result, load_fixture, path_sums

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]


def test_cpp_shim_known_answers(tmp_path):
    exe = cc.build("shim_main", tmp_path)
    res = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert res.returncode == 0, res.stdout + res.stderr
    assert res.stdout.startswith("OK")


def _check_caller_output(out, fx, expected):
    assert out["rc"] == 0
    for q, e in enumerate(expected):
        r = out[q]
        assert r["found"] == e["found"], f"task {q}: found"
        if not e["found"]:
            assert r["path"].size == 0
            continue
        assert (r["cost"], r["delay"]) == (e["cost"], e["delay"]), f"task {q}: cost/delay"
        p = r["path"]
        assert p[0] == fx["src"][q] and p[-1] == fx["dst"][q]
        assert path_sums(fx["row_ptr"], fx["col"], fx["len"], fx["delay"], p) == (e["cost"], e["delay"])


def test_reference_caller_on_a_cola_graph(tmp_path):
    """tests/cpp/ref_main.cpp repeats the reference's main.cu sequence
    (config -> read_graph (COLA) -> load_query -> adj_to_csr -> el ->
    make_gpu_graph -> cspp -> solve) against this header; its answers equal
    the reference solver's (golden fixture road_small)."""
    fx = load_fixture("road_small")
    g, qf, conf = tmp_path / "road.graph", tmp_path / "road.query", tmp_path / "config"
    cc.write_cola_graph(g, fx["row_ptr"], fx["col"], fx["len"], fx["delay"])
    cc.write_cola_queries(qf, fx["src"], fx["dst"], fx["budget"])
    cc.write_config(conf, 2, g, qf, len(fx["queries"]))
    exe = cc.build("ref_main", tmp_path, cuda=True)
    res = subprocess.run([str(exe), str(conf)], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stdout[-2000:] + res.stderr[-2000:]
    _check_caller_output(cc.parse_results(res.stdout), fx, fx["queries"])


def test_reference_caller_on_a_type1_edge_list(tmp_path, oracle_mod):
    """The same caller on the reference's type-1 format (each row added in
    both directions) with its CSV query file; expected answers from the
    reference's own solver (oracle/_ref) on the symmetric graph."""
    O = oracle_mod
    if not O.ref_available():
        pytest.fail("oracle/_ref missing")
    fx = load_fixture("chunglu_small")
    # undirected rows: one per arc u < v of the fixture graph
    src_of = np.repeat(np.arange(len(fx["row_ptr"]) - 1), np.diff(fx["row_ptr"]))
    keep = src_of < fx["col"]
    rows = np.stack([src_of[keep], fx["col"][keep], fx["len"][keep].astype(np.int64),
                     fx["delay"][keep].astype(np.int64)], axis=1)
    n = len(fx["row_ptr"]) - 1
    gpath = tmp_path / "g.txt"
    gpath.write_text(f"{n} {rows.shape[0]}\n" + "".join(f"{a} {b} {c} {d}\n" for a, b, c, d in rows))
    # the CSR read_graph builds: rows in file order, forward then backward arc
    arcs = []
    for a, b, c, d in rows:
        arcs.append((a, b, c, d))
        arcs.append((b, a, c, d))
    order = sorted(range(len(arcs)), key=lambda i: arcs[i][0])  # stable by tail
    row_ptr = np.zeros(n + 1, np.int64)
    np.add.at(row_ptr, np.array([arcs[i][0] for i in order]) + 1, 1)
    row_ptr = np.cumsum(row_ptr)
    col = np.array([arcs[i][1] for i in order], np.int32)
    ln = np.array([arcs[i][2] for i in order], np.float32)
    dl = np.array([arcs[i][3] for i in order], np.float32)
    sym = dict(row_ptr=row_ptr, col=col, len=ln, delay=dl, src=fx["src"], dst=fx["dst"])
    qpath = tmp_path / "q.csv"
    qpath.write_text("id,src,snk,delay,hop,cost\n" + "".join(
        f"{i},{s},{t},{int(b)},0,0\n" for i, (s, t, b) in enumerate(zip(fx["src"], fx["dst"], fx["budget"]))))
    conf = tmp_path / "config"
    cc.write_config(conf, 1, gpath, qpath, len(fx["src"]))
    ref = O.RefSolver(O.CsrGraph(row_ptr, col, ln, dl))
    rr = ref.solve(fx["src"], fx["dst"], np.floor(fx["budget"]), nthreads=O.cpu_count())
    ref.close()
    expected = [{"found": bool(rr["found"][q]), "cost": float(rr["cost"][q]),
                 "delay": float(rr["delay"][q])} for q in range(len(fx["src"]))]
    exe = cc.build("ref_main", tmp_path, cuda=True)
    res = subprocess.run([str(exe), str(conf)], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stdout[-2000:] + res.stderr[-2000:]
    _check_caller_output(cc.parse_results(res.stdout), sym, expected)
