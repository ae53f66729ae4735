"""CPU tests of the boundary: the C-ABI library loads and exports every
function the headers declare; generators are deterministic and produce the
advertised shapes; host-side argument checking (no device needed)."""
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(vine_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_library_exports_every_declared_function():
    import ctypes
    lib = ctypes.CDLL(str(ROOT / "vine_b200" / "libvine.so"))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"
    assert len(declared_functions()) >= 25


def test_binding_covers_every_declared_function():
    from vine_b200 import _lib
    assert set(declared_functions()) <= set(_lib.SIGNATURES)


def test_library_is_built_for_sm100a():
    import subprocess
    out = subprocess.run(["/usr/local/cuda/bin/cuobjdump", "--list-elf",
                          str(ROOT / "vine_b200" / "libvine.so")],
                         capture_output=True, text=True).stdout
    assert "sm_100a" in out


def test_config_defaults_and_names():
    import vine_b200 as v
    c = v.Config(engine="plain", mode="pareto", policy="ar", bucket_width=50.0)
    d = v.config_dict(c)
    assert d["engine"] == 1 and d["mode"] == 1 and d["policy"] == 1
    assert d["bucket_width"] == 50.0 and d["block_threads"] == 512
    with pytest.raises(TypeError):
        v.Config(not_a_field=1)


def test_grid_workload_shape_and_determinism():
    import vine_b200 as v
    a = v.Workload.generate(1)
    b = v.Workload.generate(1)
    assert a.n == 10000 and a.m == 39600 and a.nq == 16
    for k in ("row_ptr", "col", "len", "delay", "src", "dst", "budget"):
        assert np.array_equal(getattr(a, k), getattr(b, k))
    assert a.len.min() >= 1 and a.len.max() <= 100 and np.all(a.len == np.round(a.len))
    assert np.all(a.src != a.dst)


def test_road_workload_shape():
    import vine_b200 as v
    w = v.Workload.generate(2, rows=50, cols=60, m_target=8400, n_pairs=4)
    assert w.n == 3000
    assert abs(w.m - 8400) < 600
    # symmetric arcs with equal length both ways
    src = np.repeat(np.arange(w.n), np.diff(w.row_ptr))
    fwd = {(int(u), int(x)): l for u, x, l in zip(src, w.col, w.len)}
    assert all(fwd[(x, u)] == l for (u, x), l in fwd.items())
    assert w.nq == 12 and set(np.round(w.alpha.astype(float), 2).tolist()) == {0.2, 0.5, 0.8}
    assert np.all(w.budget >= 0)


def test_chunglu_and_batch_workloads():
    import vine_b200 as v
    w = v.Workload.generate(4, n=3000, m_target=40000, n_pairs=8)
    deg = np.diff(w.row_ptr)
    assert deg.max() > 20 * max(1, np.median(deg))  # heavy-tailed
    assert w.nq == 8
    b = v.Workload.generate(5, rows=30, cols=30, m_target=2500, n_pairs=20, hop_hi=40)
    assert b.nq == 20 and np.all((b.alpha >= 0.1) & (b.alpha < 0.9))


def test_budget_rule_matches_dijkstra(oracle_mod):
    import vine_b200 as v
    w = v.Workload.generate(2, rows=20, cols=25, m_target=1400, n_pairs=5)
    g = oracle_mod.CsrGraph(w.row_ptr, w.col, w.len, w.delay)
    for q in range(w.nq):
        dmin, _, _ = oracle_mod.dijkstra(g, int(w.src[q]), "delay")
        _, dlen, _ = oracle_mod.dijkstra(g, int(w.src[q]), "len")
        t = int(w.dst[q])
        want = np.floor(dmin[t] + np.float32(w.alpha[q]) * (dlen[t] - dmin[t]))
        assert abs(float(w.budget[q]) - float(want)) <= 1.0


@pytest.mark.parametrize("name", ["tech_routers_rf", "tech_internet_as"])
def test_mtx_loader_reproduces_the_real_graph_fixtures(name):
    """The 5-column loader on the reference's own inputs/tech-*.mtx.txt files
    gives exactly the arrays committed in the full-size fixtures (which the
    GPU tests use where the reference tree is absent)."""
    import hashlib
    import json
    import vine_b200 as v
    from golden_util import GOLDEN, load_scale
    from oracle import oracle as O
    meta = json.loads((GOLDEN / f"scale_{name}.json").read_text())
    path = Path(O.REF_TREE) / meta["source_file"]
    if not path.exists():
        pytest.skip("reference inputs not present")
    assert hashlib.sha256(path.read_bytes()).hexdigest() == meta["source_sha256"]
    w = v.Workload.load_mtx(str(path), n_pairs=meta.get("n_pairs", 3) or 3, alpha=(0.5,),
                            seed=meta["query_seed"])
    fx = load_scale(name)
    for k in ("row_ptr", "col", "len", "delay"):
        assert np.array_equal(getattr(w, k), fx[k]), k
    n = len(fx["queries"])
    w2 = v.Workload.load_mtx(str(path), n_pairs=n, alpha=(0.5,), seed=meta["query_seed"])
    assert np.array_equal(w2.src, fx["src"]) and np.array_equal(w2.dst, fx["dst"])
    assert np.array_equal(w2.budget, fx["budget"])


def test_cola_loader_roundtrip(tmp_path):
    import vine_b200 as v
    g = tmp_path / "g.graph"
    g.write_text("3\n0: 1 5 2 2 20 1 -1\n1: 2 7 3 -1\n2: -1\n")
    q = tmp_path / "q.txt"
    q.write_text("0 2 1 1 100\n0 2 1 1 4\n")
    w = v.Workload.load_cola(str(g), str(q))
    assert w.n == 3 and w.m == 3 and w.nq == 2
    assert w.budget.tolist() == [100.0, 4.0]
    assert w.col.tolist() == [1, 2, 2] and w.len.tolist() == [5, 20, 7]


def test_loader_errors_are_status_codes(tmp_path):
    import vine_b200 as v
    with pytest.raises(v.VineError) as e:
        v.Workload.load_mtx(str(tmp_path / "missing.mtx"))
    assert e.value.status == v._lib.VINE_ERR_IO


def test_graph_validation_without_device():
    import vine_b200 as v
    # a malformed graph is rejected before any device work
    g = v.Graph([0, 2, 1], [1, 0], [1, 1], [1, 1])
    with pytest.raises(v.VineError) as e:
        g.make_gpu_graph()
    assert e.value.status == v._lib.VINE_ERR_INVALID
    g = v.Graph([0, 1, 1], [1], [-1.0], [1])
    with pytest.raises(v.VineError):
        g.make_gpu_graph()


def test_dropin_graph_model_builds_the_csr(tmp_path):
    """The C++ drop-in's read_graph (COLA format) + adj_to_csr, built and run
    on the host: the CSR equals the one the file was written from, with edge
    ids in file order (include/io.hpp:61-91, include/graph.hpp:136-167)."""
    import cpp_callers as cc
    from golden_util import load_fixture
    fx = load_fixture("road_small")
    gpath = tmp_path / "g.graph"
    cc.write_cola_graph(gpath, fx["row_ptr"], fx["col"], fx["len"], fx["delay"])
    exe = cc.build("csr_dump", tmp_path)
    res = subprocess.run([str(exe), str(gpath), "2"], capture_output=True, text=True, timeout=60)
    assert res.returncode == 0, res.stderr
    lines = res.stdout.split("\n")
    n, m = map(int, lines[0].split())
    assert (n, m) == (len(fx["row_ptr"]) - 1, len(fx["col"]))
    row = np.array([int(x) for x in lines[1:n + 2]])
    assert np.array_equal(row, fx["row_ptr"])
    slots = np.array([[float(x) for x in ln.split()] for ln in lines[n + 2:n + 2 + m]])
    assert np.array_equal(slots[:, 0].astype(np.int64), fx["col"])
    assert np.array_equal(slots[:, 1].astype(np.float32), fx["len"])
    assert np.array_equal(slots[:, 2].astype(np.float32), fx["delay"])
    assert np.array_equal(slots[:, 3].astype(np.int64), np.arange(m))  # edge ids in file order


def test_reference_arm_loads_no_engine_library(tmp_path):
    """bench.py --impl reference times the reference's CPU solver on the same
    seeded workload without loading the engine's library (it builds the
    workload with the generator copy in oracle/_ref)."""
    import json
    import sys
    from oracle import oracle as O
    if not O.ref_available():
        pytest.skip("oracle/_ref not built")
    code = (
        "import sys, json, types\n"
        "sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '0', '--nq', '48']\n"
        "import bench\n"
        "bench.main()\n"
        "mods = [m for m in sys.modules if m.startswith('vine_b200')]\n"
        "maps = open('/proc/self/maps').read()\n"
        "print(json.dumps({'mods': mods, 'libvine': 'libvine.so' in maps}))\n")
    root = Path(__file__).resolve().parents[1]
    res = subprocess.run([sys.executable, "-c", code], cwd=root, capture_output=True, text=True,
                         timeout=600)
    assert res.returncode == 0, res.stderr[-3000:]
    lines = [ln for ln in res.stdout.splitlines() if ln.startswith("{")]
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["value"] > 0
    check = json.loads(lines[-1])
    assert check == {"mods": [], "libvine": False}
