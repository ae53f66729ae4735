"""CPU tests of the oracle (no GPU): the restatement of the reference solver
against the golden vectors generated from the reference's own code, the
label-setting search under the engine's pruning rules, and lower bounds."""
import numpy as np
import pytest

from golden_util import FIXTURES, csr_digest, load_fixture

SMALL = ["kat3", "diamond", "line", "cycle", "road_small", "road_anticorr_small",
         "chunglu_small", "road_batch_small", "grid"]


@pytest.mark.parametrize("name", SMALL)
def test_restatement_matches_reference_golden(oracle_mod, name):
    O = oracle_mod
    fx = load_fixture(name)
    assert csr_digest(fx["row_ptr"], fx["col"], fx["len"], fx["delay"]) == fx["digest"], \
        "workload generator drifted from the golden fixture"
    g = O.CsrGraph(fx["row_ptr"], fx["col"], fx["len"], fx["delay"])
    qs = fx["queries"] if name != "grid" else fx["queries"][:6]
    for q, e in enumerate(qs):
        a = O.solve_reference_rules(g, e["src"], e["dst"], e["budget"])
        assert a["found"] == e["found"]
        assert a["R"] == e["expand_calls"] and a["dom_calls"] == e["dominate_calls"]
        if e["found"]:
            assert (float(a["cost"]), float(a["delay"])) == (e["cost"], e["delay"])
        if "pareto" in e:
            assert np.array_equal(a["pareto"], np.array(e["pareto"], np.float32).reshape(-1, 2))


@pytest.mark.parametrize("name", SMALL)
def test_label_setting_matches_reference_golden(oracle_mod, name):
    O = oracle_mod
    fx = load_fixture(name)
    g = O.CsrGraph(fx["row_ptr"], fx["col"], fx["len"], fx["delay"])
    qs = fx["queries"] if name != "grid" else fx["queries"][:6]
    for e in qs:
        full = O.solve_label_setting(g, e["src"], e["dst"], e["budget"], use_incumbent=False)
        hl, hd = O.lower_bounds(g, e["dst"])
        pruned = O.solve_label_setting(g, e["src"], e["dst"], e["budget"], h_len=hl, h_del=hd,
                                       use_incumbent=True)
        for r in (full, pruned):
            assert r["found"] == e["found"]
            if e["found"]:
                assert (float(r["cost"]), float(r["delay"])) == (e["cost"], e["delay"])
        if "pareto" in e:
            assert np.array_equal(full["pareto"],
                                  np.array(e["pareto"], np.float32).reshape(-1, 2))
        assert pruned["R"] <= full["R"]


def test_known_answers_by_hand(oracle_mod):
    O = oracle_mod
    # 0->1 (5,2), 1->2 (7,3), 0->2 (20,1)
    g = O.CsrGraph([0, 2, 3, 3], [1, 2, 2], [5, 20, 7], [2, 1, 3])
    r = O.solve_reference_rules(g, 0, 2, 100.0)
    assert (r["cost"], r["delay"]) == (12.0, 5.0)
    assert r["path"].tolist() == [0, 1, 2]
    assert r["pareto"].tolist() == [[12.0, 5.0], [20.0, 1.0]]
    r = O.solve_reference_rules(g, 0, 2, 4.0)
    assert (r["cost"], r["delay"]) == (20.0, 1.0) and r["path"].tolist() == [0, 2]
    assert not O.solve_reference_rules(g, 0, 2, 0.0)["found"]
    r = O.solve_reference_rules(g, 1, 1, 0.0)
    assert r["found"] and r["cost"] == 0.0 and r["path"].tolist() == [1]


def test_reference_build_agrees_with_restatement(oracle_mod):
    """Runs the reference's own template when it has been built here."""
    O = oracle_mod
    if not O.ref_available():
        pytest.skip("oracle/_ref not built")
    fx = load_fixture("road_small")
    g = O.CsrGraph(fx["row_ptr"], fx["col"], fx["len"], fx["delay"])
    ref = O.RefSolver(g)
    rr = ref.solve(fx["src"], fx["dst"], fx["budget"], nthreads=4, record_paths=True)
    for q, e in enumerate(fx["queries"]):
        a = O.solve_reference_rules(g, e["src"], e["dst"], e["budget"])
        assert bool(rr["found"][q]) == a["found"]
        assert tuple(rr["calls"][q]) == (a["R"], a["dom_calls"])
        if a["found"]:
            assert (rr["cost"][q], rr["delay"][q]) == (a["cost"], a["delay"])
            assert np.array_equal(rr["paths"][q], a["path"])


def test_lower_bounds_are_exact_distances(oracle_mod):
    O = oracle_mod
    fx = load_fixture("road_small")
    g = O.CsrGraph(fx["row_ptr"], fx["col"], fx["len"], fx["delay"])
    t = int(fx["dst"][0])
    hl, hd = O.lower_bounds(g, t)
    assert hl[t] == 0 and hd[t] == 0
    # consistency: h(u) <= w(u,v) + h(v) on every arc
    src = np.repeat(np.arange(g.n), np.diff(g.row_ptr))
    ok = np.isinf(hl[g.col]) | (hl[src] <= g.len + hl[g.col])
    assert ok.all()
    ok = np.isinf(hd[g.col]) | (hd[src] <= g.delay + hd[g.col])
    assert ok.all()


def test_bytes_per_query_formula(oracle_mod):
    assert oracle_mod.bytes_per_query({"P": 1, "R": 2, "S": 3, "I": 4}) == 20 + 24 + 24 + 96


@pytest.mark.parametrize("cid,over", [(1, {}), (2, dict(rows=30, cols=30, m_target=2500, n_pairs=12)),
                                      (3, dict(rows=28, cols=32, m_target=2300, n_pairs=16)),
                                      (4, dict(n=2000, m_target=30000, n_pairs=16)),
                                      (5, dict(rows=40, cols=40, m_target=4400, n_pairs=32,
                                               hop_lo=2, hop_hi=60))])
def test_host_generator_copy_matches_library(oracle_mod, cid, over):
    """The generator copy linked into the reference library (used by the CPU
    reference timing) builds the same arrays as the engine library's."""
    O = oracle_mod
    if not O.ref_available():
        pytest.skip("oracle/_ref not built")
    import vine_b200 as v
    a = O.HostWorkload(cid, **over)
    b = v.Workload.generate(cid, **over)
    for k in ("row_ptr", "col", "len", "delay", "src", "dst", "budget", "alpha"):
        assert np.array_equal(getattr(a, k), getattr(b, k)), k


def test_variant_golden_reproduces_and_hand_answers(oracle_mod):
    """tests/golden/variants.json is what the reference's solver (built with
    the variant labels) returns, and its 3-vertex cases are the hand-checked
    answers: hop limit 1 forces the direct arc (20), the QoS floor 3 leaves
    only the direct arc (bandwidth 1 < 3 fails, so no path) ..."""
    import json
    O = oracle_mod
    if not O.ref_available():
        pytest.skip("oracle/_ref not built")
    from golden_util import GOLDEN
    var = json.loads((GOLDEN / "variants.json").read_text())
    for name in ("kat3", "road_small"):
        fx = load_fixture(name)
        g = O.CsrGraph(fx["row_ptr"], fx["col"], fx["len"], fx["delay"])
        ref = O.RefSolver(g)
        for kind, k in (("hop", 2), ("maxcost", 3), ("qos", 6)):
            qs = var[name][kind]
            r = ref.solve_variant(k, [e["src"] for e in qs], [e["dst"] for e in qs],
                                  [e["delay_L"] for e in qs], [e.get("hop_L", 100) for e in qs],
                                  [e.get("max_L", 10000.0) for e in qs], nthreads=4)
            for q, e in enumerate(qs):
                assert bool(r["found"][q]) == e["found"]
                if e["found"]:
                    assert [float(x) for x in r["best"][q]] == e["best"]
        ref.close()
    r = O.RefSolver(O.CsrGraph(*[load_fixture("kat3")[k] for k in ("row_ptr", "col", "len", "delay")]))
    hop = r.solve_variant(2, [0, 0], [2, 2], [100, 100], [2, 1])
    assert hop["best"][0][:3].tolist() == [12, 5, 2] and hop["best"][1][:3].tolist() == [20, 1, 1]
    qos = r.solve_variant(6, [0, 0], [2, 2], [2, 3])
    # 0-1-2 has bandwidth min(2, 3) = 2; the direct arc has bandwidth 1
    assert qos["best"][0][:2].tolist() == [12, 2] and not qos["found"][1]
    r.close()
