"""CPU tests of the race-free multi-core host engine (vine_solve_host, the
fixed RUN_CSPP_OMP): answers, paths and sink Pareto sets equal the
reference solver's (golden fixtures), for every thread count and both ways
of spreading the work.  Needs no GPU."""
import numpy as np
import pytest

from golden_util import FIXTURES, check_result, load_fixture, load_scale

SMALL = [f for f in FIXTURES if f != "grid"]


@pytest.mark.parametrize("threads,across", [(1, False), (3, False), (8, False), (4, True)])
@pytest.mark.parametrize("name", SMALL)
def test_host_engine_matches_reference(name, threads, across):
    import vine_b200 as v
    fx = load_fixture(name)
    g = v.Graph(fx["row_ptr"], fx["col"], fx["len"], fx["delay"])
    stride = 1024
    res = v.solve_host(g, fx["src"], fx["dst"], fx["budget"], nthreads=threads,
                       across_queries=across, pareto_stride=stride, raise_on_error=False)
    for q, e in enumerate(fx["queries"]):
        if e["src"] < 0 or e["dst"] < 0:
            continue
        check_result(fx, res, q, e)
        if "pareto" in e:
            want = np.array(e["pareto"], np.float32).reshape(-1, 2)
            got = np.stack([res.pareto_d[q, :res.pareto_n[q]], res.pareto_delay[q, :res.pareto_n[q]]], 1)
            assert np.array_equal(got, want), f"q{q}: Pareto sets differ"


def test_host_engine_on_a_real_graph():
    """The reference's tech-routers-rf graph, answers from the reference's
    own solver (full-size fixture)."""
    import vine_b200 as v
    fx = load_scale("tech_routers_rf")
    g = v.Graph(fx["row_ptr"], fx["col"], fx["len"], fx["delay"])
    res = v.solve_host(g, fx["src"], fx["dst"], fx["budget"], nthreads=0)
    for q, e in enumerate(fx["queries"]):
        check_result(fx, res, q, e)


def test_host_engine_rejects_bad_queries():
    import vine_b200 as v
    fx = load_fixture("kat3")
    g = v.Graph(fx["row_ptr"], fx["col"], fx["len"], fx["delay"])
    res = v.solve_host(g, [0, 9, 0], [2, 0, -1], [100, 5, 5], raise_on_error=False)
    assert res.status[0] == 0 and res.cost[0] == 12
    assert res.status[1] == v._lib.VINE_ERR_INVALID and res.status[2] == v._lib.VINE_ERR_INVALID


def test_cspp_solve_omp_and_cpu():
    import vine_b200 as v
    fx = load_fixture("diamond")
    g = v.Graph(fx["row_ptr"], fx["col"], fx["len"], fx["delay"])
    n = len(fx["queries"])
    for method in ("solve_omp", "solve_cpu"):
        s = v.cspp(g, n, [v.c_label(int(x)) for x in fx["src"]], list(map(int, fx["dst"])),
                   [v.c_constraint(float(b)) for b in fx["budget"]])
        assert getattr(s, method)() == 0
        for q, e in enumerate(fx["queries"]):
            assert bool(s.found_l[q]) == e["found"]
            if e["found"]:
                assert float(s.cost_l[q]) == e["cost"] and s.size_of_result_l[q] >= 1


def test_host_engine_label_cap_fails_the_query_not_the_host(monkeypatch):
    """A query that would hold more labels than the cap stops with
    VINE_ERR_CAPACITY and no answer; small queries of the same call finish
    exactly (the cap is forced low through VINE_HOST_MAX_LABELS)."""
    import vine_b200 as v
    fx = load_fixture("road_small")
    g = v.Graph(fx["row_ptr"], fx["col"], fx["len"], fx["delay"])
    full = v.solve_host(g, fx["src"], fx["dst"], fx["budget"], nthreads=2, raise_on_error=False)
    monkeypatch.setenv("VINE_HOST_MAX_LABELS", "200")
    for across in (False, True):
        res = v.solve_host(g, fx["src"], fx["dst"], fx["budget"], nthreads=2, across_queries=across,
                           raise_on_error=False)
        capped = res.status == v._lib.VINE_ERR_CAPACITY
        assert capped.any() and not capped.all()
        assert (res.found[capped] == 0).all()
        ok = res.status == 0
        assert np.array_equal(res.found[ok], full.found[ok])
        assert np.array_equal(np.where(res.found[ok] == 1, res.cost[ok], 0),
                              np.where(full.found[ok] == 1, full.cost[ok], 0))
    monkeypatch.delenv("VINE_HOST_MAX_LABELS")
    again = v.solve_host(g, fx["src"], fx["dst"], fx["budget"], nthreads=2, raise_on_error=False)
    assert np.array_equal(again.status, full.status)
