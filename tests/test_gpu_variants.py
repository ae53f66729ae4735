"""GPU parity of the label variants (vine_solve_labels) with the reference's
solver: hop-constrained (CSP=2), max-cost (CSP=3) and network-QoS labels.

Expected answers come from the reference's RUN_CSPP_CPU instantiated with
each variant's label (tests/golden/variants.json, written by
tests/golden/make_variant_golden.py).  The best feasible sink label must
match bit-exactly; the returned path must exist, respect every limit and
recompute to the reported label (sums for d and delay, the path's arc
count for hop, its largest arc length for maxcost, its smallest arc delay
for the QoS bandwidth)."""
import json

import numpy as np
import pytest

from golden_util import GOLDEN, check_result, load_fixture, load_scale

pytestmark = pytest.mark.gpu

VARIANTS = json.loads((GOLDEN / "variants.json").read_text()) if (GOLDEN / "variants.json").exists() else {}
CASES = [(g, k) for g in VARIANTS for k in ("hop", "maxcost", "qos")]


def _along(fx, path):
    """(d, delay sum, hop count, max len, min delay) along a vertex path."""
    d = np.float32(0)
    dl = np.float32(0)
    mx = np.float32(0)
    mn = np.float32(21474836.0)
    for u, v in zip(path[:-1], path[1:]):
        a, b = fx["row_ptr"][u], fx["row_ptr"][u + 1]
        hit = np.nonzero(fx["col"][a:b] == v)[0]
        assert hit.size, f"arc {u}->{v} missing"
        j = a + hit[0]
        d = np.float32(d + fx["len"][j])
        dl = np.float32(dl + fx["delay"][j])
        mx = max(mx, fx["len"][j])
        mn = min(mn, fx["delay"][j])
    return float(d), float(dl), len(path) - 1, float(mx), float(mn)


@pytest.fixture(scope="module")
def graphs():
    import vine_b200 as v
    cache = {}

    def get(name):
        if name not in cache:
            for old in list(cache):
                cache.pop(old)[1].close()
            fx = load_scale(name) if name.startswith("tech_") else load_fixture(name)
            cache[name] = (fx, v.Graph(fx["row_ptr"], fx["col"], fx["len"], fx["delay"]))
        return cache[name]
    yield get
    for _, g in cache.values():
        g.close()


@pytest.mark.parametrize("name,kind", CASES)
def test_variant_matches_reference(graphs, name, kind):
    import vine_b200 as v
    fx, g = graphs(name)
    qs = VARIANTS[name][kind]
    src = [e["src"] for e in qs]
    dst = [e["dst"] for e in qs]
    dL = [e["delay_L"] for e in qs]
    hL = [e.get("hop_L", 100) for e in qs] if kind != "qos" else None
    mL = [e.get("max_L", 10000.0) for e in qs] if kind == "maxcost" else None
    res = v.solve_labels(g, kind, src, dst, dL, hL, mL)
    for q, e in enumerate(qs):
        assert res.status[q] == 0
        assert bool(res.found[q]) == e["found"], f"q{q}: found {res.found[q]} vs {e['found']}"
        if not e["found"]:
            continue
        best = e["best"]
        got = (float(res.cost[q]), float(res.delay[q]), float(res.extra[q, 0]), float(res.extra[q, 1]))
        if kind == "qos":
            assert got[:2] == tuple(best[:2]), f"q{q}: {got[:2]} vs {best[:2]}"
        elif kind == "hop":
            assert got[:3] == tuple(best[:3]), f"q{q}: {got[:3]} vs {best[:3]}"
        else:
            assert got == tuple(best), f"q{q}: {got} vs {best}"
        p = res.path(q)
        assert p[0] == e["src"] and p[-1] == e["dst"]
        d, dl, hops, mx, mn = _along(fx, p)
        assert d == got[0]
        if kind == "qos":
            bw = mn if len(p) > 1 else 21474836.0
            assert bw == got[1] and not (bw < e["delay_L"])
        else:
            assert dl == got[1] and hops == got[2] and dl <= e["delay_L"] and hops <= e["hop_L"]
            if kind == "maxcost":
                assert mx == got[3] and mx <= e["max_L"]


@pytest.mark.parametrize("name", ["kat3", "road_small", "chunglu_small"])
def test_csp_kind_matches_the_csp_engine_golden(graphs, name):
    """The variant engine with the CSP=1 label equals the reference's answers
    of the main fixtures (the same ones the CSP engines are held to)."""
    import vine_b200 as v
    fx, g = graphs(name)
    res = v.solve_labels(g, "csp", fx["src"], fx["dst"], fx["budget"], raise_on_error=False)
    for q, e in enumerate(fx["queries"]):
        if e["src"] < 0 or e["dst"] < 0 or e["src"] >= g.N or e["dst"] >= g.N:
            assert res.status[q] == v._lib.VINE_ERR_INVALID
            continue
        check_result(fx, res, q, e)


def test_variant_rejects_unknown_kind(graphs):
    import vine_b200 as v
    fx, g = graphs("kat3")
    with pytest.raises(v.VineError):
        v.solve_labels(g, 5, [0], [2], [10.0])
