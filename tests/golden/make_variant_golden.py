"""Expected answers for the label variants, from the reference's own solver.

Writes tests/golden/variants.json.  For each graph (the hand-made ones and
small generated workloads of the other fixtures) and each label kind -- hop
constrained (the reference's CSP=2 label), max cost (CSP=3) and network QoS
-- it runs the reference's RUN_CSPP_CPU (algorithm/cspp_cpu.hpp:44-125),
compiled from its sources into oracle/_ref with the variant label types of
oracle/ref_oracle.cpp, and records per query the best feasible sink label:
(d, delay, hop, maxcost), or (d, bandwidth) for QoS, and feasibility.

Limits: the hop limit is taken from the hop count of the unconstrained CSP
answer (so that it binds for some queries), the max-cost limit from the
arc-length distribution, the QoS bandwidth floor from the arc-delay
distribution.  Run in a tree with the reference sources:

    python tests/golden/make_variant_golden.py
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path[:0] = [str(ROOT), str(ROOT / "tests")]

from golden_util import load_fixture, load_scale  # noqa: E402
from oracle import oracle as O  # noqa: E402

OUT = Path(__file__).resolve().parent / "variants.json"
GRAPHS = ["kat3", "diamond", "line", "cycle", "road_small", "road_anticorr_small", "chunglu_small",
          "road_batch_small", "tech_routers_rf", "tech_internet_as"]
SCALE = {"tech_routers_rf", "tech_internet_as"}  # the reference's real graphs (full-size fixtures)
CAP_S = 60.0


def main():
    if not O.ref_available():
        O.build()
    out = {}
    for name in GRAPHS:
        fx = load_scale(name) if name in SCALE else load_fixture(name)
        ok = (fx["src"] >= 0) & (fx["dst"] >= 0) & (fx["src"] < len(fx["row_ptr"]) - 1) & \
             (fx["dst"] < len(fx["row_ptr"]) - 1) & (fx["budget"] >= 0)
        src, dst, bud = fx["src"][ok], fx["dst"][ok], fx["budget"][ok]
        g = O.CsrGraph(fx["row_ptr"], fx["col"], fx["len"], fx["delay"])
        ref = O.RefSolver(g)
        nq = len(src)
        base = ref.solve(src, dst, bud, nthreads=O.cpu_count(), record_paths=True)
        hops = np.array([max(1, len(p) - 1) if f else 3 for p, f in zip(base["paths"], base["found"])])
        cases = {
            # hop limits at, just under and far above the CSP answer's hop count
            "hop": dict(kind=2, delay_L=np.concatenate([bud, bud, bud]),
                        hop_L=np.concatenate([hops, np.maximum(hops - 2, 1), np.full(nq, 100)]),
                        rep=3),
            "maxcost": dict(kind=3, delay_L=np.concatenate([bud, bud]),
                            hop_L=np.full(2 * nq, 100),
                            max_L=np.concatenate([np.full(nq, float(np.percentile(fx["len"], 60))),
                                                  np.full(nq, float(np.percentile(fx["len"], 90)))]),
                            rep=2),
            "qos": dict(kind=6, delay_L=np.concatenate([np.full(nq, float(np.percentile(fx["delay"], q)))
                                                        for q in (10, 30, 50)]), rep=3),
        }
        rec = {}
        for kname, cs in cases.items():
            rep = cs["rep"]
            s2, d2 = np.tile(src, rep), np.tile(dst, rep)
            r = ref.solve_variant(cs["kind"], s2, d2, cs["delay_L"], cs.get("hop_L"), cs.get("max_L"),
                                  nthreads=O.cpu_count(), cap_seconds=CAP_S)
            qs = []
            for q in range(len(s2)):
                if not r["finished"][q]:
                    continue
                e = {"src": int(s2[q]), "dst": int(d2[q]), "delay_L": float(cs["delay_L"][q]),
                     "found": bool(r["found"][q]), "expand_calls": int(r["calls"][q])}
                if "hop_L" in cs:
                    e["hop_L"] = int(cs["hop_L"][q])
                if "max_L" in cs:
                    e["max_L"] = float(cs["max_L"][q])
                if r["found"][q]:
                    e["best"] = [float(x) for x in r["best"][q]]
                qs.append(e)
            rec[kname] = qs
            print(name, kname, len(qs), "of", len(s2), "feasible", sum(e["found"] for e in qs))
        ref.close()
        out[name] = rec
    OUT.write_text(json.dumps(out, separators=(",", ":")))
    print("wrote", OUT)


if __name__ == "__main__":
    main()
