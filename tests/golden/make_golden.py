"""Generates tests/golden/*.json from the reference's own CPU solver.

Run in a tree that has the reference sources (oracle/_ref/libvine_ref.so is
built from them by oracle/Makefile):

    python tests/golden/make_golden.py

Each fixture holds a small workload (hand-made graphs inline; generated
workloads by their generator parameters plus a CSR checksum that detects
generator drift) and, per query, what the reference's RUN_CSPP_CPU
(algorithm/cspp_cpu.hpp:44-125, instantiated with an additive label)
reaches: the lexicographically smallest feasible (cost, delay), feasibility,
the number of expand_cpu / dominate_cpu calls, and the sink Pareto set taken
from the restatement (whose call counts must equal the reference's).
"""
from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import oracle as O  # noqa: E402

OUT = Path(__file__).resolve().parent


def csr_digest(row_ptr, col, length, delay) -> str:
    h = hashlib.sha256()
    for a, dt in ((row_ptr, np.int64), (col, np.int32), (length, np.float32), (delay, np.float32)):
        h.update(np.ascontiguousarray(a, dt).tobytes())
    return h.hexdigest()


def from_arcs(n, arcs):
    arcs = sorted(arcs, key=lambda a: a[0])  # stable: keeps listed order per source
    row = np.zeros(n + 1, np.int64)
    for u, _, _, _ in arcs:
        row[u + 1] += 1
    row = np.cumsum(row)
    col = np.array([a[1] for a in arcs], np.int32)
    ln = np.array([a[2] for a in arcs], np.float32)
    dl = np.array([a[3] for a in arcs], np.float32)
    return row, col, ln, dl


HAND = {
    # 3 vertices: 0->1 (5,2), 1->2 (7,3), 0->2 (20,1)
    "kat3": (3, [(0, 1, 5, 2), (1, 2, 7, 3), (0, 2, 20, 1)],
             [(0, 2, 100), (0, 2, 4), (0, 2, 0), (0, 0, 5), (2, 0, 100), (1, 1, -1), (0, 2, 5)]),
    # diamond with equal-cost ties and a direct arc
    "diamond": (4, [(0, 1, 1, 5), (0, 2, 2, 2), (1, 3, 2, 1), (2, 3, 1, 4), (0, 3, 4, 3)],
                [(0, 3, 10), (0, 3, 5), (0, 3, 6), (0, 3, 2), (3, 0, 50)]),
    # a line of 10 vertices, unit weights
    "line": (10, [(i, i + 1, 1, 1) for i in range(9)],
             [(0, 9, 9), (0, 9, 8), (0, 5, 100), (9, 0, 100)]),
    # a cycle back to the source and a zero-weight arc
    "cycle": (4, [(0, 1, 1, 1), (1, 0, 1, 1), (1, 2, 0, 3), (2, 3, 2, 0), (0, 3, 9, 9), (3, 1, 1, 1)],
              [(0, 3, 10), (0, 3, 3), (0, 3, 2), (1, 1, 0), (2, 1, 10)]),
}

GENERATED = {
    # name: (config_id, overrides, pareto)
    "grid": (1, {}, True),
    "road_small": (2, dict(rows=30, cols=30, m_target=2500, n_pairs=12), True),
    "road_anticorr_small": (3, dict(rows=28, cols=32, m_target=2300, n_pairs=16), True),
    "chunglu_small": (4, dict(n=2000, m_target=30000, n_pairs=16), True),
    "road_batch_small": (5, dict(rows=40, cols=40, m_target=4400, n_pairs=32, hop_lo=2,
                                 hop_hi=60), False),
}


def run(name, row, col, ln, dl, src, dst, bud, pareto: bool, gen=None):
    g = O.CsrGraph(row, col, ln, dl)
    ref = O.RefSolver(g)
    rr = ref.solve(src, dst, bud, nthreads=O.cpu_count(), record_paths=False)
    queries = []
    for q in range(len(src)):
        a = O.solve_reference_rules(g, int(src[q]), int(dst[q]), float(bud[q]))
        if (a["R"], a["dom_calls"]) != tuple(int(x) for x in rr["calls"][q]):
            raise SystemExit(f"{name} q{q}: restatement call counts differ from the reference")
        if bool(a["found"]) != bool(rr["found"][q]) or (
                a["found"] and (a["cost"], a["delay"]) != (rr["cost"][q], rr["delay"][q])):
            raise SystemExit(f"{name} q{q}: restatement result differs from the reference")
        rec = {"src": int(src[q]), "dst": int(dst[q]), "budget": float(bud[q]),
               "found": bool(rr["found"][q]),
               "cost": float(rr["cost"][q]) if rr["found"][q] else None,
               "delay": float(rr["delay"][q]) if rr["found"][q] else None,
               "expand_calls": int(rr["calls"][q][0]), "dominate_calls": int(rr["calls"][q][1])}
        if pareto:
            rec["pareto"] = a["pareto"].tolist()
        queries.append(rec)
    fx = {"name": name, "generator": gen, "digest": csr_digest(row, col, ln, dl),
          "n": int(g.n), "m": int(col.shape[0]), "queries": queries}
    if gen is None:
        fx["graph"] = {"row_ptr": row.tolist(), "col": col.tolist(), "len": ln.tolist(),
                       "delay": dl.tolist()}
    (OUT / f"{name}.json").write_text(json.dumps(fx, separators=(",", ":")))
    print(name, g.n, col.shape[0], len(queries))


def main():
    if not O.ref_available():
        O.build()
    for name, (n, arcs, qs) in HAND.items():
        row, col, ln, dl = from_arcs(n, arcs)
        src = np.array([q[0] for q in qs], np.int32)
        dst = np.array([q[1] for q in qs], np.int32)
        bud = np.array([q[2] for q in qs], np.float32)
        run(name, row, col, ln, dl, src, dst, bud, True)
    import vine_b200 as v
    for name, (cid, over, pareto) in GENERATED.items():
        w = v.Workload.generate(cid, **over)
        run(name, w.row_ptr, w.col, w.len, w.delay, w.src, w.dst, w.budget, pareto,
            gen={"config_id": cid, "overrides": over})


if __name__ == "__main__":
    main()
