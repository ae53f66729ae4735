"""Algorithmic work of the 4096-query road workload, from the CPU oracle.

Writes tests/golden/road264k_work.json: for every query of the benchmark
workload (264k-vertex road graph, 4096 hop-sampled queries) the counters of
the oracle's exact label-setting search under the GPU engine's pruning rules
(delay and A* length lower bounds from the sink, incumbent pruning):

  P  labels expanded      R  arcs relaxed
  S  stored-label reads   I  labels inserted

plus the work of the two bounded reverse searches that compute the bounds
(vertices settled and arcs scanned).  bench.py turns these into the
algorithmic bytes of one launch:

  forward: 20 P + 12 R + 8 S + 24 I
  bounds:  per pass 20 bytes per settled vertex + 16 bytes per scanned arc

The length bound is restricted, as in the engine, to the vertices whose
delay bound fits the budget.  Usage: python tests/golden/make_work_counts.py
"""
from __future__ import annotations

import json
import multiprocessing as mp
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
OUT = Path(__file__).resolve().parent / "road264k_work.json"

_G = None


def _init(arrays):
    global _G
    from oracle import oracle as O
    row, col, ln, dl = arrays
    g = O.CsrGraph(row, col, ln, dl)
    rg = g.reverse()
    indeg = np.diff(rg.row_ptr)
    _G = (O, g, rg, indeg)


def _one(args):
    q, s, t, L = args
    O, g, rg, indeg = _G
    hd, _, _ = O.dijkstra(rg, t, "delay")
    feas = hd <= L
    # length bound restricted to the delay-feasible vertices
    keep = feas[rg.col] & feas[np.repeat(np.arange(g.n), np.diff(rg.row_ptr))]
    counts = np.zeros(g.n + 1, np.int64)
    src_of = np.repeat(np.arange(g.n), np.diff(rg.row_ptr))
    np.add.at(counts, src_of[keep] + 1, 1)
    rp = np.cumsum(counts)
    sub = O.CsrGraph(rp, rg.col[keep], rg.len[keep], rg.delay[keep])
    hl, _, _ = O.dijkstra(sub, t, "len")
    hl = np.where(feas, hl, np.inf).astype(np.float32)
    hd = np.where(feas, hd, np.inf).astype(np.float32)
    r = O.solve_label_setting(g, s, t, L, h_len=hl, h_del=hd, use_incumbent=True)
    nv = int(feas.sum())
    na = int(indeg[feas].sum())
    return q, {"P": int(r["P"]), "R": int(r["R"]), "S": int(r["S"]), "I": int(r["I"]),
               "bound_vertices": 2 * nv, "bound_arcs": 2 * na, "found": bool(r["found"]),
               "cost": float(r["cost"]) if r["found"] else None}


def main():
    import vine_b200 as v
    w = v.Workload.generate(5)
    t0 = time.time()
    jobs = [(q, int(w.src[q]), int(w.dst[q]), float(w.budget[q])) for q in range(w.nq)]
    ctx = mp.get_context("spawn")
    out = [None] * w.nq
    with ctx.Pool(processes=mp.cpu_count(), initializer=_init,
                  initargs=((w.row_ptr, w.col, w.len, w.delay),)) as pool:
        for k, (q, rec) in enumerate(pool.imap_unordered(_one, jobs, chunksize=4)):
            out[q] = rec
            if k % 256 == 0:
                print(f"{k}/{w.nq} {time.time() - t0:.0f}s", flush=True)
    tot = {k: int(sum(r[k] for r in out)) for k in ("P", "R", "S", "I", "bound_vertices", "bound_arcs")}
    OUT.write_text(json.dumps({"workload": "road264k-4096q", "n": w.n, "m": w.m, "nq": w.nq,
                               "totals": tot, "queries": out}, separators=(",", ":")))
    print("wrote", OUT, tot, f"{time.time() - t0:.0f}s")


if __name__ == "__main__":
    main()
