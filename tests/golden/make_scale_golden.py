"""Expected answers for the workloads at their full stated sizes.

Writes tests/golden/scale_<case>.json (and, for the reference's two real
graphs, tests/golden/<case>_graph.npz).  Run in a tree that has the reference
sources (oracle/_ref/libvine_ref.so is built from them by oracle/Makefile):

    python tests/golden/make_scale_golden.py [case ...]

Cases:
  c2_road264k       the 264,000-vertex road-like graph, 300 pairs x alpha {0.2, 0.5, 0.8}
  c3_road1500k      the 1.5M-vertex road-like graph, anti-correlated delay, 200 queries
  c4_chunglu100k    the Chung-Lu graph (100k vertices, exponent 2.2), 64 queries 3-6 hops apart
  c5_sample256      256 seeded random queries of the 4096-query benchmark batch
  tech_routers_rf   the reference's inputs/tech-routers-rf.mtx.txt, 48 random pairs, alpha 0.5
  tech_internet_as  the reference's inputs/tech-internet-as.mtx.txt, 32 random pairs, alpha 0.5

Every query gets the lexicographically smallest feasible (cost, delay) and
feasibility from three solvers, tried in this order; the first that finishes
is recorded as the query's `source`, and every one that finishes must agree:

  reference           the reference's own RUN_CSPP_CPU (algorithm/cspp_cpu.hpp:44-125),
                      compiled from its sources, stopped after REF_CAP seconds
  label_setting_plain exhaustive Pareto label setting (Martins' method) with no lower
                      bounds and no incumbent pruning -- none of the GPU engine's pruning
                      rules -- stopped after PLAIN_CAP seconds
  label_setting_bounds the label-setting search under the engine's own pruning rules
                      (exact reverse delay / length bounds, incumbent), always run

The exhaustive reference search needs minutes to hours for long queries on
these graphs, so many queries fall through to the second or third solver;
the counts per source are stored in the fixture (`sources`).
"""
from __future__ import annotations

import hashlib
import json
import multiprocessing as mp
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
OUT = Path(__file__).resolve().parent

REF_CAP = 10.0
THREADS = max(1, mp.cpu_count() - 1)

CASES = {
    "c4_chunglu100k": dict(config_id=4, plain_cap=60.0),
    "tech_routers_rf": dict(mtx="inputs/tech-routers-rf.mtx.txt", n_pairs=48, plain_cap=60.0),
    "tech_internet_as": dict(mtx="inputs/tech-internet-as.mtx.txt", n_pairs=32, plain_cap=60.0),
    "c5_sample256": dict(config_id=5, sample=256, sample_seed=2024, plain_cap=60.0),
    "c2_road264k": dict(config_id=2, plain_cap=60.0),
    "c3_road1500k": dict(config_id=3, plain_cap=30.0),
}


def csr_digest(row_ptr, col, length, delay) -> str:
    h = hashlib.sha256()
    for a, dt in ((row_ptr, np.int64), (col, np.int32), (length, np.float32), (delay, np.float32)):
        h.update(np.ascontiguousarray(a, dt).tobytes())
    return h.hexdigest()


_W = None


def _init(arrays):
    global _W
    from oracle import oracle as O
    g = O.CsrGraph(*arrays)
    _W = (O, g, g.reverse())


def _bounds_job(args):
    q, s, t, L = args
    O, g, rg = _W
    hl, _, _ = O.dijkstra(rg, t, "len")
    hd, _, _ = O.dijkstra(rg, t, "delay")
    r = O.solve_label_setting(g, s, t, L, h_len=hl, h_del=hd, use_incumbent=True)
    return q, (bool(r["found"]), float(r["cost"]), float(r["delay"]))


def _plain_job(args):
    q, s, t, L, cap = args
    O, g, _ = _W
    t0 = time.time()
    r = O.solve_label_setting(g, s, t, L, use_incumbent=False, time_limit=cap)
    if r is None:
        return q, None, time.time() - t0
    return q, (bool(r["found"]), float(r["cost"]), float(r["delay"])), time.time() - t0


def _same(a, b) -> bool:
    if a[0] != b[0]:
        return False
    return (not a[0]) or (a[1], a[2]) == (b[1], b[2])


def load_case_workload(name: str, spec: dict):
    """(row_ptr, col, len, delay, src, dst, budget, meta) of a case."""
    import vine_b200 as v
    if "mtx" in spec:
        from oracle import oracle as O
        path = Path(O.REF_TREE) / spec["mtx"]
        w = v.Workload.load_mtx(str(path), n_pairs=spec["n_pairs"], alpha=(0.5,), seed=1)
        np.savez_compressed(OUT / f"{name}_graph.npz", row_ptr=w.row_ptr, col=w.col,
                            len=w.len.astype(np.uint16), delay=w.delay.astype(np.uint16))
        assert np.array_equal(w.len.astype(np.uint16).astype(np.float32), w.len)
        assert np.array_equal(w.delay.astype(np.uint16).astype(np.float32), w.delay)
        file_sha = hashlib.sha256(path.read_bytes()).hexdigest()
        meta = {"graph_file": f"{name}_graph.npz", "source_file": spec["mtx"],
                "source_sha256": file_sha, "query_seed": 1, "alpha": 0.5}
        return w.row_ptr, w.col, w.len, w.delay, w.src, w.dst, w.budget, meta
    w = v.Workload.generate(spec["config_id"])
    meta = {"generator": {"config_id": spec["config_id"], "overrides": {}}}
    src, dst, bud = w.src, w.dst, w.budget
    if "sample" in spec:
        sel = np.sort(np.random.default_rng(spec["sample_seed"]).choice(w.nq, spec["sample"],
                                                                        replace=False))
        meta["sample_index"] = sel.tolist()
        src, dst, bud = src[sel], dst[sel], bud[sel]
    return w.row_ptr, w.col, w.len, w.delay, src, dst, bud, meta


def run_case(name: str, spec: dict) -> None:
    from oracle import oracle as O
    t0 = time.time()
    row, col, ln, dl, src, dst, bud, meta = load_case_workload(name, spec)
    nq = len(src)
    print(f"[{name}] {len(row) - 1} V, {len(col)} arcs, {nq} queries", flush=True)
    g = O.CsrGraph(row, col, ln, dl)
    ref = O.RefSolver(g)
    rr = ref.solve_capped(src, dst, bud, THREADS, REF_CAP)
    ref.close()
    print(f"[{name}] reference finished {int(rr['finished'].sum())}/{nq} "
          f"({time.time() - t0:.0f}s)", flush=True)
    ctx = mp.get_context("spawn")
    with ctx.Pool(THREADS, initializer=_init, initargs=((row, col, ln, dl),)) as pool:
        jobs = [(q, int(src[q]), int(dst[q]), float(bud[q])) for q in range(nq)]
        bnd = dict(pool.imap_unordered(_bounds_job, jobs, chunksize=1))
        print(f"[{name}] bounded label setting done ({time.time() - t0:.0f}s)", flush=True)
        pj = [(q, int(src[q]), int(dst[q]), float(bud[q]), spec["plain_cap"])
              for q in range(nq) if not rr["finished"][q]]
        plain = {}
        for q, res, _ in pool.imap_unordered(_plain_job, pj, chunksize=1):
            plain[q] = res
    print(f"[{name}] plain label setting finished "
          f"{sum(r is not None for r in plain.values())}/{len(pj)} ({time.time() - t0:.0f}s)",
          flush=True)
    queries, sources = [], {"reference": 0, "label_setting_plain": 0, "label_setting_bounds": 0}
    for q in range(nq):
        found = []
        if rr["finished"][q]:
            found.append(("reference", (bool(rr["found"][q]), float(rr["cost"][q]),
                                        float(rr["delay"][q]))))
        if plain.get(q) is not None:
            found.append(("label_setting_plain", plain[q]))
        found.append(("label_setting_bounds", bnd[q]))
        for tag, res in found[1:]:
            if not _same(found[0][1], res):
                raise SystemExit(f"{name} q{q}: {found[0][0]} {found[0][1]} != {tag} {res}")
        tag, (f, c, d) = found[0]
        sources[tag] += 1
        queries.append({"src": int(src[q]), "dst": int(dst[q]), "budget": float(bud[q]),
                        "found": f, "cost": c if f else None, "delay": d if f else None,
                        "source": tag, "agree": [t for t, _ in found]})
    fx = dict(meta, name=name, digest=csr_digest(row, col, ln, dl), n=int(len(row) - 1),
              m=int(len(col)), ref_cap_s=REF_CAP, plain_cap_s=spec["plain_cap"],
              sources=sources, queries=queries)
    (OUT / f"scale_{name}.json").write_text(json.dumps(fx, separators=(",", ":")))
    print(f"[{name}] wrote scale_{name}.json sources={sources} ({time.time() - t0:.0f}s)",
          flush=True)


def main():
    from oracle import oracle as O
    if not O.ref_available():
        O.build()
    names = sys.argv[1:] or list(CASES)
    for name in names:
        run_case(name, CASES[name])


if __name__ == "__main__":
    main()
