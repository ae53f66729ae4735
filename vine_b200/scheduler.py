"""Learned bucket scheduler: trace collection, training and evaluation.

The batch engine chooses, at every bucket boundary of every query, the width
of the next bucket.  The reference sets it with an AR forecast of bucket
sizes (algorithm/cspp.cuh:254-284): widen 1.5x while sizes fall, otherwise
steer the forecast size to a quarter of the shared table.  Here a 16-64-64-2
FP32 MLP, evaluated by one warp inside the persistent kernel, scales the AR
rule's width for the next bucket by 2^y (y clamped to [-1.5, 1.5]) from 16
frontier statistics.  It only changes how work is grouped into buckets, so
answers stay exact whatever it predicts.

Training data comes from the plain method itself: the engine runs query sets
under the AR policy with every global width multiplier in SCALES
(vine_config.ar_scale), with tracing on.  Each trace row holds the 16
features the scheduler saw when a bucket was opened.  For every query the
multiplier with the fewest SM cycles (VINE_STAT_CYCLES) is its label, kept
at the AR rule's own width (1) unless another saves at least MARGIN of the
query's cycles; every trace row of that query, from every run, becomes one
training example: features -> (log2(best multiplier), gate), gate = 1 when
the best multiplier is not the AR rule's.  The kernel applies the first
output only where the second says the departure pays: a network that
strays on a query it does not know falls back to the AR rule there (an
ungated network made a few mid-sized queries several times slower, and
those, started late in the longest-first order, stretched the batch).
Rows from all runs keep the network from reading the answer off the width
feature.  Training runs on the GPU through libvine's own forward/backward
and Adam kernels.

Usage: ``python -m vine_b200.scheduler [--train-configs 1,2,5] [--eval-configs 5,3]``
Training traces come from the 100x100 grid (config 1), the 264k-vertex road
graph's random pairs (config 2) and a hop-sampled batch on the same graph
with its own query seed (config 5); evaluation runs on a held-out 4096-query
batch (config 5, another seed) and on the 1.5M-vertex anti-correlated road
graph (config 3).  Writes vine_b200/models/scheduler_mlp.npy and
scheduler_mlp.json.
"""
from __future__ import annotations

import argparse
import json
import time
from pathlib import Path

import numpy as np

from . import api as v

SCALES = (0.35, 0.5, 0.7, 1.0, 1.4, 2.0, 2.8)  # multipliers on the AR width
BASE_MULT = 0.3          # initial bucket width / mean arc length
MARGIN = 0.03            # a multiplier other than 1 must save this share of a query's cycles
TABLE_LOG2 = 13
MODEL_DIR = Path(__file__).resolve().parent / "models"
MODEL_NPY = MODEL_DIR / "scheduler_mlp.npy"
MODEL_JSON = MODEL_DIR / "scheduler_mlp.json"

STAT_CYCLES = 7  # VINE_STAT_CYCLES


def base_config(mean_len: float, **kw):
    """Batch engine settings shared by every arm of the comparison."""
    d = dict(engine="batch", use_bounds=1, block_threads=512, table_log2=TABLE_LOG2,
             bucket_width=BASE_MULT * mean_len)
    d.update(kw)
    return v.Config(**d)


def collect(graph: v.Graph, src, dst, budget, mean_len: float):
    """Runs the AR policy at every multiplier in SCALES with tracing on.
    Returns (cycles[setting, q], traces: list of arrays, settings)."""
    settings = list(SCALES)
    cycles = np.zeros((len(settings), len(src)), np.float64)
    traces = []
    for k, sc in enumerate(settings):
        cfg = base_config(mean_len, policy="ar", ar_scale=sc, trace=1)
        r = v.solve(graph, src, dst, budget, cfg, paths=False, stats=True)
        cycles[k] = r.stats[:, STAT_CYCLES]
        traces.append(v.fetch_trace(graph))
    return cycles, traces, settings


def make_dataset(cycles, traces, settings, rows_per_setting: int = 200000, seed: int = 0,
                 margin: float = MARGIN):
    """Features of every trace row -> (log2 of the best multiplier of the
    row's query, gate).  A query keeps the AR rule's own width (multiplier
    1, gate 0) unless another multiplier saves at least `margin` of its
    cycles (gate 1), so the network departs from the rule it refines only
    where that clearly pays.  Half of the rows are drawn with probability
    proportional to their query's cost (the heavy queries decide most of a
    batch's time), half uniformly over queries (so the light and mid-sized
    ones, which run late in a longest-first batch, are learnt too)."""
    best = np.argmin(cycles, axis=0)
    ar = settings.index(1.0)
    keep_ar = cycles[best, np.arange(cycles.shape[1])] > (1.0 - margin) * cycles[ar]
    best = np.where(keep_ar, ar, best)
    qcost = cycles.min(axis=0)
    rng = np.random.default_rng(seed)
    xs, ys = [], []
    for tr in traces:
        if tr.shape[0] == 0:
            continue
        q = tr[:, 16].astype(np.int64)
        rows_of_q = np.maximum(np.bincount(q, minlength=cycles.shape[1]).astype(np.float64), 1.0)
        p_cost = qcost[q] / rows_of_q[q]
        p_query = 1.0 / rows_of_q[q]
        p = 0.5 * p_cost / p_cost.sum() + 0.5 * p_query / p_query.sum()
        tr = tr[rng.choice(tr.shape[0], min(rows_per_setting, 4 * tr.shape[0]), replace=True, p=p)]
        q = tr[:, 16].astype(np.int64)
        sc = np.array([settings[b] for b in best[q]], np.float32)
        gate = (best[q] != ar).astype(np.float32)
        xs.append(tr[:, :16])
        ys.append(np.stack([np.log2(sc), gate], axis=1))
    x = np.concatenate(xs).astype(np.float32)
    y = np.concatenate(ys).astype(np.float32)
    ok = np.isfinite(x).all(1) & np.isfinite(y).all(1)
    return x[ok], y[ok]


def train(x, y, device: int = 0, epochs: int = 30, batch: int = 512, lr: float = 1e-3,
          seed: int = 0):
    mlp = v.MLP(device=device, seed=seed)
    loss0, _ = mlp.loss_grad(x[:65536], y[:65536])
    loss = mlp.train(x, y, epochs=epochs, batch=batch, lr=lr, seed=seed)
    return mlp, float(loss0), float(loss)


def evaluate(graph: v.Graph, src, dst, budget, mean_len: float, mlp, repeats: int = 5,
             answers=None, warm_up: bool = True):
    """Times the batch engine under the fixed, AR and MLP policies (same base
    width); returns {policy: {ms, cycles, expanded}} and checks every arm
    returns identical costs.  The arms are interleaved (fixed, AR, MLP,
    fixed, AR, ...) and each arm's time is the median of its runs, so a
    drift of the machine's speed during the evaluation does not favour one
    arm."""
    import torch
    out = {}
    arms = {"fixed": base_config(mean_len, policy="fixed"),
            "ar": base_config(mean_len, policy="ar")}
    if mlp is not None:
        arms["mlp"] = base_config(mean_len, policy="mlp", mlp=mlp)
    if warm_up:
        for cfg in arms.values():
            v.solve(graph, src, dst, budget, cfg, paths=False)
    times = {name: [] for name in arms}
    last = {}
    for _ in range(repeats):
        for name, cfg in arms.items():
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            r = v.solve(graph, src, dst, budget, cfg, paths=False, stats=True)
            times[name].append((time.perf_counter() - t0) * 1e3)
            last[name] = r
    ref = answers
    for name, r in last.items():
        if ref is None:
            ref = (r.cost.copy(), r.found.copy())
        same = bool(np.array_equal(r.found, ref[1]) and
                    np.array_equal(np.where(r.found == 1, r.cost, 0), np.where(ref[1] == 1, ref[0], 0)))
        out[name] = {"ms": float(np.median(times[name])),
                     "ms_all": [round(t, 1) for t in times[name]],
                     "retried": int(r.retried),
                     "cycles": float(r.stats[:, STAT_CYCLES].sum()),
                     "cycles_max": float(r.stats[:, STAT_CYCLES].max()),
                     "expanded": int(r.stats[:, 0].sum()), "rounds": int(r.stats[:, 5].sum()),
                     "same_answers": same}
    return out


def save(mlp, meta: dict):
    MODEL_DIR.mkdir(exist_ok=True)
    np.save(MODEL_NPY, mlp.params)
    MODEL_JSON.write_text(json.dumps(meta, indent=1, sort_keys=True) + "\n")


def load(device: int = 0):
    """The trained scheduler (or None) and its metadata."""
    if not MODEL_NPY.exists():
        return None, {}
    meta = json.loads(MODEL_JSON.read_text()) if MODEL_JSON.exists() else {}
    return v.MLP(device=device, params=np.load(MODEL_NPY)), meta


def _evaluate_batch(a, mlp, config: int):
    """Fixed / AR / network on a whole batch (config 5: drawn with its own
    query seed, held out from training and from the bench batch)."""
    over = {"n_pairs": a.eval_queries, "query_seed": a.eval_seed} if config == 5 else {}
    ev = v.Workload.generate(config, **over)
    n = len(ev.src)
    ge = ev.graph()
    # the 1.5M-vertex batch takes minutes per arm: one timed run each
    heavy = config == 3
    res = evaluate(ge, ev.src, ev.dst, ev.budget, float(ev.len.mean()), mlp,
                   repeats=1 if heavy else 5, warm_up=not heavy)
    ge.close()
    return res, n


def _evaluate_all(a, mlp) -> dict:
    out = {}
    for cfg in a.eval_configs:
        res, n = _evaluate_batch(a, mlp, cfg)
        out[str(cfg)] = dict(res, queries=n)
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--train-configs", default="1,2,5",
                    help="workloads whose traces train the network")
    ap.add_argument("--train-queries", type=int, default=4096,
                    help="queries of the config-5 training batch")
    ap.add_argument("--train-queries-c3", type=int, default=48,
                    help="queries of a config-3 training batch (own query seed), when 3 is "
                         "among the training configs")
    ap.add_argument("--train-seed", type=int, default=0x7EA1,
                    help="query seed of the training batch (the bench batch uses the default seed)")
    ap.add_argument("--eval-configs", default="5,3",
                    help="held-out evaluation workloads (the first one decides `mlp_faster`)")
    ap.add_argument("--eval-queries", type=int, default=4096)
    ap.add_argument("--eval-seed", type=int, default=0xE7A1,
                    help="query seed of the evaluation batch (neither the training nor the bench batch)")
    ap.add_argument("--eval-only", action="store_true",
                    help="re-evaluate the committed network without training")
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--margin", type=float, default=MARGIN,
                    help="share of a query's cycles another multiplier must save to be its label")
    ap.add_argument("--model-dir", default=None,
                    help="write the network and its record here instead of vine_b200/models")
    ap.add_argument("--out", default=None, help="write the evaluation JSON here")
    a = ap.parse_args(argv)
    a.eval_configs = [int(x) for x in a.eval_configs.split(",") if x]
    a.train_configs = [int(x) for x in a.train_configs.split(",") if x]

    t0 = time.time()
    if a.eval_only:
        mlp, meta = load()
        if mlp is None:
            raise SystemExit("no trained scheduler to evaluate")
        ev = _evaluate_all(a, mlp)
        first = ev[str(a.eval_configs[0])]
        by_config = dict(meta.get("eval_by_config", {}))
        by_config.update(ev)  # configs not re-evaluated keep their record
        meta.update({"eval_config": a.eval_configs[0], "eval_queries": first["queries"],
                     "eval_seed": a.eval_seed,
                     "eval": {k: v_ for k, v_ in first.items() if k != "queries"},
                     "eval_by_config": by_config})
        MODEL_JSON.write_text(json.dumps(meta, indent=1, sort_keys=True) + "\n")
        text = json.dumps(meta, indent=1, sort_keys=True)
        if a.out:
            Path(a.out).write_text(text + "\n")
        print(text)
        return
    xs, ys, per_config = [], [], {}
    for tc in a.train_configs:
        over = {}
        if tc == 5:
            over = {"n_pairs": a.train_queries, "query_seed": a.train_seed}
        elif tc == 3:  # the 1.5M-vertex graph: a small batch with its own query seed
            over = {"n_pairs": a.train_queries_c3, "query_seed": a.train_seed}
        wl = v.Workload.generate(tc, **over)
        g = wl.graph()
        cycles, traces, settings = collect(g, wl.src, wl.dst, wl.budget, float(wl.len.mean()))
        g.close()
        x, y = make_dataset(cycles, traces, settings, margin=a.margin)
        xs.append(x)
        ys.append(y)
        best = np.argmin(cycles, axis=0)
        static_best = int(np.argmin(cycles.sum(1)))
        per_config[str(tc)] = {
            "queries": int(len(wl.src)), "rows": int(x.shape[0]),
            "best_setting_histogram": {str(settings[k]): int((best == k).sum())
                                       for k in range(len(settings))},
            "gate_share": float(y[:, 1].mean()),
            "best_static_setting": settings[static_best],
            "oracle_best_per_query_cycles": float(cycles.min(0).sum()),
            "best_static_cycles": float(cycles[static_best].sum()),
            "ar_cycles": float(cycles[settings.index(1.0)].sum())}
    x = np.concatenate(xs)
    y = np.concatenate(ys)
    perm = np.random.default_rng(1).permutation(x.shape[0])
    x, y = x[perm], y[perm]
    mlp, loss0, loss = train(x, y, epochs=a.epochs)

    ev = _evaluate_all(a, mlp)
    first = ev[str(a.eval_configs[0])]
    meta = {"base_mult": BASE_MULT, "table_log2": TABLE_LOG2, "block_threads": 512,
            "margin": a.margin, "train_configs": a.train_configs, "rows": int(x.shape[0]),
            "train_queries_c5": a.train_queries,
            "loss_initial": loss0, "loss_final": loss, "epochs": a.epochs,
            "training": per_config,
            "eval_config": a.eval_configs[0], "eval_queries": first["queries"],
            "eval_seed": a.eval_seed,
            "eval": {k: v_ for k, v_ in first.items() if k != "queries"},
            "eval_by_config": ev,
            "seconds": time.time() - t0}
    if a.model_dir:
        d = Path(a.model_dir)
        d.mkdir(parents=True, exist_ok=True)
        np.save(d / MODEL_NPY.name, mlp.params)
        (d / MODEL_JSON.name).write_text(json.dumps(meta, indent=1, sort_keys=True) + "\n")
    else:
        save(mlp, meta)
    text = json.dumps(meta, indent=1, sort_keys=True)
    if a.out:
        Path(a.out).write_text(text + "\n")
    print(text)


if __name__ == "__main__":
    main()
