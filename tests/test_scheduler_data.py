"""Host logic of the scheduler trainer (no GPU): how trace rows become
training examples."""
import numpy as np


def _traces(nq, rows_per_q, seed=0):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(3):
        q = np.repeat(np.arange(nq), rows_per_q)
        tr = np.zeros((q.size, 20), np.float32)
        tr[:, :16] = rng.normal(size=(q.size, 16))
        tr[:, 16] = q
        out.append(tr)
    return out


def test_labels_follow_the_best_multiplier_with_a_margin():
    from vine_b200 import scheduler as S
    settings = [0.5, 1.0, 2.0]
    # query 0: 0.5 saves 20 % -> label 0.5; query 1: 2.0 saves 2 % -> keeps 1.0
    cycles = np.array([[80.0, 120.0], [100.0, 100.0], [130.0, 98.0]])
    x, y = S.make_dataset(cycles, _traces(2, 50), settings, rows_per_setting=4000, seed=1)
    assert x.shape[1] == 16 and y.shape[1] == 2
    assert set(np.unique(y[:, 0]).tolist()) <= {np.log2(0.5), 0.0}
    # the gate is 1 exactly where the label departs from the AR rule's width
    assert np.array_equal(y[:, 1], (y[:, 0] != 0.0).astype(np.float32))
    # half the rows by query cost (query 0: 80 of 178), half uniform by query:
    # about 0.5 * 80 / 178 + 0.5 * 0.5 = 0.47 of the rows belong to query 0
    frac0 = float(np.mean(y[:, 0] == np.log2(0.5)))
    assert 0.40 < frac0 < 0.55


def test_rows_with_non_finite_features_are_dropped():
    from vine_b200 import scheduler as S
    tr = _traces(1, 20)
    for t in tr:
        t[::2, 3] = np.nan
    x, y = S.make_dataset(np.array([[1.0], [1.0], [1.0]]), tr, [0.5, 1.0, 2.0],
                          rows_per_setting=500, seed=2)
    assert np.isfinite(x).all() and np.isfinite(y).all() and x.shape[0] > 0


def test_auto_policy_needs_a_faster_median_and_no_worse_tail(tmp_path, monkeypatch):
    import json
    import bench
    from vine_b200 import scheduler as S

    def record(mlp_runs, ar_runs):
        def arm(runs):
            return {"ms": float(np.median(runs)), "ms_all": runs, "cycles": 1.0}
        meta = {"eval": {"fixed": arm([3000.0]), "ar": arm(ar_runs), "mlp": arm(mlp_runs)}}
        path = tmp_path / "m.json"
        path.write_text(json.dumps(meta))
        monkeypatch.setattr(S, "MODEL_JSON", path)
        monkeypatch.setattr(bench, "MODEL_PATH", path)
        return bench.scheduler_record()

    r = record([1600.0, 1610.0, 1620.0], [1670.0, 1671.0, 1672.0])
    assert r["mlp_faster"] and r["mlp_tail_ok"]
    r = record([1600.0, 1610.0, 5774.0], [1670.0, 1671.0, 1672.0])   # one blown-up run
    assert r["mlp_median_faster"] and not r["mlp_tail_ok"] and not r["mlp_faster"]
    r = record([1690.0, 1690.0, 1690.0], [1670.0, 1671.0, 1672.0])   # slower median
    assert r["mlp_tail_ok"] and not r["mlp_faster"]


def test_trainer_defaults_reproduce_the_shipped_network_recipe():
    """`python -m vine_b200.scheduler` with no options trains the network the
    way the committed one was trained (its record holds the recipe)."""
    import json
    from vine_b200 import scheduler as S
    meta = json.loads(S.MODEL_JSON.read_text())
    assert S.MARGIN == meta["margin"]
    parser_defaults = {}
    import argparse
    orig = argparse.ArgumentParser.parse_args

    def capture(self, argv=None, namespace=None):
        ns = orig(self, [], namespace)
        parser_defaults.update(vars(ns))
        raise SystemExit(0)
    try:
        argparse.ArgumentParser.parse_args = capture
        try:
            S.main([])
        except SystemExit:
            pass
    finally:
        argparse.ArgumentParser.parse_args = orig
    assert parser_defaults["margin"] == meta["margin"]
    assert parser_defaults["train_queries"] == meta["train_queries_c5"]
    assert [int(x) for x in parser_defaults["train_configs"].split(",")] == meta["train_configs"]
    assert parser_defaults["epochs"] == meta["epochs"]
    assert parser_defaults["eval_seed"] == meta["eval_seed"]
