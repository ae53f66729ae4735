"""The batch-engine autotuner: it times its candidate settings on a sample of
queries, returns the fastest one that solved every query, caches it per graph
(a second call reads the cache instead of timing again), and the settings it
returns give the reference's answers."""
import time

import numpy as np
import pytest

from golden_util import check_result, load_fixture

pytestmark = pytest.mark.gpu


def test_autotune_picks_a_candidate_and_caches_it(tmp_path):
    import vine_b200 as v
    fx = load_fixture("road_batch_small")
    g = v.Graph(fx["row_ptr"], fx["col"], fx["len"], fx["delay"])
    try:
        cache = str(tmp_path / "tune.txt")
        base = v.Config(engine="batch", use_bounds=1)
        best = v.autotune(g, fx["src"], fx["dst"], fx["budget"], base, cache_path=cache)
        d = v.config_dict(best)
        assert d["block_threads"] == 512 and d["table_log2"] in (12, 13)
        assert d["band_mult"] in (8, 16)
        mean_len = float(np.mean(fx["len"]))
        assert any(abs(d["bucket_width"] - m * mean_len) <= 1e-4 * mean_len for m in (0.2, 0.3, 0.5))
        lines = open(cache).read().splitlines()
        assert len(lines) == 1 and "|" in lines[0]
        t0 = time.perf_counter()
        again = v.autotune(g, fx["src"], fx["dst"], fx["budget"], base, cache_path=cache)
        assert time.perf_counter() - t0 < 1.0  # read from the cache, not timed again
        assert v.config_dict(again) == d
        assert len(open(cache).read().splitlines()) == 1
        res = v.solve(g, fx["src"], fx["dst"], fx["budget"], best)
        for q, e in enumerate(fx["queries"]):
            check_result(fx, res, q, e)
    finally:
        g.close()
