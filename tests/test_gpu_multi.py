"""Query sharding over several graph handles (vine_solve_multi).  This run
has one GPU, so the shares go to two handles of the same graph on device 0:
the split, the concurrent solves and the scatter back into query order are
the same code a multi-GPU machine runs (the solves never wait on each
other)."""
import numpy as np
import pytest

from golden_util import check_result, load_fixture

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nshares", [1, 2, 3])
def test_sharded_batch_matches_reference(nshares):
    import vine_b200 as v
    fx = load_fixture("road_batch_small")
    graphs = [v.Graph(fx["row_ptr"], fx["col"], fx["len"], fx["delay"], device=0)
              for _ in range(nshares)]
    # every handle sizes its own label arena; on one shared device they get a
    # fixed one so that all of them fit
    cfg = v.Config(use_bounds=1, pool_labels=1 << 24)
    res = v.solve_multi(graphs, fx["src"], fx["dst"], fx["budget"], cfg, stats=True)
    for q, e in enumerate(fx["queries"]):
        check_result(fx, res, q, e)
    one = v.solve(graphs[0], fx["src"], fx["dst"], fx["budget"], cfg)
    assert np.array_equal(res.cost, one.cost) and np.array_equal(res.found, one.found)
    assert (res.stats[:, v._lib.STAT_CYCLES] > 0).all()  # every query was solved by some share
    for g in graphs:
        g.close()


def test_sharded_batch_reports_per_query_errors():
    import vine_b200 as v
    fx = load_fixture("kat3")
    graphs = [v.Graph(fx["row_ptr"], fx["col"], fx["len"], fx["delay"]) for _ in range(2)]
    res = v.solve_multi(graphs, [0, 7, 0, 0], [2, 1, 2, 2], [100, 5, 4, 0],
                        v.Config(pool_labels=1 << 24), raise_on_error=False)
    assert res.status.tolist() == [0, v._lib.VINE_ERR_INVALID, 0, 0]
    assert res.cost[0] == 12 and res.cost[2] == 20 and res.found[3] == 0
    for g in graphs:
        g.close()
