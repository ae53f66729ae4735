"""GPU parity: the engine (through the C ABI) against the reference's results.

Golden values come from the reference's own RUN_CSPP_CPU (tests/golden);
costs and delays must match bit-exactly, returned paths must exist, respect
the budget and re-add to the reported cost and delay, and in Pareto mode the
sink Pareto set must equal the reference's final sink store."""
import numpy as np
import pytest

from golden_util import FIXTURES, check_result, csr_digest, load_fixture

pytestmark = pytest.mark.gpu

CONFIGS = {
    "batch_fixed": dict(engine="batch", policy="fixed"),
    "batch_ar": dict(engine="batch", policy="ar"),
    "batch_small_table": dict(engine="batch", table_log2=6, spill_log2=12, split_threshold=64),
    "batch_wide": dict(engine="batch", bucket_width=100000.0),
    "batch_narrow": dict(engine="batch", bucket_width=1.0, block_threads=128),
    "batch_bounds": dict(engine="batch", use_bounds=1),
    "batch_bounds_narrow": dict(engine="batch", use_bounds=1, bucket_width=5.0, block_threads=256),
    "batch_sync_rounds": dict(engine="batch", use_bounds=1, sync_rounds=1),
    "batch_sync_small": dict(engine="batch", sync_rounds=1, table_log2=6, split_threshold=64),
    # bucket opening through bulk-copied label tiles (tiles span several
    # bins; narrow buckets rebuild the band from the rest pile often)
    "batch_staged": dict(engine="batch", use_bounds=1, split_staging=1),
    "batch_staged_small": dict(engine="batch", split_staging=1, bucket_width=20.0, block_threads=256,
                               table_log2=8),
    "plain": dict(engine="plain"),
    "plain_bounds": dict(engine="plain", use_bounds=1),
}


@pytest.fixture(scope="module")
def graphs():
    import vine_b200 as v
    cache = {}

    def get(name):
        # one graph alive at a time: each holds its engines' device workspaces
        if name not in cache:
            for old in list(cache):
                cache.pop(old)[1].close()
            fx = load_fixture(name)
            assert csr_digest(fx["row_ptr"], fx["col"], fx["len"], fx["delay"]) == fx["digest"]
            cache[name] = (fx, v.Graph(fx["row_ptr"], fx["col"], fx["len"], fx["delay"]))
        return cache[name]
    yield get
    for fx, g in cache.values():
        g.close()


@pytest.mark.parametrize("cfg", list(CONFIGS))
@pytest.mark.parametrize("name", FIXTURES)
def test_optimal_matches_reference(graphs, name, cfg):
    import vine_b200 as v
    fx, g = graphs(name)
    res = v.solve(g, fx["src"], fx["dst"], fx["budget"], v.Config(**CONFIGS[cfg]))
    for q, expect in enumerate(fx["queries"]):
        check_result(fx, res, q, expect)


@pytest.mark.parametrize("engine", ["batch", "plain"])
@pytest.mark.parametrize("name", [f for f in FIXTURES if f != "road_batch_small"])
def test_pareto_set_matches_reference(graphs, name, engine):
    import vine_b200 as v
    fx, g = graphs(name)
    res = v.solve(g, fx["src"], fx["dst"], fx["budget"], v.Config(engine=engine, mode="pareto"),
                  pareto_stride=1024)
    for q, expect in enumerate(fx["queries"]):
        check_result(fx, res, q, expect)
        want = np.array(expect["pareto"], np.float32).reshape(-1, 2)
        got = res.pareto(q)
        assert res.pareto_n[q] == want.shape[0], f"q{q}: {res.pareto_n[q]} vs {want.shape[0]}"
        assert np.array_equal(got, want), f"q{q}: Pareto sets differ"


def test_repeat_calls_are_identical(graphs):
    import vine_b200 as v
    fx, g = graphs("grid")
    cfg = v.Config()
    a = v.solve(g, fx["src"], fx["dst"], fx["budget"], cfg)
    b = v.solve(g, fx["src"], fx["dst"], fx["budget"], cfg)
    assert np.array_equal(a.cost, b.cost) and np.array_equal(a.delay, b.delay)


def test_cspp_class_shim(graphs):
    import vine_b200 as v
    fx, g = graphs("kat3")
    n = len(fx["queries"])
    solver = v.cspp(g, n, [v.c_label(int(s)) for s in fx["src"]], list(map(int, fx["dst"])),
                    [v.c_constraint(float(b)) for b in fx["budget"]])
    assert solver.solve() == 0
    for q, e in enumerate(fx["queries"]):
        assert bool(solver.found_l[q]) == e["found"]
        if e["found"]:
            assert float(solver.cost_l[q]) == e["cost"]
            assert solver.size_of_result_l[q] == len(solver.path_l[q]) >= 1


def test_invalid_queries_get_status(graphs):
    import vine_b200 as v
    fx, g = graphs("kat3")
    res = v.solve(g, [0, 7, 0], [2, 1, -1], [100, 5, 5], raise_on_error=False)
    assert res.status[0] == 0 and res.found[0] == 1 and res.cost[0] == 12
    assert res.status[1] == v._lib.VINE_ERR_INVALID and res.found[1] == 0
    assert res.status[2] == v._lib.VINE_ERR_INVALID


@pytest.mark.parametrize("use_graph", [0, 1])
@pytest.mark.parametrize("name", ["road_small", "road_batch_small"])
def test_device_entry_matches_reference(graphs, name, use_graph):
    """vine_solve_device (device buffers, caller's stream, optionally a
    captured CUDA graph replayed on the second call) gives the same answers
    and packed paths as the host entry and the reference."""
    import torch
    import vine_b200 as v
    fx, g = graphs(name)
    nq = len(fx["queries"])
    dev = torch.device("cuda", 0)
    src = torch.from_numpy(np.asarray(fx["src"], np.int32)).to(dev)
    dst = torch.from_numpy(np.asarray(fx["dst"], np.int32)).to(dev)
    bud = torch.from_numpy(np.asarray(fx["budget"], np.float32)).to(dev)
    out = {"cost": torch.empty(nq, dtype=torch.float32, device=dev),
           "delay": torch.empty(nq, dtype=torch.float32, device=dev),
           "found": torch.empty(nq, dtype=torch.int32, device=dev),
           "status": torch.empty(nq, dtype=torch.int32, device=dev),
           "path_offsets": torch.empty(nq + 1, dtype=torch.int64, device=dev),
           "path": torch.empty(nq * 4096, dtype=torch.int32, device=dev)}
    cfg = v.Config(engine="batch", use_bounds=1, use_cuda_graph=use_graph)
    side = torch.cuda.Stream(dev)
    host = v.solve(g, fx["src"], fx["dst"], fx["budget"], cfg)
    for _ in range(2):
        for t in out.values():
            t.fill_(-7)
        with torch.cuda.stream(side):
            v.solve_device(g, src, dst, bud, out, cfg, side.cuda_stream)
        side.synchronize()
        r = v.Results(cost=out["cost"].cpu().numpy(), delay=out["delay"].cpu().numpy(),
                      found=out["found"].cpu().numpy(), status=out["status"].cpu().numpy())
        r.path_offsets = out["path_offsets"].cpu().numpy()
        r.path_vertices = out["path"].cpu().numpy()
        for q, expect in enumerate(fx["queries"]):
            check_result(fx, r, q, expect)
        assert np.array_equal(r.cost, host.cost) and np.array_equal(r.found, host.found)
        assert np.array_equal(r.path_offsets, host.path_offsets)
        total = int(r.path_offsets[nq])
        assert np.array_equal(r.path_vertices[:total], host.path_vertices[:total])


def test_empty_batch(graphs):
    import vine_b200 as v
    fx, g = graphs("kat3")
    res = v.solve(g, np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros(0, np.float32))
    assert res.rc == 0 and res.cost.shape == (0,) and res.path_offsets.shape == (1,)


@pytest.mark.parametrize("engine", ["batch", "plain"])
def test_repeated_queries_in_one_batch(graphs, engine):
    """Many workers solving copies of the same queries at once agree with
    each other and with the reference."""
    import vine_b200 as v
    fx, g = graphs("road_small")
    reps = 40 if engine == "batch" else 3
    nq = len(fx["queries"])
    src = np.tile(np.asarray(fx["src"], np.int32), reps)
    dst = np.tile(np.asarray(fx["dst"], np.int32), reps)
    bud = np.tile(np.asarray(fx["budget"], np.float32), reps)
    res = v.solve(g, src, dst, bud, v.Config(engine=engine, use_bounds=1))
    tiled = dict(fx, src=src, dst=dst, budget=bud)
    for k in range(reps * nq):
        # equal-cost paths may differ between copies; each must be valid
        check_result(tiled, res, k, fx["queries"][k % nq])
