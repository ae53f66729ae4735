"""GPU tests of the failure paths, made without faulting the device.

* Capacity: per-worker structures sized too small for some queries make them
  fail with VINE_ERR_CAPACITY (an abort-site code says where); vine_solve
  solves those again with roomier structures (`retried`) and every answer
  still equals the reference's.  The device entry, which does not retry,
  reports the per-query status.
* Time and wait limits: `time_limit_ms` and `wait_limit` set tiny make
  queries stop with VINE_ERR_TIMEOUT instead of running on; the call returns,
  statuses are readable, and the next call on the same graph is correct.
"""
import numpy as np
import pytest

from golden_util import check_result, load_fixture

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    import vine_b200 as v
    return v


def _graph(v, name):
    fx = load_fixture(name)
    return fx, v.Graph(fx["row_ptr"], fx["col"], fx["len"], fx["delay"])


def _device_solve(v, g, fx, cfg):
    import torch
    dev = torch.device("cuda", 0)
    nq = len(fx["queries"])
    src = torch.from_numpy(np.asarray(fx["src"], np.int32)).to(dev)
    dst = torch.from_numpy(np.asarray(fx["dst"], np.int32)).to(dev)
    bud = torch.from_numpy(np.asarray(fx["budget"], np.float32)).to(dev)
    out = {"cost": torch.empty(nq, dtype=torch.float32, device=dev),
           "delay": torch.empty(nq, dtype=torch.float32, device=dev),
           "found": torch.empty(nq, dtype=torch.int32, device=dev),
           "status": torch.empty(nq, dtype=torch.int32, device=dev),
           "stats": torch.zeros((nq, v._lib.STAT_COUNT), dtype=torch.int64, device=dev)}
    v.solve_device(g, src, dst, bud, out, cfg)
    torch.cuda.synchronize()
    return {k: t.cpu().numpy() for k, t in out.items()}


def test_arena_overflow_is_retried_and_exact(lib):
    """An arena of 2^20 labels holds 16 of the 65,536-label chunks the
    workers take; the other queries overflow it, are solved again with a
    4x arena, and all 32 answers equal the reference's."""
    v = lib
    fx, g = _graph(v, "road_batch_small")
    cfg = v.Config(pool_labels=1 << 20)
    res = v.solve(g, fx["src"], fx["dst"], fx["budget"], cfg, stats=True)
    assert res.retried > 0, "no query overflowed the small arena"
    for q, e in enumerate(fx["queries"]):
        check_result(fx, res, q, e)
    dev = _device_solve(v, g, fx, cfg)
    cap = dev["status"] == v._lib.VINE_ERR_CAPACITY
    assert cap.any()
    assert set(dev["stats"][cap, v._lib.STAT_ABORT_SITE].tolist()) <= {1, 2}  # arena sites
    ok = dev["status"] == 0
    assert ok.any() and (ok | cap).all()
    for q in np.nonzero(ok)[0]:
        e = fx["queries"][q]
        assert bool(dev["found"][q]) == e["found"]
        if e["found"]:
            assert (float(dev["cost"][q]), float(dev["delay"][q])) == (e["cost"], e["delay"])
    g.close()


@pytest.mark.parametrize("name,far", [("chunglu_small", 2048), ("road_batch_small", 1024)])
def test_far_pile_overflow_is_retried_and_exact(lib, name, far):
    """Far piles of `far` labels per worker (the minimum allowed is 1024):
    queries whose pending labels outgrow them fail with VINE_ERR_CAPACITY at
    a pile site and are solved again with 8x piles, which hold every label
    such a query inserts; every answer equals the reference's."""
    v = lib
    fx, g = _graph(v, name)
    cfg = v.Config(far_capacity=far, use_bounds=0)
    res = v.solve(g, fx["src"], fx["dst"], fx["budget"], cfg)
    for q, e in enumerate(fx["queries"]):
        check_result(fx, res, q, e)
    # the device entry does not retry: the same overflows show as statuses
    # (their number can differ by a few from the host entry's first attempt:
    # how full the piles get depends on the order the warps run in)
    dev = _device_solve(v, g, fx, cfg)
    cap = dev["status"] == v._lib.VINE_ERR_CAPACITY
    assert set(dev["status"].tolist()) <= {0, v._lib.VINE_ERR_CAPACITY}
    assert set(dev["stats"][cap, v._lib.STAT_ABORT_SITE].tolist()) <= {4, 5}  # band / rest
    if res.retried > 0:
        assert cap.any()
    g.close()
    if name == "chunglu_small":
        assert res.retried > 0, "no query overflowed the small far piles"


def test_time_limit_stops_queries(lib):
    """time_limit_ms = 1 on the 10,000-vertex grid (queries insert up to
    1.5M labels): queries stop with VINE_ERR_TIMEOUT at the time site; the
    ones that finished are exact; the next call without the limit is exact."""
    v = lib
    fx, g = _graph(v, "grid")
    res = v.solve(g, fx["src"], fx["dst"], fx["budget"], v.Config(time_limit_ms=1), stats=True,
                  raise_on_error=False)
    st = res.status
    assert set(st.tolist()) <= {0, v._lib.VINE_ERR_TIMEOUT}
    late = st == v._lib.VINE_ERR_TIMEOUT
    assert late.any()
    assert set(res.stats[late, v._lib.STAT_ABORT_SITE].tolist()) == {v._lib.SITE_TIME}
    assert (res.found[late] == 0).all()
    for q in np.nonzero(~late)[0]:
        check_result(fx, res, q, fx["queries"][q])
    again = v.solve(g, fx["src"], fx["dst"], fx["budget"], v.Config())
    for q, e in enumerate(fx["queries"]):
        check_result(fx, again, q, e)
    g.close()


@pytest.mark.parametrize("engine", ["batch", "plain"])
def test_time_limit_on_both_engines(lib, engine):
    v = lib
    fx, g = _graph(v, "grid")
    n = 4
    res = v.solve(g, fx["src"][:n], fx["dst"][:n], fx["budget"][:n],
                  v.Config(engine=engine, time_limit_ms=1), stats=True, raise_on_error=False)
    assert (res.status == v._lib.VINE_ERR_TIMEOUT).any()
    assert set(res.status.tolist()) <= {0, v._lib.VINE_ERR_TIMEOUT}
    g.close()


def test_wait_limit_stops_waits(lib):
    """wait_limit = 1: a warp that finds the bucket queue empty while other
    warps still expand gives up at once, so queries fail with
    VINE_ERR_TIMEOUT at a wait site instead of waiting; the next call with the
    default limit is exact."""
    v = lib
    fx, g = _graph(v, "grid")
    res = v.solve(g, fx["src"], fx["dst"], fx["budget"], v.Config(wait_limit=1), stats=True,
                  raise_on_error=False)
    st = res.status
    assert set(st.tolist()) <= {0, v._lib.VINE_ERR_TIMEOUT}
    late = st == v._lib.VINE_ERR_TIMEOUT
    assert late.any()
    sites = set(res.stats[late, v._lib.STAT_ABORT_SITE].tolist())
    assert sites <= {v._lib.SITE_LOCK, v._lib.SITE_ASYNC, 1}  # 1: arena chunk wait
    for q in np.nonzero(~late)[0]:
        check_result(fx, res, q, fx["queries"][q])
    again = v.solve(g, fx["src"], fx["dst"], fx["budget"], v.Config())
    for q, e in enumerate(fx["queries"]):
        check_result(fx, again, q, e)
    g.close()


def test_limits_are_validated(lib):
    v = lib
    fx, g = _graph(v, "kat3")
    with pytest.raises(v.VineError):
        v.solve(g, fx["src"], fx["dst"], fx["budget"], v.Config(wait_limit=-3))
    res = v.solve(g, fx["src"], fx["dst"], fx["budget"], v.Config(time_limit_ms=-1))  # no limit
    for q, e in enumerate(fx["queries"]):
        check_result(fx, res, q, e)
    g.close()
