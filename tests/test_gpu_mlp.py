"""The learned scheduler's network on the GPU against the FP64 CPU oracle
(oracle/mlp_ref.py): forward outputs, loss and every parameter gradient of
the hand-written backward kernel, one Adam step, and that training lowers
the loss.  Then the scheduler inside the engine: answers under the MLP
policy are bit-identical to the reference's, whatever the network predicts.
"""
import numpy as np
import pytest

from golden_util import check_result, load_fixture

pytestmark = pytest.mark.gpu


def _data(n=300, seed=3):
    rng = np.random.default_rng(seed)
    x = rng.normal(0, 1.5, (n, 16)).astype(np.float32)
    y = np.stack([np.sin(x[:, 0]) + 0.3 * x[:, 3], 0.5 * x[:, 1] - 0.2 * x[:, 7]], 1).astype(np.float32)
    return x, y


def test_forward_matches_fp64():
    import vine_b200 as v
    from oracle import mlp_ref
    x, _ = _data()
    m = v.MLP(seed=11)
    got = m.forward(x)
    want, _ = mlp_ref.forward(m.params, x)
    # FP32 dot products of length <= 64 against FP64: relative 1e-4
    np.testing.assert_allclose(got, want, rtol=1e-4, atol=1e-4)


def test_loss_and_gradient_match_fp64():
    import vine_b200 as v
    from oracle import mlp_ref
    x, y = _data(n=257)  # not a multiple of the 32-row tile
    m = v.MLP(seed=5)
    loss, grad = m.loss_grad(x, y)
    wl, wg = mlp_ref.loss_grad(m.params, x, y)
    assert abs(loss - wl) <= 1e-4 * max(1.0, abs(wl))
    scale = np.abs(wg).max()
    np.testing.assert_allclose(grad, wg, rtol=2e-3, atol=2e-5 * scale)


def test_adam_step_matches_fp64():
    import vine_b200 as v
    from oracle import mlp_ref
    x, y = _data(n=128)
    m = v.MLP(seed=7)
    p0 = m.params.astype(np.float64)
    _, g = mlp_ref.loss_grad(p0, x, y)
    m.train(x, y, epochs=1, batch=128, lr=1e-3, seed=0)  # one full-batch step
    p1, _, _ = mlp_ref.adam_step(p0, np.zeros_like(p0), np.zeros_like(p0), g, 1, 1e-3)
    # step 1 of Adam moves each parameter by ~lr*sign(g); where |g| is near
    # FP32 noise the sign is not defined, so those parameters are skipped
    ok = np.abs(g) > 1e-4 * np.abs(g).max()
    np.testing.assert_allclose(m.params[ok], p1[ok], rtol=0, atol=2e-5)


def test_training_reduces_loss():
    import vine_b200 as v
    x, y = _data(n=4096)
    m = v.MLP(seed=1)
    before, _ = m.loss_grad(x, y)
    after = m.train(x, y, epochs=40, batch=256, lr=3e-3, seed=2)
    assert after < 0.25 * before, (before, after)


@pytest.mark.parametrize("name", ["road_small", "road_batch_small", "chunglu_small"])
@pytest.mark.parametrize("seed", [0, 9])
def test_mlp_policy_is_exact(name, seed):
    """Random (untrained) networks only reorder work: answers stay exact."""
    import vine_b200 as v
    fx = load_fixture(name)
    g = v.Graph(fx["row_ptr"], fx["col"], fx["len"], fx["delay"])
    try:
        m = v.MLP(seed=seed)
        res = v.solve(g, fx["src"], fx["dst"], fx["budget"],
                      v.Config(engine="batch", policy="mlp", mlp=m, use_bounds=1))
        for q, e in enumerate(fx["queries"]):
            check_result(fx, res, q, e)
    finally:
        g.close()


def test_trained_scheduler_is_exact():
    """The committed trained network, if present, keeps answers exact."""
    import vine_b200 as v
    from vine_b200 import scheduler
    m, meta = scheduler.load()
    if m is None:
        pytest.skip("no trained scheduler committed")
    fx = load_fixture("road_batch_small")
    g = v.Graph(fx["row_ptr"], fx["col"], fx["len"], fx["delay"])
    try:
        cfg = scheduler.base_config(float(np.mean(fx["len"])), policy="mlp", mlp=m)
        res = v.solve(g, fx["src"], fx["dst"], fx["budget"], cfg)
        for q, e in enumerate(fx["queries"]):
            check_result(fx, res, q, e)
    finally:
        g.close()
