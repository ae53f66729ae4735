"""The no-allocation loss / gradient entry point (vine_mlp_loss_grad_noalloc)
against the allocating one (vine_mlp_loss_grad), both called through the C
ABI.  Collected last on purpose: it must also pass after every other test
has run in the same process (scratch state left by earlier calls)."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _data(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.normal(0, 1.5, (n, 16)).astype(np.float32)
    y = rng.normal(0, 1.0, (n, 2)).astype(np.float32)
    return x, y


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def _noalloc(lib, m, x, y, stream=None):
    loss = np.zeros(1, np.float32)
    grad = np.full(_lib().MLP_PARAMS, np.nan, np.float32)
    rc = lib.vine_mlp_loss_grad_noalloc(m.handle, x.shape[0], _ptr(x), _ptr(y), _ptr(loss),
                                        _ptr(grad), stream)
    return rc, float(loss[0]), grad


def _lib():
    from vine_b200 import _lib
    return _lib


def _alloc(lib, m, x, y):
    loss = np.zeros(1, np.float32)
    grad = np.empty(_lib().MLP_PARAMS, np.float32)
    rc = lib.vine_mlp_loss_grad(m.handle, x.shape[0], _ptr(x), _ptr(y), _ptr(loss), _ptr(grad))
    assert rc == 0
    return float(loss[0]), grad


@pytest.mark.parametrize("n", [1, 257, 4096])
def test_noalloc_matches_allocating_entry_twice(n):
    import vine_b200 as v
    lib = v._lib.lib
    m = v.MLP(seed=21)
    x, y = _data(n, seed=n)
    want_loss, want_grad = _alloc(lib, m, x, y)
    scale = float(np.abs(want_grad).max())
    # two calls in a row: the second must not see the first's accumulators
    for _ in range(2):
        rc, loss, grad = _noalloc(lib, m, x, y)
        assert rc == 0, v._lib.lib.vine_last_error().decode()
        # same kernel, same data; only the order of float atomics differs
        assert abs(loss - want_loss) <= 1e-5 * max(1.0, abs(want_loss))
        np.testing.assert_allclose(grad, want_grad, rtol=1e-4, atol=1e-6 * scale)
    m.close()


def test_noalloc_on_a_caller_stream():
    import torch
    import vine_b200 as v
    lib = v._lib.lib
    m = v.MLP(seed=4)
    x, y = _data(300, seed=9)
    want_loss, want_grad = _alloc(lib, m, x, y)
    s = torch.cuda.Stream()
    rc, loss, grad = _noalloc(lib, m, x, y, C.c_void_p(s.cuda_stream))
    assert rc == 0
    assert abs(loss - want_loss) <= 1e-5 * max(1.0, abs(want_loss))
    np.testing.assert_allclose(grad, want_grad, rtol=1e-4, atol=1e-6 * float(np.abs(want_grad).max()))
    m.close()


def test_noalloc_rejects_sizes_beyond_the_scratch():
    import vine_b200 as v
    lib = v._lib.lib
    m = v.MLP(seed=1)
    limit = 4096  # VINE_MLP_NOALLOC_MAX_ROWS
    for n in (0, limit + 1):
        x, y = _data(max(n, 1), seed=3)
        loss = np.zeros(1, np.float32)
        grad = np.zeros(_lib().MLP_PARAMS, np.float32)
        rc = lib.vine_mlp_loss_grad_noalloc(m.handle, n, _ptr(x), _ptr(y), _ptr(loss), _ptr(grad),
                                            None)
        assert rc == v._lib.VINE_ERR_INVALID
        assert "4096" in v._lib.lib.vine_last_error().decode()
    m.close()


def test_noalloc_sees_new_parameters_on_a_caller_stream():
    """set_params followed directly by the no-allocation call on a
    non-blocking stream: the kernel must read the new parameters."""
    import torch
    import vine_b200 as v
    lib = v._lib.lib
    a, b = v.MLP(seed=5), v.MLP(seed=6)
    x, y = _data(512, seed=12)
    want_loss, want_grad = _alloc(lib, b, x, y)
    s = torch.cuda.Stream()
    a.params = b.params  # no call that synchronises in between
    rc, loss, grad = _noalloc(lib, a, x, y, C.c_void_p(s.cuda_stream))
    assert rc == 0
    assert abs(loss - want_loss) <= 1e-5 * max(1.0, abs(want_loss))
    np.testing.assert_allclose(grad, want_grad, rtol=1e-4, atol=1e-6 * float(np.abs(want_grad).max()))
    a.close()
    b.close()


def test_noalloc_makes_no_device_allocation():
    """After one warm-up call, repeated calls leave the device's free memory
    unchanged (nothing is allocated, cached or freed per call)."""
    import torch
    import vine_b200 as v
    lib = v._lib.lib
    m = v.MLP(seed=8)
    x, y = _data(4096, seed=13)
    assert _noalloc(lib, m, x, y)[0] == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for n in (1, 100, 4096, 2048, 4096):
        rc, _, _ = _noalloc(lib, m, x[:n], y[:n])
        assert rc == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, f"free device memory moved by {free0 - free1} bytes"
    m.close()
