"""The learned closure's network: the numpy oracle (oracle/mlp_oracle.py) pinned by finite
differences and torch's BF16 rounding; the tensor-core forward, gradient and training
kernels (rw_mlp_*) checked against it."""
import numpy as np
import pytest

from oracle import mlp_oracle as M


def _params(seed):
    rng = np.random.default_rng(seed)
    p = np.zeros(M.NPARAM)
    for off, shp in M.SHAPES:
        n = int(np.prod(shp))
        a = np.sqrt(6.0 / sum(shp)) if len(shp) == 2 else 0.1
        p[off:off + n] = rng.uniform(-a, a, n)
    return p.astype(np.float32)


def _features(n, seed):
    """Inputs shaped like the closure's features: stress ratios around a geostatic
    state, unit strain-rate directions, relative void ratio in [0, 1], friction angle."""
    rng = np.random.default_rng(seed)
    x = np.zeros((n, 16), np.float32)
    x[:, 0:3] = -1.0 + 0.3 * rng.standard_normal((n, 3))
    x[:, 3:6] = 0.2 * rng.standard_normal((n, 3))
    d = rng.standard_normal((n, 6))
    x[:, 6:12] = d / np.linalg.norm(d, axis=1, keepdims=True)
    x[:, 12] = rng.uniform(0.0, 1.0, n)
    x[:, 13] = rng.uniform(-1.0, 1.0, n)
    return x


def _target(x):
    """A smooth synthetic target with the closure's output shape."""
    s, d = x[:, 0:6], x[:, 6:12]
    t = -0.4 * d + 0.3 * s * d.sum(1, keepdims=True) + 0.5 * (s * (0.5 + 0.5 * x[:, 12:13] ** 0.18))
    return (t * (1.0 + 0.2 * x[:, 13:14])).astype(np.float32)


def test_bf16_rounding_matches_torch():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(0)
    a = np.concatenate([rng.standard_normal(10000).astype(np.float32),
                        np.float32([1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -1.0 - 2 ** -8, 0.0, 65504.0])])
    ref = torch.from_numpy(a).to(torch.bfloat16).float().numpy()
    np.testing.assert_array_equal(M.bf16(a), ref)


def test_oracle_gradient_matches_finite_differences():
    p = _params(3).astype(np.float64)
    x = _features(24, 4).astype(np.float64)
    t = _target(x.astype(np.float32)).astype(np.float64)
    _, g = M.loss_grad(p, x, t, emulate=False)
    rng = np.random.default_rng(5)
    idx = np.concatenate([rng.choice(M.NPARAM, 60, replace=False), [M.P_B5, M.P_B1 + 3, M.P_W5 + 7]])
    eps = 1e-6
    for k in idx:
        q = p.copy()
        q[k] += eps
        lp, _ = M.loss_grad(q, x, t, emulate=False)
        q[k] -= 2 * eps
        lm, _ = M.loss_grad(q, x, t, emulate=False)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(g[k])) + 1e-9, (k, fd, g[k])


def test_emulated_arithmetic_close_to_float64():
    p = _params(7)
    x = _features(512, 8)
    t = _target(x)
    y32, _ = M.forward(p, x, emulate=True)
    y64, _ = M.forward(p, x, emulate=False)
    assert np.linalg.norm(y32 - y64) / np.linalg.norm(y64) < 2e-2
    l32, g32 = M.loss_grad(p, x, t, emulate=True)
    l64, g64 = M.loss_grad(p, x, t, emulate=False)
    assert abs(l32 - l64) / l64 < 2e-2
    assert np.linalg.norm(g32 - g64) / np.linalg.norm(g64) < 5e-2


def _block_errors(g, ref):
    errs = {}
    for off, shp in M.SHAPES:
        n = int(np.prod(shp))
        a, b = g[off:off + n], ref[off:off + n]
        errs[off] = float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))
    return errs


@pytest.mark.gpu
def test_params_roundtrip_and_forward_vs_oracle():
    from retainwall_code_b200.closure import Mlp

    net = Mlp(seed=11)
    p = _params(12)
    net.set_params(p)
    np.testing.assert_array_equal(net.params(), p)
    x = _features(3000, 13)  # 24 tiles minus a partial one
    y = net.forward(x)
    ye, _ = M.forward(p, x, emulate=True)
    y64, _ = M.forward(p, x, emulate=False)
    assert np.linalg.norm(y - ye) / np.linalg.norm(ye) < 3e-3
    assert np.linalg.norm(y - y64) / np.linalg.norm(y64) < 2e-2
    net.close()


@pytest.mark.gpu
def test_gradient_vs_oracle():
    """The tensor-core backward pass (dH = G W on tcgen05, dW and db on the CUDA
    cores) against the oracle's emulation of the same BF16 / FP32 arithmetic, block by
    block, and against float64."""
    from retainwall_code_b200.closure import Mlp

    net = Mlp(seed=21)
    p = _params(22)
    net.set_params(p)
    x = _features(1000, 23)
    t = _target(x)
    loss, g = net.grad(x, t)
    le, ge = M.loss_grad(p, x, t, emulate=True)
    l64, g64 = M.loss_grad(p, x, t, emulate=False)
    assert abs(loss - le) <= 1e-3 * le
    for off, e in _block_errors(g, ge).items():
        assert e < 2e-2, (off, e)
    assert np.linalg.norm(g - g64) / np.linalg.norm(g64) < 5e-2
    net.close()


@pytest.mark.gpu
def test_training_fits_a_smooth_target():
    from retainwall_code_b200.closure import Mlp

    net = Mlp(seed=31, sample_capacity=200_000)
    x = _features(160_000, 32)
    t = _target(x)
    net.add_samples(x, t)
    assert net.sample_count() == 160_000
    xs, ts = net.samples(10)
    np.testing.assert_array_equal(xs, x[:10])
    np.testing.assert_array_equal(ts, t[:10])
    l0 = float(np.mean((net.forward(x[:20000]) - t[:20000]) ** 2))
    loss = net.train(epochs=8, batch=128 * 64, lr=2e-3, seed=1)
    xv = _features(20000, 33)
    tv = _target(xv)
    lv = float(np.mean((net.forward(xv) - tv) ** 2))
    assert loss < 0.05 * l0 and lv < 0.05 * l0, (l0, loss, lv)
    lo, hi, tmax = net.feature_ranges()
    np.testing.assert_allclose(lo, x.min(0), rtol=0, atol=0)
    np.testing.assert_allclose(hi, x.max(0), rtol=0, atol=0)
    assert tmax == pytest.approx(float(np.abs(t).max()))
    net.close()
