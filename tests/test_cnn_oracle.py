"""The CPU restatement of the learned short-range network, checked on its own.

The network has no counterpart in the reference, so the oracle is pinned by
mathematics: finite-difference gradients, torch's float64 conv3d and Adam as
second implementations, and the trilinear weights summing to one.
"""
import numpy as np
import pytest

import cnn_oracle as co


def _batch(seed=0, B=2, D=9, n=40, c_in=2):
    rng = np.random.default_rng(seed)
    x0 = rng.normal(size=(B, D, D, D, c_in))
    Do = D - 6
    pb = rng.integers(0, B, n)
    ps = rng.uniform(0.0, Do - 1 - 1e-9, (n, 3))
    target = rng.normal(size=(n, 3))
    weight = rng.uniform(0.5, 1.5, n)
    return x0, pb, ps, target, weight


def test_conv_matches_torch_conv3d():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(1)
    x = rng.normal(size=(2, 7, 6, 5, 3))
    w = rng.normal(size=(27, 16, 3))
    b = rng.normal(size=16)
    got = co.conv_valid(x, w, b)
    wt = np.zeros((16, 3, 3, 3, 3))
    for t, (dx, dy, dz) in enumerate(co.taps()):
        wt[:, :, dz, dy, dx] = w[t]
    ref = torch.nn.functional.conv3d(torch.from_numpy(x).permute(0, 4, 1, 2, 3), torch.from_numpy(wt),
                                     torch.from_numpy(b)).permute(0, 2, 3, 4, 1).numpy()
    assert np.allclose(got, ref, rtol=1e-12, atol=1e-12)


def test_gelu_gradient():
    z = np.linspace(-5, 5, 101)
    h = 1e-6
    fd = (co.gelu(z + h) - co.gelu(z - h)) / (2 * h)
    assert np.allclose(co.gelu_grad(z), fd, rtol=1e-7, atol=1e-9)


def test_interpolation_weights_sum_to_one():
    out = np.ones((1, 4, 4, 4, 3))
    ps = np.random.default_rng(2).uniform(0, 2.999, (50, 3))
    assert np.allclose(co.interpolate(out, np.zeros(50, dtype=int), ps), 1.0)


def test_gradients_match_finite_differences():
    x0, pb, ps, target, weight = _batch()
    p = co.init_params(2, seed=3) + 0.05 * np.random.default_rng(4).normal(size=co.n_params(2))
    loss, g = co.loss_and_grads(p, x0, pb, ps, target, weight)
    rng = np.random.default_rng(5)
    idx = rng.choice(len(p), 60, replace=False)
    h = 1e-6
    for i in idx:
        e = np.zeros_like(p)
        e[i] = h
        lp, _ = co.loss_and_grads(p + e, x0, pb, ps, target, weight)
        lm, _ = co.loss_and_grads(p - e, x0, pb, ps, target, weight)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) < 1e-6 * max(1.0, abs(fd)), (i, fd, g[i])


def test_gradients_match_torch_autograd():
    torch = pytest.importorskip("torch")
    x0, pb, ps, target, weight = _batch(seed=6)
    p = co.init_params(2, seed=7)
    _, g = co.loss_and_grads(p, x0, pb, ps, target, weight)
    pt = torch.tensor(p, requires_grad=True)
    parts, o = [], 0
    for s in co.param_shapes(2):
        k = int(np.prod(s))
        parts.append(pt[o:o + k].reshape(s))
        o += k
    w1, b1, w2, b2, w3, b3, wh, bh = parts
    F = torch.nn.functional

    def conv(x, w, b):
        wt = torch.zeros((16, x.shape[1], 3, 3, 3), dtype=torch.float64)
        for t, (dx, dy, dz) in enumerate(co.taps()):
            wt[:, :, dz, dy, dx] = w[t]
        return F.conv3d(x, wt, b)

    x = torch.from_numpy(x0).permute(0, 4, 1, 2, 3)
    a = F.gelu(conv(x, w1, b1))
    a = F.gelu(conv(a, w2, b2))
    a = F.gelu(conv(a, w3, b3))
    out = (a.permute(0, 2, 3, 4, 1) @ wh.T + bh)
    i0 = np.floor(ps).astype(np.int64)
    f = torch.from_numpy(ps - i0)
    pred = torch.zeros((len(pb), 3), dtype=torch.float64)
    for c in range(8):
        ox, oy, oz = c & 1, (c >> 1) & 1, c >> 2
        wgt = ((f[:, 0] if ox else 1 - f[:, 0]) * (f[:, 1] if oy else 1 - f[:, 1]) *
               (f[:, 2] if oz else 1 - f[:, 2]))
        pred = pred + wgt[:, None] * out[pb, i0[:, 2] + oz, i0[:, 1] + oy, i0[:, 0] + ox]
    w = torch.from_numpy(weight)
    loss = (w[:, None] * (pred - torch.from_numpy(target)) ** 2).sum() / w.sum()
    loss.backward()
    assert np.allclose(pt.grad.numpy(), g, rtol=1e-9, atol=1e-12)


def test_adam_matches_torch():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(8)
    p = rng.normal(size=50)
    m = np.zeros(50)
    v = np.zeros(50)
    pt = torch.tensor(p.copy(), requires_grad=True)
    opt = torch.optim.Adam([pt], lr=1e-3)
    for step in range(1, 6):
        g = rng.normal(size=50)
        p, m, v = co.adam(p, g, m, v, step)
        pt.grad = torch.from_numpy(g.copy())
        opt.step()
    assert np.allclose(p, pt.detach().numpy(), rtol=1e-12, atol=1e-14)


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 1e-3])
    r = co.to_bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 ** -6 and r[3] == -2.5
    assert abs(r[4] - 1e-3) < 2 ** -9 * 1e-3
