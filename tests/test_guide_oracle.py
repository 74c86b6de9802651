"""CPU checks of the guiding oracle (oracle/guide_oracle.py): its analytic loss
gradient and back-propagation against central finite differences in FP64, the
normalisation of its lobe mixture, and its bf16 rounding."""
import numpy as np
import pytest

from oracle import guide_oracle as go


def _random_net(rng, scale=0.3):
    W = rng.normal(size=(5, 64, 64)) * scale / 8.0
    for l in range(4):
        W[l, 63, :] = 0.0
        W[l, 63, 63] = 1.0
    return W


def _loss(W, x, d, c):
    _, _, out = go.forward(W, x)
    _, loss = go.loss_grad_output(out, d, c)
    return loss.sum()


def _unit(rng, n):
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def test_encode_layout():
    p = np.array([[0.25, 0.5, 0.75]])
    n = np.array([[0.0, 1.0, 0.0]])
    wo = np.array([[0.6, 0.0, 0.8]])
    x = go.encode(p, n, wo)
    assert x.shape == (1, 64)
    assert np.allclose(x[0, 0:3], p[0])
    assert np.allclose(x[0, 3:6], np.sin(np.pi * p[0]))
    assert np.allclose(x[0, 6:9], np.cos(np.pi * p[0]))
    assert np.allclose(x[0, 33:36], np.sin(32 * np.pi * p[0]))
    assert np.allclose(x[0, 39:42], n[0]) and np.allclose(x[0, 42:45], wo[0])
    assert np.allclose(x[0, 45:48], np.sin(np.pi * n[0])) and np.allclose(x[0, 54:57], np.cos(np.pi * wo[0]))
    assert np.all(x[0, 57:63] == 0.0) and x[0, 63] == 1.0


def test_mixture_pdf_normalised():
    rng = np.random.default_rng(3)
    o = rng.normal(size=(2, 64))
    o[:, 3::5] = rng.uniform(-1, 4, size=o[:, 3::5].shape)
    # Monte Carlo over uniform directions: E[p / (1 / 4 pi)] = 1
    d = _unit(rng, 400000)
    for b in range(2):
        p = go.mixture_pdf(np.repeat(o[b:b + 1], d.shape[0], 0), d)
        est = p.mean() * 4 * np.pi
        assert abs(est - 1.0) < 0.02, est


def test_loss_gradient_finite_differences():
    rng = np.random.default_rng(5)
    B = 6
    W = _random_net(rng)
    x = go.encode(rng.uniform(size=(B, 3)), _unit(rng, B), _unit(rng, B))
    d = _unit(rng, B)
    c = rng.uniform(0.2, 2.0, B)
    hs, xs, out = go.forward(W, x)
    dout, _ = go.loss_grad_output(out, d, c)
    gW = go.backward(W, hs, xs, dout)
    eps = 1e-6
    for (l, i, j) in [(4, 0, 5), (4, 3, 63), (4, 9, 17), (4, 39, 2), (3, 10, 63), (2, 5, 40), (1, 0, 0), (0, 12, 63),
                      (0, 20, 45)]:
        Wp = W.copy(); Wp[l, i, j] += eps
        Wm = W.copy(); Wm[l, i, j] -= eps
        fd = (_loss(Wp, x, d, c) - _loss(Wm, x, d, c)) / (2 * eps)
        assert abs(fd - gW[l, i, j]) <= 1e-6 + 1e-4 * abs(fd), (l, i, j, fd, gW[l, i, j])


def test_output_gradient_finite_differences():
    rng = np.random.default_rng(6)
    B = 4
    o = rng.normal(size=(B, 64))
    d = _unit(rng, B)
    c = np.ones(B)
    g, _ = go.loss_grad_output(o, d, c)
    eps = 1e-6
    for k in range(40):
        op = o.copy(); op[:, k] += eps
        om = o.copy(); om[:, k] -= eps
        fd = (go.loss_grad_output(op, d, c)[1] - go.loss_grad_output(om, d, c)[1]) / (2 * eps)
        assert np.allclose(fd, g[:, k], atol=1e-6, rtol=1e-4), k
    assert np.all(g[:, 40:] == 0.0)


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 2 ** -7, 1.0 + 3 * 2 ** -8, -2.5, 3.14159265], np.float64)
    r = go.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0                     # tie -> even
    assert r[2] == 1.0 + 2 ** -7
    assert r[3] == 1.0 + 2 ** -6           # tie -> even (upward)
    assert r[4] == -2.5
    assert abs(r[5] - 3.140625) < 1e-12


@pytest.mark.parametrize("quantized", [False, True])
def test_gradient_helper_consistent(quantized):
    rng = np.random.default_rng(7)
    n = 33
    W = _random_net(rng)
    rec = np.zeros((n, 5, 4))
    rec[:, 0, :3] = rng.uniform(-1, 1, (n, 3))
    rec[:, 0, 3] = rng.uniform(0, 2, n)
    rec[:, 1, :3] = _unit(rng, n)
    rec[:, 2, :3] = _unit(rng, n)
    rec[:, 3, :3] = _unit(rng, n)
    rec[:, 4, :3] = 1.0
    rec[:3, 0, 3] = 0.0       # records without contribution give no gradient
    g, loss = go.gradient(W, rec.reshape(n, 20), [-1, -1, -1], [0.5, 0.5, 0.5], quantized=quantized)
    g2, loss2 = go.gradient(W, rec[3:].reshape(n - 3, 20), [-1, -1, -1], [0.5, 0.5, 0.5], quantized=quantized)
    assert np.allclose(g, g2) and np.isclose(loss, loss2)
    assert np.isfinite(g).all() and loss > 0
