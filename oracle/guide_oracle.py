"""Test infrastructure only: FP64 numpy restatement of the learned guiding proposal.

The guiding network has no counterpart in the reference (it is the learned
proposal added beside the plain NEE+MIS estimator); this module is the CPU
checker for the GPU kernels' feature encoding, forward pass, mixture pdf and
loss gradient. Conventions shared with the kernels (wurstrenderer_b200/csrc/wr_guide.cu):

* features (64): p in [0,1]^3 (scene box), sin/cos(2^f * pi * p) for f = 0..5
  (36), normal (3), outgoing direction (3), sin/cos(pi * n) (6), sin/cos(pi * wo)
  (6) -- 57 values -- then 6 zeros and a constant 1 at index 63;
* 5 layers, y = W x (W: 64 x 64, row = output), ReLU after layers 0..3; unit 63 of
  every hidden layer is the constant 1 (row 63 of W_l = e_63), so column 63 of
  the next layer acts as its bias;
* 8 lobes from outputs 5k..5k+4: axis r (3, normalised), sharpness
  lambda = softplus(s) + 0.5, weight = softmax over the 8 logits;
* vMF lobe pdf f(w) = lambda / (2 pi (1 - exp(-2 lambda))) exp(lambda (mu.w - 1));
* loss per sample = -c * log(sum_k w_k f_k(w)), c = target / p_sample (clamped).
"""
from __future__ import annotations

import numpy as np

N_LOBES = 8
LAMBDA_MIN = 0.5
LAMBDA_MAX = 5000.0
C_MAX = 100.0


def encode(p01, n, wo):
    """p01, n, wo: (B, 3) -> (B, 64) features."""
    p01 = np.asarray(p01, np.float64)
    B = p01.shape[0]
    out = np.zeros((B, 64))
    out[:, 0:3] = p01
    col = 3
    for f in range(6):
        a = (2.0 ** f) * np.pi * p01
        out[:, col:col + 3] = np.sin(a)
        out[:, col + 3:col + 6] = np.cos(a)
        col += 6
    out[:, col:col + 3] = n
    out[:, col + 3:col + 6] = wo
    col += 6
    out[:, col:col + 3] = np.sin(np.pi * np.asarray(n))
    out[:, col + 3:col + 6] = np.cos(np.pi * np.asarray(n))
    col += 6
    out[:, col:col + 3] = np.sin(np.pi * np.asarray(wo))
    out[:, col + 3:col + 6] = np.cos(np.pi * np.asarray(wo))
    col += 6
    assert col == 57
    out[:, 63] = 1.0
    return out


def forward(W, x, quantize=None):
    """W: (5, 64, 64); x: (B, 64). Returns (pre-activations list, inputs list, output (B, 64)).
    quantize: optional function applied to every layer input (the GPU stores them as bf16)."""
    xs, hs = [], []
    h = x
    for l in range(5):
        xin = quantize(h) if quantize is not None else h
        xs.append(xin)
        y = xin @ W[l].T
        hs.append(y)
        h = np.maximum(y, 0.0) if l < 4 else y
    return hs, xs, h


def lobes(o):
    """o: (B, 64) raw outputs -> mu (B, 8, 3), lam (B, 8), w (B, 8)."""
    o = o[:, :5 * N_LOBES].reshape(-1, N_LOBES, 5)
    r = o[..., 0:3]
    nr = np.linalg.norm(r, axis=-1, keepdims=True)
    mu = np.where(nr > 1e-12, r / np.maximum(nr, 1e-30), np.array([0.0, 1.0, 0.0]))
    s = o[..., 3]
    lam = np.minimum(np.logaddexp(0.0, s) + LAMBDA_MIN, LAMBDA_MAX)
    a = o[..., 4]
    a = a - a.max(axis=-1, keepdims=True)
    w = np.exp(a)
    w /= w.sum(axis=-1, keepdims=True)
    return mu, lam, w


def vmf(mu, lam, d):
    """mu (..., 3), lam (...), d (..., 3) -> pdf."""
    c = np.sum(mu * d, axis=-1)
    norm = lam / (2.0 * np.pi * -np.expm1(-2.0 * lam))
    return norm * np.exp(lam * (c - 1.0))


def mixture_pdf(o, d):
    mu, lam, w = lobes(o)
    return np.sum(w * vmf(mu, lam, d[:, None, :]), axis=-1)


def loss_grad_output(o, d, c, c_max=C_MAX):
    """Gradient of -c * log p(d) w.r.t. the raw outputs o (B, 64); also returns the loss (B,)."""
    B = o.shape[0]
    oo = o[:, :5 * N_LOBES].reshape(B, N_LOBES, 5)
    r = oo[..., 0:3]
    nr = np.maximum(np.linalg.norm(r, axis=-1, keepdims=True), 1e-30)
    mu = r / nr
    s = oo[..., 3]
    lam = np.logaddexp(0.0, s) + LAMBDA_MIN
    a = oo[..., 4] - oo[..., 4].max(axis=-1, keepdims=True)
    w = np.exp(a)
    w /= w.sum(axis=-1, keepdims=True)
    f = vmf(mu, lam, d[:, None, :])
    p = np.sum(w * f, axis=-1)
    resp = w * f / p[:, None]                          # posterior lobe responsibilities
    cosk = np.sum(mu * d[:, None, :], axis=-1)
    dlogf_dlam = 1.0 / lam - 2.0 * np.exp(-2.0 * lam) / (-np.expm1(-2.0 * lam)) + (cosk - 1.0)
    g = np.zeros((B, N_LOBES, 5))
    g[..., 4] = resp - w                               # d log p / d logit
    g[..., 3] = resp * dlogf_dlam / (1.0 + np.exp(-s))  # softplus' = sigmoid
    g[..., 0:3] = (resp * lam)[..., None] * (d[:, None, :] - mu * cosk[..., None]) / nr
    cc = np.minimum(np.asarray(c, np.float64), c_max)
    out = np.zeros((B, 64))
    out[:, :5 * N_LOBES] = (-cc[:, None, None] * g).reshape(B, -1)
    return out, -cc * np.log(p)


def backward(W, hs, xs, dout, quantize=None):
    """Gradient of sum(loss) w.r.t. W given d loss / d output (B, 64).
    quantize: optional function applied to every back-propagated gradient before it
    enters a product (the GPU stores them as bf16)."""
    q = quantize if quantize is not None else (lambda a: a)
    gW = np.zeros_like(W)
    dh = q(dout)
    for l in range(4, -1, -1):
        gW[l] = dh.T @ xs[l]
        if l > 0:
            dx = dh @ W[l]
            dh = q(dx * (hs[l - 1] > 0))
    return gW


def record_arrays(records):
    """Splits (n, 20) training records into position, c, normal, outgoing, direction."""
    r = np.asarray(records, np.float64).reshape(-1, 5, 4)
    return r[:, 0, :3], r[:, 0, 3], r[:, 1, :3], r[:, 2, :3], r[:, 3, :3]


def gradient(W, records, box_lo, box_inv, c_max=C_MAX, quantized=True):
    """The full training gradient of the GPU kernel for (n, 20) records: returns (gW, summed loss).
    With quantized=True the weights, layer inputs and back-propagated gradients are rounded
    to bf16 as on the GPU, and the position feature is formed in float32."""
    p, c, n, wo, d = record_arrays(records)
    p01 = ((p.astype(np.float32) - np.asarray(box_lo, np.float32)) * np.asarray(box_inv, np.float32)).astype(np.float64)
    x = encode(p01, n, wo)
    qf = bf16 if quantized else None
    Wq = bf16(W) if quantized else np.asarray(W, np.float64)
    hs, xs, out = forward(Wq, x, quantize=qf)
    dout, loss = loss_grad_output(out, d, c, c_max)
    dout[c <= 0] = 0.0
    loss[c <= 0] = 0.0
    return backward(Wq, hs, xs, dout, quantize=qf), float(loss.sum())


def eval_rows(W, rows, box_lo, box_inv, quantized=True):
    """Lobes for (n, 9) rows (position, normal, outgoing) as the inference kernel computes them."""
    rows = np.asarray(rows, np.float64)
    p01 = ((rows[:, 0:3].astype(np.float32) - np.asarray(box_lo, np.float32)) *
           np.asarray(box_inv, np.float32)).astype(np.float64)
    x = encode(p01, rows[:, 3:6], rows[:, 6:9])
    Wq = bf16(W) if quantized else np.asarray(W, np.float64)
    _, _, out = forward(Wq, x, quantize=bf16 if quantized else None)
    return lobes(out)


def bf16(x):
    """Round to bfloat16 (nearest-even) and back to float64."""
    x32 = np.asarray(x, np.float32)
    u = x32.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)
