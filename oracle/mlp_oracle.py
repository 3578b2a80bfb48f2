"""FP64 NumPy oracle of the per-satellite NLOS network (test infrastructure:
used only by tests/ and the learned-likelihood checks; never on a product
path).

Network 12 -> 64 -> 64 -> 2 with ReLU; p = sigmoid(o0), mu = 20 m *
softplus(o1); loss per row BCE(p, nlos) + nlos ((mu - bias) / 20)^2, mean
over rows.  Parameters in the library's order
    W1t[64][16] b1[64] W2t[64][64] b2[64] W3t[2][64] b3[2]   (Wt[out][in]).

`bf16=True` rounds, as the tensor-core kernels do, every MMA operand to
BF16 (round to nearest even): the inputs, the weights, the hidden
activations after ReLU, and the backward signals dL/do, dL/dH2, dL/dH1
before they enter a product; sums stay in FP64 here (FP32 on the GPU).
"""
from __future__ import annotations

import numpy as np

IN, FEAT, H, OUT = 16, 12, 64, 2
OFF_W1 = 0
OFF_B1 = OFF_W1 + H * IN
OFF_W2 = OFF_B1 + H
OFF_B2 = OFF_W2 + H * H
OFF_W3 = OFF_B2 + H
OFF_B3 = OFF_W3 + OUT * H
N_PARAMS = OFF_B3 + OUT
MU_SCALE = 20.0


def bf16(x):
    """Round to BF16 (nearest even) and return as float64."""
    a = np.asarray(x, np.float32)
    b = a.view(np.uint32).astype(np.uint64)
    lsb = (b >> 16) & 1
    r = ((b + 0x7FFF + lsb) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(prm):
    prm = np.asarray(prm, np.float64)
    W1t = prm[OFF_W1:OFF_B1].reshape(H, IN)
    b1 = prm[OFF_B1:OFF_W2]
    W2t = prm[OFF_W2:OFF_B2].reshape(H, H)
    b2 = prm[OFF_B2:OFF_W3]
    W3t = prm[OFF_W3:OFF_B3].reshape(OUT, H)
    b3 = prm[OFF_B3:N_PARAMS]
    return W1t, b1, W2t, b2, W3t, b3


def init_params(seed=0):
    """He-style initial weights (FP32)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(N_PARAMS, np.float32)
    p[OFF_W1:OFF_B1] = (rng.normal(0, np.sqrt(2.0 / FEAT), (H, IN)) * (np.arange(IN) < FEAT)).ravel()
    p[OFF_W2:OFF_B2] = rng.normal(0, np.sqrt(2.0 / H), H * H)
    p[OFF_W3:OFF_B3] = rng.normal(0, np.sqrt(1.0 / H), OUT * H)
    p[OFF_B3:N_PARAMS] = [-1.0, 0.0]
    return p


def softplus(x):
    return np.where(x > 20.0, x, np.log1p(np.exp(np.minimum(x, 20.0))))


def sigmoid(x):
    return 1.0 / (1.0 + np.exp(-x))


def forward(prm, X, bf=True):
    """Returns (o (n,2), cache)."""
    r = bf16 if bf else (lambda v: np.asarray(v, np.float64))
    W1t, b1, W2t, b2, W3t, b3 = unpack(prm)
    W1t, W2t, W3t = r(W1t), r(W2t), r(W3t)
    Xp = np.zeros((len(X), IN))
    Xp[:, :FEAT] = X
    Xb = r(Xp)
    a1 = Xb @ W1t.T + b1
    h1 = r(np.maximum(a1, 0.0))
    a2 = h1 @ W2t.T + b2
    h2 = r(np.maximum(a2, 0.0))
    o = h2 @ W3t.T + b3
    return o, (Xb, h1, h2, W1t, W2t, W3t)


def predict(prm, X, bf=True):
    o, _ = forward(prm, X, bf)
    return sigmoid(o[:, 0]), MU_SCALE * softplus(o[:, 1])


def loss_grad(prm, X, Y, bf=True):
    """Mean loss and its gradient (N_PARAMS,) in the library's layout."""
    r = bf16 if bf else (lambda v: np.asarray(v, np.float64))
    n = len(X)
    o, (Xb, h1, h2, W1t, W2t, W3t) = forward(prm, X, bf)
    y, b = Y[:, 0].astype(np.float64), Y[:, 1].astype(np.float64)
    o0, o1 = o[:, 0], o[:, 1]
    p = sigmoid(o0)
    mu = MU_SCALE * softplus(o1)
    e = (mu - b) / MU_SCALE
    bce = np.maximum(o0, 0) - o0 * y + np.log1p(np.exp(-np.abs(o0)))
    loss = np.mean(bce + y * e * e)
    do = np.zeros((n, 2))
    do[:, 0] = (p - y) / n
    do[:, 1] = y * 2.0 * e * sigmoid(o1) / n
    do = r(do)
    g2 = r((do @ W3t) * (h2 > 0))
    g1 = r((g2 @ W2t) * (h1 > 0))
    grad = np.zeros(N_PARAMS)
    grad[OFF_W3:OFF_B3] = (do.T @ h2).ravel()
    grad[OFF_B3:N_PARAMS] = do.sum(0)
    grad[OFF_W2:OFF_B2] = (g2.T @ h1).ravel()
    grad[OFF_B2:OFF_W3] = g2.sum(0)
    grad[OFF_W1:OFF_B1] = (g1.T @ Xb).ravel()
    grad[OFF_B1:OFF_W2] = g1.sum(0)
    return loss, grad


def loss_only(prm, X, Y):
    o, _ = forward(prm, X, bf=False)
    y, b = Y[:, 0], Y[:, 1]
    e = (MU_SCALE * softplus(o[:, 1]) - b) / MU_SCALE
    bce = np.maximum(o[:, 0], 0) - o[:, 0] * y + np.log1p(np.exp(-np.abs(o[:, 0])))
    return np.mean(bce + y * e * e)
