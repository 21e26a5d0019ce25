"""numpy restatement of the per-group opening-angle MLP (the checker for the
CUDA forward/backward kernels in bonsai2_b200/csrc/learned.cu).

TEST INFRASTRUCTURE ONLY.  The network has no counterpart in the reference
(its opening angle is one number, computeMultipoles.cu:168-177); this file
restates the project's own definition: 16 -> 64 -> 64 -> 1, tanh hidden
units, theta = lo + (hi - lo) sigmoid(z), loss = mean over samples of
0.5 (theta - y)^2 (1 + over [theta > y]).  Weight layout W1[64][16], b1[64],
W2[64][64], b2[64], w3[64], b3.
"""
import numpy as np

F, H = 16, 64
NW = H * F + H + H * H + H + H + 1


def unpack(w):
    w = np.asarray(w, np.float64)
    o = 0
    W1 = w[o:o + H * F].reshape(H, F); o += H * F
    b1 = w[o:o + H]; o += H
    W2 = w[o:o + H * H].reshape(H, H); o += H * H
    b2 = w[o:o + H]; o += H
    w3 = w[o:o + H]; o += H
    b3 = w[o]
    return W1, b1, W2, b2, w3, b3


def forward(X, w, lo, hi):
    W1, b1, W2, b2, w3, b3 = unpack(w)
    h1 = np.tanh(X @ W1.T + b1)
    h2 = np.tanh(h1 @ W2.T + b2)
    z = h2 @ w3 + b3
    s = 1.0 / (1.0 + np.exp(-z))
    return lo + (hi - lo) * s, (h1, h2, s)


def loss_grad(X, y, w, lo, hi, over):
    X = np.asarray(X, np.float64)
    y = np.asarray(y, np.float64)
    S = X.shape[0]
    th, (h1, h2, s) = forward(X, w, lo, hi)
    e = th - y
    wgt = np.where(e > 0, 1.0 + over, 1.0)
    loss = np.mean(0.5 * e * e * wgt)
    gz = e * wgt * (hi - lo) * s * (1 - s) / S
    W1, b1, W2, b2, w3, b3 = unpack(w)
    d2 = gz[:, None] * w3[None, :] * (1 - h2 * h2)
    d1 = (d2 @ W2) * (1 - h1 * h1)
    g = np.concatenate([(d1.T @ X).ravel(), d1.sum(0), (d2.T @ h1).ravel(), d2.sum(0), gz @ h2, [gz.sum()]])
    return loss, g
