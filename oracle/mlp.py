"""CPU restatement of the candidate-screen MLP and its training step.

TEST INFRASTRUCTURE ONLY: the checker for the GPU forward, loss and backward
kernels (tagore_b200/csrc/mlp.cu). The screen has no counterpart in the
reference; it is the learned part of this project's chosen kNN path.

Network: z = W2^T relu(W1^T x + b1) + b2, x in R^d, hidden 128, output 32.
Loss per triplet (a, p, m) whose exact distances order d(a,p) < d(a,m):
    u = log(Dp + eps) - log(Dm + eps),  L = softplus(u),
    Dp = |z_a - z_p|^2,  Dm = |z_a - z_m|^2,
mean over the batch. It depends only on the ratio Dp / Dm, so it asks the
projection to keep the order of exact distances, not their scale.
Everything is float64 here; the GPU works in float32. In a build the GPU
first subtracts the mean of the base rows from x; the checked batches use a
zero mean, which is this formula.
"""
import numpy as np

HIDDEN, OUT, EPS = 128, 32, 1e-6


def forward(x, w1, b1, w2, b2):
    pre = x @ w1 + b1
    h = np.maximum(pre, 0.0)
    return pre, h, h @ w2 + b2


def loss_and_grads(x, tri, w1, b1, w2, b2):
    """x: (n, d) rows; tri: (B, 3) row indices (a, p, m). Returns (loss, grads)."""
    x = np.asarray(x, np.float64)
    w1, b1, w2, b2 = (np.asarray(v, np.float64) for v in (w1, b1, w2, b2))
    rows = tri.reshape(-1)
    xr = x[rows]
    pre, h, z = forward(xr, w1, b1, w2, b2)
    B = tri.shape[0]
    za, zp, zm = z[0::3], z[1::3], z[2::3]
    dp = ((za - zp) ** 2).sum(1)
    dm = ((za - zm) ** 2).sum(1)
    u = np.log(dp + EPS) - np.log(dm + EPS)
    loss = np.logaddexp(0.0, u).mean()
    s = 1.0 / (1.0 + np.exp(-u)) / B
    gdp = s / (dp + EPS)
    gdm = -s / (dm + EPS)
    dz = np.zeros_like(z)
    dz[0::3] = 2 * gdp[:, None] * (za - zp) + 2 * gdm[:, None] * (za - zm)
    dz[1::3] = -2 * gdp[:, None] * (za - zp)
    dz[2::3] = -2 * gdm[:, None] * (za - zm)
    gw2 = h.T @ dz
    gb2 = dz.sum(0)
    dh = (dz @ w2.T) * (pre > 0)
    gw1 = xr.T @ dh
    gb1 = dh.sum(0)
    return loss, (gw1, gb1, gw2, gb2)
