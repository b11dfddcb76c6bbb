"""The CPU checker of the screen MLP (oracle/mlp.py) against central finite
differences, so that the GPU gradients are compared with a checker that is
itself right."""
import numpy as np

from oracle import mlp


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(3)
    n, d, B = 40, 12, 16
    x = rng.normal(size=(n, d))
    tri = rng.integers(0, n, size=(B, 3))
    w1 = rng.normal(0, 0.4, size=(d, mlp.HIDDEN))
    b1 = rng.normal(0, 0.1, size=mlp.HIDDEN)
    w2 = rng.normal(0, 0.2, size=(mlp.HIDDEN, mlp.OUT))
    b2 = rng.normal(0, 0.1, size=mlp.OUT)
    params = [w1, b1, w2, b2]
    _, grads = mlp.loss_and_grads(x, tri, *params)
    h = 1e-6
    for which, (p, g) in enumerate(zip(params, grads)):
        flat = p.reshape(-1)
        for i in rng.choice(flat.size, size=6, replace=False):
            old = flat[i]
            flat[i] = old + h
            lp, _ = mlp.loss_and_grads(x, tri, *params)
            flat[i] = old - h
            lm, _ = mlp.loss_and_grads(x, tri, *params)
            flat[i] = old
            num = (lp - lm) / (2 * h)
            assert abs(num - g.reshape(-1)[i]) <= 1e-6 + 1e-4 * abs(num), (which, i)


def test_loss_prefers_order_preserving_projection():
    rng = np.random.default_rng(4)
    x = rng.normal(size=(3, 8))
    tri = np.array([[0, 1, 2]])
    # a projection that keeps x's order scores lower than one that reverses it
    w1 = np.eye(8, mlp.HIDDEN)
    w2 = np.eye(mlp.HIDDEN, mlp.OUT)
    z0 = np.zeros(mlp.HIDDEN)
    x[1] = x[0] + 0.1
    x[2] = x[0] + 2.0
    good, _ = mlp.loss_and_grads(np.abs(x), tri, w1, z0, w2, np.zeros(mlp.OUT))
    bad, _ = mlp.loss_and_grads(np.abs(x), tri[:, [0, 2, 1]], w1, z0, w2, np.zeros(mlp.OUT))
    assert good < bad
