"""Why the d = 960 join screens with FP16 Gram tiles and not FP8 E4M3.

On the GIST-like configuration's data (512 components, sigma 0.05, values in
[0, 1]) a node's near neighbours lie at squared distances of about 2 % of the
squared norms, while FP8 E4M3 keeps 3 mantissa bits. For sampled nodes of a
50K-point sample, the 100 nearest points stand in for a join list; the screen
keeps each row's two best partners by the low-precision distance (norms and
Gram both from the quantized rows). Measured: with per-vector scales the FP8
ranking misses 48 % of the exact best two, 20 % after centring the data on its
mean; the FP16 tile the build uses misses none, since its products are exact
and only FP32 accumulation rounds. Denser data (1M points) only narrows the
gaps between neighbours.
"""
import numpy as np
import pytest

from tagore_b200 import synth


def miss_rate(x, q, samp, width=100):
    missed = 0
    for u in samp:
        d = ((x - x[u]) ** 2).sum(1)
        d[u] = np.inf
        ids = np.argsort(d)[:width]
        exact = d[ids]
        approx = (q[u] ** 2).sum() + (q[ids] ** 2).sum(1) - 2.0 * (q[ids] @ q[u])
        missed += len(set(np.argsort(exact)[:2]) - set(np.argsort(approx)[:2]))
    return missed / (2 * len(samp))


def test_fp8_screen_misses_the_nearest_partners():
    torch = pytest.importorskip("torch")
    if not hasattr(torch, "float8_e4m3fn"):
        pytest.skip("no float8 type in this torch")
    x, _ = synth.config(2, n=50_000)
    x = x.astype(np.float16).astype(np.float64)
    samp = np.random.default_rng(0).choice(x.shape[0], 60, replace=False)

    def fp8(v, center):
        mu = v.mean(0) if center else 0.0
        c = v - mu
        s = np.abs(c).max(1, keepdims=True) / 448.0
        t = torch.from_numpy((c / s).astype(np.float32)).to(torch.float8_e4m3fn)
        return t.to(torch.float64).numpy() * s

    m8 = miss_rate(x, fp8(x, False), samp)
    m8c = miss_rate(x, fp8(x, True), samp)
    m16 = miss_rate(x, x, samp)  # the build's tile holds the FP16 rows themselves
    print(f"best-2 partners missed: FP8 {m8:.2f}, FP8 centred {m8c:.2f}, FP16 {m16:.2f}")
    assert m16 == 0.0
    assert m8 > 0.3 and m8c > 0.1
