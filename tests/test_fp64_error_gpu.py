"""FP32 distance error against FP64 at d = 960 on about a million seeded
pairs: every stored kNN distance of a GIST-like base (16,384 points x 64
neighbours) against the same squared L2 of the same FP16 rows in FP64.

The reference order sums each lane's 960 / 128 = 7.5 chunks into two
accumulators (at most 16 fused multiply-adds each), then five tree levels and
one final add. Each product's rounded difference contributes at most 2^-23
relative error, and each of the at most 22 sequential roundings on a path
2^-24, so every stored value lies within 22 * 2^-24 + 2^-23 (about 1.4e-6) of
the FP64 sum relative to it; the test allows 2e-6."""
import numpy as np
import pytest

from tagore_b200 import synth

pytestmark = pytest.mark.gpu


def test_fp32_distances_against_fp64_at_960(capi):
    base, _ = synth.mixture("gist", 16384, 960, 64, 0x7A6E + 2)
    K = 64
    st = capi.gnn_descent_host(base, K, 4)
    n = base.shape[0]
    g = st.download(0).reshape(n, K).astype(np.int64)
    d32 = st.download(3).reshape(n, K).astype(np.float64)
    half = st.download(2).reshape(n, -1).astype(np.float64)
    st.free()
    rel = np.empty(n * K)
    rows = np.repeat(np.arange(n), K)
    cols = g.reshape(-1)
    for s in range(0, n * K, 1 << 14):
        a, b = rows[s:s + (1 << 14)], cols[s:s + (1 << 14)]
        d64 = ((half[a] - half[b]) ** 2).sum(1)
        rel[s:s + len(a)] = np.abs(d32.reshape(-1)[s:s + len(a)] - d64) / np.maximum(d64, 1e-30)
    print(f"pairs {n * K}: relative error mean {rel.mean():.2e}, max {rel.max():.2e}")
    assert n * K >= 1_000_000
    assert rel.max() < 2e-6
