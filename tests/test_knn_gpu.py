"""kNN graph build on the GPU: structure, exact stored distances, recall."""
import numpy as np
import pytest

from tagore_b200 import synth

pytestmark = pytest.mark.gpu


def recall_at(ids, truth, k):
    hit = 0
    for a, b in zip(ids[:, :k], truth[:, :k]):
        hit += len(set(a.tolist()) & set(b.tolist()))
    return hit / (truth.shape[0] * k)


def build(capi, base, K, iters, mode):
    st = capi.gnn_descent_host(base, K, iters, mode=mode)
    n = base.shape[0]
    g = st.download(0).reshape(n, K)
    d = st.download(3).reshape(n, K)
    half = st.download(2).reshape(n, -1)
    st.free()
    return g, d, half


@pytest.mark.parametrize("mode", ["plain", "chosen"])
def test_knn_structure_and_exact_distances(capi, orc, mode):
    base, _ = synth.mixture("sift", 8000, 128, 32, 21)
    K = 32
    g, d, half = build(capi, base, K, 6, capi.KNN_PLAIN if mode == "plain" else capi.KNN_CHOSEN)
    n = base.shape[0]
    assert (g < n).all()
    assert not (g == np.arange(n)[:, None]).any()
    assert (np.diff(d, axis=1) >= 0).all()
    for r in g[:200]:
        assert len(set(r.tolist())) == K
    exp = orc.dist_pairs(half, np.repeat(np.arange(n), K), g.reshape(-1)).reshape(n, K)
    assert np.array_equal(d.view(np.uint32), exp.view(np.uint32))


@pytest.mark.parametrize("mode", ["plain", "chosen"])
def test_knn_recall(capi, orc, mode):
    base, _ = synth.mixture("sift", 20000, 128, 64, 22)
    K = 32
    g, d, half = build(capi, base, K, 10, capi.KNN_PLAIN if mode == "plain" else capi.KNN_CHOSEN)
    truth, _ = orc.exact_knn(half, K)
    r = recall_at(g, truth, 10)
    assert r > 0.95, r


@pytest.mark.parametrize("kind,dim", [("deep", 96), ("gist", 960), ("sift", 200), ("deep", 136),
                                      ("gist", 1024)])
@pytest.mark.parametrize("mode", ["plain", "chosen"])
def test_knn_other_widths(capi, orc, kind, dim, mode):
    """Row widths beside 128: 96 (one tensor-core tile) and, above 128, the
    K-streamed tensor-core join in the chosen mode: 960, 200, 136 (a last
    column block mostly zero-filled) and 1024 (sixteen full blocks); the plain
    mode reads rows from the cache hierarchy."""
    base, _ = synth.mixture(kind, 4000, dim, 16, 23)
    K = 32
    g, d, half = build(capi, base, K, 8, capi.KNN_PLAIN if mode == "plain" else capi.KNN_CHOSEN)
    n = base.shape[0]
    assert (g < n).all()
    assert not (g == np.arange(n)[:, None]).any()
    assert (np.diff(d, axis=1) >= 0).all()
    exp = orc.dist_pairs(half, np.repeat(np.arange(n), K), g.reshape(-1)).reshape(n, K)
    assert np.array_equal(d.view(np.uint32), exp.view(np.uint32))
    truth, _ = orc.exact_knn(half, K)
    assert recall_at(g, truth, 10) > 0.9
