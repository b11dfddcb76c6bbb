"""GPU prune vs the CPU oracle at the configurations' full sizes.

The small-N tests in test_prune_gpu.py cover the rules and the edge cases;
these repeat the comparison on the graphs the bench and the configurations
actually prune, where reverse lists overflow on hubs and the beam's hash set
and the reverse-edge sort run at full load:

  * 100,000 x 128 SIFT-like (64 components), K = 32, 10 iterations, NSG at
    degree 32, TOPM 64;
  * 1,000,000 x 128 SIFT-like (256 components), K = 96, 10 iterations:
    Pruning_with_CFS('path', 'dist', 1.0), Vamana with alpha 1.2 and CAGRA,
    all at degree 32, TOPM 64;
  * 500,000 x 96 Deep-like (the 2M configuration's generator), K = 64, 10
    iterations: Vamana with alpha 1.2 at degree 32 (the cooperative filter and
    the fixed 96-dim tree);
  * 200,000 x 960 GIST-like (the 1M configuration's generator), K = 64, 12
    iterations: NSSG (2-hop collect, angle filter at 60 degrees) and DPG at
    degree 32 (the cooperative filter and two-hop scoring, the block-per-node
    DPG select).

The oracle's time at the two larger configurations' own sizes (several
minutes of CPU each) sets the smaller sizes here; both bases stay above L2.

The kNN graph comes from this library's own GNN_descent; the prune must then
equal the oracle on every buffer it touches, bit for bit.
"""
import numpy as np
import pytest

from tagore_b200 import synth

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

NAMES = ("graph", "nei_distance", "reverse_graph", "reverse_distance", "reverse_num",
         "hybrid_list")


def knn_buffers(capi, n, dim, k, iters, comps, seed):
    base, _ = synth.mixture("sift", n, dim, comps, seed)
    st = capi.gnn_descent_host(base, k, iters)
    bufs = st.buffers()
    st.free()
    return bufs


def compare(capi, orc, bufs, n, dim, k, fd, what, topm=64, thre=1.0):
    st = capi.State.alloc(n, dim, k)
    for i, (name, _) in enumerate(capi.BUFFERS[:8]):
        st.upload(i, bufs[name])
    buf = orc.Buffers(bufs["graph"].reshape(n, k), bufs["nei_distance"].reshape(n, k),
                      bufs["data"].reshape(n, dim), bufs["center"], bufs["reverse_graph"],
                      bufs["reverse_distance"], bufs["reverse_num"], bufs["hybrid_list"])
    if what[0] == "index":
        ep_g = capi.pruning(st, fd, what[1], topm=topm, thre=thre)
        ep_c = orc.prune(buf, fd, what[1], topm=topm, thre=thre)
    else:
        ep_g = capi.pruning_cfs(st, fd, what[1], what[2], topm=topm, thre=thre)
        ep_c = orc.prune_cfs(buf, fd, what[1], what[2], topm=topm, thre=thre)
    assert ep_g == ep_c, (what, ep_g, ep_c)
    for i, (name, _) in enumerate(capi.BUFFERS[:8]):
        if name not in NAMES:
            continue
        g = st.download(i)
        e = getattr(buf, name)
        g32 = g.view(np.uint32) if g.dtype == np.float32 else g
        e32 = e.view(np.uint32) if e.dtype == np.float32 else e
        if not np.array_equal(g32, e32):
            bad = np.nonzero(g32 != e32)[0]
            pytest.fail(f"{what}: buffer {name} differs at {bad[:8]} (of {bad.size})")
    rows = st.download(0).reshape(n, k)
    st.free()
    return rows


def knn_buffers_config(capi, cfg, n, k, iters):
    base, _ = synth.config(cfg, n=n)
    st = capi.gnn_descent_host(base, k, iters)
    bufs = st.buffers()
    st.free()
    return bufs


@pytest.fixture(scope="module")
def knn_1m(capi):
    return knn_buffers(capi, 1_000_000, 128, 96, 10, 256, 0x7A6E + 1)


def test_config1_nsg_100k(capi, orc):
    n, k = 100_000, 32
    bufs = knn_buffers(capi, n, 128, k, 10, 64, 0x7A6E)
    rows = compare(capi, orc, bufs, n, 128, k, 32, ("index", "NSG"))
    assert rows[:, 0].max() <= 31 and rows[:, 0].mean() > 8


def test_config2_cfs_path_dist_1m(capi, orc, knn_1m):
    compare(capi, orc, knn_1m, 1_000_000, 128, 96, 32, ("cfs", "path", "dist"), thre=1.0)


def test_config2_vamana_1m(capi, orc, knn_1m):
    compare(capi, orc, knn_1m, 1_000_000, 128, 96, 32, ("index", "Vamana"), thre=1.2)


def test_config2_cagra_1m(capi, orc, knn_1m):
    rows = compare(capi, orc, knn_1m, 1_000_000, 128, 96, 32, ("index", "CAGRA"))
    assert rows.shape == (1_000_000, 96)


@pytest.fixture(scope="module")
def knn_deep_500k(capi):
    return knn_buffers_config(capi, 3, 500_000, 64, 10)


def test_config4_vamana_500k_x_96(capi, orc, knn_deep_500k):
    rows = compare(capi, orc, knn_deep_500k, 500_000, 96, 64, 32, ("index", "Vamana"), thre=1.2)
    assert rows[:, 0].max() <= 32


@pytest.fixture(scope="module")
def knn_gist_200k(capi):
    return knn_buffers_config(capi, 2, 200_000, 64, 12)


def test_config3_nssg_200k_x_960(capi, orc, knn_gist_200k):
    compare(capi, orc, knn_gist_200k, 200_000, 960, 64, 32, ("index", "NSSG"), thre=0.5)


def test_config3_dpg_200k_x_960(capi, orc, knn_gist_200k):
    compare(capi, orc, knn_gist_200k, 200_000, 960, 64, 32, ("index", "DPG"))
