"""GPU prune vs the CPU oracle, through the C ABI, on seeded inputs.

Every buffer the prune touches (graph rows, nei_distance, reverse lists,
reverse counts, hybrid_list) must be identical bit for bit."""
import numpy as np
import pytest

from tagore_b200 import synth

pytestmark = pytest.mark.gpu

_CASES = {}


def case(kind, n, dim, K, noise=0.1, seed=0):
    key = (kind, n, dim, K, noise, seed)
    if key in _CASES:
        return _CASES[key]
    from oracle import oracle as orc
    if kind == "sift":
        base, _ = synth.mixture("sift", n, dim, 32, 100 + seed)
        half = (base * np.float32(0.01)).astype(np.float16)
    elif kind == "gist":
        base, _ = synth.mixture("gist", n, dim, 64, 200 + seed)
        half = base.astype(np.float16)
    elif kind == "deep":
        base, _ = synth.mixture("deep", n, dim, 64, 300 + seed)
        half = base.astype(np.float16)
    elif kind == "int":  # small integers: many exactly tied distances
        half = np.random.default_rng(seed).integers(0, 3, size=(n, dim)).astype(np.float16)
    else:
        raise ValueError(kind)
    ids, dis = orc.knn_input(half, K, noise=noise, seed=seed + 5)
    center = half.astype(np.float32).mean(0).astype(np.float16)
    _CASES[key] = (half, ids, dis, center)
    return _CASES[key]


def run_pair(capi, orc, c, fd, what, topm=64, thre=1.0, hub=False):
    half, ids, dis, center = c
    n, K = ids.shape
    ids = ids.copy()
    if hub:  # many rows point at node 0: its reverse list overflows
        ids[1::3, -1] = 0
    rng = np.random.default_rng(99)
    rg0 = rng.integers(0, n, size=n * 128).astype(np.uint32)  # stale contents stay stale
    rd0 = rng.random(n * 128).astype(np.float32)
    st = capi.State.from_host(ids, dis, half, center, reverse_graph=rg0, reverse_distance=rd0)
    buf = orc.Buffers(ids, dis, half, center, reverse_graph=rg0, reverse_distance=rd0)
    if what[0] == "index":
        ep_g = capi.pruning(st, fd, what[1], topm=topm, thre=thre)
        ep_c = orc.prune(buf, fd, what[1], topm=topm, thre=thre)
    else:
        ep_g = capi.pruning_cfs(st, fd, what[1], what[2], topm=topm, thre=thre)
        ep_c = orc.prune_cfs(buf, fd, what[1], what[2], topm=topm, thre=thre)
    got = st.buffers()
    st.free()
    assert ep_g == ep_c
    for name in ("graph", "nei_distance", "reverse_graph", "reverse_distance", "reverse_num",
                 "hybrid_list"):
        exp = getattr(buf, name)
        g = got[name]
        if not np.array_equal(g.view(np.uint32) if g.dtype == np.float32 else g,
                              exp.view(np.uint32) if exp.dtype == np.float32 else exp):
            bad = np.nonzero((g != exp) & ~(np.isnan(g.astype(np.float64)) & np.isnan(exp.astype(np.float64))))[0]
            pytest.fail(f"{what}: buffer {name} differs at {bad[:8]} (of {bad.size})")
    return got


INDEX_TYPES = [("NSG", 1.0), ("Vamana", 1.2), ("NSSG", 0.5), ("CAGRA", 1.0)]


@pytest.mark.parametrize("itype,thre", INDEX_TYPES)
def test_index_types_config2_shape(capi, orc, itype, thre):
    run_pair(capi, orc, case("sift", 3000, 128, 96), 32, ("index", itype), thre=thre)


@pytest.mark.parametrize("mode,metric,thre", [("path", "dist", 1.0), ("path", "dist", 1.2),
                                              ("path", "angle", 0.5), ("2-hop", "dist", 1.0),
                                              ("2-hop", "angle", 0.5), ("1-hop", "rank", 1.0)])
def test_cfs_combinations(capi, orc, mode, metric, thre):
    run_pair(capi, orc, case("sift", 2500, 128, 64, seed=1), 32, ("cfs", mode, metric), thre=thre)


def test_nsg_k32_final_degree_equals_k_topm_above_k(capi, orc):
    # configuration 1: K = 32, FINAL_DEGREE = 32, TOPM = 64
    run_pair(capi, orc, case("sift", 3000, 128, 32, seed=2), 32, ("index", "NSG"), topm=64)


@pytest.mark.parametrize("itype,thre", [("NSSG", 0.5), ("DPG", 1.0), ("NSG", 1.0), ("Vamana", 1.2)])
def test_d960(capi, orc, itype, thre):
    # rows wider than 128 halves take the warp-cooperative filter
    run_pair(capi, orc, case("gist", 1200, 960, 64, seed=3), 32, ("index", itype), thre=thre)


@pytest.mark.parametrize("itype,thre", [("NSSG", 0.5), ("Vamana", 1.2), ("DPG", 1.0)])
def test_d260_odd_chunks(capi, orc, itype, thre):
    # 65 four-half chunks: lane 0 of the cooperative tree takes three, the
    # others two; the thread-serial tree walks 4-half chunks (not 16-byte units)
    run_pair(capi, orc, case("gist", 900, 260, 48, seed=8), 24, ("index", itype), thre=thre)


def test_dpg_wide_odd_k(capi, orc):
    # the block-per-node DPG select with an odd K: the reference's pair set
    # skips the middle row (a = K/2)
    run_pair(capi, orc, case("gist", 700, 200, 47, seed=9), 24, ("index", "DPG"))


def test_vamana_d96(capi, orc):
    run_pair(capi, orc, case("deep", 3000, 96, 64, seed=4), 32, ("index", "Vamana"), thre=1.2)


@pytest.mark.parametrize("itype,thre", INDEX_TYPES + [("DPG", 1.0)])
def test_ties_and_hub_overflow(capi, orc, itype, thre):
    K = 64
    run_pair(capi, orc, case("int", 2000, 32, K, noise=0.3, seed=5), 32, ("index", itype),
             thre=thre, hub=True)


def test_small_graph(capi, orc):
    run_pair(capi, orc, case("sift", 40, 16, 24, noise=0.0, seed=6), 8, ("index", "NSG"), topm=16)
    run_pair(capi, orc, case("sift", 40, 16, 24, noise=0.0, seed=6), 8, ("cfs", "2-hop", "angle"),
             thre=0.5)


def test_entry_point_matches(capi, orc):
    half, ids, dis, center = case("sift", 3000, 128, 96)
    st = capi.State.from_host(ids, dis, half, center)
    buf = orc.Buffers(ids, dis, half, center)
    assert capi.entry_point(st, 64) == orc.cal_ep(buf, 64)
    st.free()


def test_rejections(capi):
    half, ids, dis, center = case("sift", 3000, 128, 96)
    st = capi.State.from_host(ids, dis, half, center)
    with pytest.raises(capi.TagoreError) as e:
        capi.pruning(st, 32, "HNSW")
    assert e.value.code == capi.TAGORE_EINVAL
    with pytest.raises(capi.TagoreError):
        capi.pruning_cfs(st, 32, "path", "rank")
    bad = ids.copy()
    bad[5, 3] = 3000
    st.upload(0, bad)
    with pytest.raises(capi.TagoreError) as e:
        capi.pruning(st, 32, "NSG")
    assert "id >= POINTS" in str(e.value)
    st.free()


def test_host_prep_is_bit_exact(capi, orc):
    base, _ = synth.mixture("sift", 5000, 128, 16, 7)
    st = capi.gnn_descent_host(base, 16, 2, mode=capi.KNN_PLAIN)
    half, center, factor = orc.host_prep(base)
    assert st.st.norm_factor == factor
    assert np.array_equal(st.download(2).view(np.uint16), half.reshape(-1).view(np.uint16))
    assert np.array_equal(st.download(6).view(np.uint16), center.view(np.uint16))
    assert st.download(5).max() == 0  # reverse_num starts at zero, as after GNN_descent
    st.free()
