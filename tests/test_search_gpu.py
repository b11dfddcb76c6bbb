"""The GPU greedy search (tagore_search) against the oracle's sequential
search: the same ids in the same order. Graphs are pruned indexes and ragged
random graphs with duplicate and out-of-range ids; bases have integer values
(SIFT-like), so equal distances are common and the tie order is exercised."""
import numpy as np
import pytest

from tagore_b200 import synth

pytestmark = pytest.mark.gpu


def both(capi, orc, base, offs, adj, ep, queries, L, k, seed, visit_cap=0):
    import torch
    dev = torch.device("cuda:0")
    b = torch.as_tensor(np.ascontiguousarray(base, np.float32), device=dev)
    o = torch.as_tensor(offs.astype(np.int64), device=dev)
    a = torch.as_tensor(np.ascontiguousarray(adj, np.uint32).view(np.int32), device=dev)
    q = torch.as_tensor(np.ascontiguousarray(queries, np.float32), device=dev)
    got = capi.search(b, o, a, ep, q, L, k, seed, visit_cap).cpu().numpy().astype(np.uint32)
    want = orc.greedy_search(base, offs, adj, ep, queries, L, k, seed)
    return got, want


def ragged_graph(n, max_deg, rng, bad_ids=True):
    deg = rng.integers(0, max_deg + 1, size=n)
    offs = np.zeros(n + 1, np.uint64)
    offs[1:] = np.cumsum(deg)
    adj = rng.integers(0, n, size=int(offs[-1])).astype(np.uint32)
    if bad_ids and adj.size:
        pick = rng.random(adj.size)
        adj[pick < 0.02] = n + rng.integers(0, 5)      # skipped: outside the base
        dup = np.nonzero(pick > 0.97)[0]
        adj[dup[dup > 0]] = adj[dup[dup > 0] - 1]      # repeated neighbour
    return offs, adj


@pytest.fixture(scope="module")
def pruned(capi):
    base, queries = synth.mixture("sift", 20000, 128, 32, 61, nq=300)
    K, fd = 32, 24
    st = capi.gnn_descent_host(base, K, 8)
    ep = capi.pruning_cfs(st, fd, "path", "dist", topm=48, thre=1.0)
    rows = st.download(0).reshape(-1, K).copy()
    st.free()
    offs, adj = capi.rows_to_csr(rows)
    return base, queries, offs, adj, ep


@pytest.mark.parametrize("L,k,seed", [(64, 10, 0), (128, 10, 0x5EED), (100, 100, 7), (40, 50, 3)])
def test_pruned_index_matches_oracle(capi, orc, pruned, L, k, seed):
    base, queries, offs, adj, ep = pruned
    got, want = both(capi, orc, base, offs, adj, ep, queries, L, k, seed)
    assert np.array_equal(got, want), np.argwhere(got != want)[:5]


@pytest.mark.parametrize("dim,max_deg,seed", [(128, 31, 0), (96, 64, 11), (100, 40, 5), (7, 80, 0)])
def test_ragged_graphs_match_oracle(capi, orc, dim, max_deg, seed):
    rng = np.random.default_rng(dim * 1000 + max_deg)
    base, queries = synth.mixture("sift", 3000, dim, 8, 62, nq=120)
    offs, adj = ragged_graph(3000, max_deg, rng)
    got, want = both(capi, orc, base, offs, adj, 17, queries, 72, 16, seed)
    assert np.array_equal(got, want), np.argwhere(got != want)[:5]


def test_small_base_pool_covers_everything(capi, orc):
    rng = np.random.default_rng(9)
    base = rng.integers(0, 4, size=(50, 16)).astype(np.float32)   # many equal distances
    queries = rng.integers(0, 4, size=(20, 16)).astype(np.float32)
    offs, adj = ragged_graph(50, 6, rng, bad_ids=False)
    for seed in (0, 99):
        got, want = both(capi, orc, base, offs, adj, 0, queries, 64, 70, seed)
        assert np.array_equal(got, want)
        assert (got[:, 50:] == 0xFFFFFFFF).all()  # the pool holds at most n ids


def test_edgeless_graph_and_no_queries(capi, orc):
    import torch
    base = np.random.default_rng(1).random((10, 8)).astype(np.float32)
    offs = np.zeros(11, np.uint64)
    adj = np.zeros(0, np.uint32)
    q = base[:3] + 0.01
    got, want = both(capi, orc, base, offs, adj, 4, q, 8, 3, 0)
    assert np.array_equal(got, want)
    assert (got[:, 0] == 4).all() and (got[:, 1:] == 0xFFFFFFFF).all()
    dev = torch.device("cuda:0")
    empty = torch.zeros((0, 8), dtype=torch.float32, device=dev)
    out = capi.search(torch.as_tensor(base, device=dev), torch.as_tensor(offs.astype(np.int64), device=dev),
                      torch.zeros(1, dtype=torch.int32, device=dev), 0, empty, 8, 3)
    assert out.shape == (0, 3)


def test_visited_overflow_is_an_error_not_a_wrong_answer(capi):
    import torch
    rng = np.random.default_rng(4)
    n = 40000
    base = rng.random((n, 16)).astype(np.float32)
    offs, adj = ragged_graph(n, 64, rng, bad_ids=False)
    dev = torch.device("cuda:0")
    args = (torch.as_tensor(base, device=dev), torch.as_tensor(offs.astype(np.int64), device=dev),
            torch.as_tensor(adj.view(np.int32), device=dev), 0,
            torch.as_tensor(base[:4] + 0.5, device=dev))
    with pytest.raises(capi.TagoreError, match="visit_cap"):
        capi.search(*args, 2048, 10, 0, visit_cap=16384)
    capi.search(*args, 64, 10, 0, visit_cap=1 << 17)  # enough room: no error


def test_rejects_bad_arguments(capi):
    import torch
    dev = torch.device("cuda:0")
    base = torch.zeros((10, 8), dtype=torch.float32, device=dev)
    offs = torch.zeros(11, dtype=torch.int64, device=dev)
    adj = torch.zeros(1, dtype=torch.int32, device=dev)
    with pytest.raises(capi.TagoreError):
        capi.search(base, offs, adj, 10, base[:2].contiguous(), 8, 3)   # entry point outside
    with pytest.raises(capi.TagoreError):
        capi.search(base, offs, adj, 0, base[:2].contiguous(), 0, 3)    # empty pool
