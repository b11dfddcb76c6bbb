"""The opt-in connectivity fix on a pruned graph of separated clusters: every
node becomes reachable from the entry point, the pruned rows are kept as
prefixes (edges are only appended), and a search from the entry point alone
finds far more true neighbours."""
import numpy as np
import pytest

from tagore_b200 import synth

pytestmark = pytest.mark.gpu


def reachable(rows, ep):
    n = rows.shape[0]
    seen = np.zeros(n, bool)
    seen[ep] = True
    stack = [ep]
    while stack:
        u = stack.pop()
        for v in rows[u, 1:1 + rows[u, 0]].tolist():
            if not seen[v]:
                seen[v] = True
                stack.append(v)
    return seen


def search_recall(orc, rows, ep, base, queries, k=10):
    n = rows.shape[0]
    deg = rows[:, 0].astype(np.int64)
    offs = np.zeros(n + 1, np.uint64)
    offs[1:] = np.cumsum(deg)
    adj = np.concatenate([rows[i, 1:1 + deg[i]] for i in range(n)]).astype(np.uint32)
    found = orc.greedy_search(base, offs, adj, ep, queries, 64, k, 0)  # ep only, no random starts
    d2 = ((queries[:, None, :] - base[None]) ** 2).sum(-1)
    truth = np.argsort(d2, 1)[:, :k]
    return float(np.mean([len(set(a) & set(b)) / k for a, b in zip(found.tolist(), truth.tolist())]))


def test_connect_makes_every_node_reachable(capi, orc):
    base, queries = synth.mixture("sift", 6000, 64, 24, 51, nq=200)
    K, fd = 32, 16
    st = capi.gnn_descent_host(base, K, 8)
    ep = capi.pruning_cfs(st, fd, "path", "dist", topm=48, thre=1.0)
    before = st.download(0).reshape(-1, K).copy()
    seen0 = reachable(before, ep)
    assert not seen0.all()  # separated clusters leave nodes unreachable
    added = capi.connect(st, ep)
    after = st.download(0).reshape(-1, K).copy()
    st.free()
    assert reachable(after, ep).all()
    assert 0 < added <= (~seen0).sum()
    assert int(after[:, 0].sum() - before[:, 0].sum()) == added
    for u in range(before.shape[0]):  # rows only grow
        d0 = before[u, 0]
        assert np.array_equal(after[u, 1:1 + d0], before[u, 1:1 + d0])
    r0 = search_recall(orc, before, ep, base, queries)
    r1 = search_recall(orc, after, ep, base, queries)
    print(f"search recall@10 from ep: {r0:.3f} -> {r1:.3f}, {added} edges added")
    # the kNN build is not deterministic; over repeated runs the gain measured
    # 0.19 to 0.30 (from about 0.47)
    assert r1 > r0 + 0.15


def test_connect_rejects_bad_entry_point(capi):
    base, _ = synth.mixture("sift", 500, 32, 4, 52)
    st = capi.gnn_descent_host(base, 16, 4)
    capi.pruning_cfs(st, 8, "path", "dist", topm=16)
    with pytest.raises(capi.TagoreError):
        capi.connect(st, 10_000)
    st.free()
