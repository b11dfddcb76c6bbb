"""The GIST-like configuration end to end at 100,000 points (d = 960, k = 64,
12 iterations): the K-streamed tensor-core kNN graph, then both of the
configuration's index types -- NSSG (the reference's 2-hop collect with the
angle filter at 60 degrees) and DPG, at final_degree 32 and m = 64 -- written,
read back and searched on the GPU (pool 128, seeded random starts) against
brute force on 500 held-out queries.

At this size the 512 components hold about 195 points each and lie far apart
(squared centre distance about 160 against about 4.8 within one), so the
pruned graph splits into about one piece per component and a search reaches
the query's component only through a random start: recall is bounded near
1 - (1 - 1/512)^128 = 0.22. With the opt-in connectivity fix, searched from its
root, the same 2-hop/angle graph is one piece."""
import ctypes as C

import numpy as np
import pytest

from tagore_b200 import synth

pytestmark = pytest.mark.gpu


def search_recall(capi, path, kind, base, queries):
    import torch
    info, offs, adj = capi.index_read(path, kind)
    cuda = torch.device("cuda:0")
    xb = torch.as_tensor(base, device=cuda)
    xq = torch.as_tensor(queries, device=cuda)
    ep = info.eps[0] if info.n_eps else 0
    found = capi.search(xb, torch.as_tensor(offs.astype(np.int64), device=cuda),
                        torch.as_tensor(adj.view(np.int32), device=cuda), ep, xq, 128, 10,
                        0x5EED).cpu().numpy()
    d2 = (xq * xq).sum(1, keepdim=True) + (xb * xb).sum(1)[None] - 2.0 * (xq @ xb.T)
    truth = torch.topk(d2, 10, largest=False).indices.cpu().numpy()
    return info, float(np.mean([len(set(a.tolist()) & set(b.tolist())) / 10
                                for a, b in zip(found, truth)]))


def test_gist_configuration_nssg_and_dpg(capi, tmp_path):
    base, queries = synth.config(2, n=100_000, nq=500)
    n = base.shape[0]
    results = {}
    for kind, thre in (("NSSG", 0.5), ("DPG", 1.0)):
        st = capi.gnn_descent_host(base, 64, 12)
        path = tmp_path / f"index.{kind}"
        capi.pruning(st, 32, kind, topm=64, thre=thre, index_path=str(path))
        st.free()
        info, recall = search_recall(capi, path, kind, base, queries)
        assert info.n == n
        results[kind] = (recall, info.edges / n, info.max_degree)
    print("d=960, n=100000: " + "; ".join(f"{k} recall@10 {r:.4f} ({e:.1f} edges per node, max {m})"
                                          for k, (r, e, m) in results.items()))
    assert results["NSSG"][2] <= 31 and results["DPG"][2] == 32
    assert results["NSSG"][0] > 0.1 and results["DPG"][0] > 0.1  # measured 0.17 / 0.16

    st = capi.gnn_descent_host(base, 64, 12)
    ep = capi.entry_point(st)
    capi.pruning_cfs(st, 32, "2-hop", "angle", topm=64, thre=0.5)
    added = capi.connect(st, ep)
    rows = st.download(0).reshape(n, 64)
    st.free()
    path = tmp_path / "connected.nsg"
    capi.check(capi.lib().tagore_store_nsg(str(path).encode(), rows.ctypes.data_as(C.c_void_p),
                                           32, ep, n, 64))
    info, recall = search_recall(capi, path, "NSG", base, queries)
    print(f"2-hop/angle with the connectivity fix ({added} edges added): recall@10 {recall:.4f}")
    assert recall > results["NSSG"][0] + 0.25  # measured 0.17 -> 0.52
