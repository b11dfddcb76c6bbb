"""The small configuration end to end at its own size: 100,000 SIFT-like
vectors (64 components), GNN_descent k = 32 for 10 iterations, Pruning 'NSG'
at final_degree 32 and m = 64, the index file written and read back, and
recall@10 of a GPU greedy search over it on 1,000 held-out queries against
brute force. The chosen and plain kNN graphs reach equal recall on sampled
nodes."""
import numpy as np
import pytest

from tagore_b200 import synth

pytestmark = pytest.mark.gpu


def knn_recall(g, half, samp):
    import torch
    x = torch.as_tensor(half, device="cuda").float()
    q = x[samp]
    d2 = (q * q).sum(1, keepdim=True) + (x * x).sum(1)[None] - 2.0 * (q @ x.T)
    d2[torch.arange(len(samp)), torch.as_tensor(samp, device="cuda")] = float("inf")
    truth = torch.topk(d2, 10, largest=False).indices.cpu().numpy()
    return float(np.mean([len(set(g[s, :10].tolist()) & set(truth[i].tolist())) / 10
                          for i, s in enumerate(samp)]))


def test_small_configuration_nsg_index(capi, tmp_path):
    import torch
    base, queries = synth.config(0, nq=1000)
    n, dim, K = base.shape[0], base.shape[1], 32
    samp = np.random.default_rng(3).choice(n, 2000, replace=False)
    recalls = {}
    for mode, name in ((capi.KNN_PLAIN, "plain"), (capi.KNN_CHOSEN, "chosen")):
        st = capi.gnn_descent_host(base, K, 10, mode=mode)
        recalls[name] = knn_recall(st.download(0).reshape(n, K), st.download(2).reshape(n, dim), samp)
        if name == "chosen":
            path = tmp_path / "index.nsg"
            ep = capi.pruning(st, 32, "NSG", topm=64, index_path=str(path))
        st.free()
    info, offs, adj = capi.index_read(path, "NSG")
    assert info.n == n and info.eps[0] == ep and info.max_degree <= 31 and info.width == 32
    cuda = torch.device("cuda:0")
    xb = torch.as_tensor(base, device=cuda)
    xq = torch.as_tensor(queries, device=cuda)
    found = capi.search(xb, torch.as_tensor(offs.astype(np.int64), device=cuda),
                        torch.as_tensor(adj.view(np.int32), device=cuda), ep, xq, 128, 10,
                        0x5EED).cpu().numpy()
    d2 = (xq * xq).sum(1, keepdim=True) + (xb * xb).sum(1)[None] - 2.0 * (xq @ xb.T)
    truth = torch.topk(d2, 10, largest=False).indices.cpu().numpy()
    recall = float(np.mean([len(set(a.tolist()) & set(b.tolist())) / 10
                            for a, b in zip(found, truth)]))
    print(f"kNN recall@10 plain {recalls['plain']:.4f} chosen {recalls['chosen']:.4f}; "
          f"NSG index recall@10 {recall:.4f} (L=128, {info.edges / n:.1f} edges per node)")
    assert abs(recalls["chosen"] - recalls["plain"]) < 0.01
    assert recall > 0.8  # measured 0.876
