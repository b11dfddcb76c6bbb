"""largeIndex on one device, end to end: cluster files -> per-cluster kNN graph
and CFS path prune on the GPU -> two-copy merge -> final index file.

GNN-Descent keeps the first reverse samples that arrive (as the reference
does), so two builds of a cluster need not be identical; the merge itself is
checked byte for byte on the CPU. Here the file must be well formed, every
edge must stay inside the clusters of its node (local graphs are built per
cluster), degrees must respect max_degree, and the index must be searchable."""
import ctypes as C
import struct

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def clustered(n, dim, c, seed):
    rng = np.random.default_rng(seed)
    centers = rng.normal(0, 4, size=(c, dim)).astype(np.float32)
    x = (centers[rng.integers(0, c, n)] + rng.normal(0, 1.5, size=(n, dim))).astype(np.float32)
    d = ((x[:, None, :] - centers[None]) ** 2).sum(-1)
    order = np.argsort(d, 1)
    return x, order[:, 0].astype(np.uint32), order[:, 1].astype(np.uint32)


def params(capi, tmp, dim, k, cn, n, maxd, bs, fd, topm, thre, iters, out):
    p = capi.LargeParams()
    p.dim, p.k, p.cluster_num, p.max_points = dim, k, cn, n
    p.data_prefix = str(tmp / "cluster_").encode()
    p.local_prefix = str(tmp / "spill_").encode()
    p.index_store_path = str(out).encode()
    p.max_degree, p.buffer_size, p.num = maxd, bs, n
    p.centers_path = str(tmp / "centers.bin").encode()
    p.thre, p.final_degree, p.topm, p.knn_iters, p.mode = thre, fd, topm, iters, capi.KNN_CHOSEN
    return p


def read_index(path):
    raw = open(path, "rb").read()
    size, maxd, medoid, _ = struct.unpack_from("<QIIQ", raw, 0)
    off, rows = 24, []
    while off < len(raw):
        (deg,) = struct.unpack_from("<I", raw, off)
        rows.append(np.frombuffer(raw, np.uint32, deg, off + 4).copy())
        off += 4 + 4 * deg
    return size, maxd, medoid, rows, len(raw)


def test_large_index_single_device(capi, orc, tmp_path):
    n, dim, cn, k = 6000, 32, 6, 24
    maxd, bs, fd, topm, thre, iters = 20, 3, 16, 32, 1.2, 6
    x, first, second = clustered(n, dim, cn, 5)
    np.stack([first, second], 1).astype(np.uint32).tofile(tmp_path / "centers.bin")
    members = [np.sort(np.concatenate([np.nonzero(first == c)[0], np.nonzero(second == c)[0]]))
               for c in range(cn)]
    for c in range(cn):
        with open(tmp_path / f"cluster_{c}", "wb") as f:
            f.write(struct.pack("<I", len(members[c])))
            f.write(np.ascontiguousarray(x[members[c]]).tobytes())
    out = tmp_path / "final.index"
    p = params(capi, tmp_path, dim, k, cn, n, maxd, bs, fd, topm, thre, iters, out)
    dev = (C.c_uint32 * 1)(0)
    capi.check(capi.lib().tagore_large_index(C.byref(p), dev, 1))

    size, md, medoid, adj, nbytes = read_index(out)
    assert size == nbytes and md == maxd and len(adj) == n and medoid < n
    assert all(len(a) <= maxd and (a < n).all() for a in adj)
    # an edge u -> v needs u and v in a common cluster
    home = [{int(first[i]), int(second[i])} for i in range(n)]
    for u in range(0, n, 7):
        for v in adj[u].tolist():
            assert home[u] & home[v], (u, v)
    assert sum(len(a) for a in adj) > n * fd // 2
    # searchable: the reference's NSG search from the medoid with random starts
    offs = np.zeros(n + 1, np.uint64)
    offs[1:] = np.cumsum([len(a) for a in adj])
    flat = np.concatenate(adj).astype(np.uint32)
    q = x[::60] + np.random.default_rng(9).normal(0, 0.5, size=(n // 60, dim)).astype(np.float32)
    found = orc.greedy_search(x, offs, flat, medoid, q, 64, 10, 0x5EED)
    d2 = ((q[:, None, :] - x[None]) ** 2).sum(-1)
    truth = np.argsort(d2, 1)[:, :10]
    rec = np.mean([len(set(a) & set(b)) / 10 for a, b in zip(found.tolist(), truth.tolist())])
    assert rec > 0.8, rec


def test_large_index_uneven_clusters_recall_and_rate(capi, tmp_path):
    """The configuration's shape at a smaller scale: 24 clusters of lognormal
    sizes, unit-normalised d = 96 points each stored in its two nearest of 24
    centres, k = 64, max_degree 22, alpha 1.2. The merged file is read back
    with the Vamana reader (the same layout), searched on the GPU from its
    medoid, and scored by recall@10 against brute force on 2,000 held-out
    queries; the build rate is printed."""
    import time

    import torch
    rng = np.random.default_rng(5)
    cn, dim = 24, 96
    sizes = np.clip(np.exp(rng.normal(np.log(25000), 0.8, cn)), 5000, 120000).astype(int)
    n = int(sizes.sum()) // 2
    centers = rng.normal(0, 1, size=(cn, dim)).astype(np.float32)

    def draw(m):
        y = centers[rng.integers(0, cn, m)] + rng.normal(0, 0.35, size=(m, dim)).astype(np.float32)
        return (y / np.linalg.norm(y, axis=1, keepdims=True)).astype(np.float32)

    x, queries = draw(n), draw(2000)
    order = np.argsort(-(x @ centers.T), 1)
    first, second = order[:, 0].astype(np.uint32), order[:, 1].astype(np.uint32)
    np.stack([first, second], 1).astype(np.uint32).tofile(tmp_path / "centers.bin")
    members = [np.sort(np.concatenate([np.nonzero(first == c)[0], np.nonzero(second == c)[0]]))
               for c in range(cn)]
    for c in range(cn):
        with open(tmp_path / f"cluster_{c}", "wb") as f:
            f.write(struct.pack("<I", len(members[c])))
            f.write(np.ascontiguousarray(x[members[c]]).tobytes())
    builds = sum(len(m) for m in members)
    capi.gnn_descent_host(x[:max(len(m) for m in members)], 64, 2).free()  # pool warm-up
    cuda = torch.device("cuda:0")
    xb = torch.as_tensor(x, device=cuda)
    xq = torch.as_tensor(queries, device=cuda)
    d2 = (xq * xq).sum(1, keepdim=True) + (xb * xb).sum(1)[None] - 2.0 * (xq @ xb.T)
    truth = torch.topk(d2, 10, largest=False).indices.cpu().numpy()
    # devicelist [0]: one builder; [0, 0]: two builder threads sharing the GPU
    # (their kernels never wait on each other), as several devices would
    for devs in ([0], [0, 0]):
        out = tmp_path / f"final_{len(devs)}.index"
        p = params(capi, tmp_path, dim, 64, cn, max(len(m) for m in members), 22, 8, 32, 64, 1.2,
                   0, out)
        p.num = n
        dev = (C.c_uint32 * len(devs))(*devs)
        t = time.perf_counter()
        capi.check(capi.lib().tagore_large_index(C.byref(p), dev, len(devs)))
        el = time.perf_counter() - t
        info, offs, adj = capi.index_read(out, "Vamana")
        assert info.n == n and info.max_degree <= 22 and info.eps[0] < n
        found = capi.search(xb, torch.as_tensor(offs.astype(np.int64), device=cuda),
                            torch.as_tensor(adj.view(np.int32), device=cuda), info.eps[0], xq, 128,
                            10, 0x5EED).cpu().numpy()
        recall = float(np.mean([len(set(a.tolist()) & set(b.tolist())) / 10
                                for a, b in zip(found, truth)]))
        print(f"largeIndex devicelist {devs}: {cn} clusters ({min(len(m) for m in members)}-"
              f"{max(len(m) for m in members)} points), {n} points, {builds} point-builds in "
              f"{el:.2f} s ({builds / el / 1e6:.2f} M/s); recall@10 {recall:.4f}")
        # measured 0.82 at pool size 128 (rows truncated to 22 neighbours by the merge)
        assert recall > 0.75
