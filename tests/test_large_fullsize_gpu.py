"""largeIndex at the clustered configuration's scale on one device.

120 clusters of unit-normalised d = 96 points, each point stored in its two
nearest of 120 seeded centres. Home-cluster counts are lognormal (median
75,000, clamped to 10,000-300,000), so the clusters themselves (both copies
counted) span roughly 20,000-600,000 points around a median of 150,000: about
12M points and 24M point-builds. k = 64, max_degree 22, alpha 1.2, degree 32,
TOPM 64, buffer_size 30. The merged file is read back and searched on the GPU
from its medoid; recall@10 against brute force on 2,000 held-out queries. The
build rate, the cluster-size spread and the recall at two search widths are
printed.
"""
import ctypes as C
import struct
import time

import numpy as np
import pytest

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

CN, DIM = 120, 96


def generate(tmp, seed=0x7A6E + 4):
    rng = np.random.default_rng(seed)
    centres = rng.normal(0, 1, size=(CN, DIM)).astype(np.float32)
    homes = np.clip(np.exp(rng.normal(np.log(75_000), 0.7, CN)), 10_000, 300_000).astype(np.int64)
    n = int(homes.sum())
    x = np.empty((n, DIM), np.float32)
    home = np.repeat(np.arange(CN), homes)
    for s in range(0, n, 1 << 20):
        e = min(n, s + (1 << 20))
        y = centres[home[s:e]] + rng.normal(0, 0.35, size=(e - s, DIM)).astype(np.float32)
        x[s:e] = y / np.linalg.norm(y, axis=1, keepdims=True)
    q = centres[rng.integers(0, CN, 2000)] + rng.normal(0, 0.35, size=(2000, DIM)).astype(np.float32)
    q = (q / np.linalg.norm(q, axis=1, keepdims=True)).astype(np.float32)
    first = np.empty(n, np.uint32)
    second = np.empty(n, np.uint32)
    for s in range(0, n, 1 << 20):
        e = min(n, s + (1 << 20))
        order = np.argsort(-(x[s:e] @ centres.T), 1)[:, :2]
        first[s:e], second[s:e] = order[:, 0], order[:, 1]
    np.stack([first, second], 1).astype(np.uint32).tofile(tmp / "centers.bin")
    sizes = []
    for c in range(CN):
        m = np.sort(np.concatenate([np.nonzero(first == c)[0], np.nonzero(second == c)[0]]))
        sizes.append(len(m))
        with open(tmp / f"cluster_{c}", "wb") as f:
            f.write(struct.pack("<I", len(m)))
            f.write(np.ascontiguousarray(x[m]).tobytes())
    return x, q, np.array(sizes)


def test_large_index_at_configuration_scale(capi, tmp_path):
    import torch
    x, queries, sizes = generate(tmp_path)
    n = x.shape[0]
    p = capi.LargeParams()
    p.dim, p.k, p.cluster_num, p.max_points = DIM, 64, CN, int(sizes.max())
    p.data_prefix = str(tmp_path / "cluster_").encode()
    p.local_prefix = str(tmp_path / "spill_").encode()
    out = tmp_path / "final.index"
    p.index_store_path = str(out).encode()
    p.max_degree, p.buffer_size, p.num = 22, 30, n
    p.centers_path = str(tmp_path / "centers.bin").encode()
    p.thre, p.final_degree, p.topm, p.knn_iters, p.mode = 1.2, 32, 64, 0, capi.KNN_CHOSEN
    capi.gnn_descent_host(x[:int(sizes.max())], 64, 2).free()  # pool warm-up
    dev = (C.c_uint32 * 1)(0)
    t = time.perf_counter()
    capi.check(capi.lib().tagore_large_index(C.byref(p), dev, 1))
    el = time.perf_counter() - t
    info, offs, adj = capi.index_read(out, "Vamana")
    assert info.n == n and info.max_degree <= 22 and info.eps[0] < n
    cuda = torch.device("cuda:0")
    xb = torch.as_tensor(x, device=cuda)
    xq = torch.as_tensor(queries, device=cuda)
    best_d, best_i = None, None
    for s in range(0, n, 1 << 20):  # brute force in column chunks of 1M points
        xc = xb[s:s + (1 << 20)]
        d2 = (xq * xq).sum(1, keepdim=True) + (xc * xc).sum(1)[None] - 2.0 * (xq @ xc.T)
        v, i = torch.topk(d2, 10, largest=False)
        i = i + s
        if best_d is not None:
            v, j = torch.topk(torch.cat([best_d, v], 1), 10, largest=False)
            i = torch.gather(torch.cat([best_i, i], 1), 1, j)
        best_d, best_i = v, i
    truth = best_i.cpu().numpy()
    rec = {}
    for L in (128, 512):
        found = capi.search(xb, torch.as_tensor(offs.astype(np.int64), device=cuda),
                            torch.as_tensor(adj.view(np.int32), device=cuda), info.eps[0], xq, L,
                            10, 0x5EED).cpu().numpy()
        rec[L] = float(np.mean([len(set(a.tolist()) & set(b.tolist())) / 10
                                for a, b in zip(found, truth)]))
    builds = int(sizes.sum())
    print(f"largeIndex devicelist [0]: {CN} clusters (min {sizes.min()}, median "
          f"{int(np.median(sizes))}, max {sizes.max()} points), {n} points, {builds} point-builds "
          f"in {el:.1f} s ({builds / el / 1e6:.2f} M/s); recall@10 {rec[128]:.4f} at L=128, "
          f"{rec[512]:.4f} at L=512")
    # The clusters are far apart and cross only through points stored in their
    # second-nearest cluster, so a search from the file's single medoid reaches
    # the query's cluster only some of the time (0.33 at L = 128 when measured);
    # the bound catches a broken graph, not a weak search.
    assert rec[128] > 0.2 and rec[512] >= rec[128] - 0.01
