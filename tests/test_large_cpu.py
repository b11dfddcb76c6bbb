"""largeIndex host half (cluster order, two-copy merge, spills, final index)
against the Python restatement in oracle/large_merge.py, byte for byte, on
given local graphs (no GPU needed)."""
import ctypes as C
import os

import numpy as np
import pytest


def scenario(seed, N=2500, Cn=7, K=16):
    rng = np.random.default_rng(seed)
    first = rng.integers(0, Cn, size=N)
    second = (first + rng.integers(1, Cn, size=N)) % Cn  # a different cluster
    clusters = [[] for _ in range(Cn)]
    for i in range(N):
        clusters[first[i]].append(i)
        clusters[second[i]].append(i)
    rows, medoids = [], []
    for c in range(Cn):
        n = len(clusters[c])
        r = np.zeros((n, K), np.uint32)
        for j in range(n):
            deg = int(rng.integers(0, K))
            r[j, 0] = deg
            r[j, 1:1 + deg] = rng.choice(clusters[c], size=deg, replace=False)
            r[j, 1 + deg:] = rng.integers(0, N, size=K - 1 - deg)
        rows.append(r)
        medoids.append(int(rng.choice(clusters[c])))
    return first, second, clusters, rows, medoids


@pytest.mark.parametrize("seed,bs,maxd", [(1, 2, 10), (2, 3, 12), (3, 7, 15), (4, 12, 8)])
def test_merge_matches_reference_restatement(capi, tmp_path, seed, bs, maxd):
    from oracle import large_merge as lm
    K = 16
    first, second, clusters, rows, medoids = scenario(seed, K=K)
    N, Cn = len(first), len(clusters)
    cpath = tmp_path / "centers.bin"
    np.stack([first, second], 1).astype(np.uint32).tofile(cpath)
    local = str(tmp_path / "local_")
    index = str(tmp_path / "final.index")
    p = capi.LargeParams()
    p.dim, p.k, p.cluster_num, p.max_points = 8, K, Cn, 10_000
    p.data_prefix = str(tmp_path / "unused_").encode()
    p.local_prefix = local.encode()
    p.index_store_path = index.encode()
    p.max_degree, p.buffer_size, p.num = maxd, bs, N
    p.centers_path = str(cpath).encode()
    p.thre, p.final_degree, p.topm, p.knn_iters, p.mode = 1.2, 12, 16, 4, 0
    keep = [np.ascontiguousarray(r) for r in rows]
    arr = (C.c_void_p * Cn)(*[r.ctypes.data for r in keep])
    meds = np.asarray(medoids, np.uint32)
    capi.check(capi.lib().tagore_large_merge(C.byref(p), arr, meds.ctypes.data_as(C.c_void_p)))
    f, s, cl = lm.clusters_from_centers(str(cpath), N, Cn)
    order, position, bs2 = lm.reorder(f, s, Cn, bs)
    exp_index, exp_files = lm.merge(rows, medoids, f, s, cl, order, position, bs2, K, maxd, None)
    assert open(index, "rb").read() == exp_index
    for cid, data in exp_files.items():
        assert open(local + str(cid), "rb").read() == data, f"spill file {cid}"


def test_large_rejections(capi, tmp_path):
    p = capi.LargeParams()
    p.k, p.cluster_num, p.num, p.buffer_size, p.max_degree = 16, 3, 10, 2, 8
    p.data_prefix = p.local_prefix = p.index_store_path = b"/tmp/x"
    p.centers_path = b"/nonexistent/centers"
    dev = (C.c_uint32 * 1)(0)
    assert capi.lib().tagore_large_index(C.byref(p), dev, 1) == capi.TAGORE_EIO
    p.max_degree = 16  # must stay below K
    assert capi.lib().tagore_large_index(C.byref(p), dev, 1) == capi.TAGORE_EINVAL
    assert capi.lib().tagore_large_index(C.byref(p), dev, 2) == capi.TAGORE_EINVAL


@pytest.mark.parametrize("missing", [0, 3, 6])
def test_a_failed_cluster_stops_every_builder(capi, tmp_path, missing):
    """One cluster's local graph is missing: the builder that takes it fails,
    the other builder threads and the merger stop, and the call returns the
    error instead of hanging or writing a partial index."""
    K = 16
    first, second, clusters, rows, medoids = scenario(5, K=K)
    N, Cn = len(first), len(clusters)
    cpath = tmp_path / "centers.bin"
    np.stack([first, second], 1).astype(np.uint32).tofile(cpath)
    p = capi.LargeParams()
    p.dim, p.k, p.cluster_num, p.max_points = 8, K, Cn, 10_000
    p.data_prefix = str(tmp_path / "unused_").encode()
    p.local_prefix = str(tmp_path / "local_").encode()
    p.index_store_path = str(tmp_path / "final.index").encode()
    p.max_degree, p.buffer_size, p.num = 10, 3, N
    p.centers_path = str(cpath).encode()
    p.thre, p.final_degree, p.topm, p.knn_iters, p.mode = 1.2, 12, 16, 4, 0
    keep = [np.ascontiguousarray(r) for r in rows]
    arr = (C.c_void_p * Cn)(*[None if c == missing else keep[c].ctypes.data for c in range(Cn)])
    meds = np.asarray(medoids, np.uint32)
    rc = capi.lib().tagore_large_merge(C.byref(p), arr, meds.ctypes.data_as(C.c_void_p))
    assert rc == capi.TAGORE_EINVAL
    assert f"no local graph for cluster {missing}".encode() in capi.lib().tagore_last_error()
