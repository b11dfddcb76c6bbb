"""The largeIndex host half against the reference's own code.

oracle/_ref/merge_ref is the reference's order_merge_main and order_merge_new
(src/large_index.cu:86-106, :286-522), compiled from its sources by
oracle/build_ref.sh, driven on given local graphs the way gpu_construct hands
them over (:255-277). This library's tagore_large_merge gets the same cluster
assignment, local graphs and entry points; the final index file and every
spill file must be identical byte for byte. Local rows hold at most
max_degree ids: the reference's final merge reads a spilled row into a
max_degree-sized buffer and overflows it on longer rows. Skipped where the
reference was not built.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MERGE_REF = os.path.join(ROOT, "oracle", "_ref", "merge_ref")

pytestmark = pytest.mark.skipif(not os.path.exists(MERGE_REF),
                                reason="reference merger not built (oracle/build_ref.sh)")


def scenario(seed, N, Cn, K, maxd):
    rng = np.random.default_rng(seed)
    first = rng.integers(0, Cn, size=N)
    second = (first + rng.integers(1, Cn, size=N)) % Cn  # a different cluster
    clusters = [[] for _ in range(Cn)]
    for i in range(N):
        clusters[first[i]].append(i)
        clusters[second[i]].append(i)
    rows, eps = [], []
    for c in range(Cn):
        n = len(clusters[c])
        r = rng.integers(0, N, size=(n, K)).astype(np.uint32)
        # local degrees up to max_degree: longer rows overflow the reference's
        # buffers in its final merge (neighbors(max_degree), :483-497)
        deg = rng.integers(0, maxd + 1, size=n)
        for j in range(n):
            r[j, 0] = deg[j]
            r[j, 1:1 + deg[j]] = rng.choice(clusters[c], size=deg[j], replace=False)
        rows.append(r)
        eps.append(int(rng.choice(clusters[c])))
    return first.astype(np.uint32), second.astype(np.uint32), clusters, rows, eps


@pytest.mark.parametrize("seed,N,Cn,K,bs,maxd",
                         [(1, 3000, 7, 16, 2, 10), (2, 4000, 9, 24, 3, 12), (3, 2500, 6, 16, 6, 15),
                          (4, 5000, 12, 32, 4, 22),
                          # the final pass splits the points into ranges of at least 4,096,
                          # merged on separate threads: several ranges here
                          (5, 40000, 16, 24, 5, 16)])
def test_merge_equals_reference_merger(capi, tmp_path, seed, N, Cn, K, bs, maxd):
    first, second, clusters, rows, eps = scenario(seed, N, Cn, K, maxd)
    ref_dir, our_dir = tmp_path / "ref", tmp_path / "ours"
    ref_dir.mkdir()
    our_dir.mkdir()
    inp = tmp_path / "input.bin"
    with open(inp, "wb") as f:
        np.array([N, Cn, K, maxd, bs], np.uint32).tofile(f)
        np.stack([first, second], 1).astype(np.uint32).tofile(f)
        for r in rows:
            r.tofile(f)
        np.array(eps, np.uint32).tofile(f)
    out = subprocess.run([MERGE_REF, str(inp), str(ref_dir / "final.index"), str(ref_dir / "local_")],
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]

    np.stack([first, second], 1).astype(np.uint32).tofile(tmp_path / "centers.bin")
    p = capi.LargeParams()
    p.dim, p.k, p.cluster_num, p.max_points = 8, K, Cn, max(len(c) for c in clusters)
    p.data_prefix = str(tmp_path / "unused_").encode()
    p.local_prefix = str(our_dir / "local_").encode()
    p.index_store_path = str(our_dir / "final.index").encode()
    p.max_degree, p.buffer_size, p.num = maxd, bs, N
    p.centers_path = str(tmp_path / "centers.bin").encode()
    arrs = [np.ascontiguousarray(r) for r in rows]
    ptrs = (C.c_void_p * Cn)(*[a.ctypes.data for a in arrs])
    meds = np.array(eps, np.uint32)
    capi.check(capi.lib().tagore_large_merge(C.byref(p), ptrs, meds.ctypes.data_as(C.c_void_p)))

    ref_final = open(ref_dir / "final.index", "rb").read()
    our_final = open(our_dir / "final.index", "rb").read()
    assert len(ref_final) == len(our_final) and ref_final == our_final
    for c in range(Cn):
        a = open(ref_dir / f"local_{c}", "rb").read()
        b = open(our_dir / f"local_{c}", "rb").read()
        assert a == b, f"spill file of cluster {c} differs"
