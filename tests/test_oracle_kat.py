"""Known-answer tests that pin the CPU oracle independently of the GPU code.

* The reference-order FP32 distance is recomputed with exact rational
  arithmetic and explicit IEEE float32 rounding.
* The bitonic network is restated a second time in Python from the
  reference's loop (src/Tagore_src.cu:29-44) and compared on inputs with ties.
* A line graph, whose NSG prune keeps exactly the nearest neighbour on each
  side of every node, gives hand-derived prune results.
* CAGRA and DPG detour counts are recomputed from their definitions.
* The host preparation follows pybind.cu:24-61 step by step.
"""
import math
from fractions import Fraction

import numpy as np
import pytest


def round_f32(x):
    """Nearest float32 of an exact rational (ties to even), as a Fraction."""
    if x == 0:
        return Fraction(0)
    sign = -1 if x < 0 else 1
    a = abs(x)
    e = a.numerator.bit_length() - a.denominator.bit_length()
    if Fraction(2) ** e > a:
        e -= 1
    if Fraction(2) ** (e + 1) <= a:
        e += 1
    e = max(e, -126)
    q = a * Fraction(2) ** (23 - e)
    n = q.numerator // q.denominator
    r = q - n
    if r > Fraction(1, 2) or (r == Fraction(1, 2) and n % 2 == 1):
        n += 1
    return sign * Fraction(n) * Fraction(2) ** (e - 23)


def lane_order_dist(a16, b16):
    a = [Fraction(float(v)) for v in a16]
    b = [Fraction(float(v)) for v in b16]
    lx = [Fraction(0)] * 32
    ly = [Fraction(0)] * 32
    for j in range(len(a) // 4):
        l = j % 32
        d = [round_f32(a[4 * j + t] - b[4 * j + t]) for t in range(4)]
        lx[l] = round_f32(d[0] * d[0] + lx[l])
        ly[l] = round_f32(d[1] * d[1] + ly[l])
        lx[l] = round_f32(d[2] * d[2] + lx[l])
        ly[l] = round_f32(d[3] * d[3] + ly[l])
    off = 16
    while off:
        for l in range(off):
            lx[l] = round_f32(lx[l] + lx[l + off])
            ly[l] = round_f32(ly[l] + ly[l + off])
        off //= 2
    return round_f32(lx[0] + ly[0])


@pytest.mark.parametrize("dim", [4, 16, 96, 128, 960])
def test_distance_is_reference_lane_order(orc, dim):
    rng = np.random.default_rng(dim)
    for trial in range(3):
        a = (rng.random(dim) * 3).astype(np.float16)
        b = (rng.random(dim) * 3).astype(np.float16)
        got = Fraction(float(np.float32(orc.dist(a, b))))
        assert got == lane_order_dist(a, b)


def test_distance_close_to_exact(orc):
    rng = np.random.default_rng(7)
    a = (rng.random((50, 128)) * 2.5).astype(np.float16)
    b = (rng.random((50, 128)) * 2.5).astype(np.float16)
    for x, y in zip(a, b):
        ref = float(((x.astype(np.float64) - y.astype(np.float64)) ** 2).sum())
        assert abs(orc.dist(x, y) - ref) <= 1e-5 * ref + 1e-6


def py_network(keys, payload):
    """Second restatement of the reference's bitonic loop."""
    keys = list(keys)
    payload = list(payload)
    n = len(keys)
    stride = 1
    while stride < n:
        step = stride
        while step > 0:
            for k in range(n // 2):
                a = 2 * step * (k // step)
                b = k % step
                u = a + step - 1 - b if step == stride else a + b
                d = a + b + step
                if d < n and keys[u] > keys[d]:
                    keys[u], keys[d] = keys[d], keys[u]
                    payload[u], payload[d] = payload[d], payload[u]
            step //= 2
        stride *= 2
    return keys, payload


@pytest.mark.parametrize("n", [0, 1, 2, 3, 5, 31, 64, 96, 160, 576])
def test_network_sorts_and_places_ties_like_reference(orc, n):
    rng = np.random.default_rng(n)
    keys = rng.integers(0, max(2, n // 4), size=n).astype(np.uint32)
    pay = np.arange(n, dtype=np.uint32)
    k2, p2 = keys.copy(), pay.copy()
    import ctypes as C
    orc.lib().orc_network_sort_u32(k2.ctypes.data_as(C.c_void_p), p2.ctypes.data_as(C.c_void_p), n)
    ek, ep = py_network(keys.tolist(), pay.tolist())
    assert k2.tolist() == sorted(keys.tolist()) == ek
    assert p2.tolist() == ep


def line_points(n):
    """Points on a line with strictly growing gaps (distinct, exact in FP16)."""
    pos = np.cumsum(np.arange(1, n + 1)) / 8.0
    x = np.zeros((n, 4), np.float16)
    x[:, 0] = pos
    return x


@pytest.mark.parametrize("fd", [3, 4, 6])
def test_nsg_on_a_line_keeps_nearest_per_side(orc, fd):
    n, K = 30, 24
    x = line_points(n)
    ids, dis = orc.knn_input(x, K)
    buf = orc.Buffers(ids, dis, x, center_f16=x[n // 2])
    orc.prune_cfs(buf, fd, "path", "dist", topm=16, thre=1.0)
    g = buf.graph.reshape(n, K)
    for u in range(n):
        side = [v for v in (u - 1, u + 1) if 0 <= v < n]
        side.sort(key=lambda v: abs(float(x[v, 0]) - float(x[u, 0])))
        deg = int(g[u, 0])
        assert deg == len(side), (u, g[u, :4])
        assert g[u, 1:1 + deg].tolist() == side
        # slots past the degree keep the kNN row (rows are rewritten in place)
        assert g[u, 1 + deg:].tolist() == ids[u, 1 + deg:].tolist()


def test_entry_point_is_nearest_to_center(orc):
    n, K = 30, 24
    x = line_points(n)
    ids, dis = orc.knn_input(x, K)
    buf = orc.Buffers(ids, dis, x, center_f16=x[17])
    assert orc.cal_ep(buf, topm=16) == 17


def detours(graph, u, K):
    nei0 = graph[u]
    det = [0] * K
    pairs = set()
    for i in range(K // 2):
        for a in (i, K - 1 - i):
            for m in range(a + 1, K):
                pairs.add((a, m))
    for a, m in pairs:
        if nei0[m] in set(graph[nei0[a]].tolist()):
            det[m] += 1
    return det


def test_cagra_forward_lists_follow_detour_counts(orc):
    rng = np.random.default_rng(3)
    n, K, d = 200, 32, 16
    x = (rng.random((n, 16)) * 2).astype(np.float16)
    ids, dis = orc.knn_input(x, K)
    buf = orc.Buffers(ids, dis, x)
    orc.prune(buf, d, "CAGRA")
    hyb = buf.hybrid_list[:n * K].reshape(n, K)  # new_list rows have stride K (:1708)
    for u in range(0, n, 7):
        det = detours(ids, u, K)
        _, order = py_network(det, list(ids[u]))
        assert hyb[u, :d].tolist() == order[:d]


def dpg_detours(orc, x, ids, dis, u, K):
    """DPG's detour rule (src/Tagore_src.cu:1713-1785) from its definition: for
    the i-th nearest and the i-th farthest neighbour a (i < K/2), every later
    neighbour m of the row counts one detour when d(a, m) < d(u, m); the near
    one is compared with every m after it, the far one with the i entries
    after it. Each warp of the rule stages its own vector a."""
    nei0 = ids[u]
    det = [0] * K
    for i in range(K // 2):
        for a, later in ((i, range(i + 1, K)), (K - 1 - i, range(K - i, K))):
            for m in later:
                if orc.dist(x[nei0[a]], x[nei0[m]]) < dis[u, m]:
                    det[m] += 1
    return det


def test_dpg_forward_lists_follow_detour_counts(orc):
    rng = np.random.default_rng(5)
    n, K, d = 120, 40, 24
    x = (rng.random((n, 16)) * 2).astype(np.float16)
    ids, dis = orc.knn_input(x, K)
    buf = orc.Buffers(ids, dis, x)
    orc.prune(buf, d, "DPG")
    hyb = buf.hybrid_list[:n * K].reshape(n, K)
    for u in range(0, n, 5):
        det = dpg_detours(orc, x, ids, dis, u, K)
        _, order = py_network(det, list(ids[u]))
        assert hyb[u, :d].tolist() == order[:d], u


def test_host_prep_matches_reference_steps(orc):
    from tagore_b200 import synth
    base, _ = synth.mixture("sift", 3000, 128, 8, 11)
    half, center, factor = orc.host_prep(base)
    ave = np.float32(0)
    for v in base[0]:
        ave = np.float32(ave + np.float32(abs(v)))
    ave = np.float32(ave / np.float32(128))
    f = np.float32(1)
    while ave < 0.5:
        ave, f = np.float32(ave * 10), np.float32(f * 10)
    while ave > 5:
        ave, f = np.float32(ave / 10), np.float32(f / 10)
    assert factor == f
    c = np.cumsum(base, axis=0, dtype=np.float32)[-1] / np.float32(base.shape[0])
    assert np.array_equal(center, (c.astype(np.float32) * f).astype(np.float16))
    assert np.array_equal(half, (base * f).astype(np.float16))


def test_greedy_search_walks_a_line(orc):
    """NSG's search on a hand-checkable graph: ten points on a line, each
    linked to its two neighbours. From node 0 with a pool of 3 and no random
    starts, the search must expand along the line and end with the three
    nodes nearest to a query past node 9, in distance order; with a pool of
    1 it still reaches node 9, since every step finds a closer neighbour."""
    base = np.zeros((10, 4), np.float32)
    base[:, 0] = np.arange(10)
    offs, adj = [0], []
    for i in range(10):
        adj += [j for j in (i - 1, i + 1) if 0 <= j < 10]
        offs.append(len(adj))
    offs = np.array(offs, np.uint64)
    adj = np.array(adj, np.uint32)
    q = np.array([[9.4, 0, 0, 0]], np.float32)
    assert orc.greedy_search(base, offs, adj, 0, q, 3, 3, 0).tolist() == [[9, 8, 7]]
    assert orc.greedy_search(base, offs, adj, 0, q, 1, 1, 0).tolist() == [[9]]
    # k past the pool: the slots the pool cannot fill hold 0xFFFFFFFF
    assert orc.greedy_search(base, offs, adj, 0, q, 2, 4, 0).tolist() == [[9, 8, 0xFFFFFFFF,
                                                                          0xFFFFFFFF]]


def test_reference_gnn_descent_model_runs(orc):
    """The CPU model of the reference's GNN_descent: sorted rows of valid,
    non-self ids whose recall is well above chance after two iterations."""
    from tagore_b200 import synth
    n, d, K = 2000, 128, 32
    base, _ = synth.mixture("sift", n, d, 8, 13)
    half, _, _ = orc.host_prep(base)
    ids, dis = orc.gnn_descent_model(half.reshape(n, d), K, 2)
    assert ids.max() < n and not (ids == np.arange(n)[:, None]).any()
    assert (np.diff(dis, axis=1) >= 0).all()
    gt = orc.bruteforce_knn(base, base, 10, exclude_self=np.arange(n, dtype=np.uint32))
    hit = (ids[:, :10, None] == gt[:, None, :]).any(-1).sum(1).mean() / 10
    assert hit > 0.5
    with pytest.raises(ValueError):
        orc.gnn_descent_model(half.reshape(n, d), 40, 2)
