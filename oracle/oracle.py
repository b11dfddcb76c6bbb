"""ctypes binding of the CPU oracle (tagore_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py as the checker. The product never imports it.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libtagore_oracle.so")


class OrcState(C.Structure):
    _fields_ = [("n", C.c_uint32), ("k", C.c_uint32), ("dim", C.c_uint32),
                ("graph", C.c_void_p), ("reverse_graph", C.c_void_p), ("data", C.c_void_p),
                ("nei_distance", C.c_void_p), ("reverse_distance", C.c_void_p),
                ("reverse_num", C.c_void_p), ("center", C.c_void_p), ("hybrid_list", C.c_void_p)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} missing; run `make -C oracle`")
        L = C.CDLL(LIB_PATH)
        vp, u32, f32 = C.c_void_p, C.c_uint32, C.c_float
        S = C.POINTER(OrcState)
        sigs = {
            "orc_dist": (f32, [vp, vp, u32]),
            "orc_dist_pairs": (None, [vp, u32, vp, vp, C.c_uint64, vp]),
            "orc_f2h": (C.c_uint16, [f32]),
            "orc_h2f": (f32, [C.c_uint16]),
            "orc_network_sort_u32": (None, [vp, vp, u32]),
            "orc_cal_ep": (C.c_int, [S, u32, C.POINTER(u32)]),
            "orc_select_path": (C.c_int, [S, u32, u32, u32, f32]),
            "orc_select_2hop": (C.c_int, [S, u32, f32]),
            "orc_filter_reverse": (C.c_int, [S, u32, C.c_int, f32]),
            "orc_select_1hop_cagra": (C.c_int, [S, u32]),
            "orc_select_1hop_dpg": (C.c_int, [S, u32]),
            "orc_filter_reverse_1hop": (C.c_int, [S, u32]),
            "orc_prune": (C.c_int, [S, u32, u32, C.c_char_p, f32, C.POINTER(u32)]),
            "orc_prune_cfs": (C.c_int, [S, u32, u32, C.c_char_p, C.c_char_p, f32, C.POINTER(u32)]),
            "orc_host_prep": (C.c_int, [vp, u32, u32, vp, vp, C.POINTER(f32)]),
            "orc_bruteforce_knn": (C.c_int, [vp, u32, u32, vp, u32, u32, vp, vp]),
            "orc_greedy_search": (C.c_int, [vp, u32, u32, vp, vp, u32, vp, u32, u32, u32, C.c_uint64, vp]),
            "orc_nndescent": (C.c_int, [vp, u32, u32, u32, u32, u32, C.c_uint64, vp, vp]),
            "orc_num_threads": (C.c_int, []),
            "orc_gnn_descent_model": (C.c_int, [vp, u32, u32, u32, u32, C.c_uint64, vp, vp]),
        }
        for name, (res, args) in sigs.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class Buffers:
    """Host copies of the reference's eight buffers, as the oracle mutates them."""

    def __init__(self, graph, nei_distance, data_f16, center_f16=None, reverse_graph=None,
                 reverse_distance=None, reverse_num=None, hybrid_list=None):
        n, k = graph.shape
        dim = data_f16.shape[1]
        self.n, self.k, self.dim = n, k, dim
        self.graph = np.ascontiguousarray(graph, dtype=np.uint32).reshape(-1).copy()
        self.nei_distance = np.ascontiguousarray(nei_distance, dtype=np.float32).reshape(-1).copy()
        self.data = np.ascontiguousarray(data_f16, dtype=np.float16).reshape(-1).copy()
        self.center = (np.zeros(dim, np.float16) if center_f16 is None
                       else np.ascontiguousarray(center_f16, dtype=np.float16).copy())
        z = lambda m, dt: np.zeros(m, dtype=dt)
        self.reverse_graph = z(n * 128, np.uint32) if reverse_graph is None else \
            np.ascontiguousarray(reverse_graph, dtype=np.uint32).reshape(-1).copy()
        self.reverse_distance = z(n * 128, np.float32) if reverse_distance is None else \
            np.ascontiguousarray(reverse_distance, dtype=np.float32).reshape(-1).copy()
        self.reverse_num = z(n, np.uint32) if reverse_num is None else \
            np.ascontiguousarray(reverse_num, dtype=np.uint32).copy()
        self.hybrid_list = z(n * 128, np.uint32) if hybrid_list is None else \
            np.ascontiguousarray(hybrid_list, dtype=np.uint32).reshape(-1).copy()

    def state(self):
        return OrcState(self.n, self.k, self.dim, _p(self.graph).value,
                        _p(self.reverse_graph).value, _p(self.data).value,
                        _p(self.nei_distance).value, _p(self.reverse_distance).value,
                        _p(self.reverse_num).value, _p(self.center).value,
                        _p(self.hybrid_list).value)


def dist(a_f16, b_f16):
    a = np.ascontiguousarray(a_f16, dtype=np.float16)
    b = np.ascontiguousarray(b_f16, dtype=np.float16)
    return lib().orc_dist(_p(a), _p(b), a.shape[-1])


def dist_pairs(data_f16, ia, ib):
    data = np.ascontiguousarray(data_f16, dtype=np.float16)
    ia = np.ascontiguousarray(ia, dtype=np.uint32).reshape(-1)
    ib = np.ascontiguousarray(ib, dtype=np.uint32).reshape(-1)
    out = np.empty(ia.shape[0], np.float32)
    lib().orc_dist_pairs(_p(data), data.shape[1], _p(ia), _p(ib), ia.shape[0], _p(out))
    return out


def prune(buf, final_degree, index_type, topm=64, thre=1.0):
    st = buf.state()
    ep = C.c_uint32(0)
    rc = lib().orc_prune(C.byref(st), final_degree, topm, index_type.encode(), thre, C.byref(ep))
    if rc:
        raise ValueError(f"oracle rejected {index_type}")
    return ep.value


def prune_cfs(buf, final_degree, mode, metric, topm=64, thre=1.0):
    st = buf.state()
    ep = C.c_uint32(0)
    rc = lib().orc_prune_cfs(C.byref(st), final_degree, topm, mode.encode(), metric.encode(), thre,
                             C.byref(ep))
    if rc:
        raise ValueError(f"oracle rejected {mode}/{metric}")
    return ep.value


def cal_ep(buf, topm=64):
    st = buf.state()
    ep = C.c_uint32(0)
    lib().orc_cal_ep(C.byref(st), topm, C.byref(ep))
    return ep.value


def host_prep(data):
    data = np.ascontiguousarray(data, dtype=np.float32)
    n, dim = data.shape
    half = np.empty((n, dim), np.float16)
    center = np.empty(dim, np.float16)
    f = C.c_float(0)
    lib().orc_host_prep(_p(data), n, dim, _p(half), _p(center), C.byref(f))
    return half, center, f.value


def bruteforce_knn(base, queries, k, exclude_self=None):
    base = np.ascontiguousarray(base, dtype=np.float32)
    q = np.ascontiguousarray(queries, dtype=np.float32)
    out = np.empty((q.shape[0], k), np.uint32)
    ex = None
    if exclude_self is not None:
        ex = np.ascontiguousarray(exclude_self, dtype=np.uint32)
    lib().orc_bruteforce_knn(_p(base), base.shape[0], base.shape[1], _p(q), q.shape[0], k,
                             _p(ex) if ex is not None else None, _p(out))
    return out


def greedy_search(base, offsets, adj, ep, queries, L, k, seed=0):
    base = np.ascontiguousarray(base, dtype=np.float32)
    q = np.ascontiguousarray(queries, dtype=np.float32)
    offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
    adj = np.ascontiguousarray(adj, dtype=np.uint32)
    out = np.empty((q.shape[0], k), np.uint32)
    lib().orc_greedy_search(_p(base), base.shape[0], base.shape[1], _p(offsets), _p(adj), ep, _p(q),
                            q.shape[0], L, k, seed, _p(out))
    return out


def nndescent(base, k, iters, sample=32, seed=0x7A6E):
    base = np.ascontiguousarray(base, dtype=np.float32)
    n, dim = base.shape
    ids = np.empty((n, k), np.uint32)
    dis = np.empty((n, k), np.float32)
    rc = lib().orc_nndescent(_p(base), n, dim, k, iters, sample, seed, _p(ids), _p(dis))
    if rc:
        raise ValueError("bad nndescent arguments")
    return ids, dis


def gnn_descent_model(data_f16, K, iters, seed=0x7A6E):
    """The reference's two-phase GNN_descent restated on the CPU
    (gnn_descent_model.cpp): returns (ids, dists), each n x K."""
    data = np.ascontiguousarray(data_f16, dtype=np.float16)
    n, dim = data.shape
    ids = np.empty((n, K), np.uint32)
    dis = np.empty((n, K), np.float32)
    rc = lib().orc_gnn_descent_model(_p(data), n, dim, K, iters, seed, _p(ids), _p(dis))
    if rc:
        raise ValueError("gnn_descent_model needs K in {32, 64, 96}, dim % 4 == 0 and n > K")
    return ids, dis


def num_threads():
    return lib().orc_num_threads()


def exact_knn(data_f16, K):
    """Exact kNN rows of an FP16 base (self excluded), ranked by FP32 distance
    of the FP16 values, with the oracle's reference-order distances."""
    x = np.asarray(data_f16, dtype=np.float32)
    n = x.shape[0]
    sq = (x * x).sum(1)
    ids = np.empty((n, K), np.uint32)
    for s in range(0, n, 4096):
        e = min(n, s + 4096)
        d2 = sq[s:e, None] + sq[None, :] - 2.0 * (x[s:e] @ x.T)
        d2[np.arange(e - s), np.arange(s, e)] = np.inf
        part = np.argpartition(d2, K, axis=1)[:, :K]
        order = np.take_along_axis(d2, part, 1).argsort(1, kind="stable")
        ids[s:e] = np.take_along_axis(part, order, 1)
    dis = dist_pairs(data_f16, np.repeat(np.arange(n, dtype=np.uint32), K), ids.reshape(-1))
    dis = dis.reshape(n, K)
    order = np.argsort(dis, axis=1, kind="stable")
    return np.take_along_axis(ids, order, 1), np.take_along_axis(dis, order, 1)


def knn_input(data_f16, K, noise=0.0, seed=1):
    """A kNN graph for prune tests: exact rows, then a fraction `noise` of the
    entries replaced by random ids (as an approximate build would leave),
    rows re-sorted by distance."""
    ids, dis = exact_knn(data_f16, K)
    n = ids.shape[0]
    if noise > 0:
        rng = np.random.default_rng(seed)
        mask = rng.random(ids.shape) < noise
        repl = rng.integers(0, n, size=ids.shape).astype(np.uint32)
        ids = np.where(mask, repl, ids).astype(np.uint32)
        dis = dist_pairs(data_f16, np.repeat(np.arange(n, dtype=np.uint32), K),
                         ids.reshape(-1)).reshape(n, K)
        order = np.argsort(dis, axis=1, kind="stable")
        ids = np.take_along_axis(ids, order, 1)
        dis = np.take_along_axis(dis, order, 1)
    return np.ascontiguousarray(ids), np.ascontiguousarray(dis)
