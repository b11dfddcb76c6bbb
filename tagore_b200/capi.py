"""ctypes binding of the C ABI in include/tagore_b200.h.

This is how tests and benchmarks call the library; users of the reference's
API import the compiled `Tagore` module instead. Loading fails loudly when the
library has not been built: there is no fallback.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libtagore_b200.so")

TAGORE_OK, TAGORE_EINVAL, TAGORE_EIO, TAGORE_ENOMEM, TAGORE_ECUDA, TAGORE_ETIMEOUT = range(6)
KNN_CHOSEN, KNN_PLAIN, KNN_LEARNED = 0, 1, 2
LEARN_FIXED_T, LEARN_NO_TRAIN = 1, 2

# Buffer index -> (name, numpy dtype); the reference's capsule order.
BUFFERS = [("graph", np.uint32), ("reverse_graph", np.uint32), ("data", np.float16),
           ("nei_distance", np.float32), ("reverse_distance", np.float32),
           ("reverse_num", np.uint32), ("center", np.float16), ("hybrid_list", np.uint32),
           ("norms", np.float32)]


class KnnState(C.Structure):
    _fields_ = [("n", C.c_uint32), ("dim", C.c_uint32), ("k", C.c_uint32), ("device", C.c_int32),
                ("norm_factor", C.c_float), ("ep", C.c_uint32),
                ("graph", C.c_void_p), ("reverse_graph", C.c_void_p), ("data", C.c_void_p),
                ("nei_distance", C.c_void_p), ("reverse_distance", C.c_void_p),
                ("reverse_num", C.c_void_p), ("center", C.c_void_p), ("hybrid_list", C.c_void_p),
                ("norms", C.c_void_p), ("owns", C.c_uint32), ("pad_", C.c_uint32)]


class KnnParams(C.Structure):
    _fields_ = [("k", C.c_uint32), ("n", C.c_uint32), ("dim", C.c_uint32), ("iters", C.c_uint32),
                ("mode", C.c_uint32), ("sample", C.c_uint32), ("per_row", C.c_uint32),
                ("rescale", C.c_uint32), ("seed", C.c_uint64), ("learn_steps", C.c_uint32),
                ("learn_flags", C.c_uint32)]


class PruneParams(C.Structure):
    _fields_ = [("k", C.c_uint32), ("n", C.c_uint32), ("dim", C.c_uint32),
                ("final_degree", C.c_uint32), ("topm", C.c_uint32), ("thre", C.c_float)]


class LargeParams(C.Structure):
    _fields_ = [("dim", C.c_uint32), ("k", C.c_uint32), ("cluster_num", C.c_uint32),
                ("max_points", C.c_uint32), ("data_prefix", C.c_char_p),
                ("local_prefix", C.c_char_p), ("index_store_path", C.c_char_p),
                ("max_degree", C.c_uint32), ("buffer_size", C.c_uint32), ("num", C.c_uint32),
                ("centers_path", C.c_char_p), ("thre", C.c_float), ("final_degree", C.c_uint32),
                ("topm", C.c_uint32), ("knn_iters", C.c_uint32), ("mode", C.c_uint32)]


class Timings(C.Structure):
    _fields_ = [("knn_ms", C.c_double), ("prune_ms", C.c_double), ("prep_ms", C.c_double),
                ("total_ms", C.c_double), ("kernel_launches", C.c_uint64)]


class ScreenStats(C.Structure):
    _fields_ = [("used", C.c_uint32), ("steps", C.c_uint32), ("screened_iters", C.c_uint32),
                ("per_row", C.c_uint32), ("fallback", C.c_uint32), ("pad_", C.c_uint32),
                ("loss_first", C.c_float), ("loss_last", C.c_float), ("last_miss", C.c_double),
                ("last_best_kept", C.c_double)]


class SearchParams(C.Structure):
    _fields_ = [("L", C.c_uint32), ("k", C.c_uint32), ("seed", C.c_uint64),
                ("visit_cap", C.c_uint32), ("pad_", C.c_uint32)]


class IndexInfo(C.Structure):
    _fields_ = [("n", C.c_uint64), ("edges", C.c_uint64), ("max_degree", C.c_uint32),
                ("width", C.c_uint32), ("n_eps", C.c_uint32), ("eps", C.c_uint32 * 16),
                ("pad_", C.c_uint32)]


class StageStat(C.Structure):
    _fields_ = [("name", C.c_char * 32), ("ms", C.c_double), ("launches", C.c_uint64),
                ("bytes", C.c_uint64), ("items", C.c_uint64)]


# Every exported entry point with its C signature (restype, argtypes).
SIGNATURES = {
    "tagore_gnn_descent": (C.c_int, [C.POINTER(KnnParams), C.c_char_p, C.POINTER(KnnState)]),
    "tagore_gnn_descent_host": (C.c_int, [C.POINTER(KnnParams), C.c_void_p, C.c_uint32,
                                          C.c_uint32, C.POINTER(KnnState)]),
    "tagore_pruning": (C.c_int, [C.POINTER(PruneParams), C.POINTER(KnnState), C.c_char_p,
                                 C.c_char_p]),
    "tagore_pruning_cfs": (C.c_int, [C.POINTER(PruneParams), C.POINTER(KnnState), C.c_char_p,
                                     C.c_char_p]),
    "tagore_pruning_cfs_noalloc": (C.c_int, [C.POINTER(PruneParams), C.POINTER(KnnState),
                                             C.c_char_p, C.c_char_p, C.c_void_p]),
    "tagore_large_index": (C.c_int, [C.POINTER(LargeParams), C.c_void_p, C.c_int]),
    "tagore_large_merge": (C.c_int, [C.POINTER(LargeParams), C.POINTER(C.c_void_p), C.c_void_p]),
    "tagore_entry_point": (C.c_int, [C.POINTER(KnnState), C.c_uint32, C.POINTER(C.c_uint32)]),
    "tagore_connect": (C.c_int, [C.POINTER(KnnState), C.c_uint32, C.POINTER(C.c_uint64)]),
    "tagore_search": (C.c_int, [C.POINTER(SearchParams), C.c_void_p, C.c_uint64, C.c_uint32,
                                C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint32, C.c_void_p,
                                C.c_uint32, C.c_void_p, C.c_void_p]),
    "tagore_index_info": (C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(IndexInfo)]),
    "tagore_index_read": (C.c_int, [C.c_char_p, C.c_char_p, C.c_uint64, C.c_uint64, C.c_void_p,
                                    C.c_void_p]),
    "tagore_state_alloc": (C.c_int, [C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(KnnState)]),
    "tagore_state_free": (C.c_int, [C.POINTER(KnnState)]),
    "tagore_state_upload": (C.c_int, [C.POINTER(KnnState), C.c_int, C.c_void_p, C.c_size_t]),
    "tagore_state_download": (C.c_int, [C.POINTER(KnnState), C.c_int, C.c_void_p, C.c_size_t]),
    "tagore_state_bytes": (C.c_size_t, [C.POINTER(KnnState), C.c_int]),
    "tagore_build_index_host": (C.c_int, [C.POINTER(KnnParams), C.c_void_p, C.c_uint32,
                                          C.c_uint32, C.c_uint32, C.c_uint32, C.c_float,
                                          C.c_void_p, C.POINTER(C.c_uint32)]),
    "tagore_store_nsg": (C.c_int, [C.c_char_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32,
                                   C.c_uint32]),
    "tagore_store_vamana": (C.c_int, [C.c_char_p, C.c_void_p, C.c_uint32, C.c_uint32,
                                      C.c_uint32]),
    "tagore_store_nssg": (C.c_int, [C.c_char_p, C.c_void_p, C.c_uint32, C.c_uint32,
                                    C.c_uint32]),
    "tagore_store_dpg": (C.c_int, [C.c_char_p, C.c_void_p, C.c_uint32, C.c_uint32]),
    "tagore_store_cagra": (C.c_int, [C.c_char_p, C.c_void_p, C.c_uint32, C.c_uint32]),
    "tagore_load_fvecs_header": (C.c_int, [C.c_char_p, C.POINTER(C.c_uint32),
                                           C.POINTER(C.c_uint32)]),
    "tagore_load_fvecs": (C.c_int, [C.c_char_p, C.c_void_p, C.c_uint32, C.c_uint32]),
    "tagore_last_timings": (C.c_int, [C.POINTER(Timings)]),
    "tagore_gnn_descent_device": (C.c_int, [C.POINTER(KnnParams), C.c_void_p, C.c_void_p,
                                            C.c_uint32, C.c_uint32, C.POINTER(KnnState)]),
    "tagore_set_stream": (C.c_int, [C.c_void_p]),
    "tagore_reset_counters": (C.c_int, []),
    "tagore_set_profiling": (C.c_int, [C.c_int]),
    "tagore_stage_stats": (C.c_int, [C.POINTER(StageStat), C.c_int, C.POINTER(C.c_int)]),
    "tagore_device_free": (C.c_int, [C.c_void_p]),
    "tagore_allocation_count": (C.c_uint64, []),
    "tagore_trim_cache": (C.c_int, []),
    "tagore_wait_selftest": (C.c_int, [C.POINTER(C.c_int)]),
    "tagore_last_screen": (C.c_int, [C.POINTER(ScreenStats)]),
    "tagore_mlp_loss_grad": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_uint32,
                                       C.c_void_p, C.c_void_p, C.POINTER(C.c_double)]),
    "tagore_last_error": (C.c_char_p, []),
    "tagore_version": (C.c_char_p, []),
}

_lib = None


class TagoreError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"tagore error {code}: {msg}")
        self.code = code


def lib():
    """Loads libtagore_b200.so once; raises if it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing; build it with `python -m tagore_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc):
    if rc != TAGORE_OK:
        raise TagoreError(rc, lib().tagore_last_error().decode())


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


class State:
    """Owns a TagoreKnnState (the eight device buffers plus norms)."""

    def __init__(self, st=None):
        self.st = st if st is not None else KnnState()

    @classmethod
    def alloc(cls, n, dim, k):
        s = cls()
        check(lib().tagore_state_alloc(n, dim, k, C.byref(s.st)))
        return s

    @classmethod
    def from_host(cls, graph, nei_distance, data_f16, center_f16=None, reverse_graph=None,
                  reverse_distance=None, reverse_num=None, hybrid_list=None):
        n, k = graph.shape
        dim = data_f16.shape[1]
        s = cls.alloc(n, dim, k)
        s.upload(0, graph)
        s.upload(3, nei_distance)
        s.upload(2, data_f16)
        if center_f16 is not None:
            s.upload(6, center_f16)
        for idx, arr in ((1, reverse_graph), (4, reverse_distance), (5, reverse_num),
                         (7, hybrid_list)):
            if arr is not None:
                s.upload(idx, arr)
        return s

    def upload(self, which, arr):
        arr = np.ascontiguousarray(arr, dtype=BUFFERS[which][1])
        check(lib().tagore_state_upload(C.byref(self.st), which, _ptr(arr), arr.nbytes))

    def download(self, which):
        nbytes = lib().tagore_state_bytes(C.byref(self.st), which)
        dt = np.dtype(BUFFERS[which][1])
        out = np.empty(nbytes // dt.itemsize, dtype=dt)
        check(lib().tagore_state_download(C.byref(self.st), which, _ptr(out), out.nbytes))
        return out

    def buffers(self):
        """All nine buffers as host arrays, keyed by name."""
        return {BUFFERS[i][0]: self.download(i) for i in range(9)}

    def free(self):
        lib().tagore_state_free(C.byref(self.st))

    def __del__(self):
        try:
            if self.st.owns:
                self.free()
        except Exception:
            pass


def knn_params(k, n, dim, iters, mode=KNN_CHOSEN, sample=0, per_row=0, rescale=1, seed=0x7A6E,
               learn_steps=0, learn_flags=0):
    return KnnParams(k, n, dim, iters, mode, sample, per_row, rescale, seed, learn_steps,
                     learn_flags)


def gnn_descent_host(data, k, iters, mode=KNN_CHOSEN, rescale=1, seed=0x7A6E, sample=0, per_row=0,
                     learn_steps=0, learn_flags=0):
    data = np.ascontiguousarray(data, dtype=np.float32)
    n, dim = data.shape
    p = knn_params(k, n, dim, iters, mode, sample, per_row, rescale, seed, learn_steps, learn_flags)
    s = State()
    check(lib().tagore_gnn_descent_host(C.byref(p), _ptr(data), n, dim, C.byref(s.st)))
    return s


def gnn_descent_file(path, k, iters, mode=KNN_CHOSEN, rescale=1, seed=0x7A6E):
    """GNN_descent from an fvecs file; the file is parsed on the device."""
    n, dim = C.c_uint32(), C.c_uint32()
    check(lib().tagore_load_fvecs_header(str(path).encode(), C.byref(n), C.byref(dim)))
    p = knn_params(k, n.value, dim.value, iters, mode, 0, 0, rescale, seed)
    s = State()
    check(lib().tagore_gnn_descent(C.byref(p), str(path).encode(), C.byref(s.st)))
    return s


def pruning(state, final_degree, index_type, topm=64, thre=1.0, index_path=None):
    st = state.st
    p = PruneParams(st.k, st.n, st.dim, final_degree, topm, thre)
    path = index_path.encode() if index_path else None
    check(lib().tagore_pruning(C.byref(p), C.byref(st), index_type.encode(), path))
    return st.ep


def pruning_cfs(state, final_degree, mode, metric, topm=64, thre=1.0):
    st = state.st
    p = PruneParams(st.k, st.n, st.dim, final_degree, topm, thre)
    check(lib().tagore_pruning_cfs(C.byref(p), C.byref(st), mode.encode(), metric.encode()))
    return st.ep


def pruning_cfs_noalloc(state, final_degree, mode, metric, topm=64, thre=1.0, stream=None):
    st = state.st
    p = PruneParams(st.k, st.n, st.dim, final_degree, topm, thre)
    check(lib().tagore_pruning_cfs_noalloc(C.byref(p), C.byref(st), mode.encode(), metric.encode(),
                                           stream))
    return st.ep


def connect(state, ep):
    """Opt-in connectivity fix; returns the number of edges added."""
    added = C.c_uint64(0)
    check(lib().tagore_connect(C.byref(state.st), ep, C.byref(added)))
    return added.value


def rows_to_csr(rows):
    """[deg, ids...] rows (the pruned graph) as CSR: offs (n+1 u64), adj (u32)."""
    rows = np.asarray(rows, dtype=np.uint32)
    deg = rows[:, 0].astype(np.int64)
    if np.any(deg >= rows.shape[1]):
        raise ValueError("a row's degree exceeds its width")
    offs = np.zeros(rows.shape[0] + 1, np.uint64)
    offs[1:] = np.cumsum(deg)
    mask = np.arange(rows.shape[1] - 1)[None, :] < deg[:, None]
    return offs, np.ascontiguousarray(rows[:, 1:][mask], dtype=np.uint32)


def search(base, offs, adj, ep, queries, L, k, seed=0, visit_cap=0, stream=None):
    """Greedy search on the current CUDA device. base (n x dim f32), offs
    (n+1 u64 as int64), adj (u32 as int32), queries (nq x dim f32) are CUDA
    tensors; returns an nq x k int64 tensor of ids (-1 where the pool ran
    short)."""
    import torch
    for t in (base, offs, adj, queries):
        if not t.is_cuda or not t.is_contiguous():
            raise ValueError("search takes contiguous CUDA tensors")
    if base.dtype != torch.float32 or queries.dtype != torch.float32:
        raise ValueError("base and queries are float32")
    n, dim = base.shape
    nq = queries.shape[0] if queries.numel() else 0
    out = torch.empty((nq, k), dtype=torch.int32, device=base.device)
    p = SearchParams(L, k, seed, visit_cap, 0)
    check(lib().tagore_search(C.byref(p), base.data_ptr(), n, dim, offs.data_ptr(),
                              adj.data_ptr(), adj.numel(), ep, queries.data_ptr(), nq,
                              out.data_ptr(), stream))
    return out.to(torch.int64) & 0xFFFFFFFF


def index_info(path, index_type):
    info = IndexInfo()
    check(lib().tagore_index_info(str(path).encode(), index_type.encode(), C.byref(info)))
    return info


def index_read(path, index_type):
    """Reads an index file back: (info, offs n+1 u64, adj u32)."""
    info = index_info(path, index_type)
    offs = np.zeros(info.n + 1, np.uint64)
    adj = np.zeros(max(info.edges, 1), np.uint32)
    check(lib().tagore_index_read(str(path).encode(), index_type.encode(), info.n, info.edges,
                                  _ptr(offs), _ptr(adj)))
    return info, offs, adj[:info.edges]


def entry_point(state, topm=64):
    ep = C.c_uint32(0)
    check(lib().tagore_entry_point(C.byref(state.st), topm, C.byref(ep)))
    return ep.value


def build_index_host(data, k, iters, final_degree, topm=64, thre=1.0, mode=KNN_CHOSEN,
                     seed=0x7A6E, out=None):
    data = np.ascontiguousarray(data, dtype=np.float32)
    n, dim = data.shape
    p = knn_params(k, n, dim, iters, mode, 0, 0, 1, seed)
    if out is None:
        out = np.empty((n, k), dtype=np.uint32)
    ep = C.c_uint32(0)
    check(lib().tagore_build_index_host(C.byref(p), _ptr(data), n, dim, final_degree, topm, thre,
                                        _ptr(out), C.byref(ep)))
    return out, ep.value


def last_screen():
    t = ScreenStats()
    check(lib().tagore_last_screen(C.byref(t)))
    return t


def mlp_loss_grad(rows_f16, tri, params):
    """Loss and gradients of the screen MLP on the GPU (host arrays in and out)."""
    rows_f16 = np.ascontiguousarray(rows_f16, dtype=np.float16)
    n, dim = rows_f16.shape
    tri = np.ascontiguousarray(tri, dtype=np.uint32)
    params = np.ascontiguousarray(params, dtype=np.float32)
    grads = np.zeros_like(params)
    loss = C.c_double(0.0)
    check(lib().tagore_mlp_loss_grad(_ptr(rows_f16), n, dim, _ptr(tri), tri.shape[0],
                                     _ptr(params), _ptr(grads), C.byref(loss)))
    return loss.value, grads


def last_timings():
    t = Timings()
    check(lib().tagore_last_timings(C.byref(t)))
    return t
