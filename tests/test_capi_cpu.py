"""C ABI checks that need no GPU: exports, index-file layouts, fvecs loader
errors, argument validation, and the `Tagore` module's surface."""
import ctypes as C
import os
import re
import struct

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "tagore_b200.h")


def header_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(tagore_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol(capi):
    L = capi.lib()
    names = header_functions()
    assert len(names) >= 20
    for name in names:
        assert hasattr(L, name), name
    assert set(names) == set(capi.SIGNATURES), set(names) ^ set(capi.SIGNATURES)


def test_version_and_error_string(capi):
    assert b"sm_100a" in capi.lib().tagore_version()
    st = capi.KnnState()
    p = capi.PruneParams(8, 10, 4, 4, 8, 1.0)
    rc = capi.lib().tagore_pruning(C.byref(p), C.byref(st), b"NSG", None)
    assert rc == capi.TAGORE_EINVAL
    assert b"missing buffers" in capi.lib().tagore_last_error()


def rows(n, k, rng):
    g = np.zeros((n, k), np.uint32)
    for i in range(n):
        deg = int(rng.integers(0, k))
        g[i, 0] = deg
        g[i, 1:1 + deg] = rng.integers(0, n, size=deg)
        g[i, 1 + deg:] = rng.integers(0, n, size=k - 1 - deg)
    return g


def expected_rows(g):
    out = b""
    for r in g:
        deg = int(r[0])
        out += struct.pack("<I", deg) + r[1:1 + deg].astype("<u4").tobytes()
    return out


def test_nsg_layout(capi, tmp_path):
    g = rows(50, 12, np.random.default_rng(0))
    path = str(tmp_path / "a.nsg")
    capi.check(capi.lib().tagore_store_nsg(path.encode(), g.ctypes.data_as(C.c_void_p), 11, 7, 50, 12))
    assert open(path, "rb").read() == struct.pack("<II", 11, 7) + expected_rows(g)


def test_vamana_layout_backpatches_size_and_max_degree(capi, tmp_path):
    g = rows(40, 10, np.random.default_rng(1))
    path = str(tmp_path / "a.vamana")
    capi.check(capi.lib().tagore_store_vamana(path.encode(), g.ctypes.data_as(C.c_void_p), 3, 40, 10))
    body = expected_rows(g)
    head = struct.pack("<QIIQ", 24 + len(body), int(g[:, 0].max()), 3, 0)
    assert open(path, "rb").read() == head + body


def test_nssg_layout(capi, tmp_path):
    g = rows(30, 9, np.random.default_rng(2))
    path = str(tmp_path / "a.nssg")
    capi.check(capi.lib().tagore_store_nssg(path.encode(), g.ctypes.data_as(C.c_void_p), 8, 30, 9))
    raw = open(path, "rb").read()
    width, n_ep = struct.unpack("<II", raw[:8])
    eps = struct.unpack("<10I", raw[8:48])
    assert (width, n_ep) == (8, 10)
    assert len(set(eps)) == 10 and max(eps) < 30
    assert raw[48:] == expected_rows(g)


def test_dpg_and_cagra_layouts(capi, tmp_path):
    n, d = 20, 6
    dense = np.random.default_rng(3).integers(0, n, size=(n, d)).astype(np.uint32)
    p1, p2 = str(tmp_path / "a.dpg"), str(tmp_path / "a.cagra")
    ptr = dense.ctypes.data_as(C.c_void_p)
    capi.check(capi.lib().tagore_store_dpg(p1.encode(), ptr, n, d))
    capi.check(capi.lib().tagore_store_cagra(p2.encode(), ptr, n, d))
    exp_dpg = b"KNNGRAPH" + struct.pack("<III", 2, 0, n)
    exp_cagra = b""
    for r in dense:
        exp_dpg += struct.pack("<II", d, d) + r.astype("<u4").tobytes()
        exp_cagra += struct.pack("<I", d) + r.astype("<u4").tobytes()
    assert open(p1, "rb").read() == exp_dpg
    assert open(p2, "rb").read() == exp_cagra


def test_writer_rejects_unwritable_path(capi):
    g = np.zeros((2, 4), np.uint32)
    rc = capi.lib().tagore_store_nsg(b"/nonexistent-dir/x", g.ctypes.data_as(C.c_void_p), 4, 0, 2, 4)
    assert rc == capi.TAGORE_EIO


def test_fvecs_roundtrip_and_errors(capi, tmp_path):
    from tagore_b200 import synth
    x = np.random.default_rng(4).random((37, 12)).astype(np.float32)
    path = str(tmp_path / "a.fvecs")
    synth.write_fvecs(path, x)
    n, d = C.c_uint32(), C.c_uint32()
    capi.check(capi.lib().tagore_load_fvecs_header(path.encode(), C.byref(n), C.byref(d)))
    assert (n.value, d.value) == (37, 12)
    out = np.empty_like(x)
    capi.check(capi.lib().tagore_load_fvecs(path.encode(), out.ctypes.data_as(C.c_void_p), 37, 12))
    assert np.array_equal(out, x)
    assert capi.lib().tagore_load_fvecs_header(b"/no/such/file", C.byref(n), C.byref(d)) == capi.TAGORE_EIO
    with open(path, "r+b") as f:
        f.truncate(os.path.getsize(path) - 3)
    assert capi.lib().tagore_load_fvecs_header(path.encode(), C.byref(n), C.byref(d)) == capi.TAGORE_EIO


def test_bad_build_arguments_are_rejected_before_any_device_work(capi):
    x = np.zeros((10, 6), np.float32)
    p = capi.knn_params(4, 10, 6, 2)
    st = capi.KnnState()
    assert capi.lib().tagore_gnn_descent_host(C.byref(p), x.ctypes.data_as(C.c_void_p), 10, 6,
                                              C.byref(st)) == capi.TAGORE_EINVAL
    p = capi.knn_params(10, 10, 8, 2)
    assert capi.lib().tagore_gnn_descent_host(C.byref(p), x.ctypes.data_as(C.c_void_p), 10, 8,
                                              C.byref(st)) == capi.TAGORE_EINVAL


def test_tagore_module_surface():
    import tagore_b200
    T = tagore_b200.load_tagore()
    for name in ("GNN_descent", "Pruning", "Pruning_with_CFS", "largeIndex"):
        assert hasattr(T, name)
    doc = T.Pruning.__doc__
    for arg in ("K", "POINTS", "DIM", "FINAL_DEGREE", "TOPM", "ptrs", "index_type", "thre",
                "index_path"):
        assert arg in doc
    with pytest.raises(ValueError):
        T.Pruning(8, 10, 4, 4, 8, (), "NSG")


def csr_of_rows(g):
    deg = g[:, 0].astype(np.int64)
    offs = np.zeros(len(g) + 1, np.uint64)
    offs[1:] = np.cumsum(deg)
    return offs, np.concatenate([r[1:1 + r[0]] for r in g]).astype(np.uint32)


@pytest.mark.parametrize("kind", ["NSG", "Vamana", "NSSG"])
def test_index_reader_roundtrip_rows(capi, tmp_path, kind):
    g = rows(64, 12, np.random.default_rng(5))
    path = str(tmp_path / f"a.{kind}")
    ptr = g.ctypes.data_as(C.c_void_p)
    if kind == "NSG":
        capi.check(capi.lib().tagore_store_nsg(path.encode(), ptr, 11, 9, 64, 12))
    elif kind == "Vamana":
        capi.check(capi.lib().tagore_store_vamana(path.encode(), ptr, 9, 64, 12))
    else:
        capi.check(capi.lib().tagore_store_nssg(path.encode(), ptr, 11, 64, 12))
    info, offs, adj = capi.index_read(path, kind)
    want_offs, want_adj = csr_of_rows(g)
    assert info.n == 64 and info.edges == len(want_adj)
    assert info.max_degree == int(g[:, 0].max())
    assert np.array_equal(offs, want_offs) and np.array_equal(adj, want_adj)
    if kind == "NSSG":
        assert info.n_eps == 10 and len(set(info.eps[:10])) == 10
    else:
        assert info.n_eps == 1 and info.eps[0] == 9
    assert info.width == (int(g[:, 0].max()) if kind == "Vamana" else 11)


@pytest.mark.parametrize("kind", ["DPG", "CAGRA"])
def test_index_reader_roundtrip_dense(capi, tmp_path, kind):
    dense = np.random.default_rng(6).integers(0, 30, size=(30, 7)).astype(np.uint32)
    path = str(tmp_path / f"a.{kind}")
    fn = capi.lib().tagore_store_dpg if kind == "DPG" else capi.lib().tagore_store_cagra
    capi.check(fn(path.encode(), dense.ctypes.data_as(C.c_void_p), 30, 7))
    info, offs, adj = capi.index_read(path, kind)
    assert (info.n, info.edges, info.max_degree, info.n_eps) == (30, 210, 7, 0)
    assert np.array_equal(offs, np.arange(31, dtype=np.uint64) * 7)
    assert np.array_equal(adj, dense.reshape(-1))


def test_index_reader_errors(capi, tmp_path):
    g = rows(20, 8, np.random.default_rng(7))
    path = str(tmp_path / "a.vamana")
    capi.check(capi.lib().tagore_store_vamana(path.encode(), g.ctypes.data_as(C.c_void_p), 0, 20, 8))
    info = capi.IndexInfo()
    L = capi.lib()
    assert L.tagore_index_info(path.encode(), b"HNSW", C.byref(info)) == capi.TAGORE_EINVAL
    assert L.tagore_index_info(b"/no/such/index", b"NSG", C.byref(info)) == capi.TAGORE_EIO
    with open(path, "r+b") as f:                      # a row cut short
        f.truncate(os.path.getsize(path) - 2)
    assert L.tagore_index_info(path.encode(), b"Vamana", C.byref(info)) == capi.TAGORE_EIO
    with open(path, "ab") as f:                       # whole rows, but the header's size is stale
        f.write(b"\0\0")
        f.write(struct.pack("<I", 0))
    assert L.tagore_index_info(path.encode(), b"Vamana", C.byref(info)) == capi.TAGORE_EIO
    dpg = str(tmp_path / "a.dpg")
    open(dpg, "wb").write(b"KNNGRAPX" + struct.pack("<III", 2, 0, 0))
    assert L.tagore_index_info(dpg.encode(), b"DPG", C.byref(info)) == capi.TAGORE_EIO
    nsg = str(tmp_path / "b.nsg")
    capi.check(L.tagore_store_nsg(nsg.encode(), g.ctypes.data_as(C.c_void_p), 8, 0, 20, 8))
    info = capi.index_info(nsg, "NSG")
    offs = np.zeros(info.n + 1, np.uint64)
    adj = np.zeros(info.edges, np.uint32)
    assert L.tagore_index_read(nsg.encode(), b"NSG", info.n - 1, info.edges,         # arrays too small
                               offs.ctypes.data_as(C.c_void_p),
                               adj.ctypes.data_as(C.c_void_p)) == capi.TAGORE_EINVAL


def test_search_argument_checks_need_no_device(capi):
    p = capi.SearchParams(16, 4, 0, 0, 0)
    L = capi.lib()
    # n = 0, and an entry point outside the base: rejected before any device call
    assert L.tagore_search(C.byref(p), None, 0, 8, None, None, 0, 0, None, 0, None, None) == capi.TAGORE_EINVAL
    assert L.tagore_search(C.byref(p), None, 5, 8, None, None, 0, 5, None, 1, None, None) == capi.TAGORE_EINVAL
    # no queries: nothing to do
    assert L.tagore_search(C.byref(p), None, 5, 8, None, None, 0, 0, None, 0, None, None) == capi.TAGORE_OK
