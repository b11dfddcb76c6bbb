"""The capsule tuple between this library's `Tagore` module and the reference's.

The reference's `Pruning` reads elements 0-7 of the tuple `GNN_descent`
returns (pybind.cu:132-141, :151-158), and so does this module's. Both modules
are loaded into one process and the tuples cross over:

  * the reference's GNN_descent tuple goes into this module's Pruning, whose
    rows must equal the oracle's prune of the same buffers bit for bit;
  * this module's GNN_descent tuple goes into the reference's Pruning, whose
    rows must be well formed and agree with the oracle's edge sets (the
    reference scores candidates in FP16 and rewrites rows while other blocks
    read them, so only near-equality is expected).

The reference module is built from its own sources into oracle/_ref by
oracle/build_ref.sh; without it these tests are skipped. Its GNN_descent runs
only on the input it has already run on (2,000 x 128 SIFT-like, K = 96, two
iterations). The recall of both kNN graphs on that input is recorded.
"""
import ctypes
import glob
import importlib.machinery
import os

import numpy as np
import pytest

from tagore_b200 import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_SO = sorted(glob.glob(os.path.join(ROOT, "oracle", "_ref", "Tagore*.so")))

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not REF_SO, reason="reference module not built (oracle/_ref)")]

N, D, K, ITERS, FD, TOPM = 2000, 128, 96, 2, 32, 64


def load_reference():
    """The reference's module beside this library's, in one process. Both are
    pybind11 modules named `Tagore`, and pybind11 hands a second import of a
    name back the module it cached under that name. So the reference's
    PyModuleDef (multi-phase init) is instantiated here under its own spec
    name, as the import system would do it."""
    path = REF_SO[0]
    api = ctypes.pythonapi
    init = ctypes.PyDLL(path).PyInit_Tagore
    init.restype = ctypes.py_object
    mdef = init()
    api.Py_IncRef.argtypes = [ctypes.py_object]
    api.Py_IncRef(mdef)  # a static object: ctypes must never release it
    api.PyModule_FromDefAndSpec2.restype = ctypes.py_object
    api.PyModule_FromDefAndSpec2.argtypes = [ctypes.py_object, ctypes.py_object, ctypes.c_int]
    api.PyModule_ExecDef.restype = ctypes.c_int
    api.PyModule_ExecDef.argtypes = [ctypes.py_object, ctypes.py_object]
    spec = importlib.machinery.ModuleSpec("Tagore_reference", None, origin=path)
    mod = api.PyModule_FromDefAndSpec2(mdef, spec, 1013)
    mod.__spec__ = spec
    mod.__file__ = path
    assert api.PyModule_ExecDef(mod, mdef) == 0
    return mod


@pytest.fixture(scope="module")
def modules():
    import tagore_b200
    ours = tagore_b200.load_tagore()
    ref = load_reference()
    assert ref is not ours and ref.__file__ != ours.__file__
    return ours, ref


@pytest.fixture(scope="module")
def fvecs(tmp_path_factory):
    base, _ = synth.mixture("sift", N, D, 8, 13)
    path = str(tmp_path_factory.mktemp("interop") / "base.fvecs")
    synth.write_fvecs(path, base)
    return base, path


def pointer(cap):
    get = ctypes.pythonapi.PyCapsule_GetPointer
    get.restype = ctypes.c_void_p
    get.argtypes = [ctypes.py_object, ctypes.c_char_p]
    return get(cap, None)


def view(capi, caps):
    """A non-owning state over the tuple's device buffers."""
    st = capi.KnnState()
    st.n, st.dim, st.k, st.device = N, D, K, 0
    for i, (name, _) in enumerate(capi.BUFFERS[:8]):
        setattr(st, name, pointer(caps[i]))
    st.owns = 0
    s = capi.State()
    s.st = st
    return s


def host_buffers(capi, caps):
    s = view(capi, caps)
    return {name: s.download(i) for i, (name, _) in enumerate(capi.BUFFERS[:8])}


def oracle_nsg(orc, b):
    buf = orc.Buffers(b["graph"].reshape(N, K), b["nei_distance"].reshape(N, K),
                      b["data"].reshape(N, D), b["center"], b["reverse_graph"],
                      b["reverse_distance"], b["reverse_num"], b["hybrid_list"])
    ep = orc.prune(buf, FD, "NSG", topm=TOPM, thre=1.0)
    return ep, buf


def knn_recall10(orc, base, graph):
    gt = orc.bruteforce_knn(base, base, 10, exclude_self=np.arange(N, dtype=np.uint32))
    g = graph.reshape(N, K)[:, :10]
    return float(np.mean([len(set(g[i]) & set(gt[i])) / 10 for i in range(N)]))


def test_reference_tuple_into_our_pruning(capi, orc, modules, fvecs, tmp_path):
    ours, ref = modules
    base, path = fvecs
    caps = ref.GNN_descent(K, N, D, ITERS, path)
    assert len(caps) == 8
    before = host_buffers(capi, caps)
    ep_c, buf = oracle_nsg(orc, before)
    index = str(tmp_path / "ours.nsg")
    ours.Pruning(K, N, D, FD, TOPM=TOPM, ptrs=caps, index_type="NSG", thre=1.0,
                 index_path=index)
    after = host_buffers(capi, caps)
    for name in ("graph", "nei_distance", "reverse_graph", "reverse_distance", "reverse_num",
                 "hybrid_list"):
        a, e = after[name], getattr(buf, name)
        assert np.array_equal(a.view(np.uint32), e.view(np.uint32)), name
    info = capi.index_info(index, "NSG")
    assert info.eps[0] == ep_c


def test_our_tuple_into_reference_pruning(capi, orc, modules, fvecs, tmp_path):
    ours, ref = modules
    base, path = fvecs
    caps = ours.GNN_descent(K, N, D, ITERS, path)
    assert len(caps) == 9
    before = host_buffers(capi, caps)
    _, buf = oracle_nsg(orc, before)
    ref.Pruning(K, N, D, FD, TOPM, caps, "NSG", 1.0, str(tmp_path / "ref.nsg"))
    rows = host_buffers(capi, caps)["graph"].reshape(N, K)
    want = buf.graph.reshape(N, K)
    deg = rows[:, 0]
    assert deg.max() <= FD - 1 and deg.min() >= 1
    jac = []
    for i in range(N):
        a = set(rows[i, 1:1 + deg[i]].tolist())
        b = set(want[i, 1:1 + want[i, 0]].tolist())
        assert max(a) < N
        jac.append(len(a & b) / len(a | b))
    assert np.mean(jac) > 0.9, np.mean(jac)


def test_knn_recall_against_reference_same_input(orc, modules, fvecs, capi):
    """Recall@10 of both GNN_descent graphs on the same file at equal
    iterations, and of the CPU model of the reference's algorithm
    (oracle/gnn_descent_model.cpp), which stands in for the reference on
    inputs it does not run on: the model must land within 0.01 of the
    reference (both are nondeterministic)."""
    ours, ref = modules
    base, path = fvecs
    r_ref = [knn_recall10(orc, base, host_buffers(capi, ref.GNN_descent(K, N, D, ITERS, path))["graph"])
             for _ in range(3)]
    r_our = knn_recall10(orc, base, host_buffers(capi, ours.GNN_descent(K, N, D, ITERS, path))["graph"])
    half, _, _ = orc.host_prep(base)
    r_model = [knn_recall10(orc, base, orc.gnn_descent_model(half.reshape(N, D), K, ITERS, seed=s)[0])
               for s in (1, 2, 3)]
    print(f"kNN recall@10 at {N}x{D}, K={K}, {ITERS} iterations: ours {r_our:.4f}, "
          f"reference {np.round(r_ref, 4).tolist()}, model {np.round(r_model, 4).tolist()}")
    # At two iterations this build has measured 0.0019 and 0.0028 below the
    # reference's mean here; at ten iterations it is well above it (test_knn_vs_
    # reference_model_gpu.py). The bound checks it stays in that range.
    assert r_our >= np.mean(r_ref) - 0.005
    assert abs(np.mean(r_model) - np.mean(r_ref)) < 0.01
