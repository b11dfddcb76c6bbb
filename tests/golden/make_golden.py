"""Generates golden fixtures by running the reference Tagore module itself
(built from its own sources by oracle/build_ref.sh into oracle/_ref) on a GPU.

    python tests/golden/make_golden.py OUTDIR

Inputs are chosen so the reference is deterministic where it can be:
  * a base of small integers (exact in FP16, every partial sum < 2048, so its
    FP16 arithmetic equals FP32) in which every node's distances to all other
    nodes are distinct (no ties for any sort to break);
  * TOPM <= K (no uninitialised beam slots), K >= 22 (2-hop collect stays in
    its own row), reverse lists that never overflow.
Each prune case runs three times on fresh buffers; an output that differs
between runs (the reference's cross-block races) is stored as unstable.
A second set of cases runs on a base of quarter values (non-integer, still
exact in FP16) at a larger degree, with NSSG and CAGRA index files.
Outputs: OUTDIR/golden_prune.npz, OUTDIR/golden_prune_quarter.npz and
OUTDIR/golden_prep.npz.
"""
import ctypes
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle", "_ref"))
sys.path.insert(0, ROOT)

N, D, K, FD, TOPM = 40, 16, 24, 8, 16


def distinct_integer_base(seed=7, n=N, d=D, hi=11):
    """Greedy: add random integer points while every node's distances stay
    distinct and all squared distances stay below 2048."""
    rng = np.random.default_rng(seed)
    pts = [rng.integers(0, hi, size=d)]
    dists = [set()]
    while len(pts) < n:
        c = rng.integers(0, hi, size=d)
        dd = [int(((c - p) ** 2).sum()) for p in pts]
        if len(set(dd)) != len(dd) or max(dd) >= 2048 or min(dd) == 0:
            continue
        if any(dd[i] in dists[i] for i in range(len(pts))):
            continue
        for i in range(len(pts)):
            dists[i].add(dd[i])
        dists.append(set(dd))
        pts.append(c)
    return np.array(pts, np.float32)


def exact_knn(x, k):
    d2 = ((x[:, None, :] - x[None, :, :]) ** 2).sum(-1)
    np.fill_diagonal(d2, np.inf)
    ids = np.argsort(d2, axis=1)[:, :k].astype(np.uint32)
    dis = np.take_along_axis(d2, ids.astype(np.int64), 1).astype(np.float32)
    return ids, dis


def capsule(ptr):
    f = ctypes.pythonapi.PyCapsule_New
    f.restype = ctypes.py_object
    f.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_void_p]
    return f(ptr, None, None)


def run_reference(T, torch, x, center, call):
    ids, dis = exact_knn(x, K)
    bufs = [torch.from_numpy(ids.reshape(-1).astype(np.int32)).cuda(),
            torch.zeros(N * 128, dtype=torch.int32, device="cuda"),
            torch.from_numpy(x.astype(np.float16).reshape(-1)).cuda(),
            torch.from_numpy(dis.reshape(-1)).cuda(),
            torch.zeros(N * 128, dtype=torch.float32, device="cuda"),
            torch.zeros(N, dtype=torch.int32, device="cuda"),
            torch.from_numpy(center.astype(np.float16)).cuda(),
            torch.zeros(N * 128, dtype=torch.int32, device="cuda")]
    torch.cuda.synchronize()
    ptrs = tuple(capsule(b.data_ptr()) for b in bufs)
    out = call(T, ptrs)
    torch.cuda.synchronize()
    res = {"graph": bufs[0].cpu().numpy().view(np.uint32), "nei_distance": bufs[3].cpu().numpy(),
           "reverse_num": bufs[5].cpu().numpy().view(np.uint32),
           "hybrid_list": bufs[7].cpu().numpy().view(np.uint32)}
    if out is not None:
        res["file"] = np.frombuffer(out, np.uint8)
    return ids, dis, res


def distinct_quarter_base(seed=17, n=N, d=D):
    """Like distinct_integer_base, on multiples of 1/4 in [0, 2.5]: every
    difference, square and partial sum is a multiple of 1/16 below 128, so the
    reference's FP16 arithmetic is exact and equals the oracle's FP32."""
    rng = np.random.default_rng(seed)
    pts = [rng.integers(0, 11, size=d) / 4.0]
    dists = [set()]
    while len(pts) < n:
        c = rng.integers(0, 11, size=d) / 4.0
        dd = [float(((c - p) ** 2).sum()) for p in pts]
        if len(set(dd)) != len(dd) or max(dd) >= 128 or min(dd) == 0:
            continue
        if any(dd[i] in dists[i] for i in range(len(pts))):
            continue
        for i in range(len(pts)):
            dists[i].add(dd[i])
        dists.append(set(dd))
        pts.append(c)
    return np.array(pts, np.float32)


QFD = 16  # a larger degree than the integer cases, so most filter_reverse rows take the union branch


def quarter_cases(T, torch, outdir, tmp):
    """NSG, Vamana, NSSG (2-hop + angle at 60 degrees) and CAGRA, each with its
    index file, on the quarter-valued base. DPG is left out: its four warps
    share one staging vector (src/Tagore_src.cu:1715-1720) and its writer takes
    each row's count from the dense rows (src/common.cu:219-237), so its output
    pins nothing."""
    x = distinct_quarter_base()
    rng = np.random.default_rng(19)
    while True:
        center = rng.integers(0, 11, size=D) / 4.0
        dc = ((x - center) ** 2).sum(1)
        if len(set(dc.tolist())) == N and dc.min() > 0 and dc.max() < 128:
            break
    center = center.astype(np.float32)

    def file_call(kind, thre):
        def call(T, ptrs):
            path = os.path.join(tmp, f"q_{kind}.index")
            T.Pruning(K, N, D, QFD, TOPM, ptrs, kind, thre, path)
            return open(path, "rb").read()
        return call

    cases = {"nsg": file_call("NSG", 1.0), "vamana": file_call("Vamana", 1.2),
             "nssg": file_call("NSSG", 0.5), "cagra": file_call("CAGRA", 1.0)}
    arrays = {"x": x, "center": center, "meta": np.array([N, D, K, QFD, TOPM], np.int64)}
    for name, call in cases.items():
        runs = [run_reference(T, torch, x, center, call)[2] for _ in range(3)]
        for key in runs[0]:
            vals = [r[key] for r in runs]
            stable = all(np.array_equal(vals[0], v) for v in vals[1:])
            arrays[f"{name}/{key}"] = vals[0]
            arrays[f"{name}/{key}/stable"] = np.array(stable)
            print("quarter", name, key, "stable" if stable else "UNSTABLE", flush=True)
    np.savez_compressed(os.path.join(outdir, "golden_prune_quarter.npz"), **arrays)


def main():
    outdir = sys.argv[1]
    os.makedirs(outdir, exist_ok=True)
    import torch
    import Tagore as T
    x = distinct_integer_base()
    # centre: an integer point with distinct distances to every node
    rng = np.random.default_rng(11)
    while True:
        center = rng.integers(0, 11, size=D).astype(np.float32)
        dc = ((x - center) ** 2).sum(1)
        if len(set(dc.tolist())) == N and dc.min() > 0:
            break
    tmp = tempfile.mkdtemp()

    def file_call(kind, thre):
        def call(T, ptrs):
            path = os.path.join(tmp, f"{kind}.index")
            T.Pruning(K, N, D, FD, TOPM, ptrs, kind, thre, path)
            return open(path, "rb").read()
        return call

    def cfs_call(mode, metric, thre):
        def call(T, ptrs):
            T.Pruning_with_CFS(K, N, D, FD, TOPM, ptrs, mode, metric, thre)
            return None
        return call

    cases = {"nsg": file_call("NSG", 1.0), "vamana": file_call("Vamana", 1.2),
             "cfs_path_dist_1.0": cfs_call("path", "dist", 1.0),
             "cfs_path_dist_1.2": cfs_call("path", "dist", 1.2),
             "cfs_2hop_dist_0.5": cfs_call("2-hop", "dist", 0.5),
             "cfs_1hop_rank": cfs_call("1-hop", "rank", 1.0)}
    arrays = {"x": x, "center": center, "meta": np.array([N, D, K, FD, TOPM], np.int64)}
    for name, call in cases.items():
        runs = [run_reference(T, torch, x, center, call)[2] for _ in range(3)]
        for key in runs[0]:
            vals = [r[key] for r in runs]
            stable = all(np.array_equal(vals[0], v) for v in vals[1:])
            arrays[f"{name}/{key}"] = vals[0]
            arrays[f"{name}/{key}/stable"] = np.array(stable)
            print(name, key, "stable" if stable else "UNSTABLE", flush=True)
    np.savez_compressed(os.path.join(outdir, "golden_prune.npz"), **arrays)
    quarter_cases(T, torch, outdir, tmp)

    # Host preparation of GNN_descent: FP16 base and centre (capsules 2 and 6).
    from tagore_b200 import synth
    base, _ = synth.mixture("sift", 2000, 128, 8, 13)
    path = os.path.join(tmp, "base.fvecs")
    synth.write_fvecs(path, base)
    caps = T.GNN_descent(96, 2000, 128, 2, path)
    get = ctypes.pythonapi.PyCapsule_GetPointer
    get.restype = ctypes.c_void_p
    get.argtypes = [ctypes.py_object, ctypes.c_char_p]
    cuda = ctypes.CDLL("libcudart.so.12")
    half = np.empty(2000 * 128, np.uint16)
    cen = np.empty(128, np.uint16)
    cuda.cudaMemcpy(half.ctypes.data_as(ctypes.c_void_p), ctypes.c_void_p(get(caps[2], None)),
                    ctypes.c_size_t(half.nbytes), 2)
    cuda.cudaMemcpy(cen.ctypes.data_as(ctypes.c_void_p), ctypes.c_void_p(get(caps[6], None)),
                    ctypes.c_size_t(cen.nbytes), 2)
    np.savez_compressed(os.path.join(outdir, "golden_prep.npz"), base=base, data_half=half,
                        center_half=cen)
    print("done", flush=True)


if __name__ == "__main__":
    main()
