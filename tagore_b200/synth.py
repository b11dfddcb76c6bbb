"""Seeded synthetic bases with the shapes and value ranges of the workloads the
builder is measured on. No public dataset is reproduced: each generator draws a
Gaussian mixture with the stated parameters.

    sift_like  d=128, centres U[0,128)^d, sigma 20, clipped to [0,255], rounded
    gist_like  d=960, centres U[0,1)^d, sigma 0.05, clipped to [0,1]
    deep_like  d=96, unit-normalised mixture

Seeds follow 0x7A6E + config index. Held-out queries come from the same
mixture centres with their own stream (seed + 1000).
"""
import numpy as np

SEED0 = 0x7A6E

# config index -> (kind, n, d, components)
CONFIGS = {0: ("sift", 100_000, 128, 64), 1: ("sift", 1_000_000, 128, 256),
           2: ("gist", 1_000_000, 960, 512), 3: ("deep", 2_000_000, 96, 1024)}


def _centers(kind, d, comps, seed):
    rng = np.random.default_rng(seed)
    if kind == "sift":
        return rng.uniform(0.0, 128.0, size=(comps, d)).astype(np.float32)
    if kind == "gist":
        return rng.uniform(0.0, 1.0, size=(comps, d)).astype(np.float32)
    return rng.uniform(-1.0, 1.0, size=(comps, d)).astype(np.float32)


def _draw(kind, centers, n, seed, chunk=1 << 16):
    rng = np.random.default_rng(seed)
    comps, d = centers.shape
    sigma = {"sift": 20.0, "gist": 0.05, "deep": 0.35}[kind]
    out = np.empty((n, d), np.float32)
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        lab = rng.integers(0, comps, size=e - s)
        out[s:e] = centers[lab] + rng.standard_normal((e - s, d), dtype=np.float32) * sigma
    if kind == "sift":
        np.clip(out, 0, 255, out=out)
        np.rint(out, out=out)
    elif kind == "gist":
        np.clip(out, 0, 1, out=out)
    else:
        out /= np.maximum(np.linalg.norm(out, axis=1, keepdims=True), 1e-12)
    return out


def mixture(kind, n, d, comps, seed, nq=0):
    """(base, queries) drawn from one mixture; queries are held out."""
    c = _centers(kind, d, comps, seed)
    base = _draw(kind, c, n, seed + 1)
    q = _draw(kind, c, nq, seed + 1000) if nq else None
    return base, q


def config(i, n=None, nq=0):
    kind, n0, d, comps = CONFIGS[i]
    return mixture(kind, n or n0, d, comps, SEED0 + i, nq)


def write_fvecs(path, x):
    x = np.ascontiguousarray(x, dtype=np.float32)
    n, d = x.shape
    rec = np.empty((n, d + 1), np.float32)
    rec[:, 0] = np.frombuffer(np.uint32(d).tobytes(), dtype=np.float32)[0]
    rec[:, 1:] = x
    rec.tofile(path)


def read_fvecs(path):
    raw = np.fromfile(path, dtype=np.float32)
    d = int(raw[:1].view(np.uint32)[0])
    return raw.reshape(-1, d + 1)[:, 1:].copy()
