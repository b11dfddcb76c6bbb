"""Builds the sm_100a library, the `Tagore` Python module and the CPU oracle.

    python -m tagore_b200.build          # incremental
    python -m tagore_b200.build --clean

Outputs stay in the source tree (tagore_b200/libtagore_b200.so,
tagore_b200/Tagore*.so, oracle/libtagore_oracle.so) so they travel with the
repository to the GPU host.
"""
import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libtagore_b200.so")
EXT = os.path.join(HERE, "Tagore" + sysconfig.get_config_var("EXT_SUFFIX"))

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-ccbin", "/usr/bin/g++",
           "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include")]
SOURCES = ["capi.cu", "prune.cu", "knn.cu", "knn_tc.cu", "mlp.cu", "connect.cu", "prep.cu", "search.cu",
           "io.cpp", "large_index.cpp"]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd[:3]) + " ...")
    return r


def build_library(verbose=False):
    os.makedirs(OBJ, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(ROOT, "include", "tagore_b200.h"))
    objs = []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(OBJ, src + ".o")
        objs.append(obj)
        if _newer(obj, [path] + headers + [__file__]):
            cmd = [NVCC] + ARCH + NVFLAGS + ["-c", path, "-o", obj]
            if src.endswith(".cu") and verbose:
                cmd += ["-Xptxas", "-v"]
            r = _run(cmd)
            if verbose:
                sys.stderr.write(r.stderr)
    if _newer(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-Xcompiler", "-fPIC", "-lpthread"])
    return LIB


def build_extension():
    import pybind11
    src = os.path.join(CSRC, "pybind_tagore.cpp")
    if not os.path.exists(src):
        return None
    if _newer(EXT, [src, LIB, os.path.join(ROOT, "include", "tagore_b200.h")]):
        inc = sysconfig.get_paths()["include"]
        _run(["/usr/bin/g++", "-O2", "-shared", "-fPIC", "-std=c++17", src, "-o", EXT,
              "-I" + pybind11.get_include(), "-I" + inc, "-I" + os.path.join(ROOT, "include"),
              "-L" + HERE, "-ltagore_b200", "-Wl,-rpath,$ORIGIN"])
    return EXT


def build_oracle():
    _run(["make", "-s", "-C", os.path.join(ROOT, "oracle")])
    return os.path.join(ROOT, "oracle", "libtagore_oracle.so")


def clean():
    for p in [LIB, EXT]:
        if os.path.exists(p):
            os.remove(p)
    if os.path.isdir(OBJ):
        for f in os.listdir(OBJ):
            os.remove(os.path.join(OBJ, f))


def build_all(verbose=False):
    build_library(verbose)
    build_extension()
    build_oracle()


if __name__ == "__main__":
    if "--clean" in sys.argv:
        clean()
    build_all(verbose="-v" in sys.argv)
    print("built", LIB)
