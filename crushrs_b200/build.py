"""In-tree build of the engine library (crushrs_b200/libcrush_b200.so).

CUDA sources are compiled for sm_100a only, with --fmad=false so no
multiply-add is contracted (the element arithmetic must round exactly as the
reference's Rust code does). Objects go to crushrs_b200/_build/.

Usage: python -m crushrs_b200.build [--force] [--ptxas-verbose]
"""
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libcrush_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_SOURCES = ["kernels.cu", "engine.cu", "contact_static.cu", "history.cu", "frames.cu"]
HOST_SOURCES = ["host/scenario.cpp", "host/errors.cpp", "host/server.cpp", "host/signal.cpp"]
HEADERS = ["common.cuh", "element.cuh", "kernels.cuh", "hencky.cuh", "host/errors.hpp"]
INCLUDE = ["-I", os.path.join(ROOT, "include"), "-I", CSRC]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _compile(src, extra):
    path = os.path.join(CSRC, src)
    obj = os.path.join(BUILD, src.replace("/", "_") + ".o")
    deps = [path] + [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", h) for h in os.listdir(os.path.join(ROOT, "include"))]
    if not _newer(obj, deps) and "--force" not in sys.argv:
        return obj, ""
    if src.endswith(".cu"):
        cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "--fmad=false", "-std=c++17", "-Xcompiler", "-fPIC", *INCLUDE, *extra, "-c", path, "-o", obj]
    else:
        cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-Wall", *INCLUDE, "-I", "/usr/local/cuda/include", "-c", path, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build_library(verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    extra = ["-Xptxas", "-v"] if ("--ptxas-verbose" in sys.argv or verbose) else []
    with cf.ThreadPoolExecutor(max_workers=4) as ex:
        results = list(ex.map(lambda s: _compile(s, extra), CUDA_SOURCES + HOST_SOURCES))
    objs = [o for o, _ in results]
    if extra:
        for _, log in results:
            if log:
                print(log)
    if _newer(LIB, objs) or "--force" in sys.argv:
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build_library())
