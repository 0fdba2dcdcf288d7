"""Build libkhz_b200.so in-tree with nvcc for sm_100a.

    python -m openkhuzdulgraph_b200.build [--verbose]

Each .cu under csrc/ is compiled to an object with
`-gencode arch=compute_100a,code=sm_100a -O3 -lineinfo` and linked into one shared
library next to this file.  Objects are rebuilt only when a source or header is newer.
"""
import glob
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libkhz_b200.so")
APP = os.path.join(HERE, "khz_app")
HOST_CXX = os.environ.get("KHZ_HOST_CXX", "g++")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr",
                "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, ptxas_verbose=False):
    os.makedirs(OBJ, exist_ok=True)
    headers = (glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(ROOT, "include", "*.h")) +
               glob.glob(os.path.join(ROOT, "include", "*.cuh")))
    objs, cmds = [], []
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cu"))):
        obj = os.path.join(OBJ, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        if _newer(obj, [src] + headers) or ptxas_verbose:
            cmd = [NVCC] + FLAGS + (["-Xptxas", "-v"] if ptxas_verbose else []) + ["-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd), flush=True)
            cmds.append(cmd)
    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        for f in [ex.submit(subprocess.check_call, c) for c in cmds]:
            f.result()
    if _newer(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    # the reference-style command-line program over the C ABI (host C++ only)
    app_src = os.path.join(HERE, "host", "khz_app.cpp")
    hpp = os.path.join(ROOT, "include", "khz_khuzdul.hpp")
    if _newer(APP, [app_src, hpp, LIB]):
        cmd = [HOST_CXX, "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"), app_src, "-o", APP,
               "-L" + HERE, "-lkhz_b200", "-Wl,-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, ptxas_verbose="--ptxas" in sys.argv)
    print(LIB)
