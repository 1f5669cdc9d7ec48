"""Builds n2p2_b200/libn2p2b200.so for sm_100a (nvcc cross-compiles; no GPU
needed).  Incremental: a translation unit is recompiled when it or any header
in csrc/ or include/ is newer than its object.

    python -m n2p2_b200.build            # or n2p2_b200.build.build()
"""
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libn2p2b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc():
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build n2p2_b200")
    return cand


def _headers():
    return (glob.glob(os.path.join(CSRC, "*.hpp")) + glob.glob(os.path.join(CSRC, "*.cuh")) +
            glob.glob(os.path.join(ROOT, "include", "*.h")))


def _stale(obj, src, headers):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(p) > t for p in [src] + headers)


def build(verbose=False, jobs=8):
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    headers = _headers()
    cuda_inc = os.path.join(os.path.dirname(os.path.dirname(nvcc)), "include")
    cmds, objs = [], []
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cu"))):
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        if _stale(obj, src, headers):
            cmds.append([nvcc, "-std=c++17", *ARCH, "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off",
                         "-I", CSRC, "-c", src, "-o", obj])
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cpp"))):
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        if _stale(obj, src, headers):
            cmds.append(["g++", "-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-I", CSRC, "-I", cuda_inc,
                         "-c", src, "-o", obj])
    procs = []
    for c in cmds:
        if verbose:
            print(" ".join(c), flush=True)
        procs.append((c, subprocess.Popen(c, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        if len(procs) >= jobs:
            _wait(procs.pop(0))
    for p in procs:
        _wait(p)
    if cmds or not os.path.exists(LIB):
        link = [nvcc, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart", "-lpthread"]
        if verbose:
            print(" ".join(link), flush=True)
        r = subprocess.run(link, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stdout)
    return LIB


def _wait(item):
    cmd, p = item
    out, _ = p.communicate()
    if p.returncode != 0:
        raise RuntimeError("compile failed: " + " ".join(cmd) + "\n" + out.decode(errors="replace"))


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
