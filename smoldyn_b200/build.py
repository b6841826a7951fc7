"""Build libsmoldyn_b200.so in-tree with nvcc for sm_100a.

Usage: python -m smoldyn_b200.build [--force]
The rxnparam tables header is generated first (from the reference checkout
named by $SMOLDYN_REF, default /root/reference) unless it already exists.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libsmoldyn_b200.so")
SOURCES = ["engine.cu", "surrogate.cu", "noalloc.cu", "rdf.cu", "sim.cpp", "surface.cpp", "api.cpp", "ensemble.cpp",
           "autotune.cpp"]
HEADERS = ["engine.h", "devcommon.cuh", "rxnparam.cuh", "panelgeom.cuh", "sim.h", "surrogate.h", "autotune.h", "_gen/rxntables.h",
           "boundgeom.cuh", "surfparam.h", "_gen/srftables.h",
           os.path.join("..", "..", "include", "smoldyn_b200.h")]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    for f in SOURCES + HEADERS:
        p = os.path.join(CSRC, f)
        if os.path.exists(p) and os.path.getmtime(p) > t:
            return True
    return False


def gen_tables():
    gen = os.path.join(CSRC, "gen_rxntables.py")
    rc = subprocess.call([sys.executable, gen])
    if rc != 0:
        raise RuntimeError("rxnparam tables generation failed")


def build(force=False, verbose=False):
    gen_tables()
    if not force and not needs_build():
        return LIB
    cmd = [nvcc()] + ARCH + [
        "-O3", "-lineinfo", "-std=c++17", "--shared", "-Xcompiler", "-fPIC,-O3",
        "-Xptxas", "-v" if verbose else "-O3",
        "-o", LIB + ".tmp",
    ] + [os.path.join(CSRC, s) for s in SOURCES] + ["-lcudart"]
    print(" ".join(cmd))
    subprocess.check_call(cmd)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
