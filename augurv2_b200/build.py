"""Builds the CUDA library libaugur_b200.so in-tree for sm_100a.

Each translation unit under csrc/ is compiled by nvcc with its own flags
(the Gibbs units that must be bit-exact against the reference's CPU sampler
are compiled with -fmad=false), then linked into augurv2_b200/_lib/.
Usage: python -m augurv2_b200.build [--force]
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
OBJ_DIR = os.path.join(OUT_DIR, "obj")
LIB = os.path.join(OUT_DIR, "libaugur_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
BASE = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
        "-I" + INCLUDE, "-I" + CSRC]
# Units whose binary64 arithmetic must match the reference without
# contraction into fused multiply-adds.
NO_FMAD = {"lda.cu", "gmm.cu", "conj.cu", "ll.cu"}


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))


def headers_mtime():
    paths = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    paths += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE)]
    return max((os.path.getmtime(p) for p in paths), default=0.0)


def build(force=False, verbose=True):
    os.makedirs(OBJ_DIR, exist_ok=True)
    hdr_t = headers_mtime()
    objs = []
    changed = False
    for src in sources():
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ_DIR, src[:-3] + ".o")
        objs.append(o)
        if (not force and os.path.exists(o) and os.path.getmtime(o) >= os.path.getmtime(s)
                and os.path.getmtime(o) >= hdr_t):
            continue
        flags = list(BASE) + ARCH
        flags += ["-fmad=false"] if src in NO_FMAD else []
        cmd = [nvcc()] + flags + ["-c", s, "-o", o]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
        changed = True
    if changed or force or not os.path.exists(LIB):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart", "-lcuda"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv)
