"""Builds librtfmm_b200.so in place with nvcc for sm_100a.

    python exafmm-rd_b200/build.py

The library holds the host set-up (C++/OpenMP), the CUDA kernels and the C
ABI declared in include/rtfmm_b200.h.  It is written next to this file so
that it travels with the source tree.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "librtfmm_b200.so")
SOURCES = ["rtfmm_plan.cpp", "rtfmm_kernels.cu", "rtfmm_capi.cu", "rtfmm_noalloc.cu", "rtfmm_ewald.cu",
           "rtfmm_tree.cu", "rtfmm_lists.cu", "rtfmm_precompute.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
         "-Xcompiler", "-fPIC,-fopenmp,-O3", "--expt-relaxed-constexpr"]


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(ROOT, "include", "rtfmm_b200.h"))
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    if not force and not _stale():
        return LIB
    odir = os.path.join(HERE, "_build")
    os.makedirs(odir, exist_ok=True)
    objs = [os.path.join(odir, src + ".o") for src in SOURCES]

    def compile_one(k):
        cmd = [NVCC] + FLAGS + ["-I", os.path.join(ROOT, "include"), "-c", os.path.join(CSRC, SOURCES[k]), "-o",
                                objs[k]]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)

    # the translation units are independent: compile them side by side
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=min(len(SOURCES), os.cpu_count() or 1)) as ex:
        list(ex.map(compile_one, range(len(SOURCES))))
    tmp = LIB + ".tmp"
    # every symbol resolved at link time, so a missing definition fails here
    cmd = [NVCC] + FLAGS + ["-shared", "-o", tmp] + objs + ["-lgomp", "-Xlinker", "--no-undefined"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
