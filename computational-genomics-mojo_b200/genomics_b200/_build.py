"""Builds libgenomics_b200.so (nvcc, sm_100a) and libgenomics_synth.so (gcc)
in-tree under computational-genomics-mojo_b200/lib/."""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REPO_ROOT = os.path.dirname(PKG_ROOT)
CSRC = os.path.join(PKG_ROOT, "csrc")
LIBDIR = os.path.join(PKG_ROOT, "lib")
OBJDIR = os.path.join(PKG_ROOT, "_build")
INCLUDE = os.path.join(REPO_ROOT, "include")

LIB = os.path.join(LIBDIR, "libgenomics_b200.so")
SYNTH = os.path.join(LIBDIR, "libgenomics_synth.so")

CU_SOURCES = ["api.cu", "sw_kernels.cu", "wfa_kernels.cu", "wfa_tiers.cu", "wfa_cigar.cu",
              "nw.cu", "noalloc.cu", "server.cu", "pack.cu", "multi.cu"]
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
    "-I" + INCLUDE, "-I" + CSRC,
]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def _deps():
    deps = [os.path.join(CSRC, f) for f in CU_SOURCES]
    deps += [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cuh")]
    deps.append(os.path.join(INCLUDE, "genomics_b200.h"))
    return deps


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile every CUDA source for sm_100a and link the C-ABI library."""
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(OBJDIR, exist_ok=True)
    nvcc = _nvcc()
    if force or _stale(LIB, _deps()):
        def compile_one(src):
            obj = os.path.join(OBJDIR, src.replace(".cu", ".o"))
            cmd = [nvcc, *NVCC_FLAGS, "-c", os.path.join(CSRC, src), "-o", obj]
            if verbose:
                print(" ".join(cmd))
            subprocess.check_call(cmd)
            return obj

        with cf.ThreadPoolExecutor(len(CU_SOURCES)) as ex:
            objs = list(ex.map(compile_one, CU_SOURCES))
        cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", LIB, *objs,
               "-cudart", "static"]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    synth_src = os.path.join(CSRC, "synth.c")
    if force or _stale(SYNTH, [synth_src]):
        subprocess.check_call(["gcc", "-O3", "-fPIC", "-shared", "-o", SYNTH, synth_src, "-lm"])
    return LIB


if __name__ == "__main__":
    build(force=True, verbose=True)
    print(LIB)
