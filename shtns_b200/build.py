"""Build the shtns_b200 C-ABI library (libshtns_b200.so) for sm_100a in-tree.

Compiles shtns_b200/csrc/*.cu with nvcc into shtns_b200/libshtns_b200.so.
Run as `python -m shtns_b200.build` or through __graft_entry__.build().
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libshtns_b200.so")
OBJDIR = os.path.join(HERE, "_build")

SOURCES = ["sht_plan.cu", "sht_gauss.cu", "sht_api.cu", "sht_legendre.cu", "sht_legendre_simt.cu", "sht_fft.cu", "sht_noalloc.cu", "sht_split.cu", "sht_ptab.cu", "sht_ftab.cu", "sht_local.cu", "sht_rotation.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2"]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, ptxas_info=False):
    os.makedirs(OBJDIR, exist_ok=True)
    headers = [os.path.join(CSRC, "sht_internal.h")] + [
        os.path.join(HERE, "..", "include", h) for h in ("shtns.h", "shtns_cuda.h", "shtns_b200.h")]
    objs = []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJDIR, src.replace(".cu", ".o"))
        objs.append(o)
        if _stale(o, [s] + headers) or ptxas_info:
            cmd = [nvcc()] + ARCH + FLAGS + (["-Xptxas", "-v"] if ptxas_info else []) + ["-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd))
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                sys.stderr.write(r.stdout + r.stderr)
                raise RuntimeError(f"nvcc failed on {src}")
            if ptxas_info:
                sys.stdout.write(r.stderr)
    if _stale(LIB, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        if verbose:
            print(" ".join(cmd))
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link of libshtns_b200.so failed")
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_info="-v" in sys.argv)
