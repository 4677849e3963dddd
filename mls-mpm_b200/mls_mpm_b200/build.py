"""Builds libmpm_b200.so in-tree with nvcc for sm_100a.

Numerics flags: --fmad=false (no multiply-add contraction) with nvcc's IEEE
division and square root defaults; see csrc/mpm_device.cuh.
"""
import os
import subprocess
import sys

from .abi import LIB_PATH, PKG_DIR

CSRC = os.path.join(os.path.dirname(PKG_DIR), "csrc")
INCLUDE = os.path.join(os.path.dirname(os.path.dirname(PKG_DIR)), "include")

SOURCES = ["mpm_alloc.cu", "mpm_capi.cu", "mpm_kernels.cu", "mpm_world.cu", "mpm_edit.cu", "mpm_noalloc.cu", "mpm_batch.cu", "mpm_server.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "--fmad=false", "-prec-div=true", "-prec-sqrt=true", "-lineinfo",
              "-Xcompiler", "-fPIC", "-Xcompiler", "-O3", "--expt-relaxed-constexpr"]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.exists(c) or c == "nvcc"):
            return c
    return "nvcc"


def sources():
    return [os.path.join(CSRC, s) for s in SOURCES]


def deps():
    out = sources()
    for d in (CSRC, INCLUDE):
        for f in os.listdir(d):
            if f.endswith((".h", ".cuh", ".hpp")):
                out.append(os.path.join(d, f))
    return out


def up_to_date():
    if not os.path.exists(LIB_PATH):
        return False
    t = os.path.getmtime(LIB_PATH)
    return all(os.path.getmtime(f) <= t for f in deps())


def build(force=False, verbose=False, extra=()):
    """Compile every CUDA source into libmpm_b200.so (sm_100a)."""
    if not force and up_to_date():
        return LIB_PATH
    cmd = [nvcc(), *ARCH, *NVCC_FLAGS, *extra, "-shared", "-o", LIB_PATH, *sources(), "-I", INCLUDE]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + r.stdout + r.stderr)
    return LIB_PATH


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB_PATH)
