"""Build libcosmonpc_b200.so in-tree with nvcc for sm_100a.

    python -m cosmonpc_b200.build [--force] [--verbose]

The library is a plain C-ABI shared object (see include/cosmonpc_b200.h); it is
rebuilt when any source under csrc/ or include/ is newer than the .so.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(REPO, "include")
LIB = os.path.join(PKG, "libcosmonpc_b200.so")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))
    deps += glob.glob(os.path.join(INCLUDE, "*.h"))
    return any(os.path.getmtime(p) > t for p in deps)


def nvcc_command(out=LIB, ptxas_verbose=False):
    nvcc = os.path.join(CUDA_HOME, "bin", "nvcc")
    cmd = [nvcc, "-O3", "-std=c++17", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC,-O3", "-shared",
           "-I", INCLUDE, "-I", CSRC, "-o", out, *sources(),
           "-L", os.path.join(CUDA_HOME, "lib64"), "-lcufft",
           "-Xlinker", "-rpath," + os.path.join(CUDA_HOME, "lib64")]
    if ptxas_verbose:
        cmd.insert(1, "-Xptxas=-v")
    return cmd


def build(force=False, verbose=False):
    """Compile the library if it is missing or older than its sources."""
    if not force and not _stale():
        return LIB
    cmd = nvcc_command(ptxas_verbose=verbose)
    tmp = LIB + ".tmp"
    cmd[cmd.index(LIB)] = tmp
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + res.stdout + res.stderr)
    if verbose:
        sys.stdout.write(res.stdout + res.stderr)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="--verbose" in sys.argv)
    print(LIB)
