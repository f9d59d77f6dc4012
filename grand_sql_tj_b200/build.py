"""Builds libtjb200.so in-tree with nvcc for sm_100a (B200 only)."""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libtjb200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


def cutlass_include() -> str:
    """CUTLASS/CuTe headers (only the sm100 UMMA descriptor definitions are used)."""
    import glob as _g
    import site
    for d in site.getsitepackages() + [os.path.join(os.path.dirname(os.__file__), "site-packages")]:
        for cand in (os.path.join(d, "flashinfer", "data", "cutlass", "include"),):
            if os.path.exists(os.path.join(cand, "cute", "arch", "mma_sm100_desc.hpp")):
                return cand
    hits = _g.glob("/opt/**/cutlass/include/cute/arch/mma_sm100_desc.hpp", recursive=True)
    if hits:
        return os.path.dirname(os.path.dirname(os.path.dirname(hits[0])))
    raise RuntimeError("CUTLASS headers with sm100 UMMA descriptors not found")
FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-gencode", "arch=compute_100a,code=sm_100a",
         "-Xcompiler", "-fPIC,-O3", "-Xptxas", "-O3", "--expt-relaxed-constexpr"]


def sources():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")) + glob.glob(os.path.join(HERE, "csrc", "*.cpp")))


def deps():
    return sources() + sorted(glob.glob(os.path.join(HERE, "csrc", "*.h")) + glob.glob(os.path.join(HERE, "csrc", "*.cuh"))) + \
        [os.path.join(HERE, "..", "include", "tj_b200.h")]


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(d) <= t for d in deps())


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    bdir = os.path.join(HERE, "_build")
    os.makedirs(bdir, exist_ok=True)
    objs = []
    for src in sources():
        obj = os.path.join(bdir, os.path.basename(src) + ".o")
        cmd = [NVCC] + FLAGS + ["-I", os.path.join(HERE, "..", "include"), "-I", cutlass_include(), "-c", src, "-o", obj]
        if src.endswith(".cpp"):
            cmd[1:1] = ["-x", "cu"]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        objs.append(obj)
    cmd = [NVCC] + FLAGS + ["-shared", "-o", LIB] + objs + ["-lcudart"]
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
