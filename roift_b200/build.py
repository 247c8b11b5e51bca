"""Build liboift_b200.so in-tree with nvcc for sm_100a (no JIT cache, no torch types)."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "liboift_b200.so")
# gft::ift drop-ins (OIFT_Multi, ORelax_1_Multi and their per-class forms) over the C ABI
SHIM = os.path.join(HERE, "libgft_oift_b200.so")
SHIM_SRC = os.path.join(CSRC, "gft_shims.cpp")
SOURCES = ["api.cu", "weights.cu", "oift.cu", "relax.cu", "selftest.cu", "noalloc.cu", "prepost.cu", "adjoint.cu", "imagegraph.cu", "volume_io.cu", "costgrad.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
         "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden", "--expt-relaxed-constexpr"]


def _stale() -> bool:
    if not os.path.exists(LIB) or not os.path.exists(SHIM):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [
        os.path.join(HERE, "..", "include", "oift_b200.h"), __file__]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


# (source, object, extra flags): the tile sweep is compiled once per class count
UNITS = [(s, s.replace(".cu", ".o"), []) for s in SOURCES] + [
    ("relax_tiles_inst.cu", f"relax_tiles_c{c}.o", [f"-DRELAX_TILE_C={c}"]) for c in range(1, 9)]


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    from concurrent.futures import ThreadPoolExecutor

    def compile_unit(unit):
        src, obj, extra = unit
        obj = os.path.join(CSRC, obj)
        cmd = [NVCC, *FLAGS, *extra, "-dc", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        subprocess.run(cmd, check=True)
        return obj

    workers = max(1, min(len(UNITS), os.cpu_count() or 1))
    with ThreadPoolExecutor(workers) as ex:
        objs = list(ex.map(compile_unit, UNITS))
    subprocess.run([NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *objs,
                    "-o", LIB, "-lcudart", "-lz"], check=True)
    for o in objs:
        os.remove(o)
    subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", SHIM_SRC, "-o", SHIM,
                    "-L" + HERE, "-loift_b200", "-Wl,-rpath,$ORIGIN"], check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
