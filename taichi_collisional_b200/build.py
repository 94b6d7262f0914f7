"""Compile the CUDA library in-tree for sm_100a (no JIT cache; the .so sits next to this file)."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libtaichi_b200.so")
# every source of the single translation unit (tc_lib.cu includes the rest)
SOURCE_EXT = (".cu", ".cuh", ".h")
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
              "-Xcompiler", "-fPIC", "-shared"]


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, s) for s in os.listdir(CSRC) if s.endswith(SOURCE_EXT)]
    deps.append(os.path.join(HERE, "..", "include", "taichi_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, verbose=False):
    swap = os.path.join(CSRC, "swap_tables.h")
    if not os.path.exists(swap):
        subprocess.check_call([sys.executable, os.path.join(CSRC, "gen_swap_tables.py"), "20"])
    if not force and not _stale():
        return LIB
    cmd = ["nvcc"] + NVCC_FLAGS + ["-o", LIB + ".tmp", os.path.join(CSRC, "tc_lib.cu")]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
