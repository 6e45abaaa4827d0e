"""Build the gstb CUDA library in-tree (sm_100a) with nvcc."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libgstb.so")
SOURCES = ["gst_kernels.cu", "gst_engine.cu"]
HEADERS = ["gst_device.cuh", os.path.join("..", "..", "include", "gstb.h")]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
         "-Xcompiler", "-fPIC,-O3", "-shared", "--cudart", "static", "--expt-relaxed-constexpr"]
CLI = os.path.join(HERE, "gstb")
CLI_SRC = os.path.join(CSRC, "gstb_cli.cpp")


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, s) for s in SOURCES] + [os.path.join(CSRC, h) for h in HEADERS]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build_cli(force: bool = False) -> str:
    """The reference-argv command-line driver, linked against libgstb.so."""
    if force or not os.path.exists(CLI) or os.path.getmtime(CLI) < max(os.path.getmtime(CLI_SRC),
                                                                       os.path.getmtime(LIB)):
        subprocess.check_call(["g++", "-O2", "-std=c++17", "-o", CLI, CLI_SRC, "-L" + HERE, "-lgstb",
                               "-Wl,-rpath,$ORIGIN"])
    return CLI


def build(force: bool = False, verbose: bool = False) -> str:
    if force or _stale():
        cmd = [NVCC, *FLAGS, "-o", LIB, *[os.path.join(CSRC, s) for s in SOURCES]]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd), file=sys.stderr)
        subprocess.check_call(cmd)
    build_cli(force)
    return LIB


if __name__ == "__main__":
    build(force=True, verbose="-v" in sys.argv)
