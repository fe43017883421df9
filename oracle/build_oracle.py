"""Build recipe for the C restatement of the oracle (oracle/afid_cpu.c) -> oracle/libafid_cpu.so.

Test infrastructure: the timed CPU baseline and a second oracle.  gcc -O3 with OpenMP,
x86-64-v3 so the library built here also runs on the GPU hosts.
"""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "afid_cpu.c")
LIB = os.path.join(HERE, "libafid_cpu.so")


def build(verbose: bool = False, force: bool = False) -> str:
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    cmd = ["gcc", "-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-shared", "-std=gnu11", SRC, "-o", LIB, "-lm"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force=True)
