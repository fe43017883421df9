"""Build the sm_100a library ``libafidgpu.so`` and the ``afid_run`` driver in-tree.

nvcc cross-compiles for sm_100a without a GPU; objects go to ``_build/`` next to this file and
the outputs next to this file, so they travel with the source tree.
"""
from __future__ import annotations

import concurrent.futures
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INC = os.path.join(ROOT, "include")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libafidgpu.so")
RUNNER = os.path.join(HERE, "afid_run")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUFLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-I" + INC, "-I" + CSRC] + ARCH
CXXFLAGS = ["-std=c++17", "-O2", "-fPIC", "-I" + INC, "-I/usr/local/cuda/include"]

SOURCES = ["afid_k1_fp64.cu", "afid_k1_mixed.cu", "afid_k1_sal.cu", "afid_kernels.cu", "afid_api.cu", "afid_noalloc.cu",
           "afid_batch.cu", "afid_stats.cu", "afid_salinity.cu", "afid_host.cpp", "afid_mgrd.cpp",
           "afid_serve.cpp", "afid_continua.cpp", "afid_restart.cpp"]


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs += [os.path.join(INC, f) for f in os.listdir(INC) if f.endswith(".h")]
    return hs


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = _headers()
    objs, jobs = [], []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if not force and _newer(o, [s] + headers):
            continue
        if src.endswith(".cu"):
            jobs.append([NVCC] + CUFLAGS + ["-c", s, "-o", o])
        else:
            jobs.append(["g++"] + CXXFLAGS + ["-c", s, "-o", o])
    # translation units compile independently: run them side by side
    with concurrent.futures.ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        for f in [ex.submit(_run, cmd, verbose) for cmd in jobs]:
            f.result()
    if force or not _newer(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-cudart", "static"], verbose)
    run_src = os.path.join(CSRC, "afid_run.cpp")
    if force or not _newer(RUNNER, [run_src, LIB] + headers):
        _run(["g++"] + CXXFLAGS + [run_src, "-o", RUNNER, "-L" + HERE, "-lafidgpu",
                                   "-Wl,-rpath,$ORIGIN"], verbose)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
