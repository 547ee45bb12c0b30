"""Build libtigerci_sigma.so in-tree for sm_100a.

Host C++ (CSF space, spin functions, coupling engine, plan builder, C ABI) is
compiled with g++ -O3 -fopenmp; CUDA sources with
nvcc -gencode arch=compute_100a,code=sm_100a.  The CUDA runtime is linked
statically so the library loads on machines without a GPU (host-only entry
points) and on the GPU box without extra search paths.

    python -m tigerci_b200.build [--force]
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libtigerci_sigma.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _stale(obj, srcs):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(s) > t for s in srcs)


def _run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout)
        raise RuntimeError(f"build step failed: {os.path.basename(cmd[-1])}")
    return r.stdout


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    headers = (glob.glob(os.path.join(CSRC, "**", "*.h"), recursive=True) +
               glob.glob(os.path.join(CSRC, "**", "*.cuh"), recursive=True) +
               glob.glob(os.path.join(HERE, "..", "include", "*.h")))
    objs = []
    for src in sorted(glob.glob(os.path.join(CSRC, "host", "*.cpp"))):
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        if force or _stale(obj, [src] + headers):
            _run(["g++", "-std=c++17", "-O3", "-fPIC", "-fopenmp", "-Wall", "-c", "-o", obj, src])
        objs.append(obj)
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cu"))):
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        if force or _stale(obj, [src] + headers):
            out = _run([nvcc, "-std=c++17", "-O3", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC,-fopenmp",
                        "-Xptxas", "-v", "--expt-relaxed-constexpr", "-c", "-o", obj, src])
            with open(obj + ".ptxas.txt", "w") as f:
                f.write(out)
            if verbose:
                print(out)
        objs.append(obj)
    if force or _stale(LIB, objs):
        _run([nvcc, "-shared", *ARCH, "-cudart", "static", "-Xcompiler", "-fopenmp", "-o", LIB, *objs,
              "-lgomp", "-lpthread", "-ldl", "-lrt"])
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
