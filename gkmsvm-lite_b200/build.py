"""Build recipe of the CUDA library: nvcc for sm_100a, output in-tree.

``python -m gkmsvm_lite_b200.build`` (or ``build()``) compiles every
``csrc/*.cu`` (nvcc) and ``csrc/*.cpp`` (host C++, g++) into an object and
links ``_build/libgkm_b200.so`` next to this file.  Objects are rebuilt only
when their source or a header is newer.
"""

from __future__ import annotations

import glob
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_build")
LIB = os.path.join(OUT, "libgkm_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
    "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills",
]
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-Wall"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _stale(obj: str, src: str, headers: list[str]) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(p) > t for p in [src, *headers])


def build(verbose: bool = False, extra: list[str] | None = None) -> str:
    os.makedirs(OUT, exist_ok=True)
    nvcc = _nvcc()
    headers = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h"))
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu"))) + sorted(glob.glob(os.path.join(CSRC, "*.cpp")))
    cxx = os.environ.get("CXX", "g++")
    jobs = []
    objs = []
    for src in srcs:
        obj = os.path.join(OUT, os.path.splitext(os.path.basename(src))[0] + ".o")
        objs.append(obj)
        if _stale(obj, src, headers):
            if src.endswith(".cu"):
                jobs.append([nvcc, *NVCC_FLAGS, *(extra or []), "-c", src, "-o", obj])
            else:
                jobs.append([cxx, *CXX_FLAGS, "-I", INCLUDE, "-c", src, "-o", obj])

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        if verbose or r.returncode:
            sys.stderr.write(r.stdout + r.stderr)
        if r.returncode:
            raise RuntimeError(f"{os.path.basename(cmd[0])} failed: {' '.join(cmd[-3:])}")
        return r.stderr

    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        list(ex.map(run, jobs))
    if jobs or not os.path.exists(LIB):
        run([nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *objs, "-o", LIB,
             "-lcudart"])
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
