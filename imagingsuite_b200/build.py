"""Build the mrcuda library in-tree (``imagingsuite_b200/libmrcuda.so``) for sm_100a.

``python -m imagingsuite_b200.build`` compiles every ``csrc/*.cu`` with nvcc and links one
shared library. The CUDA runtime is linked statically so the library does not depend on
which ``libcudart.so.12`` another framework in the process loaded first; device pointers
and streams from any runtime in the process are valid (one driver context per device).
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libmrcuda.so")
OBJ = os.path.join(HERE, "_build")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = [
    "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
    "-ccbin", "/usr/bin/g++",
    "-I" + os.path.join(ROOT, "include"), "-I" + CSRC,
]


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("command failed: " + " ".join(cmd))


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    headers = sorted(glob.glob(os.path.join(CSRC, "*.cuh"))) + [os.path.join(ROOT, "include", "mrcuda.h")]
    objs = []
    for src in sources:
        obj = os.path.join(OBJ, os.path.basename(src) + ".o")
        objs.append(obj)
        if ptxas_info or _stale(obj, [src] + headers + [__file__]):
            cmd = [NVCC, *ARCH, *FLAGS, "-c", src, "-o", obj]
            if ptxas_info:
                cmd.insert(1, "-Xptxas=-v")
            if verbose:
                print(" ".join(cmd))
            _run(cmd)
    if _stale(OUT, objs):
        _run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", OUT, *objs, "-lpthread", "-ldl", "-lrt"])
    return OUT


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv))
