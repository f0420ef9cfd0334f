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
OUT_CHECKED = os.path.join(HERE, "libmrcuda_checked.so")
OBJ = os.path.join(HERE, "_build")
OBJ_CHECKED = os.path.join(HERE, "_build_checked")

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


def build(verbose: bool = False, ptxas_info: bool = False, bounds_check: bool = False) -> str:
    """Compile the library; bounds_check builds libmrcuda_checked.so with -DMR_BOUNDS_CHECK
    (index checks at the gather sites that record the first failure and skip the access)."""
    obj_dir = OBJ_CHECKED if bounds_check else OBJ
    out = OUT_CHECKED if bounds_check else OUT
    os.makedirs(obj_dir, exist_ok=True)
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    headers = sorted(glob.glob(os.path.join(CSRC, "*.cuh"))) + [os.path.join(ROOT, "include", "mrcuda.h")]
    objs = []
    for src in sources:
        obj = os.path.join(obj_dir, os.path.basename(src) + ".o")
        objs.append(obj)
        if ptxas_info or _stale(obj, [src] + headers + [__file__]):
            cmd = [NVCC, *ARCH, *FLAGS, *(["-DMR_BOUNDS_CHECK"] if bounds_check else []), "-c", src, "-o", obj]
            if ptxas_info:
                cmd.insert(1, "-Xptxas=-v")
            if verbose:
                print(" ".join(cmd))
            _run(cmd)
    if _stale(out, objs):
        _run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", out, *objs, "-lpthread", "-ldl", "-lrt"])
    return out


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv, bounds_check="--bounds-check" in sys.argv))
