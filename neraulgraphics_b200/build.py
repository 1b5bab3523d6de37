"""Builds libngb.so, the renderer's shared library, in-tree for sm_100a (B200).

    python -m neraulgraphics_b200.build

Every kernel file is compiled with -fmad=false and IEEE division and square root: the arithmetic rules the
kernels rely on for bit-exact parity (see csrc/device.cuh). The CUDA runtime is linked statically, so the
library needs only the driver.
"""

from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libngb.so")
OBJ = os.path.join(HERE, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
              "-Xcompiler", "-fPIC", "-Xptxas", "-v"]
SOURCES = ["lbvh.cu", "trace.cu", "persistent.cu", "tiles.cu", "adjoint.cu", "noalloc.cu", "blas_build.cu", "pose.cu", "host.cpp", "renderer.cpp"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _stale(target: str, deps: list) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(HERE, "..", "include", "ngb.h"))
    objs = []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(OBJ, src + ".o")
        objs.append(obj)
        if not _stale(obj, [path] + headers):
            continue
        if src.endswith(".cu") or src == "renderer.cpp":
            cmd = [nvcc(), "-x", "cu"] + ARCH + CUDA_FLAGS + ["-c", path, "-o", obj]
        else:
            cmd = [nvcc(), "-std=c++17", "-O3", "-Xcompiler", "-fPIC,-Wall", "-c", path, "-o", obj]
        res = subprocess.run(cmd, capture_output=True, text=True)
        log = os.path.join(OBJ, src + ".log")
        with open(log, "w") as f:
            f.write(" ".join(cmd) + "\n" + res.stdout + res.stderr)
        if res.returncode != 0:
            sys.stderr.write(res.stdout + res.stderr)
            raise RuntimeError(f"compiling {src} failed (see {log})")
        if verbose:
            sys.stdout.write(res.stderr)
    if _stale(LIB, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            sys.stderr.write(res.stdout + res.stderr)
            raise RuntimeError("linking libngb.so failed")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
