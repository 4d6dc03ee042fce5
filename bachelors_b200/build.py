"""Builds libfmmcuda.so in-tree with nvcc for sm_100a (no JIT, no torch extension)."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libfmmcuda.so")
SOURCES = ["fmm_api.cu", "fmm_tree.cu", "fmm_kernels.cu", "fmm_m2l_tc.cu", "fmm_adjoint.cu", "fmm_noalloc.cu", "fmm_seam.cu",
           "fmm_treecode.cu", "fmm_bem.cu", "fmm_geometry.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17", "-rdc=true",
    "--expt-relaxed-constexpr", "--extended-lambda",
    "-Xcompiler", "-fPIC", "-ccbin", "/usr/bin/g++",
]


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, "..", "include", "fmmcuda.h"))
    return all(os.path.getmtime(d) <= t for d in deps if os.path.exists(d))


OBJ = os.path.join(HERE, "_build")


def _compile(src: str, verbose: bool) -> tuple[str, subprocess.CompletedProcess]:
    obj = os.path.join(OBJ, os.path.splitext(src)[0] + ".o")
    cmd = [NVCC, *FLAGS, "-dc", "-o", obj, os.path.join(CSRC, src)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    return obj, subprocess.run(cmd, capture_output=True, text=True)


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles every translation unit in parallel (relocatable device code), then links them, with
    the device link step, into libfmmcuda.so."""
    if not force and up_to_date():
        return LIB
    from concurrent.futures import ThreadPoolExecutor
    os.makedirs(OBJ, exist_ok=True)
    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        results = list(ex.map(lambda s: _compile(s, verbose), SOURCES))
    for obj, r in results:
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"nvcc failed compiling {os.path.basename(obj)}")
        if verbose:
            sys.stderr.write(r.stderr)
    cmd = [NVCC, *FLAGS, "-shared", "-o", LIB + ".tmp", *[o for o, _ in results]]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed linking libfmmcuda.so")
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
