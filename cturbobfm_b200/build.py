"""Builds libctbfm.so in-tree: CUDA kernels for sm_100a (nvcc) and the host
C++ layer (g++), linked with the static CUDA runtime.

Flags that carry the numerical contract:
  * double kernels (kernels.cu, kernels_persist.cu, noalloc.cu): ``--fmad=false`` (no
    multiply-add contraction; IEEE double division and square root are
    nvcc's defaults);
  * float kernels (kernels_f32.cu, kernels_persist_f32.cu): contraction allowed, approximate
    float division and square root, denormals flushed (the float path is
    a stated-tolerance path; its faces run 38 % faster than with IEEE
    division); the compensated (Kahan) state update has no product to
    contract and no division;
  * host code: ``-ffp-contract=off`` (mesh metrics bit-identical to the
    reference's).
"""

from __future__ import annotations

import concurrent.futures
import os
import shutil
import subprocess
import sys
from typing import List

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(PKG, "libctbfm.so")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

# (source, float kernels: contraction and approximate division / square root)
CU_SOURCES = [("device/kernels.cu", False), ("device/kernels_f32.cu", True), ("device/kernels_persist.cu", False),
              ("device/kernels_persist_f32.cu", True), ("device/noalloc.cu", False)]
FAST_F32 = ["--fmad=true", "-prec-div=false", "-prec-sqrt=false", "-ftz=true"]
CPP_SOURCES = ["host/config.cpp", "host/mesh.cpp", "host/engine.cpp", "host/fluid_table.cpp", "host/restart.cpp",
               "host/output.cpp", "host/solver.cpp", "host/batch.cpp", "host/server.cpp", "capi.cpp"]


def _run(cmd: List[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd))


def _stale(target: str, deps: List[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _all_headers() -> List[str]:
    out = []
    for d, _, files in os.walk(CSRC):
        out += [os.path.join(d, f) for f in files if f.endswith((".hpp", ".cuh", ".h"))]
    out.append(os.path.join(ROOT, "include", "ctbfm.h"))
    return out


def build(verbose: bool = False, force: bool = False) -> str:
    """Compiles what changed and links libctbfm.so; returns its path."""
    if not os.path.exists(NVCC):
        raise RuntimeError(f"nvcc not found at {NVCC}")
    os.makedirs(BUILD, exist_ok=True)
    headers = _all_headers()
    objs = []
    jobs = []
    for src, fmad in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, os.path.basename(src) + ".o")
        if force or _stale(o, [s] + headers):
            jobs.append([NVCC, *ARCH, "-lineinfo", "-O3", *(FAST_F32 if fmad else ["--fmad=false"]), "-std=c++17",
                         "-Xcompiler", "-fPIC", "-Xptxas", "-v" if verbose else "-O3", "-c", s, "-o", o])
        objs.append(o)
    # the device units are independent: compile them side by side
    with concurrent.futures.ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as pool:
        for f in [pool.submit(_run, cmd) for cmd in jobs]:
            f.result()
    for src in CPP_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, os.path.basename(src) + ".o")
        if force or _stale(o, [s] + headers):
            _run(["g++", "-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-Wall", "-Wextra",
                  "-Wno-unused-parameter", f"-I{CUDA_HOME}/include", "-c", s, "-o", o])
        objs.append(o)
    if force or _stale(LIB, objs):
        tmp = LIB + ".tmp"
        _run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", tmp, *objs])
        shutil.move(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
