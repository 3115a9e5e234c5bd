"""Build the native libraries in-tree for sm_100a.

  si3d_b200/_lib/libsi3d_gpu.so   the CUDA core behind include/si3d_gpu.h (nvcc, sm_100a)
  si3d_b200/_lib/libsi3d_host.so  the C++ host (input readers, set-up, time loop), linked to it

Both are plain shared objects with C entry points; nothing here depends on PyTorch.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "_lib")

CUDA_SOURCES = ["si3d_gpu.cu", "k_momentum.cu", "k_zeta.cu", "k_pcg_persistent.cu", "k_transport.cu", "k_learn.cu",
                "noalloc.cu", "k_mg.cu", "k_tracer.cu", "k_output.cu", "k_turb.cu", "k_openbc.cu"]
CUDA_DEPS = CUDA_SOURCES + ["common.cuh", "coop.cuh", "kernels.h", "learn.h", "mg.h"]
HOST_SOURCES = [os.path.join("host", "si3d_host.cpp")]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    # strict IEEE FP64 arithmetic: no contraction into FMA, so the column kernels reproduce the
    # CPU restatement's operation sequence
    "-fmad=false",
    "-Xcompiler", "-fPIC", "-shared",
]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build si3d_b200")


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd: list[str], cwd: str) -> None:
    r = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build failed: {' '.join(cmd)}")


def build_gpu(force: bool = False) -> str:
    os.makedirs(LIB, exist_ok=True)
    out = os.path.join(LIB, "libsi3d_gpu.so")
    deps = [os.path.join(CSRC, f) for f in CUDA_DEPS] + [os.path.join(ROOT, "include", h)
                                                          for h in ("si3d_gpu.h", "si3d_learn.h")]
    if force or _stale(out, deps):
        _run([_nvcc(), *NVCC_FLAGS, "-o", out, *CUDA_SOURCES], CSRC)
    return out


def build_host(force: bool = False) -> str:
    os.makedirs(LIB, exist_ok=True)
    gpu = build_gpu(force)
    out = os.path.join(LIB, "libsi3d_host.so")
    deps = [os.path.join(CSRC, f) for f in HOST_SOURCES] + [gpu, os.path.join(ROOT, "include", "si3d_host.h")]
    if force or _stale(out, deps):
        cuda_lib = os.path.join(os.path.dirname(os.path.dirname(_nvcc())), "lib64")
        _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-o", out, *HOST_SOURCES,
              f"-L{LIB}", "-lsi3d_gpu", f"-L{cuda_lib}", "-Wl,-rpath,$ORIGIN"], CSRC)
    return out


def build_all(force: bool = False) -> None:
    build_gpu(force)
    build_host(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
    print("built", os.listdir(LIB))
