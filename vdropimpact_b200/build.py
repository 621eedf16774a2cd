"""Builds libvdi.so (the CUDA kernels and the C ABI of include/vdi.h) for
sm_100a with nvcc, in the package tree, so it travels with the sources.

    python -m vdropimpact_b200.build [--force]
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libvdi.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3",
                 "-I", os.path.join(ROOT, "include"), "-I", CSRC]
# Stencil and gas-layer kernels follow the reference's expression order
# exactly; FMA contraction would change their rounding.
EXACT = {"step_kernels.cu", "gas.cu", "liftoff.cu"}
SOURCES = ["mg.cu", "step_kernels.cu", "gas.cu", "liftoff.cu", "sim.cu", "unet.cu"]


def _sources():
    missing = [s for s in SOURCES if not os.path.exists(os.path.join(CSRC, s))]
    if missing:
        raise FileNotFoundError(f"CUDA sources missing from {CSRC}: {missing}")
    return list(SOURCES)


def _deps():
    hdrs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".hh", ".cuh", ".h"))]
    hdrs.append(os.path.join(ROOT, "include", "vdi.h"))
    return hdrs


def _compile(src: str) -> str:
    obj = os.path.join(OUT_DIR, src.replace(".cu", ".o"))
    path = os.path.join(CSRC, src)
    newest = max([os.path.getmtime(path)] + [os.path.getmtime(h) for h in _deps()])
    if os.path.exists(obj) and os.path.getmtime(obj) >= newest:
        return obj
    flags = COMMON + (["-fmad=false"] if src in EXACT else [])
    cmd = [NVCC] + flags + ["-c", path, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    if force:
        for f in os.listdir(OUT_DIR):
            if f.endswith((".o", ".so")):
                os.remove(os.path.join(OUT_DIR, f))
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(_compile, srcs))
    newest = max(os.path.getmtime(o) for o in objs)
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    _build_host()
    if verbose:
        print(LIB)
    return LIB


HOST = os.path.join(HERE, "host")
HOST_LIB = os.path.join(OUT_DIR, "libvdi_host.so")
HOST_CLI = os.path.join(OUT_DIR, "vdi_fluid_test")
CUDA_HOME = os.path.dirname(os.path.dirname(NVCC))
HOST_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-Wall", "-I", os.path.join(ROOT, "include"),
              "-I", os.path.join(HOST, "include"), "-I", os.path.join(CUDA_HOME, "include")]


def _build_host():
    """The C++ drop-in classes (host/include, host/src) as libvdi_host.so over
    libvdi.so, and the vdi_fluid_test driver."""
    srcs = sorted(os.path.join(HOST, "src", f) for f in os.listdir(os.path.join(HOST, "src")) if f.endswith(".cc"))
    hdrs = [os.path.join(HOST, "include", f) for f in os.listdir(os.path.join(HOST, "include"))]
    deps = srcs + hdrs + [LIB, os.path.join(ROOT, "include", "vdi.h"), os.path.join(HOST, "vdi_fluid_test.cc")]
    newest = max(os.path.getmtime(p) for p in deps)
    if os.path.exists(HOST_CLI) and os.path.getmtime(HOST_CLI) >= newest and os.path.getmtime(HOST_LIB) >= newest:
        return
    link = ["-L", OUT_DIR, "-lvdi", "-L", os.path.join(CUDA_HOME, "lib64"), "-lcudart_static", "-ldl", "-lpthread",
            "-lrt", "-Wl,-rpath,$ORIGIN"]
    cmd = ["g++"] + HOST_FLAGS + ["-shared", "-o", HOST_LIB] + srcs + link
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"host library build failed:\n{r.stdout}\n{r.stderr}")
    cmd = ["g++"] + HOST_FLAGS + ["-o", HOST_CLI, os.path.join(HOST, "vdi_fluid_test.cc"), "-L", OUT_DIR,
                                  "-lvdi_host", "-lvdi", "-Wl,-rpath,$ORIGIN"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"vdi_fluid_test build failed:\n{r.stdout}\n{r.stderr}")


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
