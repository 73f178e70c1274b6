"""Builds the native parts of warpjq_b200 in-tree.

  warpjq_b200/_lib/libwarpjq_kernels.so  -- the sm_100a device backend (C ABI)
  warpjq_b200/_lib/libwarpjq_kernels.a   -- the same, as the static library the
                                            reference's Rust crate links
  warpjq_b200/_lib/libwarpjq_host.so     -- the C++ host driver (query front-end,
                                            pipeline, formatting, serving loop)

Run: python -m warpjq_b200.build   (nvcc cross-compiles; no GPU needed)
"""

from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "_lib")
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC"]

KERNEL_SRCS = [os.path.join(CSRC, "backend.cu"), os.path.join(CSRC, "noalloc.cu"), os.path.join(CSRC, "csv.cu")]
KERNEL_DEPS = [os.path.join(CSRC, f) for f in ("kernels.cuh", "walker.cuh", "devutil.cuh", "fixsum.cuh", "plan.h",
                                               "plan_build.h", "csv_rows.cuh")]
HOST_SRCS = [os.path.join(CSRC, "host", f) for f in ("query.cc", "engine.cc", "gen.cc", "serve.cc")]
HEADERS = [os.path.join(ROOT, "include", f)
           for f in ("warpjq_kernels.h", "warpjq_ext.h", "warpjq_host.h", "warpjq_serve.h")]
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
EXPORTS = os.path.join(CSRC, "exports.map")  # only the C ABI is exported


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.exists(d) and os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(force: bool = False, verbose_ptxas: bool = False) -> None:
    os.makedirs(LIB, exist_ok=True)
    so = os.path.join(LIB, "libwarpjq_kernels.so")
    deps = KERNEL_SRCS + KERNEL_DEPS + HEADERS + [EXPORTS]
    if force or _stale(so, deps):
        extra = ["-Xptxas", "-v"] if verbose_ptxas else []
        _run([NVCC, *NVFLAGS, *extra, "-shared", "-Xlinker", "--version-script=" + EXPORTS, "-o", so,
              *KERNEL_SRCS])
    static = os.path.join(LIB, "libwarpjq_kernels.a")
    if force or _stale(static, deps):
        objs = []
        for src in KERNEL_SRCS:
            obj = os.path.join(LIB, os.path.basename(src) + ".o")
            _run([NVCC, *NVFLAGS, "-c", "-o", obj, src])
            objs.append(obj)
        if os.path.exists(static):
            os.remove(static)
        _run(["ar", "rcs", static, *objs])
        for obj in objs:
            os.remove(obj)
    host = os.path.join(LIB, "libwarpjq_host.so")
    hdeps = HOST_SRCS + [os.path.join(CSRC, "host", "query.h")] + HEADERS + [so, EXPORTS]
    if force or _stale(host, hdeps):
        _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-Wl,--version-script=" + EXPORTS, "-o", host,
              *HOST_SRCS, "-I" + os.path.join(CUDA_HOME, "include"),
              "-L" + LIB, "-lwarpjq_kernels", "-Wl,-rpath,$ORIGIN",
              # the serving loop's streams, events and copies: the CUDA runtime, linked in statically
              os.path.join(CUDA_HOME, "lib64", "libcudart_static.a"), "-ldl", "-lrt", "-lpthread"])


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose_ptxas="-v" in sys.argv)
