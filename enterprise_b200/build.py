"""Build recipe for the native parts of enterprise_b200.

Compiles the CUDA/C++ sources under ``csrc/`` for sm_100a with nvcc and links
``lib/libenterprise_b200.so`` (the C ABI declared in include/enterprise_b200.h)
and ``lib/enterprise.bin`` (the drop-in command line). Objects go to
``_build/`` at the repository root. Rebuilds only what changed.

Usage: python -m enterprise_b200.build [--force] [--verbose]
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIBDIR = os.path.join(PKG, "lib")
OBJDIR = os.path.join(ROOT, "_build", "enterprise_b200")
LIB = os.path.join(LIBDIR, "libenterprise_b200.so")
CLI = os.path.join(LIBDIR, "enterprise.bin")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-fopenmp,-Wall",
              "--expt-relaxed-constexpr", "-I" + INCLUDE, "-I" + CSRC] + ARCH
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-fopenmp", "-Wall", "-I" + INCLUDE, "-I" + CSRC,
             "-I/usr/local/cuda/include"]

SOURCES = [
    "host_graph.cpp",
    "device_graph.cu",
    "bfs_single.cu",
    "bfs_batch.cu",
    "bfs_noalloc.cu",
    "bfs_validate.cu",
    "graph_ingest.cu",
    "serve.cpp",
    "replicas.cpp",
    "tune.cpp",
]
HEADERS = ["gen_common.h", "ent_internal.h", "dev_graph.h", "dev_common.cuh", "batch_internal.h"]


def nvcc() -> str:
    p = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return p


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ...")
    if verbose and (r.stdout or r.stderr):
        sys.stderr.write(r.stdout + r.stderr)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJDIR, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "enterprise_b200.h")]
    objs = []
    for s in SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(OBJDIR, s + ".o")
        objs.append(obj)
        if force or _stale(obj, [src, __file__] + hdrs):
            if s.endswith(".cu"):
                cmd = [nvcc()] + NVCC_FLAGS + ["-c", src, "-o", obj]
            else:
                cmd = ["g++"] + CXX_FLAGS + ["-c", src, "-o", obj]
            _run(cmd, verbose)
    if force or _stale(LIB, objs):
        _run([nvcc(), "-shared"] + ARCH + ["-o", LIB] + objs + ["-lgomp", "-lpthread"], verbose)
    cli_src = os.path.join(CSRC, "cli_main.cpp")
    if force or _stale(CLI, [cli_src, LIB, os.path.join(INCLUDE, "bfs_gpu_opt.cuh")] + hdrs):
        _run(["g++", "-O2", "-std=c++17", "-I" + INCLUDE, cli_src, "-o", CLI, "-L" + LIBDIR,
              "-lenterprise_b200", "-Wl,-rpath,$ORIGIN"], verbose)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="--verbose" in sys.argv)
    print(LIB)
