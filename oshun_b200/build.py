"""Builds liboshun_b200.so (sm_100a) in-tree with nvcc.

    python -m oshun_b200.build [--verbose] [--ptxas-info]
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "liboshun_b200.so")
SOURCES = ["vlasov.cu", "stage_pipe.cu", "stage_batch.cu", "collide.cu", "adjoint.cu", "abi.cu", "noalloc.cu",
           "moments.cu", "restart.cu", "implicit_e.cu", "halo.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(INCLUDE, "oshun_b200.h")]
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, ptxas_info: bool = False, force: bool = False) -> str:
    if not force and not needs_build():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    nvcc = nvcc_path()
    common = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I", INCLUDE,
                     "--expt-relaxed-constexpr", "-Xcompiler", "-Wall"]
    if ptxas_info:
        common += ["-Xptxas", "-v"]
    # translation units compile in parallel
    def compile_one(src):
        obj = os.path.join(objdir, src.replace(".cu", ".o"))
        cmd = [nvcc] + common + ["-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        return src, obj, r

    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=min(len(SOURCES), os.cpu_count() or 1)) as ex:
        results = list(ex.map(compile_one, SOURCES))
    objs = []
    for src, obj, r in results:
        if r.returncode != 0 or (verbose and r.stderr):
            sys.stderr.write(r.stderr)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}")
        objs.append(obj)
    tmp = LIB + ".tmp"
    cmd = [nvcc] + ARCH + ["-shared", "-o", tmp] + objs + ["-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stderr)
        raise RuntimeError("link failed")
    os.replace(tmp, LIB)
    build_host(verbose)
    return LIB


def build_host(verbose: bool = False) -> str:
    """The C++ example driver over the host layer (host/oshun.hpp)."""
    src = os.path.join(HERE, "host", "oshun_main_loop.cpp")
    out = os.path.join(HERE, "host", "oshun_main_loop")
    cmd = ["g++", "-O2", "-std=c++17", "-Wall", "-Wextra", "-I", INCLUDE, "-I", os.path.join(HERE, "host"), src,
           "-L", HERE, "-loshun_b200", "-Wl,-rpath,$ORIGIN/..", "-o", out]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stderr)
        raise RuntimeError("host driver build failed")
    return out


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, ptxas_info="--ptxas-info" in sys.argv, force=True)
    print(LIB)
