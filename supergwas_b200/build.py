"""In-tree build of the CUDA library and the ``kgwas`` program.

Outputs (git-ignored, shipped with the source tree):
  supergwas_b200/lib/libkgwas_cuda.so   C ABI of include/kgwas_cuda.h
  supergwas_b200/bin/kgwas              drop-in for the reference's kgwas CLI
  supergwas_b200/bin/kgwas_2d           drop-in for the reference's kgwas_2d CLI

Everything device-side is compiled for sm_100a only.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB_DIR = os.path.join(PKG, "lib")
BIN_DIR = os.path.join(PKG, "bin")
LIB = os.path.join(LIB_DIR, "libkgwas_cuda.so")
BENCH_LIB = os.path.join(LIB_DIR, "libkgwas_bench.so")  # bench-side device code (generator, MMA-rate kernels)
BENCH_SOURCES = ["bench_synth.cu", "bench_mma_rate.cu"]
CLI = os.path.join(BIN_DIR, "kgwas")
CLI2 = os.path.join(BIN_DIR, "kgwas_2d")
MERGE = os.path.join(BIN_DIR, "kgwas_index_merge")
OBJ_DIR = os.path.join(PKG, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
LIB_SOURCES = ["kernels.cu", "kernel_ts.cu", "kernel_mp.cu", "kernel_mpb.cu", "kernel_mpb2.cu", "kernel_pairs.cu", "capi_pairs.cpp", "noalloc.cu", "probes.cu", "capi.cpp", "capi_multi.cpp", "prep.cpp"]
CLI_SOURCES = ["kgwas_main.cpp", "kgwas_io.cpp"]
CLI2_SOURCES = ["kgwas2d_main.cpp", "kgwas_io.cpp"]
MERGE_SOURCES = ["index_merge_main.cpp", "kgwas_io.cpp"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def _deps(names):
    out = [os.path.join(CSRC, s) for s in names]
    out += [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".hpp", ".cuh", ".h"))]
    out.append(os.path.join(ROOT, "include", "kgwas_cuda.h"))
    out.append(os.path.abspath(__file__))
    return out


def run(cmd, verbose=False):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build failed: {' '.join(cmd[:3])} ...")
    return r


def build_lib(force=False, verbose=False, ptxas_verbose=False) -> str:
    """Compile every source to an object in parallel, then link the shared library."""
    deps = _deps(LIB_SOURCES)
    if not force and _newer(LIB, deps):
        return LIB
    os.makedirs(LIB_DIR, exist_ok=True)
    os.makedirs(OBJ_DIR, exist_ok=True)
    base = [nvcc(), *ARCH, "-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O3"]
    if ptxas_verbose:
        base.append("-Xptxas=-v")
    objs = [os.path.join(OBJ_DIR, os.path.splitext(s)[0] + ".o") for s in LIB_SOURCES]
    cmds = [base + ["-c", os.path.join(CSRC, s), "-o", o] for s, o in zip(LIB_SOURCES, objs)]
    with ThreadPoolExecutor(max_workers=min(len(cmds), os.cpu_count() or 1)) as ex:
        results = list(ex.map(lambda c: run(c, verbose), cmds))
    if ptxas_verbose:
        for r in results:
            sys.stderr.write(r.stderr)
    run([nvcc(), *ARCH, "-shared", "-o", LIB, *objs], verbose)
    return LIB


def build_cli(force=False, verbose=False, target=None, sources=None) -> str:
    target = target or CLI
    sources = sources or CLI_SOURCES
    deps = _deps(sources) + [LIB]
    if not force and _newer(target, deps):
        return target
    os.makedirs(BIN_DIR, exist_ok=True)
    cmd = ["g++", "-O3", "-std=c++17", "-fopenmp", "-o", target,
           *[os.path.join(CSRC, s) for s in sources],
           "-L" + LIB_DIR, "-lkgwas_cuda", "-Wl,-rpath,$ORIGIN/../lib", "-lz", "-lpthread"]
    run(cmd, verbose)
    return target


def build_bench(force=False, verbose=False) -> str:
    """Bench-side device code, not the association library: the seeded
    generator of synthetic batches and the tensor-core rate kernels."""
    srcs = [os.path.join(CSRC, f) for f in BENCH_SOURCES]
    if not force and _newer(BENCH_LIB, srcs + [os.path.join(CSRC, "device.cuh"), os.path.abspath(__file__)]):
        return BENCH_LIB
    os.makedirs(LIB_DIR, exist_ok=True)
    run([nvcc(), *ARCH, "-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-shared", "-o", BENCH_LIB, *srcs],
        verbose)
    return BENCH_LIB


def build_all(force=False, verbose=False):
    build_lib(force, verbose)
    build_bench(force, verbose)
    build_cli(force, verbose)
    build_cli(force, verbose, CLI2, CLI2_SOURCES)
    build_cli(force, verbose, MERGE, MERGE_SOURCES)
    return LIB, CLI


if __name__ == "__main__":
    force = "--force" in sys.argv
    verbose = "-v" in sys.argv
    if "--ptxas" in sys.argv:
        build_lib(True, verbose, ptxas_verbose=True)
    else:
        print(build_all(force, verbose))
