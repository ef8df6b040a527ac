"""Build libsgb200.so (the C-ABI library) in-tree for sm_100a with nvcc.

Usage: python -m openfpm_data_b200.build [--force]
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libsgb200.so")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    # the reference builds its kernels with -use_fast_math (FMA contraction,
    # flush-to-zero); the stencils reproduce that arithmetic explicitly
    "-ftz=true", "-fmad=true",
    "-Xcompiler", "-fPIC", "-shared",
    "-Xptxas", "-warn-spills",
]


def sources():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + glob.glob(os.path.join(HERE, "csrc", "*.cuh")) + glob.glob(os.path.join(HERE, "csrc", "*.h"))
    deps += glob.glob(os.path.join(ROOT, "include", "*.h"))
    return any(os.path.getmtime(d) > t for d in deps)


OBJ_DIR = os.path.join(HERE, "_build")


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile every csrc/*.cu to an object in parallel, then link the shared library."""
    if not force and not _stale():
        return LIB
    from concurrent.futures import ThreadPoolExecutor
    nvcc = os.environ.get("NVCC", "nvcc")
    os.makedirs(OBJ_DIR, exist_ok=True)
    compile_flags = [f for f in NVCC_FLAGS if f != "-shared"]

    def compile_one(src):
        obj = os.path.join(OBJ_DIR, os.path.basename(src)[:-3] + ".o")
        cmd = [nvcc] + compile_flags + ["-I", os.path.join(ROOT, "include"), "-c", "-o", obj, src]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        return obj, r

    srcs = sources()
    with ThreadPoolExecutor(max_workers=max(1, min(len(srcs), os.cpu_count() or 1))) as ex:
        results = list(ex.map(compile_one, srcs))
    for obj, r in results:
        sys.stdout.write(r.stdout)
        sys.stderr.write(r.stderr)
        if r.returncode != 0:
            raise subprocess.CalledProcessError(r.returncode, r.args)
    tmp = LIB + ".tmp"
    cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-Xcompiler", "-fPIC", "-o", tmp]
    cmd += [obj for obj, _ in results]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


DROPIN_SRC = os.path.join(ROOT, "tests", "cpp", "test_dropin.cu")
DROPIN_BIN = os.path.join(ROOT, "tests", "cpp", "_build", "test_dropin")


def build_dropin_test(force: bool = False, verbose: bool = False) -> str:
    """Compile the C++ drop-in test (user code against include/openfpm_b200/SparseGridGpu.hpp)."""
    lib = build(verbose=verbose)
    deps = [DROPIN_SRC, lib] + glob.glob(os.path.join(ROOT, "include", "**", "*.h*"), recursive=True)
    if not force and os.path.exists(DROPIN_BIN) and all(os.path.getmtime(d) <= os.path.getmtime(DROPIN_BIN)
                                                         for d in deps):
        return DROPIN_BIN
    os.makedirs(os.path.dirname(DROPIN_BIN), exist_ok=True)
    nvcc = os.environ.get("NVCC", "nvcc")
    tmp = DROPIN_BIN + ".tmp"
    cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-lineinfo", "-std=c++17",
           "--extended-lambda", "-ftz=true", "-fmad=true", "-I", os.path.join(ROOT, "include"),
           "-o", tmp, DROPIN_SRC, "-L", HERE, "-lsgb200",
           # the binary sits in tests/cpp/_build; the library three levels up in openfpm_data_b200/
           "-Xlinker", "-rpath,$ORIGIN/../../../openfpm_data_b200"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, DROPIN_BIN)
    return DROPIN_BIN


CONV_BENCH_SRC = os.path.join(HERE, "bench_conv.cu")
CONV_BENCH_BIN = os.path.join(OBJ_DIR, "bench_conv")


def build_conv_bench(force: bool = False, verbose: bool = False) -> str:
    """Compile the conv2_b-vs-GS7 throughput program (user lambda code against the C++ header)."""
    lib = build(verbose=verbose)
    deps = [CONV_BENCH_SRC, lib] + glob.glob(os.path.join(ROOT, "include", "**", "*.h*"), recursive=True)
    if not force and os.path.exists(CONV_BENCH_BIN) and all(os.path.getmtime(d) <= os.path.getmtime(CONV_BENCH_BIN)
                                                            for d in deps):
        return CONV_BENCH_BIN
    os.makedirs(OBJ_DIR, exist_ok=True)
    nvcc = os.environ.get("NVCC", "nvcc")
    tmp = CONV_BENCH_BIN + ".tmp"
    cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
           "--extended-lambda", "-ftz=true", "-fmad=true", "-I", os.path.join(ROOT, "include"),
           "-o", tmp, CONV_BENCH_SRC, "-L", HERE, "-lsgb200", "-Xlinker", "-rpath,$ORIGIN/.."]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, CONV_BENCH_BIN)
    return CONV_BENCH_BIN


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
    if "--dropin" in sys.argv:
        print(build_dropin_test(force="--force" in sys.argv, verbose=True))
    if "--conv-bench" in sys.argv:
        print(build_conv_bench(force="--force" in sys.argv, verbose=True))
