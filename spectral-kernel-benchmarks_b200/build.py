"""Build libskb_cuda.so in-tree for sm_100a.

    python spectral-kernel-benchmarks_b200/build.py [--force] [--checked]

Every .cu/.cpp under csrc/ is compiled by nvcc with
``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3`` into build/ and linked
into libskb_cuda.so next to this file.  cudart and the C++ runtime are linked
statically and kept private so the library loads into any process (Python,
the C++ harness, a Go/cgo or JNI host) without clashing with another copy.
Files are rebuilt only when a source or header is newer than the object.
"""

from __future__ import annotations

import argparse
import concurrent.futures
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "build")
LIB = os.path.join(HERE, "libskb_cuda.so")
HARNESS = os.path.join(HERE, "harness")
CLI = os.path.join(HERE, "skbench-cuda")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
          "-I" + CSRC, "-I" + os.path.join(ROOT, "include")]


def nvcc():
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libskb_cuda.so")
    return path


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def headers():
    return glob.glob(os.path.join(CSRC, "*.h*")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))


def compile_one(src, force, extra):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    newest = max([os.path.getmtime(src)] + [os.path.getmtime(h) for h in headers()] +
                 [os.path.getmtime(__file__)])
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= newest:
        return obj, None
    cmd = [nvcc()] + ARCH + COMMON + extra + ["-c", src, "-o", obj]
    if src.endswith(".cu"):
        cmd += ["-Xptxas", "-v"] if os.environ.get("SKB_PTXAS_VERBOSE") else []
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, " ".join(cmd), proc.stderr))
    return obj, proc.stderr


def build(force=False, checked=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    extra = ["-DSKB_CHECKED=1"] if checked else []
    srcs = sources()
    with concurrent.futures.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as pool:
        results = list(pool.map(lambda s: compile_one(s, force, extra), srcs))
    objs = [r[0] for r in results]
    for _, log in results:
        if verbose and log:
            sys.stderr.write(log)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + [
            "-cudart", "static", "-Xcompiler", "-static-libstdc++", "-Xcompiler", "-static-libgcc",
            "-Xlinker", "--exclude-libs,ALL", "-lrt", "-lpthread", "-ldl"]
        proc = subprocess.run(cmd, capture_output=True, text=True)
        if proc.returncode != 0:
            raise RuntimeError("link failed:\n%s\n%s" % (" ".join(cmd), proc.stderr))
    build_cli(force)
    return LIB


def build_cli(force=False):
    """The skbench-cuda command line (harness/*.cpp) against the C ABI only."""
    srcs = sorted(glob.glob(os.path.join(HARNESS, "*.cpp")))
    deps = srcs + glob.glob(os.path.join(HARNESS, "*.hpp")) + [LIB, os.path.join(ROOT, "include", "skb_cuda.h")]
    if not force and os.path.exists(CLI) and os.path.getmtime(CLI) >= max(os.path.getmtime(d) for d in deps):
        return CLI
    cxx = shutil.which("g++") or "g++"
    cmd = [cxx, "-std=c++20", "-O2", "-Wall", "-I" + os.path.join(ROOT, "include")] + srcs + [
        "-o", CLI, "-L" + HERE, "-lskb_cuda", "-Wl,-rpath,$ORIGIN"]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError("harness build failed:\n%s\n%s" % (" ".join(cmd), proc.stderr))
    return CLI


if __name__ == "__main__":
    parser = argparse.ArgumentParser()
    parser.add_argument("--force", action="store_true")
    parser.add_argument("--checked", action="store_true")
    parser.add_argument("--verbose", action="store_true")
    args = parser.parse_args()
    print(build(args.force, args.checked, args.verbose))
