"""Builds the in-tree CUDA library (libinlm.so) and the iterNLM command line.

    python -m microtomodenoise_b200.build          # library + CLI
    python -m microtomodenoise_b200.build --lib    # library only

Everything is compiled for sm_100a only (``-gencode arch=compute_100a,code=sm_100a``);
nvcc cross-compiles without a GPU. Host code is built with
``-ffp-contract=off`` so the geometry tables round exactly as the reference's
g++ build does.
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
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libinlm.so")
CLI = os.path.join(LIBDIR, "iterNLM")
BUILD_DIR = os.path.join(ROOT, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
    "-I" + os.path.join(ROOT, "include"),
]

LIB_SOURCES = [
    "filter_kernels.cu",
    "filter_column.cu",
    "filter_fast.cu",
    "noise_kernels.cu",
    "api.cu",
    "proposal.cu",
    "proposal_tc.cu",
    "api_proposal.cu",
    "api_batch.cu",
    "api_stream.cu",
    "color_kernels.cu",
    "api_color.cu",
    "api_multi.cu",
    "api_blocks.cu",
    "filter_f64.cu",
    "geometry.cpp",
    "sampling.cpp",
    "tiff_io.cpp",
]


def nvcc() -> str:
    for c in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _newer(target: str, sources) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {os.path.basename(cmd[-1])}")
    return r


def build_lib(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(BUILD_DIR, exist_ok=True)
    headers = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.hpp")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))
    objs, cmds = [], []
    for src in LIB_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD_DIR, src + ".o")
        objs.append(o)
        if force or _newer(o, [s] + headers):
            cmd = [nvcc()] + NVCC_FLAGS + ["-c", s, "-o", o]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
            cmds.append(cmd)
    # translation units compile independently
    with concurrent.futures.ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        for r in ex.map(_run, cmds):
            if verbose:
                sys.stderr.write(r.stderr)
    if force or _newer(LIB, objs):
        _run([nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"])
    return LIB


def build_cli(force: bool = False) -> str:
    src = os.path.join(CSRC, "main.cpp")
    if not os.path.exists(src):
        return ""
    deps = [src, LIB, os.path.join(CSRC, "iternlm.hpp")]
    if force or _newer(CLI, [d for d in deps if os.path.exists(d)]):
        _run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-I" + os.path.join(ROOT, "include"), "-I" + CSRC,
              src, "-o", CLI, "-L" + LIBDIR, "-linlm", "-Wl,-rpath,$ORIGIN"])
    return CLI


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--lib", action="store_true")
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args(argv)
    print(build_lib(force=a.force, verbose=a.verbose))
    if not a.lib:
        print(build_cli(force=a.force))


if __name__ == "__main__":
    main()
