"""Builds libmars_b200.so in-tree with nvcc for sm_100a (B200).

Usage: python -m mars_b200.build   (or mars_b200.build.build() from Python)
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
import tempfile
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libmars_b200.so")
SOURCES = ["api.cu", "search.cu", "search_tc.cu", "decode.cu", "fisher.cu", "fisher_tc.cu", "color.cu", "refine.cu", "noalloc.cu", "codec.cpp", "format.cpp"]
# Translation units whose f64 arithmetic must match the host's operation for operation: no
# multiply-add contraction on the device (the host side is built with -ffp-contract=off).
EXACT_F64_SOURCES = ["rdprice.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found (CUDA 12.9 toolkit expected)")
    return cand


def host_compiler() -> list[str]:
    # The system g++ (its libstdc++ matches the one the Python process loads).
    return ["-ccbin", "/usr/bin/g++"] if os.path.exists("/usr/bin/g++") else []


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, "..", "include", "mars_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not stale():
        return LIB
    common = [nvcc(), *host_compiler(), "-O3", "-std=c++17", "-lineinfo", *ARCH,
              "-Xcompiler", "-fPIC,-ffp-contract=off,-fno-fast-math",
              "-Xptxas", "-v" if verbose else "-O3"]
    with tempfile.TemporaryDirectory() as tmp:
        # One object per translation unit, compiled in parallel, then one link.
        jobs = [(src, []) for src in SOURCES] + [(src, ["--fmad=false"]) for src in EXACT_F64_SOURCES]
        objects = [os.path.join(tmp, os.path.splitext(src)[0] + ".o") for src, _ in jobs]

        def compile_one(i):
            src, extra = jobs[i]
            _run([*common, *extra, "-c", "-o", objects[i], os.path.join(CSRC, src)], verbose)

        with ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 1)) as pool:
            list(pool.map(compile_one, range(len(jobs))))
        _run([*common, "-shared", "-o", LIB + ".tmp", *objects], verbose)
    os.replace(LIB + ".tmp", LIB)
    return LIB


def _run(cmd: list[str], verbose: bool) -> None:
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc failed building libmars_b200.so")
    if verbose:
        sys.stderr.write(res.stderr)


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
