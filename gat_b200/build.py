"""Build recipe for libgat_b200.so (and the test oracles under oracle/).

Host C++ is compiled by g++ through nvcc; CUDA sources are compiled for sm_100a only
(`-gencode arch=compute_100a,code=sm_100a`). The library is written in-tree next to this file
so that it travels with the source tree. Incremental: an object is rebuilt when its source or
any header under csrc/ or include/ is newer.

Usage: python gat_b200/build.py [--force] [--no-oracle] [-j N]   (run by path: importing the
package would load the library being built)
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
OBJDIR = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libgat_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-I", INCLUDE, "-I", CSRC, "-Xcompiler", "-fPIC"]
# float expressions on the host must round exactly like the reference's (no contraction)
HOST_FLAGS = ARCH + ["-Xcompiler", "-ffp-contract=off,-pthread,-Wall,-Wno-unused-function"]
# no fast-math: the EDR match test and cell assignment need IEEE float subtraction/division
CUDA_FLAGS = ARCH + ["-lineinfo", "--fmad=false", "-Xptxas", "-warn-spills"]


def sources() -> list[str]:
    out = []
    for name in sorted(os.listdir(CSRC)):
        if name.endswith((".cpp", ".cu")):
            out.append(os.path.join(CSRC, name))
    return out


def _headers() -> list[str]:
    hs = []
    for d in (CSRC, INCLUDE):
        for name in os.listdir(d):
            if name.endswith((".h", ".cuh", ".hpp")):
                hs.append(os.path.join(d, name))
    return hs


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str, force: bool) -> str:
    obj = os.path.join(OBJDIR, os.path.basename(src) + ".o")
    if not force and not _stale(obj, [src] + _headers()):
        return obj
    flags = COMMON + (CUDA_FLAGS if src.endswith(".cu") else HOST_FLAGS)
    cmd = [NVCC] + flags + ["-c", src, "-o", obj]
    if src.endswith(".cpp"):
        cmd = [NVCC] + flags + ["-x", "c++", "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if r.stderr.strip():
        sys.stderr.write(r.stderr)
    return obj


def build_library(force: bool = False, jobs: int = 8) -> str:
    os.makedirs(OBJDIR, exist_ok=True)
    srcs = sources()
    with ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, force), srcs))
    if force or _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart", "-Xcompiler", "-pthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return LIB


# checkout of the reference whose CPU sources oracle/Makefile compiles into oracle/_ref/gatref
REFERENCE_DIR = os.environ.get("GAT_REFERENCE_DIR", "/root/reference")


def build_oracle() -> None:
    """Test oracles: oracle/liboracle.so always; oracle/_ref/gatref when the reference sources
    are present (elsewhere the prebuilt binary is kept)."""
    r = subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "-j8", f"REF={REFERENCE_DIR}"],
                       capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stdout}\n{r.stderr}")


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--no-oracle", action="store_true")
    ap.add_argument("-j", type=int, default=8)
    a = ap.parse_args()
    print(build_library(a.force, a.j))
    if not a.no_oracle:
        build_oracle()


if __name__ == "__main__":
    main()
