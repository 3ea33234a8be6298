"""Build recipe for the in-tree sm_100a library (libntt_b200.so).

Compiles the translation units of ntt_gpu_b200/csrc (capi.cu, rowmac.cu,
server.cpp, keycache.cpp) with nvcc for sm_100a only, in parallel, and links
ntt_gpu_b200/lib/libntt_b200.so. The library travels with the source tree;
nothing is installed into site-packages.
"""
from __future__ import annotations

import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIB_DIR, "libntt_b200.so")
NVCC_FLAGS = ["-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
              "-Xcompiler", "-fPIC", "-shared"]


def sources() -> list[str]:
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC)
                  if f.endswith((".cu", ".cuh", ".cpp", ".h", ".hpp")))


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    built = os.path.getmtime(target)
    return any(os.path.getmtime(p) > built for p in deps if os.path.exists(p))


def stale() -> bool:
    header = os.path.join(HERE, "..", "include", "ntt_b200.h")
    return _stale(LIB, sources() + [header, __file__])


# Translation units of libntt_b200.so, compiled in parallel to objects under
# _build/ and linked by nvcc: capi.cu (host side and every other kernel),
# rowmac.cu (the fused row pass + key multiplication instantiations) and the
# host-only server and key cache.
UNITS = ("capi.cu", "rowmac.cu", "server.cpp", "keycache.cpp")
BUILD_DIR = os.path.join(HERE, "_build")


def _compile(nvcc: str, unit: str, verbose: bool) -> str:
    obj = os.path.join(BUILD_DIR, unit + ".o")
    flags = [f for f in NVCC_FLAGS if f != "-shared"]
    cmd = [nvcc, *flags, "-c", "-o", obj, os.path.join(CSRC, unit)]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not stale():
        return LIB
    header = os.path.join(HERE, "..", "include", "ntt_b200.h")
    os.makedirs(LIB_DIR, exist_ok=True)
    if force or _stale(LIB, sources() + [header, __file__]):
        from concurrent.futures import ThreadPoolExecutor
        nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
        os.makedirs(BUILD_DIR, exist_ok=True)
        with ThreadPoolExecutor(max_workers=len(UNITS)) as pool:
            objs = list(pool.map(lambda u: _compile(nvcc, u, verbose), UNITS))
        tmp = LIB + ".tmp"
        cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", tmp, *objs]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        os.replace(tmp, LIB)
    return LIB
