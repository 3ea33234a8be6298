"""Timing of minnow54426/ntt-gpu's own CUDA key switch (the second GPU comparator).

Measurement infrastructure, not part of the product: loads oracle/_ref/libntt_ref_cuda.so
(oracle/Makefile builds it from the reference's src/cuda/ntt_kernels.cu and src/resident.cpp with
oracle/ref_cuda_bridge.cpp) and times the reference's public GPU path, one key switch per call
(upload, Hybrid digits, MAC, ModDown of both channels, download), on seeded synthetic inputs
of the benchmark shape. Prints one JSON line.

    python -m oracle.ref_cuda_timing [--n 65536 --level 24 --k 8 --dnum 3 --count 5]
"""
import argparse
import ctypes
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
from ntt_gpu_b200.params import synthetic_params, uniform_residues  # noqa: E402

_U64P = ctypes.POINTER(ctypes.c_uint64)
LIB_PATH = os.path.join(HERE, "_ref", "libntt_ref_cuda.so")


def load():
    lib = ctypes.CDLL(LIB_PATH)
    lib.refcuda_last_error.restype = ctypes.c_char_p
    return lib


def reference_keyswitch(lib, prm, level, x, kb, ka, device=0, warmup=1, count=1):
    """The reference's CUDA key switch of one component: (ms per key switch, out_b, out_a)."""
    n = prm.n
    arr = lambda v: np.ascontiguousarray(np.array(v, dtype=np.uint64))  # noqa: E731
    keep = [arr(prm.q), arr(prm.q_psi), arr(prm.p), arr(prm.p_psi), np.ascontiguousarray(x, dtype=np.uint64),
            np.ascontiguousarray(kb, dtype=np.uint64), np.ascontiguousarray(ka, dtype=np.uint64)]
    ptr = lambda a: a.ctypes.data_as(_U64P)  # noqa: E731
    ob, oa = np.zeros((level, n), np.uint64), np.zeros((level, n), np.uint64)
    ms = ctypes.c_double()
    rc = lib.refcuda_keyswitch(ctypes.c_uint64(n), ptr(keep[0]), ptr(keep[1]), ctypes.c_size_t(prm.m),
                               ptr(keep[2]), ptr(keep[3]), ctypes.c_size_t(len(prm.p)), ctypes.c_size_t(prm.alpha),
                               ctypes.c_size_t(level), ptr(keep[4]), ptr(keep[5]), ptr(keep[6]), device, warmup,
                               count, ctypes.byref(ms), ptr(ob), ptr(oa))
    if rc != 0:
        raise RuntimeError(lib.refcuda_last_error().decode())
    return ms.value, ob, oa


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=65536)
    ap.add_argument("--level", type=int, default=24)
    ap.add_argument("--k", type=int, default=8)
    ap.add_argument("--dnum", type=int, default=3)
    ap.add_argument("--count", type=int, default=5)
    args = ap.parse_args()
    prm = synthetic_params(args.n, args.level, args.k, args.dnum)
    x = uniform_residues(args.n, prm.q, 5)[0]
    kb = uniform_residues(args.n, prm.q + prm.p, 7, polys=prm.full_digits())
    ka = uniform_residues(args.n, prm.q + prm.p, 9, polys=prm.full_digits())
    ms, _, _ = reference_keyswitch(load(), prm, args.level, x, kb, ka, warmup=2, count=args.count)
    print(json.dumps({"impl": "reference CUDA resident path (src/cuda/ntt_kernels.cu, resident_adapter.inc)",
                      "workload": f"key switch N={args.n}, L={args.level}, K={args.k}, dnum={args.dnum}, "
                                  "one component per call, host buffers in and out",
                      "ms_per_keyswitch": ms, "keyswitch_per_s": 1000.0 / ms, "timed": args.count}))


if __name__ == "__main__":
    main()
