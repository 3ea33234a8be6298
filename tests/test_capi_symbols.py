"""The sm_100a library loads on a host without a GPU and exports every entry
point include/ntt_b200.h declares (no compute calls)."""
import ctypes
import os
import re

import ntt_gpu_b200
from ntt_gpu_b200 import build

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "ntt_b200.h")


def declared():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(ntt_b200_\w+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared()
    assert "ntt_b200_keyswitch" in names and "ntt_b200_ntt" in names and len(names) >= 17


def test_library_exports_every_declared_symbol():
    build.build()
    lib = ctypes.CDLL(build.LIB)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_bindings_cover_header():
    assert set(declared()) <= set(ntt_gpu_b200._SIGNATURES)


def test_no_cuda_device_is_reported_as_cuda_error():
    """Without a GPU, context creation fails with a CUDA error status, not a crash."""
    import torch
    if torch.cuda.is_available():
        return
    lib = ntt_gpu_b200.load()
    h = ctypes.c_void_p()
    q = (ctypes.c_uint64 * 1)(1152921504606584833)
    psi = (ctypes.c_uint64 * 1)(18043022392882)
    rc = lib.ntt_b200_context_create(ctypes.byref(h), 0, 65536, q, psi, 1, None, None, 0, 1)
    assert rc == ntt_gpu_b200.ERR_CUDA
    assert b"CUDA" in lib.ntt_b200_last_error()


def test_contract_errors_precede_any_device_use():
    lib = ntt_gpu_b200.load()
    h = ctypes.c_void_p()
    q = (ctypes.c_uint64 * 1)(97)  # 97 % 128 != 1 at n = 64
    psi = (ctypes.c_uint64 * 1)(3)
    assert lib.ntt_b200_context_create(ctypes.byref(h), 0, 64, q, psi, 1, None, None, 0, 1) == ntt_gpu_b200.ERR_CONTRACT
    assert lib.ntt_b200_context_create(ctypes.byref(h), 0, 3, q, psi, 1, None, None, 0, 1) == ntt_gpu_b200.ERR_CONTRACT
    assert lib.ntt_b200_ntt(None, None, None, None, 1, 1, 0, 0, None) == ntt_gpu_b200.ERR_CONTRACT
