"""Allocation-free ModDown (ntt_b200_mod_down_static) through the C ABI.

Some callers cannot allocate device memory. Examples: a host whose HBM is
already owned by another caching allocator, a latency-critical request thread
that cannot afford cudaMalloc's implicit device synchronisation, and an FFI
host with no way to own device buffers across the boundary. This entry point
serves them: its scratch is a fixed device array inside the library. The test
checks, on two calls in a row, that its output equals the workspace-based
ntt_b200_mod_down bit for bit, and that the second call leaves the device's
free memory and its stream-ordered pool's usage unchanged (it allocates
nothing). It also checks that a request larger than the array is refused
before anything runs. The file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

import ntt_gpu_b200 as nb
from oracle.oracle import pinned_context, synthetic_context

pytestmark = pytest.mark.gpu


def _stream():
    import torch
    return torch.cuda.current_stream().cuda_stream


def _static_mod_down(g, level, dst, src):
    lib = nb.load()
    rc = lib.ntt_b200_mod_down_static(g._h, level, ctypes.c_void_p(dst.data_ptr()),
                                      ctypes.c_void_p(src.data_ptr()), _stream())
    return rc, lib.ntt_b200_last_error().decode()


def _device_memory():
    """(free bytes of the device, bytes in use in its stream-ordered pool)."""
    import torch
    from cuda.bindings import runtime as rt
    torch.cuda.synchronize()
    err, pool = rt.cudaDeviceGetDefaultMemPool(torch.cuda.current_device())
    assert err == rt.cudaError_t.cudaSuccess
    err, used = rt.cudaMemPoolGetAttribute(pool, rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemCurrent)
    assert err == rt.cudaError_t.cudaSuccess
    return torch.cuda.mem_get_info()[0], int(used)


def _check_two_calls(orc, ctx, level, seeds):
    import torch
    g = nb.Context.from_oracle(ctx)
    g.prepare(level)
    ws = g.workspace(nb.OP_MOD_DOWN, level)
    for call, seed in enumerate(seeds):  # two calls in a row share (and overwrite) the static scratch
        y = orc.lcg(ctx.n, ctx.qp_moduli(level), seed)
        src = nb.to_device(y)
        want = nb.empty((level, ctx.n))
        g.mod_down(level, want, src, ws)
        got = nb.empty((level, ctx.n))
        before = _device_memory()
        rc, msg = _static_mod_down(g, level, got, src)
        assert rc == nb.OK, msg
        torch.cuda.synchronize()
        if call > 0:  # after the first call's one-time set-up, a call allocates nothing
            assert _device_memory() == before
        np.testing.assert_array_equal(nb.to_host(got), nb.to_host(want))
        np.testing.assert_array_equal(nb.to_host(got), orc.mod_down(ctx, level, y))
    g.close()


def test_static_mod_down_matches_workspace_mod_down(orc, lib):
    assert nb.load().ntt_b200_mod_down_static_max_bytes() == 8 << 20
    _check_two_calls(orc, pinned_context(), 5, (101, 202))          # N = 2^16: 8 towers x 512 KiB
    _check_two_calls(orc, synthetic_context(orc, 16384, 24, 8, 3), 24, (303, 404))  # N = 2^14: 32 towers


def test_static_mod_down_refuses_oversized_requests(orc, lib):
    ctx = synthetic_context(orc, 65536, 24, 8, 3)  # (8 + 24) x 512 KiB = 16 MiB > 8 MiB
    g = nb.Context.from_oracle(ctx)
    g.prepare(24)
    src, dst = nb.empty((32, ctx.n)), nb.empty((24, ctx.n))
    rc, msg = _static_mod_down(g, 24, dst, src)
    assert rc == nb.ERR_CONTRACT and "static maximum" in msg
    g.close()
