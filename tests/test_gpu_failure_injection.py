"""Failure detection without a GPU fault.

- A bounded device wait made to expire: the tensor-core conversion's first
  mbarrier wait gets a poll limit of 0, so it gives up at once; the kernel
  waits (bounded) for its own bulk copy, frees its tensor memory and returns,
  the call completes, and ntt_b200_device_errors reports the timeout. With the
  limit restored the same conversion is exact again.
- Context setup failures injected on the host before each device allocation
  and upload (the reference's SetupResources failure steps,
  include/ntt/setup_resources.hpp:19-60): every partly built context is
  released, no device memory leaks, and the next context works."""
import numpy as np
import pytest

import ntt_gpu_b200 as nb
from oracle.oracle import synthetic_context

pytestmark = pytest.mark.gpu


def test_conversion_wait_expires_and_reports(lib, orc):
    import torch
    ctx = synthetic_context(orc, 4096, 8, 4, 2)
    g = nb.Context.from_oracle(ctx)
    assert nb.tuning_get("conv_tc") == 1
    src, tgt = list(range(8)), [8, 9, 10, 11]
    x = orc.lcg(ctx.n, ctx.q, 5)
    dx = nb.to_device(x)
    out = nb.empty((4, ctx.n))
    g.device_errors(clear=True)
    try:
        nb._check(nb.load().ntt_b200_conv_wait_polls(0))
        g.switch_basis(out, dx, src, tgt)  # returns: the kernel gives up its first wait
        torch.cuda.synchronize()
        assert g.device_errors(clear=True) > 0
    finally:
        nb._check(nb.load().ntt_b200_conv_wait_polls(1 << 20))
    g.switch_basis(out, dx, src, tgt)
    torch.cuda.synchronize()
    assert g.device_errors() == 0
    np.testing.assert_array_equal(nb.to_host(out), orc.basis_convert(x, ctx.q, ctx.p))
    with pytest.raises(nb.ContractError):
        nb._check(nb.load().ntt_b200_conv_wait_polls(-1))
    g.close()


def test_context_setup_failures_unwind(lib, orc):
    import ctypes

    import torch
    ctx = synthetic_context(orc, 65536, 8, 4, 2)  # 12 towers: 24 MiB of twiddle tables
    nb.Context.from_oracle(ctx).close()
    ops = ctypes.c_size_t()
    nb._check(nb.load().ntt_b200_setup_operations(ctypes.byref(ops)))
    assert ops.value >= 8
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for k in range(1, ops.value + 1):
        nb._check(nb.load().ntt_b200_inject_setup_failure(k))
        with pytest.raises(nb.CudaError, match=f"injected failure before setup operation {k}$"):
            nb.Context.from_oracle(ctx)
        assert torch.cuda.mem_get_info()[0] >= free0 - (2 << 20), f"setup step {k} leaked device memory"
    g = nb.Context.from_oracle(ctx)  # the injection was one-shot
    x = orc.lcg(ctx.n, ctx.q[:2], 9)
    out = nb.empty(x.shape)
    g.ntt(out, nb.to_device(x), [0, 1])
    np.testing.assert_array_equal(nb.to_host(out), orc.ntt(x, ctx.q[:2], ctx.q_psi[:2]))
    g.close()
