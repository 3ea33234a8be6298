"""Parity against the reference's own GPU path.

oracle/_ref/libntt_ref_cuda.so is minnow54426/ntt-gpu's CUDA resident backend
(src/cuda/ntt_kernels.cu with resident_adapter.inc, src/resident.cpp) compiled
for sm_100a by oracle/Makefile. Its Hybrid key switch, run on the same seeded
inputs, must equal ours bit for bit. Skipped where that library was not built
(no reference tree at build time)."""
import os

import numpy as np
import pytest

import ntt_gpu_b200 as nb
from ntt_gpu_b200.params import synthetic_params, uniform_residues

pytestmark = pytest.mark.gpu

_LIB = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                    "libntt_ref_cuda.so")


@pytest.mark.skipif(not os.path.exists(_LIB), reason="reference CUDA library not built")
@pytest.mark.parametrize("n,m,k,dnum", [(4096, 6, 3, 2), (65536, 24, 8, 3)])
def test_keyswitch_equals_the_reference_cuda_path(lib, n, m, k, dnum):
    import torch

    from oracle.ref_cuda_timing import load, reference_keyswitch
    prm = synthetic_params(n, m, k, dnum)
    level = m
    x = uniform_residues(n, prm.q[:level], 11)[0]
    kb = uniform_residues(n, prm.q + prm.p, 13, polys=prm.full_digits())
    ka = uniform_residues(n, prm.q + prm.p, 17, polys=prm.full_digits())
    _, rb, ra = reference_keyswitch(load(), prm, level, x, kb, ka, warmup=0, count=1)
    g = nb.Context(n, prm.q, prm.q_psi, prm.p, prm.p_psi, prm.alpha)
    ob, oa = nb.empty((level, n)), nb.empty((level, n))
    g.keyswitch(level, ob, oa, nb.to_device(x), nb.to_device(kb), nb.to_device(ka),
                g.workspace(nb.OP_KEYSWITCH, level))
    torch.cuda.synchronize()
    np.testing.assert_array_equal(nb.to_host(ob), rb)
    np.testing.assert_array_equal(nb.to_host(oa), ra)
    g.close()
