"""The tensor-core approximate-CRT switch (tcgen05, unsigned int8 limbs, int32
accumulators in tensor memory) against the CPU oracle, bit for bit.

The kernel multiplies the byte limbs of y_j = [x_j * Bhat_j^-1]_{b_j} by the
byte limbs of [Bhat_jt * 2^(8a)]_{m_t}, so sources 1..16 (K = 32..128 bytes),
target counts around its group size of 8, canonical and lazy outputs, and the
bounded-wait error word are all exercised."""
import numpy as np
import pytest

import ntt_gpu_b200 as nb
from oracle.oracle import synthetic_context
from test_gpu_requests import full_keys

pytestmark = pytest.mark.gpu


@pytest.fixture
def tc_on(lib):
    before = nb.tuning_get("conv_tc")
    nb.tuning_set("conv_tc", 1)
    yield
    nb.tuning_set("conv_tc", before)


@pytest.mark.parametrize("n,s,t", [(4096, 1, 1), (4096, 3, 7), (4096, 8, 8), (8192, 8, 9), (65536, 8, 24),
                                   (4096, 11, 24), (4096, 16, 40), (128, 5, 3)])
def test_switch_basis_on_tensor_cores(tc_on, orc, n, s, t):
    bits = [50 + (i % 11) for i in range(s + t)]
    q = []
    for b in bits:
        for v in orc.find_primes(n, 64, b):
            if v not in q:
                q.append(v)
                break
    src_q, tgt_q = q[:s], q[s:]
    ctx = nb.Context(n, q, [orc.find_psi(v, n) for v in q])
    x = orc.lcg(n, src_q, 300 + s + t)
    out = nb.empty((t, n))
    ctx.switch_basis(out, nb.to_device(x), list(range(s)), list(range(s, s + t)))
    np.testing.assert_array_equal(nb.to_host(out), orc.basis_convert(x, src_q, tgt_q))
    assert ctx.device_errors() == 0
    ctx.close()


@pytest.mark.parametrize("n,m,k,dnum", [(8192, 9, 3, 3), (65536, 24, 8, 3), (4096, 16, 16, 2)])
def test_keyswitch_with_tensor_core_conversions(tc_on, orc, n, m, k, dnum):
    """Digits (lazy outputs into the forward NTT) and ModDown conversions."""
    ctx = synthetic_context(orc, n, m, k, dnum)
    g = nb.Context.from_oracle(ctx)
    kb, ka = full_keys(orc, ctx, 7)
    level = m
    x, c0 = orc.lcg(n, ctx.q[:level], 11), orc.lcg(n, ctx.q[:level], 12)
    ob, oa = nb.empty((level, n)), nb.empty((level, n))
    g.keyswitch(level, ob, oa, nb.to_device(x), nb.to_device(kb), nb.to_device(ka), g.workspace(nb.OP_KEYSWITCH, level),
                c0=nb.to_device(c0), automorphism=5)
    wb, wa = orc.keyswitch(ctx, level, x, kb, ka, c0, 5)
    np.testing.assert_array_equal(nb.to_host(ob), wb)
    np.testing.assert_array_equal(nb.to_host(oa), wa)
    assert g.device_errors() == 0
    g.close()


def test_conversion_run_lengths_give_identical_key_switches(tc_on, orc):
    """One tensor-core launch converts all three Hybrid digits of 5 requests
    (3 x 5 x 512 tiles of 128 coefficients). CTAs take runs of 4, 3 or 7
    tiles; runs of 3 and 7 leave a short last run in every polynomial. Every
    run length gives the same key switches, equal to the oracle."""
    n, level, batch = 65536, 24, 5
    ctx = synthetic_context(orc, n, level, 8, 3)
    g = nb.Context.from_oracle(ctx)
    kb, ka = full_keys(orc, ctx, 19)
    dkb, dka = nb.to_device(kb), nb.to_device(ka)
    xs = np.stack([orc.lcg(n, ctx.q[:level], 40 + i) for i in range(batch)])
    dx = nb.to_device(xs)
    before = nb.tuning_get("conv_tc_tiles")
    got = {}
    try:
        for tiles in (4, 3, 7):
            nb.tuning_set("conv_tc_tiles", tiles)
            ob, oa = nb.empty((batch, level, n)), nb.empty((batch, level, n))
            g.keyswitch_batch(level, batch, ob, oa, dx, dkb, dka, g.workspace(nb.OP_KEYSWITCH, level, batch))
            got[tiles] = (nb.to_host(ob), nb.to_host(oa))
    finally:
        nb.tuning_set("conv_tc_tiles", before)
    assert g.device_errors() == 0
    for tiles in (3, 7):
        np.testing.assert_array_equal(got[tiles][0], got[4][0], err_msg=f"tiles={tiles}")
        np.testing.assert_array_equal(got[tiles][1], got[4][1], err_msg=f"tiles={tiles}")
    for i in (0, batch - 1):
        wb, wa = orc.keyswitch(ctx, level, xs[i], kb, ka)
        np.testing.assert_array_equal(got[4][0][i], wb)
        np.testing.assert_array_equal(got[4][1][i], wa)
    g.close()
