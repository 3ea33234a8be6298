"""The C oracle equals the reference's own CPU implementation (oracle/_ref,
compiled from the reference sources) on seeded inputs; skipped when the
compiled reference is not present."""
import numpy as np
import pytest

from oracle.oracle import LCG_SEED, synthetic_context


@pytest.mark.parametrize("n,m,k,dnum", [(64, 5, 3, 2), (128, 7, 3, 2), (256, 6, 2, 3), (32, 3, 1, 1)])
def test_chain_equals_reference(orc, ref, n, m, k, dnum):
    ctx = synthetic_context(orc, n, m, k, dnum)
    mods = ctx.q + ctx.p
    kb = np.stack([orc.splitmix(n, mods, 100 + d) for d in range(ctx.full_digits())])
    ka = np.stack([orc.splitmix(n, mods, 200 + d) for d in range(ctx.full_digits())])
    for level in range(1, m + 1):
        x = orc.lcg(n, ctx.q[:level], 7 + level)
        for ev in (0, 1):
            np.testing.assert_array_equal(orc.mod_up(ctx, level, x, ev), ref.mod_up(ctx, level, x, ev))
        y = orc.lcg(n, ctx.qp_moduli(level), 9 + level)
        np.testing.assert_array_equal(orc.mod_down(ctx, level, y), ref.mod_down(ctx, level, y))
        np.testing.assert_array_equal(orc.hybrid_digits(ctx, level, x), ref.hybrid_digits(ctx, level, x))
        for c0, g in [(None, 0), (orc.lcg(n, ctx.q[:level], 11), 5), (orc.lcg(n, ctx.q[:level], 12), 2 * n - 1)]:
            A = orc.keyswitch(ctx, level, x, kb, ka, c0, g)
            B = ref.keyswitch(ctx, level, x, kb, ka, c0, g)
            np.testing.assert_array_equal(A[0], B[0])
            np.testing.assert_array_equal(A[1], B[1])


@pytest.mark.parametrize("bits", [30, 50, 60, 62, 63])
def test_ntt_and_conversion_equal_reference(orc, ref, bits):
    n = 1024
    q = orc.find_primes(n, 6, bits)
    psi = [orc.find_psi(v, n) for v in q]
    x = orc.lcg(n, q, LCG_SEED)
    np.testing.assert_array_equal(orc.ntt(x, q, psi), ref.ntt(x, q, psi))
    np.testing.assert_array_equal(orc.ntt(x, q, psi, True), ref.ntt(x, q, psi, True))
    np.testing.assert_array_equal(orc.basis_convert(x[:4], q[:4], q[4:]), ref.basis_convert(x[:4], q[:4], q[4:]))
