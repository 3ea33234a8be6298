"""GPU parity: basis switch, ModUp, ModDown, Hybrid digits, MAC, rotation and
the full key switch through the C ABI against the CPU oracle."""
import numpy as np
import pytest

import ntt_gpu_b200 as nb
from oracle.oracle import LCG_SEED, pinned_context, synthetic_context

pytestmark = pytest.mark.gpu


def full_keys(orc, ctx, seed):
    mods = ctx.q + ctx.p
    kb = np.stack([orc.splitmix(ctx.n, mods, seed + 1000 * d) for d in range(ctx.full_digits())])
    ka = np.stack([orc.splitmix(ctx.n, mods, seed + 7 + 1000 * d) for d in range(ctx.full_digits())])
    return kb, ka


CASES = [("small", 256, 6, 3, 2), ("mid", 4096, 7, 2, 3), ("n8k", 8192, 5, 3, 2)]


@pytest.mark.parametrize("name,n,m,k,dnum", CASES)
def test_switch_basis_and_mod_up_down(lib, orc, name, n, m, k, dnum):
    ctx = synthetic_context(orc, n, m, k, dnum)
    g = nb.Context.from_oracle(ctx)
    for level in range(1, m + 1):
        x = orc.lcg(n, ctx.q[:level], LCG_SEED + level)
        # coefficient-domain switch Q_L -> P
        out = nb.empty((k, n))
        g.switch_basis(out, nb.to_device(x), list(range(level)), [m + j for j in range(k)])
        np.testing.assert_array_equal(nb.to_host(out), orc.basis_convert(x, ctx.q[:level], ctx.p))
        ws = g.workspace(nb.OP_MOD_UP, level)
        for is_eval in (0, 1):
            up = nb.empty((level + k, n))
            g.mod_up(level, up, nb.to_device(x), is_eval, ws)
            np.testing.assert_array_equal(nb.to_host(up), orc.mod_up(ctx, level, x, is_eval))
        y = orc.lcg(n, ctx.qp_moduli(level), 77 + level)
        down = nb.empty((level, n))
        g.mod_down(level, down, nb.to_device(y), g.workspace(nb.OP_MOD_DOWN, level))
        np.testing.assert_array_equal(nb.to_host(down), orc.mod_down(ctx, level, y))


@pytest.mark.parametrize("name,n,m,k,dnum", CASES)
def test_digits_and_keyswitch(lib, orc, name, n, m, k, dnum):
    ctx = synthetic_context(orc, n, m, k, dnum)
    g = nb.Context.from_oracle(ctx)
    kb, ka = full_keys(orc, ctx, 5)
    dkb, dka = nb.to_device(kb), nb.to_device(ka)
    for level in range(1, m + 1):
        x = orc.lcg(n, ctx.q[:level], 3 + level)
        digits = nb.empty((ctx.digits(level), level + k, n))
        g.hybrid_digits(level, digits, nb.to_device(x), g.workspace(nb.OP_DIGITS, level))
        np.testing.assert_array_equal(nb.to_host(digits), orc.hybrid_digits(ctx, level, x))
        ob, oa = nb.empty((level, n)), nb.empty((level, n))
        ws = g.workspace(nb.OP_KEYSWITCH, level)
        g.keyswitch(level, ob, oa, nb.to_device(x), dkb, dka, ws)
        wb, wa = orc.keyswitch(ctx, level, x, kb, ka)
        np.testing.assert_array_equal(nb.to_host(ob), wb)
        np.testing.assert_array_equal(nb.to_host(oa), wa)
        c0 = orc.lcg(n, ctx.q[:level], 9 + level)
        for g_auto in (5, 2 * n - 1, 25):
            g.keyswitch(level, ob, oa, nb.to_device(x), dkb, dka, ws, c0=nb.to_device(c0), automorphism=g_auto)
            wb, wa = orc.keyswitch(ctx, level, x, kb, ka, c0, g_auto)
            np.testing.assert_array_equal(nb.to_host(ob), wb)
            np.testing.assert_array_equal(nb.to_host(oa), wa)


def test_pinned_context_keyswitch_full_size(lib, orc):
    ctx = pinned_context()
    g = nb.Context.from_oracle(ctx)
    kb, ka = full_keys(orc, ctx, 21)
    dkb, dka = nb.to_device(kb), nb.to_device(ka)
    for level in (5, 4, 1):
        x = orc.lcg(ctx.n, ctx.q[:level], LCG_SEED)
        c0 = orc.lcg(ctx.n, ctx.q[:level], LCG_SEED + 1)
        ob, oa = nb.empty((level, ctx.n)), nb.empty((level, ctx.n))
        ws = g.workspace(nb.OP_KEYSWITCH, level)
        g.keyswitch(level, ob, oa, nb.to_device(x), dkb, dka, ws, c0=nb.to_device(c0), automorphism=5)
        wb, wa = orc.keyswitch(ctx, level, x, kb, ka, c0, 5)
        np.testing.assert_array_equal(nb.to_host(ob), wb)
        np.testing.assert_array_equal(nb.to_host(oa), wa)


def test_bench_shape_keyswitch_full_size(lib, orc):
    """N=2^16, L=24, K=8, dnum=3 (alpha=8): the benchmark shape."""
    ctx = synthetic_context(orc, 65536, 24, 8, 3)
    g = nb.Context.from_oracle(ctx)
    kb, ka = full_keys(orc, ctx, 99)
    x = orc.lcg(ctx.n, ctx.q, LCG_SEED)
    ob, oa = nb.empty((24, ctx.n)), nb.empty((24, ctx.n))
    g.keyswitch(24, ob, oa, nb.to_device(x), nb.to_device(kb), nb.to_device(ka), g.workspace(nb.OP_KEYSWITCH, 24))
    wb, wa = orc.keyswitch(ctx, 24, x, kb, ka)
    np.testing.assert_array_equal(nb.to_host(ob), wb)
    np.testing.assert_array_equal(nb.to_host(oa), wa)


@pytest.mark.parametrize("rotate", [False, True])
def test_keyswitch_batch_equals_per_request(lib, orc, rotate):
    """One batched launch sequence equals the oracle on every request."""
    ctx = synthetic_context(orc, 8192, 6, 3, 2)
    g = nb.Context.from_oracle(ctx)
    kb, ka = full_keys(orc, ctx, 17)
    level, batch = 5, 5
    xs = np.stack([orc.lcg(ctx.n, ctx.q[:level], 40 + r) for r in range(batch)])
    c0 = np.stack([orc.lcg(ctx.n, ctx.q[:level], 80 + r) for r in range(batch)]) if rotate else None
    ob, oa = nb.empty(xs.shape), nb.empty(xs.shape)
    g.keyswitch_batch(level, batch, ob, oa, nb.to_device(xs), nb.to_device(kb), nb.to_device(ka),
                      g.workspace(nb.OP_KEYSWITCH, level, batch),
                      c0=None if c0 is None else nb.to_device(c0), automorphism=25 if rotate else 0)
    got_b, got_a = nb.to_host(ob), nb.to_host(oa)
    for r in range(batch):
        wb, wa = orc.keyswitch(ctx, level, xs[r], kb, ka, None if c0 is None else c0[r], 25 if rotate else 0)
        np.testing.assert_array_equal(got_b[r], wb)
        np.testing.assert_array_equal(got_a[r], wa)


def test_full_size_golden_digests(lib, orc):
    """N = 65536 outputs equal the digests of the reference's own CPU path."""
    import golden_cases as gc
    d = gc.digests()
    contexts = {}
    for name, ctx, level, x, (kb, ka), c0, auto in gc.full_size_cases(orc):
        key = (ctx.n, tuple(ctx.q), tuple(ctx.p))
        if key not in contexts:
            contexts[key] = (nb.Context.from_oracle(ctx), nb.to_device(kb), nb.to_device(ka))
        g, dkb, dka = contexts[key]
        ob, oa = nb.empty((level, ctx.n)), nb.empty((level, ctx.n))
        g.keyswitch(level, ob, oa, nb.to_device(x), dkb, dka, g.workspace(nb.OP_KEYSWITCH, level),
                    c0=None if c0 is None else nb.to_device(c0), automorphism=auto)
        assert gc.sha(nb.to_host(ob)) == d[name + "_b"], name
        assert gc.sha(nb.to_host(oa)) == d[name + "_a"], name
    for name, q, psi, x in gc.ntt_cases(orc):
        g = nb.Context(65536, [q], [psi])
        out = nb.empty(x.shape)
        g.ntt(out, nb.to_device(x), [0])
        assert gc.sha(nb.to_host(out)) == d[f"ntt_{name}_forward"]
        g.ntt(out, nb.to_device(x), [0], inverse=True)
        assert gc.sha(nb.to_host(out)) == d[f"ntt_{name}_inverse"]


@pytest.mark.parametrize("q_bits,p_bits", [(60, 61), (61, 62)])
def test_keyswitch_with_wide_towers(lib, orc, q_bits, p_bits):
    """Whole key switch (digits, MAC, rotation, ModDown) with towers just below
    2^61 (fast butterflies at the top of their range) and in [2^61, 2^62) (lazy)."""
    ctx = synthetic_context(orc, 8192, 6, 3, 2, q_bits=q_bits, p_bits=p_bits)
    g = nb.Context.from_oracle(ctx)
    kb, ka = full_keys(orc, ctx, 61)
    for level in (6, 3):
        x = orc.lcg(ctx.n, ctx.q[:level], 70 + level)
        c0 = orc.lcg(ctx.n, ctx.q[:level], 71 + level)
        ob, oa = nb.empty((level, ctx.n)), nb.empty((level, ctx.n))
        g.keyswitch(level, ob, oa, nb.to_device(x), nb.to_device(kb), nb.to_device(ka),
                    g.workspace(nb.OP_KEYSWITCH, level), c0=nb.to_device(c0), automorphism=25)
        wb, wa = orc.keyswitch(ctx, level, x, kb, ka, c0, 25)
        np.testing.assert_array_equal(nb.to_host(ob), wb)
        np.testing.assert_array_equal(nb.to_host(oa), wa)
