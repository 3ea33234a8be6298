"""The CPU oracle reproduces every golden fixture made from the reference itself
(its Python big-int oracle and its compiled C++ CPU path, tests/golden/make_golden.py)."""
import numpy as np
import pytest

import golden_cases as gc


@pytest.mark.parametrize("n", [64, 1024])
def test_naive_dft_fixtures(orc, n):
    f = gc.naive(n)
    q, psi = [int(v) for v in f["q"]], [int(v) for v in f["psi"]]
    np.testing.assert_array_equal(orc.ntt(f["input"], q, psi), f["forward"])
    np.testing.assert_array_equal(orc.ntt(f["forward"], q, psi, inverse=True), f["input"])


def test_chain_fixtures(orc):
    fx = gc.chain()
    checked = 0
    for tag, (n, m, k, dnum) in gc.SMALL_CONTEXTS.items():
        for level in range(1, m + 1):
            ctx, x, y, c0 = gc.small_inputs(orc, tag, level)
            kb, ka = gc.full_keys(orc, ctx, 5)
            p = f"{tag}_L{level}_"
            np.testing.assert_array_equal(orc.mod_up(ctx, level, x, 0), fx[p + "modup_coeff"])
            np.testing.assert_array_equal(orc.mod_up(ctx, level, x, 1), fx[p + "modup_eval"])
            np.testing.assert_array_equal(orc.mod_down(ctx, level, y), fx[p + "moddown"])
            np.testing.assert_array_equal(orc.hybrid_digits(ctx, level, x), fx[p + "digits"])
            b, a = orc.keyswitch(ctx, level, x, kb, ka)
            np.testing.assert_array_equal(b, fx[p + "ks_b"])
            np.testing.assert_array_equal(a, fx[p + "ks_a"])
            b, a = orc.keyswitch(ctx, level, x, kb, ka, c0, 5)
            np.testing.assert_array_equal(b, fx[p + "rot5_b"])
            np.testing.assert_array_equal(a, fx[p + "rot5_a"])
            checked += 8
    assert checked == 8 * 9


def test_full_size_ntt_digests(orc):
    d = gc.digests()
    for name, q, psi, x in gc.ntt_cases(orc):
        assert gc.sha(orc.ntt(x, [q], [psi])) == d[f"ntt_{name}_forward"]
        assert gc.sha(orc.ntt(x, [q], [psi], inverse=True)) == d[f"ntt_{name}_inverse"]


def test_full_size_keyswitch_digests_pinned(orc):
    d = gc.digests()
    for name, ctx, level, x, (kb, ka), c0, g in gc.full_size_cases(orc):
        if not name.startswith("pinned"):
            continue
        b, a = orc.keyswitch(ctx, level, x, kb, ka, c0, g)
        assert gc.sha(b) == d[name + "_b"] and gc.sha(a) == d[name + "_a"], name


def test_config5_sixteen_source_digest(orc):
    """The oracle reproduces the reference's key switch at config 5's widest
    conversion shape (N = 65536, L = 32, dnum = 2: K = alpha = 16)."""
    d = gc.digests()
    ctx = gc.config5_context(orc, 2)
    kb, ka = gc.full_keys(orc, ctx, 302)
    name, level, x, c0, g = next(iter(gc.config5_cases(orc, 2)))
    b, a = orc.keyswitch(ctx, level, x, kb, ka, c0, g)
    assert gc.sha(b) == d[name + "_b"] and gc.sha(a) == d[name + "_a"], name
