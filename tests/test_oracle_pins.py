"""Pin the CPU oracle against independent Python big-integer arithmetic.

These are restatements of the reference's own gates, in this repository's code:
  * modular arithmetic vs Python ints - tests/oracle/test_arithmetic.py:14-90
    (edge operands, random operands, Shoup, Barrett estimate error in {0, 1}
    and middle carries in {0, 1, 2}, inverses with invalid zero/q);
  * the naive O(N^2) negacyclic DFT - tests/oracle/ntt_oracle.py:64-77;
  * closed-form monomials and inverse basis vectors with the pinned OpenFHE
    roots - tests/openfhe_representation_tests.cpp:56-109;
  * the negacyclic wrap x^(N-1) * x = -1 - tests/arithmetic_contract_tests.cpp:63-71;
  * the schoolbook product mod x^N + 1 - tests/unit_tests.cpp:62-74;
  * the unbounded CRT lift for basis conversion, including 63-bit primes,
    1..40 sources and invalid inputs - tests/oracle/test_basis_conversion.py:14-64.
No GPU is used.
"""
import math
import random

import numpy as np
import pytest

from oracle.oracle import (PINNED_N, PINNED_P, PINNED_P_PSI, PINNED_Q, PINNED_Q_PSI,
                           pinned_context, synthetic_context)

MASK = (1 << 64) - 1


def bitrev(x, lg):
    return int(format(x, f"0{lg}b")[::-1], 2) if lg else 0


def test_arithmetic_against_bigint(orc):
    rng = random.Random(0xD6)
    moduli = [1, 2, 17, 1000000007]
    for bits in [30, 32, 50, 55, 60, 63, 64]:
        moduli += [(1 << bits) - 1, (1 << bits) - 25]
    moduli += [rng.randrange(2, 1 << 63) for _ in range(24)]
    corrections, carries, checks = set(), set(), 0
    for q in moduli:
        edges = sorted({v % q for v in [0, 1, 2, q // 2, q - 2, q - 1, (1 << 32) - 1, 1 << 32, (1 << 32) + 1]})
        pairs = [(a, b) for a in edges for b in edges] + [(rng.randrange(q), rng.randrange(q)) for _ in range(256)]
        for a, b in pairs:
            if q < 1 << 63:
                assert orc.add(a, b, q) == (a + b) % q
                assert orc.sub(a, b, q) == (a - b) % q
            assert orc.mul(a, b, q) == a * b % q
            if 1 < q < 1 << 63:
                assert orc.shoup(a, b, q) == a * b % q
                assert orc.barrett(a, b, q) == a * b % q
                recip = (1 << 128) // q
                est = orc.barrett_estimate(a, b, q)
                corrections.add(a * b // q - est)
                lo, hi = (a * b) & MASK, (a * b) >> 64
                carries.add(((lo * (recip & MASK) >> 64) + ((lo * (recip >> 64)) & MASK)
                             + ((hi * (recip & MASK)) & MASK)) >> 64)
            checks += 1
        for a in edges + [MASK]:
            for e in [0, 1, 2, 63, 64, MASK]:
                assert orc.pow(a, e, q) == pow(a, e, q)
    assert corrections == {0, 1}, corrections
    assert carries == {0, 1, 2}, carries
    for q in [2, 17, 1000000007] + [orc.find_primes(65536, 1, b)[0] for b in (50, 55, 60)]:
        for x in [1, q - 1, q + 1, MASK]:
            if x % q:
                assert orc.inv(x, q) == pow(x, -1, q)
        assert orc.inv(0, q) is None and orc.inv(q, q) is None
    assert checks > 5000


def test_barrett_small_moduli_exhaustive(orc):
    for q in range(2, 33):
        recip = (1 << 128) // q
        for a in range(q):
            for b in range(q):
                assert orc.barrett(a, b, q) == a * b % q
                assert orc.barrett_estimate(a, b, q) == (a * b * recip) >> 128


def test_parameter_search_matches_reference_walk(orc):
    # find_primes walks up from the first 2n-multiple + 1 above 2^(bits-1).
    for n, bits in [(8, 20), (1024, 46), (65536, 50), (65536, 60)]:
        got = orc.find_primes(n, 5, bits)
        q = ((1 << (bits - 1)) // (2 * n) + 1) * 2 * n + 1
        want = []
        while len(want) < 5:
            if is_prime(q):
                want.append(q)
            q += 2 * n
        assert got == want
        for q in got:
            psi = orc.find_psi(q, n)
            assert pow(psi, n, q) == q - 1


def is_prime(n):
    if n < 2:
        return False
    for p in (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37):
        if n % p == 0:
            return n == p
    d, s = n - 1, 0
    while d % 2 == 0:
        d, s = d // 2, s + 1
    for a in (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37):
        x = pow(a, d, n)
        if x in (1, n - 1):
            continue
        for _ in range(s - 1):
            x = x * x % n
            if x == n - 1:
                break
        else:
            return False
    return True


def naive_negacyclic(a, q, psi):
    n = len(a)
    lg = n.bit_length() - 1
    table = [pow(psi, k, q) for k in range(2 * n)]
    evals = [sum(a[i] * table[((2 * j + 1) * i) % (2 * n)] for i in range(n)) % q for j in range(n)]
    return [evals[bitrev(k, lg)] for k in range(n)]


@pytest.mark.parametrize("n", [2, 4, 8, 64, 256])
def test_ntt_matches_naive_dft(orc, n):
    primes = orc.find_primes(n, 3, 46)
    psis = [orc.find_psi(q, n) for q in primes]
    rng = random.Random(n)
    x = np.array([[rng.randrange(q) for _ in range(n)] for q in primes], dtype=np.uint64)
    got = orc.ntt(x, primes, psis)
    for t, (q, psi) in enumerate(zip(primes, psis)):
        assert [int(v) for v in got[t]] == naive_negacyclic([int(v) for v in x[t]], q, psi)
    assert np.array_equal(orc.ntt(got, primes, psis, inverse=True), x)


def test_pinned_openfhe_roots_are_minimum_primitive_roots():
    for q, psi in zip(PINNED_Q + PINNED_P, PINNED_Q_PSI + PINNED_P_PSI):
        assert pow(psi, PINNED_N, q) == q - 1
        sq = psi * psi % q
        power, minimum = psi, psi
        for _ in range(PINNED_N):
            minimum = min(minimum, power)
            power = power * sq % q
        assert minimum == psi


def test_closed_form_monomials_and_inverse_basis(orc):
    n, q, psi = PINNED_N, PINNED_Q[0], PINNED_Q_PSI[0]
    lg = 16
    points = [pow(psi, 2 * bitrev(k, lg) + 1, q) for k in range(n)]
    assert points[0] == psi and points[1] == q - psi
    for deg in (0, 1, 17, n - 1):
        x = np.zeros((1, n), dtype=np.uint64)
        x[0, deg] = 1
        got = orc.ntt(x, [q], [psi])[0]
        assert [int(v) for v in got] == [pow(p, deg, q) for p in points]
    ninv = pow(n, -1, q)
    for slot in (0, 1, n // 2, n - 1):
        x = np.zeros((1, n), dtype=np.uint64)
        x[0, slot] = 1
        got = orc.ntt(x, [q], [psi], inverse=True)[0]
        step = pow(points[slot], -1, q)
        assert [int(v) for v in got[:64]] == [ninv * pow(step, i, q) % q for i in range(64)]
        assert int(got[n - 1]) == ninv * pow(step, n - 1, q) % q


def test_negacyclic_wrap_and_schoolbook_product(orc):
    # x^(N-1) * x = -1 at N = 65536 with a 60-bit prime.
    n = 65536
    q = orc.find_primes(n, 1, 60)[0]
    psi = orc.find_psi(q, n)
    a = np.zeros((1, n), dtype=np.uint64)
    b = np.zeros((1, n), dtype=np.uint64)
    a[0, n - 1] = 1
    b[0, 1] = 1
    fa, fb = orc.ntt(a, [q], [psi]), orc.ntt(b, [q], [psi])
    prod = np.array([[orc.mul(int(u), int(v), q) for u, v in zip(fa[0], fb[0])]], dtype=np.uint64)
    c = orc.ntt(prod, [q], [psi], inverse=True)
    assert int(c[0, 0]) == q - 1 and not c[0, 1:].any()
    # schoolbook product mod x^N + 1 at N = 64
    n = 64
    q = orc.find_primes(n, 1, 50)[0]
    psi = orc.find_psi(q, n)
    rng = random.Random(7)
    x = [rng.randrange(q) for _ in range(n)]
    y = [rng.randrange(q) for _ in range(n)]
    want = [0] * n
    for i in range(n):
        for j in range(n):
            if i + j < n:
                want[i + j] = (want[i + j] + x[i] * y[j]) % q
            else:
                want[i + j - n] = (want[i + j - n] - x[i] * y[j]) % q
    fx = orc.ntt(np.array([x], dtype=np.uint64), [q], [psi])[0]
    fy = orc.ntt(np.array([y], dtype=np.uint64), [q], [psi])[0]
    fp = np.array([[int(u) * int(v) % q for u, v in zip(fx, fy)]], dtype=np.uint64)
    assert [int(v) for v in orc.ntt(fp, [q], [psi], inverse=True)[0]] == want


def bigint_lift(values, source, target):
    """Unreduced approximate CRT: sum_i [x_i * Bhat_i^-1]_{b_i} * Bhat_i, reduced mod each target."""
    product = math.prod(source)
    hats = [product // b for b in source]
    inverses = [pow(h, -1, b) for h, b in zip(hats, source)]
    n = values.shape[1]
    lifted = [sum(h * (int(values[t, i]) * inv % b) for t, (h, inv, b) in enumerate(zip(hats, inverses, source)))
              for i in range(n)]
    return lifted, np.array([[v % m for v in lifted] for m in target], dtype=np.uint64)


def test_basis_conversion_against_unbounded_crt(orc):
    rng = random.Random(0xB09)
    witnesses, cases = 0, 0
    for bits in (30, 50, 55, 60, 63):
        primes = orc.find_primes(65536, 43, bits)
        for count in (1, 2, 3, 8, 16, 24, 40):
            source, target = primes[:count], primes[-3:]
            for reverse in (False, True):
                if reverse:
                    source, target = target, source
                for pattern in range(4):
                    vals = np.array([[0 if pattern == 0 else b - 1 if pattern == 1 else int(i == 7)
                                      if pattern == 2 else rng.randrange(b) for i in range(8)] for b in source],
                                    dtype=np.uint64)
                    lifted, want = bigint_lift(vals, source, target)
                    assert np.array_equal(orc.basis_convert(vals, source, target), want)
                    prod = math.prod(source)
                    witnesses += sum(v % target[0] != (v % prod) % target[0] for v in lifted)
                    cases += 1
    assert witnesses > 0 and cases == 5 * 7 * 2 * 4
    vals = np.array([[16] * 8, [96] * 8], dtype=np.uint64)
    assert np.array_equal(orc.basis_convert(vals, [17, 97], [5, 113]), bigint_lift(vals, [17, 97], [5, 113])[1])


@pytest.mark.parametrize("source,target,shape", [
    ([17, 17], [97], (2, 8)), ([17], [17], (1, 8)), ([15], [97], (1, 8)), ([17], [97], (1, 3)),
    ([0], [97], (1, 8)), ([1], [97], (1, 8)), ([2], [97], (1, 8))])
def test_basis_conversion_rejects_invalid(orc, source, target, shape):
    with pytest.raises(ValueError):
        orc.basis_convert(np.zeros(shape, dtype=np.uint64), source, target)


def test_basis_conversion_rejects_noncanonical_and_oversize(orc):
    with pytest.raises(ValueError):
        orc.basis_convert(np.full((1, 8), 17, dtype=np.uint64), [17], [97])
    primes = orc.find_primes(65536, 42, 30)
    with pytest.raises(ValueError):
        orc.basis_convert(np.zeros((41, 8), dtype=np.uint64), primes[:41], [primes[-1]])
    with pytest.raises(ValueError):
        orc.basis_convert(np.zeros((1, 8), dtype=np.uint64), [primes[-1]], primes[:41])


def test_hybrid_chain_composes_pinned_primitives(orc):
    """ModUp/ModDown/digits/MAC equal their definitions built from the pinned
    NTT and the big-int lift, and the reference's negative witnesses hold:
    canonical-CRT substitution, the missing reduced-level P key offset and
    ModDown inside the digit sum all change the result
    (tests/openfhe_hybrid_tests.cpp:132-134, 240-243, 766-791)."""
    ctx = synthetic_context(orc, 64, 5, 3, 2)
    n, L, K = ctx.n, 4, ctx.k
    qs, ps = ctx.q[:L], ctx.p
    x = orc.lcg(n, qs, 1234)
    coeff = orc.ntt(x, qs, ctx.q_psi[:L], inverse=True)
    # ModUp from evaluation: join(eval Q, NTT(lift(coeff Q -> P)))
    lifted, p_coeff = bigint_lift(coeff, qs, ps)
    up = orc.mod_up(ctx, L, x, 1)
    assert np.array_equal(up[:L], x)
    assert np.array_equal(up[L:], orc.ntt(p_coeff, ps, ctx.p_psi))
    prod = math.prod(qs)
    canon = np.array([[v % prod % m for v in lifted] for m in ps], dtype=np.uint64)
    assert not np.array_equal(canon, p_coeff)
    # ModDown: (Z_q - NTT(lift(INTT(Z_p)))) * P^-1
    z = orc.lcg(n, ctx.qp_moduli(L), 99)
    zp = orc.ntt(z[L:], ps, ctx.p_psi, inverse=True)
    corr = orc.ntt(bigint_lift(zp, ps, qs)[1], qs, ctx.q_psi[:L])
    P = math.prod(ps)
    want = np.array([[(int(z[t, i]) - int(corr[t, i])) * pow(P, -1, q) % q for i in range(n)]
                     for t, q in enumerate(qs)], dtype=np.uint64)
    assert np.array_equal(orc.mod_down(ctx, L, z), want)
    # digits: each digit keeps its own evaluations and lifts the rest
    digits = orc.hybrid_digits(ctx, L, x)
    qp = ctx.qp_moduli(L)
    qp_psi = ctx.q_psi[:L] + ctx.p_psi
    for d, first in enumerate(range(0, L, ctx.alpha)):
        own = list(range(first, min(first + ctx.alpha, L)))
        rest = [t for t in range(L + K) if t not in own]
        src = coeff[own[0]:own[-1] + 1]
        lifted_eval = orc.ntt(bigint_lift(src, [qs[t] for t in own], [qp[t] for t in rest])[1],
                              [qp[t] for t in rest], [qp_psi[t] for t in rest])
        assert np.array_equal(digits[d][own], x[own])
        assert np.array_equal(digits[d][rest], lifted_eval)
    # wrong P-key offset and ModDown-per-digit witnesses
    mods = ctx.q + ctx.p
    kb = np.stack([orc.splitmix(n, mods, 5 + 1000 * d) for d in range(ctx.full_digits())])
    ka = np.stack([orc.splitmix(n, mods, 12 + 1000 * d) for d in range(ctx.full_digits())])
    good_b, _ = orc.keyswitch(ctx, L, x, kb, ka)
    # pack keys without the M - L offset: P rows taken from rows L.. instead of M..
    wrong = kb.copy()
    for d in range(ctx.full_digits()):
        wrong[d, ctx.m:] = np.array([[int(v) % ps[j] for v in kb[d, L + j]] for j in range(K)], dtype=np.uint64)
    bad_b, _ = orc.keyswitch(ctx, L, x, wrong, ka)
    assert not np.array_equal(good_b, bad_b)
    per_digit = np.zeros((L, n), dtype=np.uint64)
    for d in range(ctx.digits(L)):
        rows = list(range(L)) + [ctx.m + j for j in range(K)]
        term = np.array([[int(digits[d][t, i]) * int(kb[d, rows[t], i]) % qp[t] for i in range(n)]
                         for t in range(L + K)], dtype=np.uint64)
        red = orc.mod_down(ctx, L, term)
        per_digit = np.array([[(int(per_digit[t, i]) + int(red[t, i])) % qs[t] for i in range(n)]
                              for t in range(L)], dtype=np.uint64)
    assert not np.array_equal(per_digit, good_b)


def test_context_rejects_invalid_parameters(orc):
    ctx = pinned_context()
    for bad in [dict(alpha=0), dict(alpha=6), dict(p=[]), dict(q_psi=[1] + PINNED_Q_PSI[1:]),
                dict(q=[PINNED_Q[0] + 2] + PINNED_Q[1:])]:
        kw = dict(n=ctx.n, q=ctx.q, q_psi=ctx.q_psi, p=ctx.p, p_psi=ctx.p_psi, alpha=ctx.alpha)
        kw.update(bad)
        if "p" in bad:
            kw["p_psi"] = []
        from oracle.oracle import Context
        c = Context(**kw)
        with pytest.raises(ValueError):
            orc.mod_down(c, 1, np.zeros((1 + len(c.p), c.n), dtype=np.uint64))
