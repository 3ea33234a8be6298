"""Device modular arithmetic against host 128-bit arithmetic, as the reference
probes its own (tests/basis_cuda.cu:49-65: shoup_kernel, barrett_kernel):
Shoup's precomputed-quotient product (include/ntt/shoup.hpp:7-27), Barrett's
128-bit reciprocal product (include/ntt/barrett.hpp:10-50) and the NTT's
approximate-quotient product (mode-2 butterflies: congruent, in [0, 4q))."""
import numpy as np
import pytest

import ntt_gpu_b200 as nb

pytestmark = pytest.mark.gpu


def _moduli(orc):
    out = []
    for bits in (31, 40, 50, 55, 59, 60, 61, 62, 63):
        out += orc.find_primes(1024, 2, bits)
    out += [3, 5, 65537, (1 << 61) - 1, (1 << 63) - 25]  # small primes and edges of the range
    return out


def _operands(q, rng, count):
    edge = [0, 1, 2, q - 1, q - 2, q // 2, (q + 1) // 2]
    rand = [int(v) % q for v in rng.integers(0, 1 << 63, size=count, dtype=np.uint64)]
    return [v % q for v in edge] + rand


def test_shoup_and_barrett_equal_host_128_bit(lib, orc):
    rng = np.random.default_rng(5)
    shoup, barrett, want = [], [], []
    for q in _moduli(orc):
        xs, ws = _operands(q, rng, 200), _operands(q, rng, 200)
        for i, x in enumerate(xs):
            w = ws[(i * 7) % len(ws)]
            shoup.append((x, w, (w << 64) // q, q, 0))
            mu = (1 << 128) // q
            barrett.append((x, w, q, mu & ((1 << 64) - 1), mu >> 64))
            want.append(x * w % q)
    want = np.array(want, dtype=np.uint64)
    np.testing.assert_array_equal(nb.arith_probe(0, np.array(shoup, dtype=np.uint64)), want)
    np.testing.assert_array_equal(nb.arith_probe(1, np.array(barrett, dtype=np.uint64)), want)
    # the oracle's Barrett (the reference's estimate) agrees with the device on the same operands
    for (a, b, q, _, _), w in list(zip(barrett, want))[::97]:
        assert orc.barrett(a, b, q) == int(w)


def test_approximate_quotient_product_range(lib, orc):
    """x any 64-bit word (the butterflies' lazy inputs), q < 2^61: the result
    is congruent to x*w and lies in [0, 4q)."""
    rng = np.random.default_rng(9)
    queries = []
    for bits in (40, 50, 55, 60, 61):
        for q in orc.find_primes(1024, 2, bits):
            xs = [0, 1, (1 << 64) - 1, 8 * q - 1, 4 * q, q] + [int(v) for v in
                                                              rng.integers(0, 1 << 63, 300, dtype=np.uint64) * 2]
            for i, x in enumerate(xs):
                w = (int(rng.integers(0, 1 << 62)) % q) if i % 5 else q - 1
                queries.append((x % (1 << 64), w, (w << 64) // q, q, 0))
    got = nb.arith_probe(2, np.array(queries, dtype=np.uint64))
    for (x, w, _, q, _), r in zip(queries, got):
        r = int(r)
        assert r < 4 * q and r % q == x * w % q
