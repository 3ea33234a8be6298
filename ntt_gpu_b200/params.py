"""Host-side CKKS parameter search and seeded synthetic inputs.

Prime search and root selection restate the reference's parameter generator
(include/ntt/param_gen.hpp:29-95 in minnow54426/ntt-gpu): Miller-Rabin with
bases 2..37; find_primes walks up from the first multiple of 2N above
2^(bits-1) (+1) in steps of 2N; find_psi takes a xorshift candidate walk and
accepts zeta = g^((q-1)/2N) when zeta^N == q-1. Synthetic residues come from a
counter-based SplitMix64 (the mix() of tests/openfhe_hybrid_tests.cpp:153-158)
so that large batches are generated vectorised.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

_BASES = (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37)
_M64 = (1 << 64) - 1


def is_prime(n: int) -> bool:
    if n < 2:
        return False
    for p in _BASES:
        if n % p == 0:
            return n == p
    d, s = n - 1, 0
    while d % 2 == 0:
        d, s = d // 2, s + 1
    for a in _BASES:
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


def find_primes(n: int, count: int, bits: int) -> list[int]:
    step = 2 * n
    q = ((1 << (bits - 1)) // step + 1) * step + 1
    out = []
    while len(out) < count:
        if q >= 1 << bits:
            raise ValueError("prime search exhausted the bit range")
        if is_prime(q):
            out.append(q)
        q += step
    return out


def find_psi(q: int, n: int) -> int:
    s = (q ^ n) or 1
    while True:
        s ^= (s << 13) & _M64
        s ^= s >> 7
        s ^= (s << 17) & _M64
        g = 2 + s % (q - 3)
        zeta = pow(g, (q - 1) // (2 * n), q)
        if pow(zeta, n, q) == q - 1:
            return zeta


def min_psi(q: int, n: int) -> int:
    """The smallest primitive 2N-th root of unity mod q: the minimum over the N
    odd powers of any one primitive root (OpenFHE's root convention, which the
    reference pins in tests/openfhe_representation_tests.cpp:56-62)."""
    psi = find_psi(q, n)
    sq, power, best = psi * psi % q, psi, psi
    for _ in range(n - 1):
        power = power * sq % q
        if power < best:
            best = power
    return best


@dataclass
class CkksParams:
    """N, M Q towers, K P towers, digit width alpha = ceil(M / dnum)."""
    n: int
    q: list
    q_psi: list
    p: list
    p_psi: list
    alpha: int
    dnum: int = 0
    tags: dict = field(default_factory=dict)

    @property
    def m(self) -> int:
        return len(self.q)

    @property
    def k(self) -> int:
        return len(self.p)

    def digits(self, level: int) -> int:
        return 1 + (level - 1) // self.alpha

    def full_digits(self) -> int:
        return 1 + (self.m - 1) // self.alpha

    def moduli(self, level: int | None = None) -> list:
        return list(self.q[: (self.m if level is None else level)])

    def qp_moduli(self, level: int) -> list:
        return list(self.q[:level]) + list(self.p)


def synthetic_params(n: int, m: int, k: int, dnum: int, q_bits: int = 55, p_bits: int = 60) -> CkksParams:
    """Q: m primes of q_bits, P: k primes of p_bits (ascending find_primes), alpha = ceil(m/dnum)."""
    q = find_primes(n, m, q_bits)
    p = find_primes(n, k, p_bits)
    return CkksParams(n, q, [find_psi(v, n) for v in q], p, [find_psi(v, n) for v in p], -(-m // dnum), dnum)


def splitmix(x: np.ndarray) -> np.ndarray:
    x = x + np.uint64(0x9E3779B97F4A7C15)
    x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return x ^ (x >> np.uint64(31))


def uniform_residues(n: int, moduli, seed: int, polys: int = 1) -> np.ndarray:
    """[polys][towers][n] residues, tower t uniform in [0, moduli[t]) from SplitMix64(seed + index)."""
    towers = len(moduli)
    with np.errstate(over="ignore"):
        idx = np.arange(polys * towers * n, dtype=np.uint64) + np.uint64(seed)
        v = splitmix(idx).reshape(polys, towers, n)
    return v % np.asarray(moduli, dtype=np.uint64)[None, :, None]
