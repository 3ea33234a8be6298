"""Shared regeneration of the golden-fixture inputs (see tests/golden/make_golden.py)."""
import hashlib
import json
import os

import numpy as np

from oracle.oracle import LCG_SEED, pinned_context, synthetic_context

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
SMALL_CONTEXTS = {"a": (64, 5, 3, 2), "b": (32, 4, 2, 3)}


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<u8").tobytes()).hexdigest()


def digests() -> dict:
    with open(os.path.join(GOLDEN, "digests.json")) as f:
        return json.load(f)


def chain() -> dict:
    return dict(np.load(os.path.join(GOLDEN, "chain_small.npz")))


def naive(n) -> dict:
    return dict(np.load(os.path.join(GOLDEN, f"ntt_n{n}.npz")))


def full_keys(orc, ctx, seed):
    mods = ctx.q + ctx.p
    kb = np.stack([orc.splitmix(ctx.n, mods, seed + 1000 * d) for d in range(ctx.full_digits())])
    ka = np.stack([orc.splitmix(ctx.n, mods, seed + 7 + 1000 * d) for d in range(ctx.full_digits())])
    return kb, ka


def small_inputs(orc, tag, level):
    n, m, k, dnum = SMALL_CONTEXTS[tag]
    ctx = synthetic_context(orc, n, m, k, dnum)
    x = orc.lcg(n, ctx.q[:level], LCG_SEED + level)
    y = orc.lcg(n, ctx.qp_moduli(level), 77 + level)
    c0 = orc.lcg(n, ctx.q[:level], 9 + level)
    return ctx, x, y, c0


def full_size_cases(orc):
    """(name, ctx, level, x, keys, c0, automorphism) for the N = 65536 digests."""
    ctx = pinned_context()
    kb, ka = full_keys(orc, ctx, 21)
    for level in (5, 4, 1):
        x = orc.lcg(ctx.n, ctx.q[:level], LCG_SEED)
        c0 = orc.lcg(ctx.n, ctx.q[:level], LCG_SEED + 1)
        yield f"pinned_L{level}_rot5", ctx, level, x, (kb, ka), c0, 5
        yield f"pinned_L{level}_ks", ctx, level, x, (kb, ka), None, 0
    ctx = synthetic_context(orc, 65536, 24, 8, 3)
    kb, ka = full_keys(orc, ctx, 99)
    for level in (24, 16, 8):
        x = orc.lcg(ctx.n, ctx.q[:level], LCG_SEED)
        yield f"bench_L{level}_ks", ctx, level, x, (kb, ka), None, 0
    x = orc.lcg(ctx.n, ctx.q, LCG_SEED)
    c0 = orc.lcg(ctx.n, ctx.q, LCG_SEED + 1)
    yield "bench_L24_rot5", ctx, 24, x, (kb, ka), c0, 5


def ntt_cases(orc):
    n = 65536
    q60 = orc.find_primes(n, 1, 60)[0]
    for name, q, psi in [("find_primes60", q60, orc.find_psi(q60, n)),
                         ("openfhe_q0", 1152921504606584833, 18043022392882)]:
        yield name, q, psi, orc.lcg(n, [q], LCG_SEED)


# Config 5's largest shapes: N = 65536, L = 32 Q towers, dnum in {2, 3, 4} with
# K = alpha = ceil(32 / dnum) P towers (16 / 11 / 8), as the mixed serving
# workload builds its contexts. dnum = 2 runs 16-source conversions.
CONFIG5_DNUM = (2, 3, 4)
CONFIG5_STEPS = (1, -1, 64, -64)


def rotation_index(n: int, step: int) -> int:
    """Generator-5 rotation group: 5^s mod 2N for s >= 0, (5^-1)^|s| otherwise."""
    two_n = 2 * n
    g = pow(5, abs(step), two_n)
    return g if step >= 0 else pow(g, -1, two_n)


def config5_context(orc, dnum):
    alpha = -(-32 // dnum)
    return synthetic_context(orc, 65536, 32, alpha, dnum)


def config5_cases(orc, dnum):
    """(name, level, x, c0, automorphism) of one config-5 context; keys are
    full_keys(orc, ctx, 300 + dnum). Rotations share the input of the L = 32
    key switch (one hoisted decomposition), and L = 17 leaves the last digit
    short (17 = 16 + 1, 11 + 6, 8 + 8 + 1)."""
    ctx = config5_context(orc, dnum)
    x = orc.lcg(ctx.n, ctx.q, LCG_SEED + 50 + dnum)
    c0 = orc.lcg(ctx.n, ctx.q, LCG_SEED + 60 + dnum)
    yield f"c5_d{dnum}_L32_ks", 32, x, None, 0
    for step in CONFIG5_STEPS:
        tag = f"p{step}" if step > 0 else f"m{-step}"
        yield f"c5_d{dnum}_L32_rot{tag}", 32, x, c0, rotation_index(ctx.n, step)
    x17 = orc.lcg(ctx.n, ctx.q[:17], LCG_SEED + 70 + dnum)
    yield f"c5_d{dnum}_L17_ks", 17, x17, None, 0
