"""Generate the golden fixtures in tests/golden/ from the reference itself.

Run in a container that has the reference tree (minnow54426/ntt-gpu) at
REF (argument, else $NTT_REFERENCE_TREE, else ../reference beside this
repository) and oracle/_ref built (make -C oracle ref):

    python tests/golden/make_golden.py [REF]            # every fixture
    python tests/golden/make_golden.py --config5 [REF]  # only the config-5 digests, merged

Two sources, neither of them this repository's oracle:
  * ntt_n1024.npz, ntt_n64.npz - the reference's Python big-integer oracle
    (tests/oracle/ntt_oracle.py: find_primes, find_psi, negacyclic_ntt_naive)
    imported from the reference tree: naive O(N^2) evaluation, bit-reversed.
  * chain_small.npz, digests.json - the reference's own C++ CPU implementation
    (NegacyclicNtt, ApproximateBasisPlan, Session + HostDriver), compiled from
    its sources into oracle/_ref/libntt_ref.so. Small cases keep full arrays;
    N = 65536 cases keep SHA-256 digests of the little-endian u64 outputs.

Inputs are regenerated from seeds by the tests (LCG of
include/ntt/benchmark_inputs.hpp, SplitMix64 of tests/openfhe_hybrid_tests.cpp),
so only outputs are stored.
"""
from __future__ import annotations

import hashlib
import importlib.util
import json
import os
import random
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.oracle import (LCG_SEED, Oracle, Reference, pinned_context,  # noqa: E402
                           synthetic_context)


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<u8").tobytes()).hexdigest()


def full_keys(orc, ctx, seed):
    mods = ctx.q + ctx.p
    kb = np.stack([orc.splitmix(ctx.n, mods, seed + 1000 * d) for d in range(ctx.full_digits())])
    ka = np.stack([orc.splitmix(ctx.n, mods, seed + 7 + 1000 * d) for d in range(ctx.full_digits())])
    return kb, ka


def naive_fixture(ref_root, n, num_primes, bits, seed):
    spec = importlib.util.spec_from_file_location(
        "ref_ntt_oracle", os.path.join(ref_root, "tests", "oracle", "ntt_oracle.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    primes = mod.find_primes(n, num_primes, bits)
    psis = [mod.find_psi(q, n) for q in primes]
    rng = random.Random(seed)
    q_total = 1
    for q in primes:
        q_total *= q
    coeffs = [rng.randrange(q_total) for _ in range(n)]  # as gen_vectors.py does
    lg = n.bit_length() - 1
    outs = []
    for q, psi in zip(primes, psis):
        want = mod.negacyclic_ntt_naive([c % q for c in coeffs], q, psi)
        outs.append([want[int(format(j, f"0{lg}b")[::-1], 2)] for j in range(n)])
    residues = np.array([[c % q for c in coeffs] for q in primes], dtype=np.uint64)
    return dict(q=np.array(primes, dtype=np.uint64), psi=np.array(psis, dtype=np.uint64),
                input=residues, forward=np.array(outs, dtype=np.uint64))


def chain_cases(orc, ref):
    """Small full-array chain fixtures from the compiled reference."""
    out = {}
    for tag, (n, m, k, dnum) in {"a": (64, 5, 3, 2), "b": (32, 4, 2, 3)}.items():
        ctx = synthetic_context(orc, n, m, k, dnum)
        kb, ka = full_keys(orc, ctx, 5)
        for level in range(1, m + 1):
            x = orc.lcg(n, ctx.q[:level], LCG_SEED + level)
            y = orc.lcg(n, ctx.qp_moduli(level), 77 + level)
            c0 = orc.lcg(n, ctx.q[:level], 9 + level)
            out[f"{tag}_L{level}_modup_coeff"] = ref.mod_up(ctx, level, x, 0)
            out[f"{tag}_L{level}_modup_eval"] = ref.mod_up(ctx, level, x, 1)
            out[f"{tag}_L{level}_moddown"] = ref.mod_down(ctx, level, y)
            out[f"{tag}_L{level}_digits"] = ref.hybrid_digits(ctx, level, x)
            b, a = ref.keyswitch(ctx, level, x, kb, ka)
            out[f"{tag}_L{level}_ks_b"], out[f"{tag}_L{level}_ks_a"] = b, a
            b, a = ref.keyswitch(ctx, level, x, kb, ka, c0, 5)
            out[f"{tag}_L{level}_rot5_b"], out[f"{tag}_L{level}_rot5_a"] = b, a
    return out


def full_size_digests(orc, ref):
    d = {}
    # Config 1: one 60-bit find_primes tower and the pinned OpenFHE q0.
    n = 65536
    q60 = orc.find_primes(n, 1, 60)[0]
    for name, q, psi in [("find_primes60", q60, orc.find_psi(q60, n)),
                         ("openfhe_q0", 1152921504606584833, 18043022392882)]:
        x = orc.lcg(n, [q], LCG_SEED)
        d[f"ntt_{name}_forward"] = sha(ref.ntt(x, [q], [psi]))
        d[f"ntt_{name}_inverse"] = sha(ref.ntt(x, [q], [psi], inverse=True))
    ctx = pinned_context()
    kb, ka = full_keys(orc, ctx, 21)
    for level in (5, 4, 1):
        x = orc.lcg(ctx.n, ctx.q[:level], LCG_SEED)
        c0 = orc.lcg(ctx.n, ctx.q[:level], LCG_SEED + 1)
        b, a = ref.keyswitch(ctx, level, x, kb, ka, c0, 5)
        d[f"pinned_L{level}_rot5_b"], d[f"pinned_L{level}_rot5_a"] = sha(b), sha(a)
        b, a = ref.keyswitch(ctx, level, x, kb, ka)
        d[f"pinned_L{level}_ks_b"], d[f"pinned_L{level}_ks_a"] = sha(b), sha(a)
    ctx = synthetic_context(orc, 65536, 24, 8, 3)
    kb, ka = full_keys(orc, ctx, 99)
    for level in (24, 16, 8):
        x = orc.lcg(ctx.n, ctx.q[:level], LCG_SEED)
        b, a = ref.keyswitch(ctx, level, x, kb, ka)
        d[f"bench_L{level}_ks_b"], d[f"bench_L{level}_ks_a"] = sha(b), sha(a)
    x = orc.lcg(ctx.n, ctx.q, LCG_SEED)
    c0 = orc.lcg(ctx.n, ctx.q, LCG_SEED + 1)
    b, a = ref.keyswitch(ctx, 24, x, kb, ka, c0, 5)
    d["bench_L24_rot5_b"], d["bench_L24_rot5_a"] = sha(b), sha(a)
    return d


def config5_digests(orc, ref):
    """Config 5's largest shapes (N = 65536, L = 32, dnum 2/3/4, K = alpha):
    key switch, rotations by +-1 and +-64 steps, and a short-last-digit level,
    from the compiled reference's Session + HostDriver chain."""
    sys.path.insert(0, os.path.dirname(HERE))
    import golden_cases as gc
    d = {}
    for dnum in gc.CONFIG5_DNUM:
        ctx = gc.config5_context(orc, dnum)
        kb, ka = full_keys(orc, ctx, 300 + dnum)
        for name, level, x, c0, g in gc.config5_cases(orc, dnum):
            b, a = ref.keyswitch(ctx, level, x, kb, ka, c0, g)
            d[name + "_b"], d[name + "_a"] = sha(b), sha(a)
            print(name, flush=True)
    return d


def reference_root(argv):
    if argv:
        return argv[0]
    return os.environ.get("NTT_REFERENCE_TREE", os.path.join(ROOT, "..", "reference"))


def main():
    args = sys.argv[1:]
    only5 = "--config5" in args
    args = [a for a in args if a != "--config5"]
    ref_root = reference_root(args)
    orc, ref = Oracle(), Reference()
    path = os.path.join(HERE, "digests.json")
    if only5:
        with open(path) as f:
            d = json.load(f)
        d.update(config5_digests(orc, ref))
        with open(path, "w") as f:
            json.dump(d, f, indent=1, sort_keys=True)
        print("config-5 digests merged into", path)
        return
    np.savez_compressed(os.path.join(HERE, "ntt_n1024.npz"), **naive_fixture(ref_root, 1024, 3, 46, 1))
    np.savez_compressed(os.path.join(HERE, "ntt_n64.npz"), **naive_fixture(ref_root, 64, 3, 46, 1))
    np.savez_compressed(os.path.join(HERE, "chain_small.npz"), **chain_cases(orc, ref))
    d = full_size_digests(orc, ref)
    d.update(config5_digests(orc, ref))
    with open(path, "w") as f:
        json.dump(d, f, indent=1, sort_keys=True)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
