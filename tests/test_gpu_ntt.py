"""GPU parity: forward/inverse NTT through the C ABI against the CPU oracle."""
import numpy as np
import pytest

import ntt_gpu_b200 as nb
from oracle.oracle import LCG_SEED, PINNED_N, PINNED_P, PINNED_P_PSI, PINNED_Q, PINNED_Q_PSI

pytestmark = pytest.mark.gpu


def towers_for(orc, n, bits_list):
    q = []
    for bits in bits_list:
        for v in orc.find_primes(n, 8, bits):
            if v not in q:
                q.append(v)
                break
    return q, [orc.find_psi(v, n) for v in q]


@pytest.mark.parametrize("logn", [1, 2, 3, 6, 8, 10, 11, 12, 13, 14, 15, 16])
def test_ntt_roundtrip_matches_oracle(lib, orc, logn):
    n = 1 << logn
    bits = [30, 50, 55, 60] if n >= 64 else [20, 30]
    q, psi = towers_for(orc, n, bits)
    ctx = nb.Context(n, q, psi)
    x = orc.lcg(n, q, LCG_SEED + logn)
    want_fwd = orc.ntt(x, q, psi)
    want_inv = orc.ntt(x, q, psi, inverse=True)
    d = nb.to_device(x)
    out = nb.empty(x.shape)
    ids = list(range(len(q)))
    ctx.ntt(out, d, ids)
    np.testing.assert_array_equal(nb.to_host(out), want_fwd)
    np.testing.assert_array_equal(nb.to_host(d), x)  # out-of-place leaves the source intact
    back = nb.empty(x.shape)
    ctx.ntt(back, out, ids, inverse=True)
    np.testing.assert_array_equal(nb.to_host(back), x)
    ctx.ntt(out, d, ids, inverse=True)
    np.testing.assert_array_equal(nb.to_host(out), want_inv)


@pytest.mark.parametrize("logn", [10, 16])
def test_ntt_strict_path_for_wide_moduli(lib, orc, logn):
    """Moduli in [2^62, 2^63) disable lazy reduction; results stay exact."""
    n = 1 << logn
    q = orc.find_primes(n, 2, 63)
    psi = [orc.find_psi(v, n) for v in q]
    ctx = nb.Context(n, q, psi)
    x = orc.lcg(n, q, 11)
    out = nb.empty(x.shape)
    ctx.ntt(out, nb.to_device(x), [0, 1])
    np.testing.assert_array_equal(nb.to_host(out), orc.ntt(x, q, psi))
    back = nb.empty(x.shape)
    ctx.ntt(back, out, [0, 1], inverse=True)
    np.testing.assert_array_equal(nb.to_host(back), x)


def test_pinned_openfhe_towers_edge_patterns(lib, orc):
    """The pinned OpenFHE Q/P table at N=65536: zeros, q-1, monomials, random."""
    mods = PINNED_Q + PINNED_P
    psis = PINNED_Q_PSI + PINNED_P_PSI
    n = PINNED_N
    ctx = nb.Context(n, PINNED_Q, PINNED_Q_PSI, PINNED_P, PINNED_P_PSI, 3)
    patterns = [np.zeros((len(mods), n), dtype=np.uint64),
                np.array([[q - 1] * n for q in mods], dtype=np.uint64)]
    mono = np.zeros((len(mods), n), dtype=np.uint64)
    for t, deg in enumerate([0, 1, 17, n - 1, 5, 1000, 32768, 65535]):
        mono[t, deg] = 1
    patterns += [mono, orc.lcg(n, mods, LCG_SEED)]
    ids = list(range(len(mods)))
    for x in patterns:
        out = nb.empty(x.shape)
        ctx.ntt(out, nb.to_device(x), ids)
        np.testing.assert_array_equal(nb.to_host(out), orc.ntt(x, mods, psis))
        back = nb.empty(x.shape)
        ctx.ntt(back, out, ids, inverse=True)
        np.testing.assert_array_equal(nb.to_host(back), x)


def test_batched_polys_with_stride(lib, orc):
    n = 1 << 14
    q, psi = towers_for(orc, n, [50, 55, 60])
    ctx = nb.Context(n, q, psi)
    polys = 5
    stride = (len(q) + 1) * n
    buf = np.zeros((polys, len(q) + 1, n), dtype=np.uint64)
    for p in range(polys):
        buf[p, :len(q)] = orc.lcg(n, q, 100 + p)
    d = nb.to_device(buf)
    ctx.ntt(d, d, list(range(len(q))), polys=polys, poly_stride=stride)
    got = nb.to_host(d).reshape(buf.shape)
    for p in range(polys):
        np.testing.assert_array_equal(got[p, :len(q)], orc.ntt(buf[p, :len(q)], q, psi))
        np.testing.assert_array_equal(got[p, len(q)], 0)  # the gap tower is untouched


def primes_below(orc, n, count, bound):
    """The largest NTT-friendly primes (q = 1 mod 2n) below `bound`."""
    out, q = [], (bound - 1) // (2 * n) * (2 * n) + 1
    while len(out) < count:
        if q < bound and orc.is_prime(q):
            out.append(q)
        q -= 2 * n
    return out


@pytest.mark.parametrize("bits", [[61], [62], [61, 62], [59, 61], [-57], [58], [-57, 58], [30, 45, -57]])
@pytest.mark.parametrize("logn", [12, 14, 16])
def test_butterfly_mode_boundaries(lib, orc, bits, logn):
    """Moduli just below 2^61 (fast approximate-quotient butterflies, values up to
    8q), in [2^61, 2^62) (Harvey lazy butterflies), just below 2^57 (forward
    butterflies without per-stage reductions, values up to 68q; inverse
    butterflies without the sums' reduction, up to 64q within a register phase)
    and just above it, and mixed within one launch: exact results, with
    all-(q-1) inputs driving every stage to the top of its range. logN = 14
    leaves the inverse column pass a first register phase of two stages."""
    n = 1 << logn
    q = []
    for b in bits:  # b < 0: the primes just below 2^|b|
        found = primes_below(orc, n, 2, 1 << -b) if b < 0 else orc.find_primes(n, 2, b)
        q += [v for v in found if v not in q][:2]
    psi = [orc.find_psi(v, n) for v in q]
    ctx = nb.Context(n, q, psi)
    ids = list(range(len(q)))
    for x in (orc.lcg(n, q, 5 + logn), np.array([[v - 1] * n for v in q], dtype=np.uint64)):
        out = nb.empty(x.shape)
        ctx.ntt(out, nb.to_device(x), ids)
        np.testing.assert_array_equal(nb.to_host(out), orc.ntt(x, q, psi))
        back = nb.empty(x.shape)
        ctx.ntt(back, out, ids, inverse=True)
        np.testing.assert_array_equal(nb.to_host(back), x)
        ctx.ntt(out, nb.to_device(x), ids, inverse=True)
        np.testing.assert_array_equal(nb.to_host(out), orc.ntt(x, q, psi, inverse=True))


@pytest.mark.parametrize("inplace", [False, True])
def test_cluster_forward_transform(lib, orc, inplace):
    """The one-pass forward transform over an 8-CTA cluster (ntt_cluster, N = 2^16:
    column pass, rows gathered through distributed shared memory, row pass) on
    3 polynomials of 50-, 55- and 60-bit towers (reduction-free and per-stage
    reducing butterflies in one launch) and all-(q-1) inputs, in and out of
    place: equal to the oracle and to the two-pass transform. The host-array
    forward call takes the same path."""
    n, polys = 1 << 16, 3
    q, psi = towers_for(orc, n, [50, 55, 60, 50, 60])
    q += primes_below(orc, n, 1, 1 << 57)
    psi = [orc.find_psi(v, n) for v in q]
    ctx = nb.Context(n, q, psi)
    ids = list(range(len(q)))
    xs = [orc.lcg(n, q, 300 + p) for p in range(polys - 1)]
    xs.append(np.array([[v - 1] * n for v in q], dtype=np.uint64))
    x = np.stack(xs)
    stride = len(q) * n
    got = {}
    before = nb.tuning_get("ntt_cluster")
    try:
        for cluster in (1, 0):
            nb.tuning_set("ntt_cluster", cluster)
            d = nb.to_device(x)
            out = d if inplace else nb.empty(x.shape)
            ctx.ntt(out, d, ids, polys=polys, poly_stride=stride)
            got[cluster] = nb.to_host(out)
        nb.tuning_set("ntt_cluster", 1)
        ws = ctx.host_transform_workspace(nb.HOST_FORWARD)
        h = x[0].copy()
        ctx.host_transform(nb.HOST_FORWARD, h, ids, ws)
    finally:
        nb.tuning_set("ntt_cluster", before)
    for p in range(polys):
        np.testing.assert_array_equal(got[1][p], orc.ntt(x[p], q, psi), err_msg=f"poly {p}")
    np.testing.assert_array_equal(got[1], got[0])
    np.testing.assert_array_equal(h, got[0][0])
    ctx.close()
