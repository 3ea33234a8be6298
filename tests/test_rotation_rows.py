"""The fused kernel's rotation as whole-row gathers, checked on the host.

When the fused row pass + key multiplication also runs the ModDown's inverse
row pass on the P towers (`ntt_gpu_b200/csrc/rowmac.cuh`, the `inv_rows`
block), a rotation moves whole 256-word rows of the bit-reversed evaluation
layout. The warp holding source row `row` computes in closed form the
destination row rd whose 256 words all come from `row`, and for each word of rd
the source column. This file restates those two formulas in numpy, with the
kernel's 32-bit wrap-around, and checks them for every row and column against
the automorphism's slot map: output slot k takes input slot
automorphism_source_index(k) (include/ntt/resident_conversion.hpp:15-29, as
the oracle states it), over the ring sizes the fused kernel takes
(2^12 .. 2^16). The GPU tests cover a handful of automorphisms end to end;
this covers every odd g below 2N at N = 2^12 and 2^13 and several hundred at
the larger sizes.
"""
import numpy as np
import pytest

from tests.golden_cases import rotation_index

_U32 = np.uint64(0xFFFFFFFF)
# 16-bit reversal table; brev(x, b) = reversal of the low b bits of x.
_BREV16 = np.zeros(1 << 16, dtype=np.uint64)
for _b in range(16):
    _BREV16 |= ((np.arange(1 << 16, dtype=np.uint64) >> np.uint64(_b)) & np.uint64(1)) << np.uint64(15 - _b)


def _brev(x, bits):
    return _BREV16[np.asarray(x, dtype=np.uint64)] >> np.uint64(16 - bits)


def _source_index(k, logn, g):
    """Input slot of output slot k under X -> X^g, bit-reversed order."""
    two_n_mask = np.uint64((2 << logn) - 1)
    odd = np.uint64(2) * _brev(k, logn) + np.uint64(1)
    return _brev(((odd * np.uint64(g)) & two_n_mask) >> np.uint64(1), logn)


def _kernel_gather(logn, g):
    """(destination slot, source slot) pairs as the fused kernel forms them.

    Returns two arrays over (row, u, e): the destination slot rd * 256 + 16u + e
    the warp of source row `row` writes from lane u's register e, and the source
    slot row * 256 + cs it reads there.
    """
    r_bits = logn - 8
    n = 1 << logn
    gi = pow(g, -1, 1 << 32)
    row = np.arange(1 << r_bits, dtype=np.uint64)[:, None, None]
    u = np.arange(16, dtype=np.uint64)[None, :, None]
    e = np.arange(16, dtype=np.uint64)[None, None, :]
    rbr = _brev(row, r_bits)
    prod = ((np.uint64(2) * rbr + np.uint64(1)) * np.uint64(gi)) & _U32  # 32-bit product
    rd = _brev((prod >> np.uint64(1)) & np.uint64((1 << r_bits) - 1), r_bits)
    dbr = _brev(rd, r_bits)
    carry = (((np.uint64(2) * dbr + np.uint64(1)) * np.uint64(g)) & np.uint64(2 * n - 1)) >> np.uint64(logn - 7)
    base = (_brev(u, 4) * np.uint64(g) + carry) & _U32
    g16 = np.uint64(g & 15)
    cs = _brev((base + np.uint64(16) * ((_brev(e, 4) * g16) & np.uint64(15))) & np.uint64(255), 8)
    dest = rd * np.uint64(256) + np.uint64(16) * u + e
    src = row * np.uint64(256) + cs
    return rd[:, 0, 0], np.broadcast_to(dest, (1 << r_bits, 16, 16)), np.broadcast_to(src, (1 << r_bits, 16, 16))


def _automorphisms(logn, rng, count):
    two_n = 2 << logn
    n = 1 << logn
    edge = [1, 5, 25, two_n - 1] + [rotation_index(n, s) for s in (1, -1, 64, -64, n // 4 - 1)]
    rand = [int(x) | 1 for x in rng.integers(0, two_n, size=count)]
    return sorted(set(edge + rand))


def test_source_index_matches_the_oracle(orc):
    rng = np.random.default_rng(7)
    for logn in (12, 14, 16):
        n = 1 << logn
        for g in _automorphisms(logn, rng, 8):
            ks = rng.integers(0, n, size=64, dtype=np.uint64)
            mine = _source_index(ks, logn, g)
            for k, s in zip(ks, mine):
                assert int(s) == orc.automorphism_source_index(int(k), n, g)


@pytest.mark.parametrize("logn", [12, 13, 14, 15, 16])
def test_fused_row_gather_equals_the_slot_map(logn):
    two_n = 2 << logn
    rng = np.random.default_rng(logn)
    gs = range(1, two_n, 2) if logn <= 13 else _automorphisms(logn, rng, {14: 400, 15: 200, 16: 100}[logn])
    rows = 1 << (logn - 8)
    for g in gs:
        rd, dest, src = _kernel_gather(logn, g)
        # every destination row is written by exactly one source row
        assert np.array_equal(np.sort(rd), np.arange(rows, dtype=np.uint64)), g
        # and each of its words reads the slot the automorphism names
        assert np.array_equal(_source_index(dest, logn, g), src), g
