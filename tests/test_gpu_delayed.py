"""GPU parity: the Hybrid MAC primitives and delayed QP operations.

The reference's OpenFHE tests sum several key switches' extended QP results
before one ModDown (KeySwitchExt / KeySwitchDown / KeySwitchDownFirstElement,
openfhe_hybrid_tests.cpp:728-765; docs/openfhe-hybrid-operation-graph.md:395-401).
Here that composition runs on the C ABI's primitives: ntt_b200_hybrid_digits,
ntt_b200_hybrid_mac[_digits] with `accumulate`, and ntt_b200_mod_down. The MAC
is checked against Z = sum_d D_d * K_d[key row] (resident_conversion.hpp:50-54;
key rows i for Q towers and M + j for P towers, backend_contract.hpp:112-119),
computed here in exact integers, and the ModDown of the summed extension
against the CPU oracle."""
import numpy as np
import pytest

import ntt_gpu_b200 as nb
from oracle.oracle import synthetic_context
from test_gpu_requests import full_keys

pytestmark = pytest.mark.gpu

CASES = [(4096, 7, 2, 3), (8192, 5, 3, 2)]


def key_rows(ctx, level):
    return list(range(level)) + [ctx.m + j for j in range(ctx.k)]


def mac_expected(ctx, level, digits, kb, ka):
    """Exact sum_d digits[d] * key[d][row] mod each QP modulus."""
    mods = np.array(ctx.qp_moduli(level), dtype=object)[:, None]
    rows = key_rows(ctx, level)
    out = []
    for key in (kb, ka):
        acc = np.zeros((level + ctx.k, ctx.n), dtype=object)
        for d in range(digits.shape[0]):
            acc = (acc + digits[d].astype(object) * key[d][rows].astype(object)) % mods
        out.append(acc.astype(np.uint64))
    return out


def add_qp(ctx, level, x, y):
    mods = np.array(ctx.qp_moduli(level), dtype=object)[:, None]
    return ((x.astype(object) + y.astype(object)) % mods).astype(np.uint64)


@pytest.mark.parametrize("n,m,k,dnum", CASES)
def test_mac_primitives_equal_the_digit_sum(lib, orc, n, m, k, dnum):
    ctx = synthetic_context(orc, n, m, k, dnum)
    g = nb.Context.from_oracle(ctx)
    kb, ka = full_keys(orc, ctx, 21)
    dkb, dka = nb.to_device(kb), nb.to_device(ka)
    for level in (m, max(1, m - dnum)):
        beta = ctx.digits(level)
        x = orc.lcg(n, ctx.q[:level], 40 + level)
        digits = orc.hybrid_digits(ctx, level, x)
        ddig = nb.to_device(digits)
        wb, wa = mac_expected(ctx, level, digits, kb, ka)
        # all digits in one pass, full-context keys
        ob, oa = nb.empty((level + k, n)), nb.empty((level + k, n))
        g.hybrid_mac(level, ob, oa, ddig, dkb, dka)
        np.testing.assert_array_equal(nb.to_host(ob), wb)
        np.testing.assert_array_equal(nb.to_host(oa), wa)
        # one digit per call, the reference's per-digit Driver::hybrid_mac loop
        pb, pa = nb.empty((level + k, n)), nb.empty((level + k, n))
        for d in range(beta):
            g.hybrid_mac_digits(level, pb, pa, [ddig[d]], [dkb[d]], [dka[d]], full_key_rows=True,
                                accumulate=d > 0)
        np.testing.assert_array_equal(nb.to_host(pb), wb)
        np.testing.assert_array_equal(nb.to_host(pa), wa)
        # packed active rows (Session::upload_hybrid_key's packing) instead of full-context keys
        rows = key_rows(ctx, level)
        packed_b = [nb.to_device(np.ascontiguousarray(kb[d][rows])) for d in range(beta)]
        packed_a = [nb.to_device(np.ascontiguousarray(ka[d][rows])) for d in range(beta)]
        g.hybrid_mac_digits(level, pb, pa, [ddig[d] for d in range(beta)], packed_b, packed_a,
                            full_key_rows=False)
        np.testing.assert_array_equal(nb.to_host(pb), wb)
        np.testing.assert_array_equal(nb.to_host(pa), wa)
    assert g.device_errors() == 0
    g.close()


@pytest.mark.parametrize("n,m,k,dnum", CASES)
def test_summed_extensions_then_one_mod_down(lib, orc, n, m, k, dnum):
    """Two key switches with different keys accumulate in QP; one ModDown per channel."""
    ctx = synthetic_context(orc, n, m, k, dnum)
    g = nb.Context.from_oracle(ctx)
    keys = [full_keys(orc, ctx, 31), full_keys(orc, ctx, 57)]
    dkeys = [(nb.to_device(kb), nb.to_device(ka)) for kb, ka in keys]
    level = m
    beta = ctx.digits(level)
    xs = [orc.lcg(n, ctx.q[:level], 60 + i) for i in range(2)]
    ext_b, ext_a = nb.empty((level + k, n)), nb.empty((level + k, n))
    want_b = np.zeros((level + k, n), dtype=np.uint64)
    want_a = np.zeros((level + k, n), dtype=np.uint64)
    ws = g.workspace(nb.OP_DIGITS, level)
    for i, x in enumerate(xs):
        ddig = nb.empty((beta, level + k, n))
        g.hybrid_digits(level, ddig, nb.to_device(x), ws)
        g.hybrid_mac_digits(level, ext_b, ext_a, [ddig[d] for d in range(beta)],
                            [dkeys[i][0][d] for d in range(beta)], [dkeys[i][1][d] for d in range(beta)],
                            full_key_rows=True, accumulate=i > 0)
        wb, wa = mac_expected(ctx, level, orc.hybrid_digits(ctx, level, x), *keys[i])
        want_b, want_a = add_qp(ctx, level, want_b, wb), add_qp(ctx, level, want_a, wa)
    np.testing.assert_array_equal(nb.to_host(ext_b), want_b)
    np.testing.assert_array_equal(nb.to_host(ext_a), want_a)
    down_ws = g.workspace(nb.OP_MOD_DOWN, level)
    out_b, out_a = nb.empty((level, n)), nb.empty((level, n))
    g.mod_down(level, out_b, ext_b, down_ws)  # KeySwitchDownFirstElement
    np.testing.assert_array_equal(nb.to_host(out_b), orc.mod_down(ctx, level, want_b))
    g.mod_down(level, out_a, ext_a, down_ws)
    np.testing.assert_array_equal(nb.to_host(out_a), orc.mod_down(ctx, level, want_a))
    # ModDown is linear only up to the approximate conversion's overflow term, so
    # the delayed form is compared with the oracle's ModDown of the sum, not with
    # the sum of two complete key switches.
    assert g.device_errors() == 0
    g.close()
