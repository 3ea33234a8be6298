"""The key multiplication fused into the digits' forward row pass
(ntt_fwd_row_mac) against the separate row pass + MAC pipeline.

Both forms must give the same key switches bit for bit: strided batches with
a shared key, with and without rotation, and request lists that mix keys,
rotations, relinearization addends and inputs shared by several requests
(hoisted digits, where one CTA serves every request of its input). Digit
counts 1 to 4 are covered (row_mac_max_beta selects per count)."""
import numpy as np
import pytest

import ntt_gpu_b200 as nb
from oracle.oracle import synthetic_context
from test_gpu_requests import Case, _keys

pytestmark = pytest.mark.gpu


def _sync():
    import torch
    torch.cuda.synchronize()


def _batch(g, ctx, level, batch, xs, kb, ka, c0=None, auto=0):
    ob, oa = nb.empty((batch, level, ctx.n)), nb.empty((batch, level, ctx.n))
    g.keyswitch_batch(level, batch, ob, oa, xs, kb, ka, g.workspace(nb.OP_KEYSWITCH, level, batch), c0=c0,
                      automorphism=auto)
    _sync()
    return nb.to_host(ob), nb.to_host(oa)


@pytest.mark.parametrize("n,m,k,dnum,levels", [(65536, 24, 8, 3, (24, 16, 8)), (16384, 32, 8, 4, (32, 25, 9, 3)),
                                               (4096, 12, 6, 2, (12, 6))])
def test_fused_batch_equals_separate_passes(lib, orc, n, m, k, dnum, levels):
    ctx = synthetic_context(orc, n, m, k, dnum)
    g = nb.Context.from_oracle(ctx)
    kb, ka, dkb, dka = _keys(orc, ctx, 41)
    for level in levels:
        batch = 3
        xs = nb.to_device(np.stack([orc.lcg(n, ctx.q[:level], 60 + i) for i in range(batch)]))
        c0 = nb.to_device(np.stack([orc.lcg(n, ctx.q[:level], 70 + i) for i in range(batch)]))
        got = {}
        for fused in (1, 0):
            nb.tuning_set("row_mac", fused)
            try:
                got[fused] = (_batch(g, ctx, level, batch, xs, dkb, dka), _batch(g, ctx, level, batch, xs, dkb, dka,
                                                                                    c0, 25))
            finally:
                nb.tuning_set("row_mac", 1)
        for a, b in zip(got[1], got[0]):
            np.testing.assert_array_equal(a[0], b[0], err_msg=f"L={level}")
            np.testing.assert_array_equal(a[1], b[1], err_msg=f"L={level}")
        # one request of each checked against the oracle
        x0 = orc.lcg(n, ctx.q[:level], 60)
        wb, wa = orc.keyswitch(ctx, level, x0, kb, ka, orc.lcg(n, ctx.q[:level], 70), 25)
        np.testing.assert_array_equal(got[1][1][0][0], wb)
        np.testing.assert_array_equal(got[1][1][1][0], wa)
    assert g.device_errors() == 0
    g.close()


def test_fused_request_list_with_shared_inputs(lib, orc):
    """Hoisted rotations (several keys and automorphisms over one input) next
    to distinct inputs and relinearizations, at two levels: equal to the
    oracle with the fused row pass."""
    ctx = synthetic_context(orc, 8192, 9, 3, 3)
    g = nb.Context.from_oracle(ctx)
    keysets = [_keys(orc, ctx, 300 + 7 * i) for i in range(3)]
    cases = []
    for level in (9, 5):
        base = Case(orc, ctx, level, 1000 + level, keysets[0], "rotate", 5)
        cases.append(base)
        for i, auto in enumerate((25, 2 * ctx.n - 1, 125)):
            cases.append(Case(orc, ctx, level, 1100 + 10 * level + i, keysets[(i + 1) % 3], "rotate", auto,
                              share=base))
        cases.append(Case(orc, ctx, level, 1200 + level, keysets[1], "switch", share=base))
        cases.append(Case(orc, ctx, level, 1300 + level, keysets[2], "relin"))
        cases.append(Case(orc, ctx, level, 1400 + level, keysets[0], "switch"))
    # interleave so requests of one input are not adjacent in the call
    order = cases[::2] + cases[1::2]
    reqs = [c.request() for c in order]
    g.keyswitch_requests(reqs, g.requests_workspace(reqs))
    _sync()
    for c in order:
        wb, wa = c.expected(orc, ctx)
        np.testing.assert_array_equal(nb.to_host(c.out_b), wb, err_msg=f"{c.kind} L={c.level}")
        np.testing.assert_array_equal(nb.to_host(c.out_a), wa, err_msg=f"{c.kind} L={c.level}")
    g.close()


@pytest.mark.parametrize("n", [8192, 65536])
def test_keyswitch_with_towers_at_the_reduction_free_bound(lib, orc, n):
    """Q primes just below 2^57 (reduction-free forward butterflies at their
    widest range, digits up to 68q into the key multiplication, and the ModDown
    epilogue) next to 60-bit P primes (per-stage reductions) in the same
    launches: key switch and rotation equal the oracle."""
    from oracle.oracle import Context
    from test_gpu_ntt import primes_below
    q = primes_below(orc, n, 6, 1 << 57)
    p = orc.find_primes(n, 3, 60)
    ctx = Context(n, q, [orc.find_psi(v, n) for v in q], p, [orc.find_psi(v, n) for v in p], 2)
    g = nb.Context.from_oracle(ctx)
    kb, ka, dkb, dka = _keys(orc, ctx, 97)
    for level in (6, 3):
        x = np.array([[v - 1] * n for v in ctx.q[:level]], dtype=np.uint64)  # top of every range
        c0 = orc.lcg(n, ctx.q[:level], 5)
        for rot in (False, True):
            ob, oa = nb.empty((level, n)), nb.empty((level, n))
            g.keyswitch(level, ob, oa, nb.to_device(x), dkb, dka, g.workspace(nb.OP_KEYSWITCH, level),
                        c0=nb.to_device(c0) if rot else None, automorphism=25 if rot else 0)
            _sync()
            wb, wa = orc.keyswitch(ctx, level, x, kb, ka, c0 if rot else None, 25 if rot else 0)
            np.testing.assert_array_equal(nb.to_host(ob), wb, err_msg=f"L={level} rot={rot}")
            np.testing.assert_array_equal(nb.to_host(oa), wa, err_msg=f"L={level} rot={rot}")
    g.close()


@pytest.mark.parametrize("n,m,k,dnum,levels", [(65536, 24, 8, 3, (24, 16)), (8192, 9, 3, 3, (9, 5)),
                                               (4096, 16, 4, 4, (16, 13))])
def test_inverse_row_pass_inside_the_fused_kernel(lib, orc, n, m, k, dnum, levels):
    """The fused kernel's P towers run the ModDown's inverse row pass before
    they are stored (row_mac_inv_rows, 2 to 4 digits, one request per input):
    key switches, relinearizations and rotations by steps +-1 and +-64 (whole
    rows gathered through the automorphism) equal the form with a separate
    inverse row pass, and the oracle."""
    ctx = synthetic_context(orc, n, m, k, dnum)
    g = nb.Context.from_oracle(ctx)
    keys = _keys(orc, ctx, 515)
    five_inv = pow(5, -1, 2 * n)
    autos = (5, five_inv, pow(5, 64, 2 * n), pow(five_inv, 64, 2 * n))
    for level in levels:
        cases = [Case(orc, ctx, level, 2000 + 10 * i + level, keys, "rotate", a) for i, a in enumerate(autos)]
        cases.append(Case(orc, ctx, level, 2100 + level, keys, "switch"))
        cases.append(Case(orc, ctx, level, 2200 + level, keys, "relin"))
        got = {}
        for fused in (1, 0):
            nb.tuning_set("row_mac_inv_rows", fused)
            try:
                for c in cases:
                    if c.kind == "relin":  # in place: restart from c0 / c1
                        c.out_b.copy_(nb.to_device(c.c0))
                        c.out_a.copy_(nb.to_device(c.c1))
                reqs = [c.request() for c in cases]
                g.keyswitch_requests(reqs, g.requests_workspace(reqs))
                _sync()
                got[fused] = [(nb.to_host(c.out_b), nb.to_host(c.out_a)) for c in cases]
            finally:
                nb.tuning_set("row_mac_inv_rows", 1)
        for c, a, b in zip(cases, got[1], got[0]):
            np.testing.assert_array_equal(a[0], b[0], err_msg=f"{c.kind} g={c.automorphism} L={level}")
            np.testing.assert_array_equal(a[1], b[1], err_msg=f"{c.kind} g={c.automorphism} L={level}")
        checked = cases if n <= 8192 else [cases[3], cases[5]]
        for c in checked:
            wb, wa = c.expected(orc, ctx)
            i = cases.index(c)
            np.testing.assert_array_equal(got[1][i][0], wb, err_msg=f"{c.kind} g={c.automorphism} L={level}")
            np.testing.assert_array_equal(got[1][i][1], wa, err_msg=f"{c.kind} g={c.automorphism} L={level}")
    assert g.device_errors() == 0
    g.close()
