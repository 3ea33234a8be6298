"""Every launch-tuning choice keeps every result exact.

The autotuner may pick any value of any tunable, so each non-default value (and
all of them together) runs forward and inverse NTTs at N = 2^12 and 2^16 and a
rotating key switch, checked against the CPU oracle bit for bit."""
import numpy as np
import pytest

import ntt_gpu_b200 as nb
from oracle.oracle import synthetic_context
from test_gpu_requests import full_keys

pytestmark = pytest.mark.gpu

VARIANTS = [("ntt_minb_fwd_col", 3), ("ntt_minb_fwd_row", 3), ("ntt_minb_inv_row", 3),
            ("ntt_minb_inv_col", 3), ("ntt_col_direct", 0), ("ntt_row_direct", 0), ("ntt_epi_stage", 1),
            ("intt_unscaled", 0), ("digits_lazy", 0), ("ntt_stage_tw_fwd_row", 1), ("ntt_stage_tw_inv_row", 1), ("conv_limbs", 0),
            ("conv_blocks_per_sm", 2), ("conv_tc_tiles", 3), ("conv_tc_fixed", 0), ("mac_limbs", 1),
            ("mac_approx", 0), ("mac_rotate", 0), ("conv_tc", 0), ("row_mac", 0),
            ("row_mac_max_beta", 1), ("row_mac_inv_rows", 0), ("ntt_cluster", 1)]


def _check_paths(orc):
    for logn, bits in ((12, (50, 60)), (16, (55, 60, 61))):
        n = 1 << logn
        q = [orc.find_primes(n, 1, b)[0] for b in bits]
        psi = [orc.find_psi(v, n) for v in q]
        g = nb.Context(n, q, psi)
        x = orc.lcg(n, q, 900 + logn)
        out = nb.empty(x.shape)
        g.ntt(out, nb.to_device(x), list(range(len(q))))
        np.testing.assert_array_equal(nb.to_host(out), orc.ntt(x, q, psi))
        g.ntt(out, nb.to_device(x), list(range(len(q))), inverse=True)
        np.testing.assert_array_equal(nb.to_host(out), orc.ntt(x, q, psi, inverse=True))
        g.close()
    ctx = synthetic_context(orc, 8192, 6, 3, 2)
    g = nb.Context.from_oracle(ctx)
    kb, ka = full_keys(orc, ctx, 77)
    x, c0 = orc.lcg(ctx.n, ctx.q[:5], 1), orc.lcg(ctx.n, ctx.q[:5], 2)
    ob, oa = nb.empty((5, ctx.n)), nb.empty((5, ctx.n))
    g.keyswitch(5, ob, oa, nb.to_device(x), nb.to_device(kb), nb.to_device(ka), g.workspace(nb.OP_KEYSWITCH, 5),
                c0=nb.to_device(c0), automorphism=25)
    wb, wa = orc.keyswitch(ctx, 5, x, kb, ka, c0, 25)
    np.testing.assert_array_equal(nb.to_host(ob), wb)
    np.testing.assert_array_equal(nb.to_host(oa), wa)
    g.close()


@pytest.mark.parametrize("name,value", VARIANTS + [("all", None)])
def test_tuning_choice_keeps_results_exact(lib, orc, name, value):
    pairs = VARIANTS if name == "all" else [(name, value)]
    before = {n: nb.tuning_get(n) for n, _ in pairs}
    try:
        for n, v in pairs:
            nb.tuning_set(n, v)
        _check_paths(orc)
    finally:
        for n, v in before.items():
            nb.tuning_set(n, v)
