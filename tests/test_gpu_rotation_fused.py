"""GPU parity at the benchmark shape: key-switch rotations fused into the MAC.

With the tunable `mac_rotate` on (the default), a rotating key switch adds
P * c0 and applies the automorphism inside the MAC's stores instead of a
separate gather pass over the extended result (rotated_b_value and
automorphism_source_index, include/ntt/resident_conversion.hpp:15-29). The
small-N cases of tests/test_gpu_keyswitch.py check the fused path against the
CPU oracle; here, at N = 2^16, L = 24 / 16 / 8, a request list mixing several
automorphisms (and plain switches) in one chunk must equal, bit for bit, every
request run alone through the separate rotation pass."""
import numpy as np
import pytest

import ntt_gpu_b200 as nb
from ntt_gpu_b200.params import synthetic_params, uniform_residues

pytestmark = pytest.mark.gpu

N = 65536


def _automorphisms(n):
    two_n = 2 * n
    return [5, 25, two_n - 1, pow(5, 37, two_n), pow(5, n // 2 - 1, two_n)]


@pytest.mark.parametrize("level", [24, 16, 8])
def test_fused_rotations_equal_the_rotation_pass(lib, level):
    prm = synthetic_params(N, 24, 8, 3)
    g = nb.Context(prm.n, prm.q, prm.q_psi, prm.p, prm.p_psi, prm.alpha)
    g.prepare(level)
    kb = nb.to_device(uniform_residues(N, prm.q + prm.p, 101, polys=prm.full_digits()))
    ka = nb.to_device(uniform_residues(N, prm.q + prm.p, 102, polys=prm.full_digits()))
    autos = _automorphisms(N) + [0]  # the last request is a plain switch in the same chunk
    count = len(autos)
    xs = nb.to_device(uniform_residues(N, prm.q[:level], 103, polys=count))
    c0s = nb.to_device(uniform_residues(N, prm.q[:level], 104, polys=count))
    out = nb.empty((count, 2, level, N))
    reqs = [nb.make_request(level, xs[i], out[i, 0], out[i, 1], kb, ka,
                            c0=c0s[i] if a else None, automorphism=a) for i, a in enumerate(autos)]
    before = nb.tuning_get("mac_rotate")
    try:
        nb.tuning_set("mac_rotate", 1)
        g.keyswitch_requests(reqs, g.requests_workspace(reqs))
        fused = nb.to_host(out)
        nb.tuning_set("mac_rotate", 0)
        alone = np.empty_like(fused)
        for i, r in enumerate(reqs):
            out.zero_()
            g.keyswitch_requests([r], g.requests_workspace([r]))
            alone[i] = nb.to_host(out[i])
    finally:
        nb.tuning_set("mac_rotate", before)
    for i, a in enumerate(autos):
        np.testing.assert_array_equal(fused[i], alone[i], err_msg=f"L={level} automorphism {a}")
    assert g.device_errors() == 0
    g.close()
