"""Host-buffer transforms (ntt_b200_host_transform): the reference's
CudaNttTransform public calls forward / inverse / pointwise_multiply / multiply
on host arrays (include/ntt/cuda_ntt.hpp:59-66), bit-exact against the oracle,
with the reference's host validation (non-canonical input: contract error, the
host array untouched)."""
import numpy as np
import pytest

import ntt_gpu_b200 as nb
from oracle.oracle import synthetic_context

pytestmark = pytest.mark.gpu


def _ring_product(orc, mods, psis, a, b):
    fa, fb = orc.ntt(a, mods, psis), orc.ntt(b, mods, psis)
    q = np.array(mods, dtype=object)[:, None]
    prod = ((fa.astype(object) * fb.astype(object)) % q).astype(np.uint64)
    return orc.ntt(prod, mods, psis, inverse=True)


@pytest.mark.parametrize("n,towers", [(65536, 7), (4096, 13), (1024, 3)])
def test_host_calls_match_oracle(lib, orc, n, towers):
    ctx = synthetic_context(orc, n, towers, 2, 2)
    g = nb.Context.from_oracle(ctx)
    ids = list(range(towers))
    mods, psis = ctx.q[:towers], ctx.q_psi[:towers]
    a = orc.lcg(n, mods, 31)
    b = orc.lcg(n, mods, 32)
    ws = g.host_transform_workspace(nb.HOST_MULTIPLY)
    v = a.copy()
    g.host_transform(nb.HOST_FORWARD, v, ids, ws)
    fa = orc.ntt(a, mods, psis)
    np.testing.assert_array_equal(v, fa)
    g.host_transform(nb.HOST_INVERSE, v, ids, ws)
    np.testing.assert_array_equal(v, a)
    fb = orc.ntt(b, mods, psis)
    v = fa.copy()
    g.host_transform(nb.HOST_POINTWISE, v, ids, ws, right=fb)
    q = np.array(mods, dtype=object)[:, None]
    np.testing.assert_array_equal(v, ((fa.astype(object) * fb.astype(object)) % q).astype(np.uint64))
    v = a.copy()
    g.host_transform(nb.HOST_MULTIPLY, v, ids, ws, right=b)
    np.testing.assert_array_equal(v, _ring_product(orc, mods, psis, a, b))
    # tower ids select tables: P towers after Q towers
    pid = [towers, towers + 1]
    pm, pp = ctx.p, ctx.p_psi
    c = orc.lcg(n, pm, 33)
    v = c.copy()
    g.host_transform(nb.HOST_FORWARD, v, pid, ws)
    np.testing.assert_array_equal(v, orc.ntt(c, pm, pp))
    g.close()


def test_host_validation_before_enqueue(lib, orc):
    ctx = synthetic_context(orc, 4096, 5, 2, 2)
    g = nb.Context.from_oracle(ctx)
    ids = list(range(5))
    a = orc.lcg(ctx.n, ctx.q[:5], 41)
    a[3, 100] = ctx.q[3]  # not canonical
    before = a.copy()
    ws = g.host_transform_workspace(nb.HOST_FORWARD)
    with pytest.raises(nb.ContractError, match="canonical"):
        g.host_transform(nb.HOST_FORWARD, a, ids, ws)
    np.testing.assert_array_equal(a, before)
    small = ws[:8]
    with pytest.raises(nb.WorkspaceError):
        g.host_transform(nb.HOST_FORWARD, orc.lcg(ctx.n, ctx.q[:5], 42), ids, small)
    with pytest.raises(nb.ContractError):
        g.host_transform(nb.HOST_MULTIPLY, orc.lcg(ctx.n, ctx.q[:5], 42), ids, ws)  # no right operand
    g.close()
