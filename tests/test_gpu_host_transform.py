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


@pytest.mark.parametrize("chunk", [1, 3, 128])
def test_checks_overlap_copies_and_fail_late(lib, orc, chunk):
    """The arrays are checked in chunks of 1, 3 or all towers while the checked
    chunks are copied in: the results do not depend on the chunk size. A
    non-canonical word in the last tower of the left or the right operand stops
    the call after copies have started; both arrays are unchanged, and the next
    call is exact."""
    ctx = synthetic_context(orc, 4096, 7, 2, 2)
    g = nb.Context.from_oracle(ctx)
    ids = list(range(7))
    mods, psis = ctx.q[:7], ctx.q_psi[:7]
    a, b = orc.lcg(ctx.n, mods, 51), orc.lcg(ctx.n, mods, 52)
    before = nb.tuning_get("host_chunk_towers")
    nb.tuning_set("host_chunk_towers", chunk)
    try:
        ws = g.host_transform_workspace(nb.HOST_MULTIPLY)
        for side in ("left", "right"):
            v, r = a.copy(), b.copy()
            (v if side == "left" else r)[6, ctx.n - 1] = mods[6]
            keep_v, keep_r = v.copy(), r.copy()
            with pytest.raises(nb.ContractError, match="canonical"):
                g.host_transform(nb.HOST_MULTIPLY, v, ids, ws, right=r)
            np.testing.assert_array_equal(v, keep_v)
            np.testing.assert_array_equal(r, keep_r)
        v = a.copy()
        g.host_transform(nb.HOST_MULTIPLY, v, ids, ws, right=b)
        np.testing.assert_array_equal(v, _ring_product(orc, mods, psis, a, b))
    finally:
        nb.tuning_set("host_chunk_towers", before)
    g.close()


def test_repeated_tower_ids_need_a_larger_workspace(lib, orc):
    """A call may name a tower more than once; its workspace then has to hold
    every tower of the call, more than the context's own towers."""
    import torch
    ctx = synthetic_context(orc, 4096, 7, 2, 2)  # 9 towers
    g = nb.Context.from_oracle(ctx)
    ids = [0, 1, 2, 3, 4, 5, 6, 0, 1, 2, 3]
    mods = [ctx.q[i] for i in ids]
    psis = [ctx.q_psi[i] for i in ids]
    x = orc.lcg(ctx.n, mods, 53)
    ws = g.host_transform_workspace(nb.HOST_FORWARD)
    with pytest.raises(nb.WorkspaceError):
        g.host_transform(nb.HOST_FORWARD, x.copy(), ids, ws)
    big = torch.empty(len(ids) * ctx.n, dtype=torch.int64, device="cuda:0")
    v = x.copy()
    g.host_transform(nb.HOST_FORWARD, v, ids, big)
    np.testing.assert_array_equal(v, orc.ntt(x, mods, psis))
    g.close()
