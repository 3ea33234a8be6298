"""Key switches recorded into a CUDA graph and replayed.

After ntt_b200_context_prepare(level) the compute entry points enqueue kernels
only (no allocation, no host synchronisation, no attribute or table uploads),
so a caller may capture them. Each replay here runs on fresh inputs written
into the captured buffers and must equal the CPU oracle bit for bit."""
import numpy as np
import pytest

import ntt_gpu_b200 as nb
from oracle.oracle import synthetic_context
from test_gpu_requests import Case, full_keys

pytestmark = pytest.mark.gpu


def _capture(fn, side):
    import torch
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=side):
        fn(side)
    return graph


@pytest.mark.parametrize("n,m,k,dnum,batch", [(8192, 6, 3, 2, 3), (65536, 24, 8, 3, 1)])
def test_batched_rotation_replays_from_a_graph(lib, orc, n, m, k, dnum, batch):
    import torch
    ctx = synthetic_context(orc, n, m, k, dnum)
    g = nb.Context.from_oracle(ctx)
    level = m
    g.prepare(level)
    kb, ka = full_keys(orc, ctx, 5)
    dkb, dka = nb.to_device(kb), nb.to_device(ka)
    x, c0 = nb.empty((batch, level, n)), nb.empty((batch, level, n))
    ob, oa = nb.empty((batch, level, n)), nb.empty((batch, level, n))
    ws = g.workspace(nb.OP_KEYSWITCH, level, batch)

    def fill(seed):
        xs = np.stack([orc.lcg(n, ctx.q[:level], seed + r) for r in range(batch)])
        cs = np.stack([orc.lcg(n, ctx.q[:level], seed + 50 + r) for r in range(batch)])
        x.copy_(nb.to_device(xs))
        c0.copy_(nb.to_device(cs))
        return xs, cs

    def step(stream):
        g.keyswitch_batch(level, batch, ob, oa, x, dkb, dka, ws, c0=c0, automorphism=5, stream=stream)

    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    fill(1)
    step(side)  # eager warm-up on the capture stream
    torch.cuda.synchronize()
    graph = _capture(step, side)
    for seed in (11, 21):
        xs, cs = fill(seed)
        torch.cuda.synchronize()
        graph.replay()
        torch.cuda.synchronize()
        for r in range(batch):
            wb, wa = orc.keyswitch(ctx, level, xs[r], kb, ka, cs[r], 5)
            np.testing.assert_array_equal(nb.to_host(ob[r]), wb)
            np.testing.assert_array_equal(nb.to_host(oa[r]), wa)
    assert g.device_errors() == 0
    del graph
    g.close()


def test_request_list_replays_from_a_graph(lib, orc):
    """Mixed levels, a relinearization (in place, addends) and a rotation in one captured call."""
    import torch
    ctx = synthetic_context(orc, 4096, 7, 2, 3)
    g = nb.Context.from_oracle(ctx)
    for level in (7, 4):
        g.prepare(level)
    kb, ka = full_keys(orc, ctx, 9)
    keys = (kb, ka, nb.to_device(kb), nb.to_device(ka))
    cases = [Case(orc, ctx, 7, 100, keys, "switch"), Case(orc, ctx, 4, 200, keys, "rotate", 25),
             Case(orc, ctx, 7, 300, keys, "relin")]
    reqs = [c.request() for c in cases]
    ws = g.requests_workspace(reqs)
    relin = cases[2]

    def refill(seed):
        for i, c in enumerate(cases):
            c.x = orc.lcg(ctx.n, ctx.q[:c.level], seed + 10 * i)
            c.dx.copy_(nb.to_device(c.x))
        rot = cases[1]
        rot.c0 = orc.lcg(ctx.n, ctx.q[:rot.level], seed + 7)
        rot.dc0.copy_(nb.to_device(rot.c0))
        relin.c0 = orc.lcg(ctx.n, ctx.q[:relin.level], seed + 8)
        relin.c1 = orc.lcg(ctx.n, ctx.q[:relin.level], seed + 9)
        relin.out_b.copy_(nb.to_device(relin.c0))
        relin.out_a.copy_(nb.to_device(relin.c1))

    def step(stream):
        g.keyswitch_requests(reqs, ws, stream=stream)

    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    refill(1)
    step(side)
    torch.cuda.synchronize()
    graph = _capture(step, side)
    for seed in (31, 41):
        refill(seed)
        torch.cuda.synchronize()
        graph.replay()
        torch.cuda.synchronize()
        for c in cases:
            wb, wa = c.expected(orc, ctx)
            np.testing.assert_array_equal(nb.to_host(c.out_b), wb, err_msg=c.kind)
            np.testing.assert_array_equal(nb.to_host(c.out_a), wa, err_msg=c.kind)
    assert g.device_errors() == 0
    del graph
    g.close()

