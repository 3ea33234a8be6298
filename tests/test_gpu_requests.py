"""GPU parity of the request-table key switch (ntt_b200_keyswitch_requests).

One call mixes levels, switching keys, rotations and relinearization addends;
every result must equal the CPU oracle and the same request run alone through
ntt_b200_keyswitch, bit for bit. Requests sharing an input share its digits
(hoisted rotations, include/ntt/openfhe_hybrid_adapter.hpp:309-361)."""
import numpy as np
import pytest

import ntt_gpu_b200 as nb
from oracle.oracle import LCG_SEED, synthetic_context

pytestmark = pytest.mark.gpu


def full_keys(orc, ctx, seed):
    mods = ctx.q + ctx.p
    kb = np.stack([orc.splitmix(ctx.n, mods, seed + 1000 * d) for d in range(ctx.full_digits())])
    ka = np.stack([orc.splitmix(ctx.n, mods, seed + 7 + 1000 * d) for d in range(ctx.full_digits())])
    return kb, ka


def add_mod(x, y, moduli):
    q = np.array(moduli, dtype=object)[:, None]
    return ((x.astype(object) + y.astype(object)) % q).astype(np.uint64)


class Case:
    """One request with host copies of everything the oracle needs."""

    def __init__(self, orc, ctx, level, seed, keys, kind, automorphism=0, share=None):
        n = ctx.n
        self.level, self.kind, self.keys, self.automorphism = level, kind, keys, automorphism
        self.x = share.x if share is not None else orc.lcg(n, ctx.q[:level], seed)
        self.dx = share.dx if share is not None else nb.to_device(self.x)
        self.c0 = orc.lcg(n, ctx.q[:level], seed + 1) if kind in ("rotate", "relin") else None
        self.c1 = orc.lcg(n, ctx.q[:level], seed + 2) if kind == "relin" else None
        self.out_b, self.out_a = nb.empty((level, n)), nb.empty((level, n))
        if kind == "relin":  # in place: the outputs start as c0 / c1 and receive the switch
            self.out_b.copy_(nb.to_device(self.c0))
            self.out_a.copy_(nb.to_device(self.c1))
        self.dc0 = nb.to_device(self.c0) if kind == "rotate" else None

    def request(self):
        kb, ka = self.keys[2], self.keys[3]
        if self.kind == "relin":
            return nb.make_request(self.level, self.dx, self.out_b, self.out_a, kb, ka,
                                   add_b=self.out_b, add_a=self.out_a)
        return nb.make_request(self.level, self.dx, self.out_b, self.out_a, kb, ka, c0=self.dc0,
                               automorphism=self.automorphism)

    def expected(self, orc, ctx):
        kb, ka = self.keys[0], self.keys[1]
        if self.kind == "rotate":
            return orc.keyswitch(ctx, self.level, self.x, kb, ka, self.c0, self.automorphism)
        wb, wa = orc.keyswitch(ctx, self.level, self.x, kb, ka)
        if self.kind == "relin":
            mods = ctx.q[:self.level]
            return add_mod(wb, self.c0, mods), add_mod(wa, self.c1, mods)
        return wb, wa


def _keys(orc, ctx, seed):
    kb, ka = full_keys(orc, ctx, seed)
    return kb, ka, nb.to_device(kb), nb.to_device(ka)


def _mixed_cases(orc, ctx, levels, n_req, seed):
    keysets = [_keys(orc, ctx, seed + 100 * i) for i in range(3)]
    kinds = ("switch", "rotate", "relin")
    autos = (5, 25, 2 * ctx.n - 1, 125)
    cases = []
    for r in range(n_req):
        level = levels[r % len(levels)]
        kind = kinds[(r // len(levels)) % 3]
        cases.append(Case(orc, ctx, level, seed + 10 * r, keysets[r % 3], kind, autos[r % 4]))
    return cases


def _sync():
    import torch
    torch.cuda.synchronize()


@pytest.mark.parametrize("n,m,k,dnum,levels", [(4096, 7, 2, 3, (7, 4, 2)), (8192, 9, 3, 3, (9, 5, 1)),
                                               (1024, 6, 3, 2, (6, 3))])
def test_mixed_request_list_matches_oracle(lib, orc, n, m, k, dnum, levels):
    ctx = synthetic_context(orc, n, m, k, dnum)
    g = nb.Context.from_oracle(ctx)
    cases = _mixed_cases(orc, ctx, levels, 12, 1234 + n)
    reqs = [c.request() for c in cases]
    g.keyswitch_requests(reqs, g.requests_workspace(reqs))
    _sync()
    for c in cases:
        wb, wa = c.expected(orc, ctx)
        np.testing.assert_array_equal(nb.to_host(c.out_b), wb, err_msg=f"{c.kind} L={c.level}")
        np.testing.assert_array_equal(nb.to_host(c.out_a), wa, err_msg=f"{c.kind} L={c.level}")
    g.close()


def test_each_request_equals_it_run_alone(lib, orc):
    """Mixed list vs one ntt_b200_keyswitch call per request (exact)."""
    ctx = synthetic_context(orc, 8192, 8, 3, 4)
    g = nb.Context.from_oracle(ctx)
    cases = [c for c in _mixed_cases(orc, ctx, (8, 6, 3), 9, 77) if c.kind != "relin"]
    reqs = [c.request() for c in cases]
    g.keyswitch_requests(reqs, g.requests_workspace(reqs))
    for c in cases:
        ob, oa = nb.empty((c.level, ctx.n)), nb.empty((c.level, ctx.n))
        g.keyswitch(c.level, ob, oa, c.dx, c.keys[2], c.keys[3], g.workspace(nb.OP_KEYSWITCH, c.level),
                    c0=c.dc0, automorphism=c.automorphism if c.dc0 is not None else 0)
        assert bool((ob == c.out_b).all()) and bool((oa == c.out_a).all())
    g.close()


def test_hoisted_rotations_share_one_input(lib, orc):
    """hybrid_rotate_many: several keys and automorphisms over one input."""
    ctx = synthetic_context(orc, 4096, 6, 3, 2)
    g = nb.Context.from_oracle(ctx)
    level = 6
    base = Case(orc, ctx, level, 555, _keys(orc, ctx, 9), "rotate", 5)
    cases = [base]
    for i, auto in enumerate((25, 2 * ctx.n - 1, 243)):
        cases.append(Case(orc, ctx, level, 600 + i, _keys(orc, ctx, 40 + i), "rotate", auto, share=base))
    cases.append(Case(orc, ctx, level, 700, base.keys, "switch", share=base))
    reqs = [c.request() for c in cases]
    ws_shared = g.requests_workspace_bytes(reqs)
    g.keyswitch_requests(reqs, g.requests_workspace(reqs))
    _sync()
    for c in cases:
        wb, wa = c.expected(orc, ctx)
        np.testing.assert_array_equal(nb.to_host(c.out_b), wb)
        np.testing.assert_array_equal(nb.to_host(c.out_a), wa)
    # The digits are stored once: sharing an input needs less workspace than distinct inputs.
    other = [Case(orc, ctx, level, 800 + i, base.keys, "rotate", 5) for i in range(len(cases))]
    assert ws_shared < g.requests_workspace_bytes([c.request() for c in other])
    g.close()


def test_config4_uneven_levels_full_size(lib, orc):
    """N = 2^16, K = 8, dnum = 3: one call with levels 8, 16 and 24 and one shared key."""
    ctx = synthetic_context(orc, 65536, 24, 8, 3)
    g = nb.Context.from_oracle(ctx)
    keys = _keys(orc, ctx, 99)
    cases = [Case(orc, ctx, level, LCG_SEED + level, keys, "switch") for level in (8, 16, 24)]
    cases.append(Case(orc, ctx, 16, LCG_SEED + 5, keys, "rotate", 5))
    reqs = [c.request() for c in cases]
    g.keyswitch_requests(reqs, g.requests_workspace(reqs))
    _sync()
    for c in cases:
        wb, wa = c.expected(orc, ctx)
        np.testing.assert_array_equal(nb.to_host(c.out_b), wb)
        np.testing.assert_array_equal(nb.to_host(c.out_a), wa)
    g.close()


def test_request_contract_errors(lib, orc):
    ctx = synthetic_context(orc, 1024, 4, 2, 2)
    g = nb.Context.from_oracle(ctx)
    keys = _keys(orc, ctx, 3)
    a = Case(orc, ctx, 4, 1, keys, "switch")
    b = Case(orc, ctx, 4, 2, keys, "rotate", 5)
    ws = g.requests_workspace([a.request(), b.request()])
    bad_level = a.request()
    bad_level.level = 5
    bad_auto = b.request()
    bad_auto.automorphism = 4
    overlap = b.request()
    overlap.out_b = a.request().src  # an output over another request's input
    for reqs in ([bad_level], [bad_auto], [a.request(), overlap]):
        with pytest.raises(nb.ContractError):
            g.keyswitch_requests(reqs, ws)
    with pytest.raises(nb.WorkspaceError):
        g.keyswitch_requests([a.request(), b.request()], ws[:16])
    g.close()


@pytest.mark.parametrize("batch,chunk,rotate", [(7, 2, False), (7, 3, True), (2, 4, True), (5, 1, False)])
def test_host_buffer_pipeline_matches_oracle(lib, orc, batch, chunk, rotate):
    """ntt_b200_keyswitch_host: pinned host inputs and outputs, chunks through two
    device slots with overlapped copies; two calls in a row on one stream."""
    import torch
    ctx = synthetic_context(orc, 8192, 6, 3, 2)
    g = nb.Context.from_oracle(ctx)
    kb, ka, dkb, dka = _keys(orc, ctx, 61)
    level = 5
    ws = g.host_workspace(level, chunk, rotate)
    for call in range(2):
        xs = np.stack([orc.lcg(ctx.n, ctx.q[:level], 100 * call + r) for r in range(batch)])
        c0 = np.stack([orc.lcg(ctx.n, ctx.q[:level], 500 + 100 * call + r) for r in range(batch)]) if rotate else None
        h_x = torch.from_numpy(xs.view(np.int64)).pin_memory()
        h_c0 = torch.from_numpy(c0.view(np.int64)).pin_memory() if rotate else None
        h_b = torch.zeros(xs.shape, dtype=torch.int64).pin_memory()
        h_a = torch.zeros(xs.shape, dtype=torch.int64).pin_memory()
        g.keyswitch_host(level, batch, chunk, h_x, h_b, h_a, dkb, dka, ws, h_c0=h_c0, automorphism=25 if rotate else 0)
        torch.cuda.synchronize()
        for r in range(batch):
            wb, wa = orc.keyswitch(ctx, level, xs[r], kb, ka, None if c0 is None else c0[r], 25 if rotate else 0)
            np.testing.assert_array_equal(h_b[r].numpy().view(np.uint64), wb)
            np.testing.assert_array_equal(h_a[r].numpy().view(np.uint64), wa)
    g.close()


def test_async_host_calls_back_to_back(lib, orc):
    """ntt_b200_keyswitch_host_async: four calls in a row on one stream with no
    wait between them (batch 5 in chunks of 2, so the calls start on either
    staging slot), the last one writing into the first one's host buffers;
    ntt_b200_keyswitch_host_wait then joins the stream. Synchronising that
    stream alone makes every output visible, each equal to the oracle."""
    import torch
    ctx = synthetic_context(orc, 8192, 6, 3, 2)
    g = nb.Context.from_oracle(ctx)
    kb, ka, dkb, dka = _keys(orc, ctx, 63)
    level, batch, chunk = 5, 5, 2
    ws = g.host_workspace(level, chunk)
    stream = torch.cuda.current_stream()
    xs = [np.stack([orc.lcg(ctx.n, ctx.q[:level], 700 + 10 * call + r) for r in range(batch)]) for call in range(4)]
    h_x = [torch.from_numpy(x.view(np.int64)).pin_memory() for x in xs]
    h_out = [(torch.zeros(xs[0].shape, dtype=torch.int64).pin_memory(),
              torch.zeros(xs[0].shape, dtype=torch.int64).pin_memory()) for _ in range(3)]
    torch.cuda.synchronize()
    for call in range(4):
        h_b, h_a = h_out[call % 3]
        g.keyswitch_host(level, batch, chunk, h_x[call], h_b, h_a, dkb, dka, ws, stream=stream, wait=False)
    g.keyswitch_host_wait(stream)
    stream.synchronize()
    for buf, call in ((0, 3), (1, 1), (2, 2)):
        h_b, h_a = h_out[buf]
        for r in range(batch):
            wb, wa = orc.keyswitch(ctx, level, xs[call][r], kb, ka)
            np.testing.assert_array_equal(h_b[r].numpy().view(np.uint64), wb, err_msg=f"call {call}")
            np.testing.assert_array_equal(h_a[r].numpy().view(np.uint64), wa, err_msg=f"call {call}")
    g.close()
