"""GPU parity at the serving workload's largest shapes (N = 65536, L = 32).

The mixed serving stream builds contexts with dnum in {2, 3, 4} and
K = alpha = ceil(32 / dnum) P towers (16 / 11 / 8), so its key switches run
16-, 11- and 8-source conversions into up to 32 targets and 2 to 4 digits.
Every output here is compared with SHA-256 digests of the reference's own CPU
Session + HostDriver chain (src/resident.cpp:458-617, compiled from its sources
by tests/golden/make_golden.py), which the oracle reproduces bit for bit:
  - key switch, rotations by +-1 and +-64 steps (automorphisms 5^s mod 2N)
    over one shared input, and a level whose last digit is short;
  - relinearization = key switch plus the (c0, c1) addends, in place;
  - through one request-table call, and through the continuous-batching
    server with concurrent arrivals where the three contexts' requests mix:
    each result equals the request alone."""
import threading
import time

import numpy as np
import pytest

import golden_cases as gc
import ntt_gpu_b200 as nb
from test_gpu_requests import add_mod

pytestmark = pytest.mark.gpu


class Shape:
    """One config-5 context on the GPU with its key and golden cases."""

    def __init__(self, orc, dnum):
        self.dnum = dnum
        self.ctx = gc.config5_context(orc, dnum)
        self.g = nb.Context.from_oracle(self.ctx)
        kb, ka = gc.full_keys(orc, self.ctx, 300 + dnum)
        self.kb, self.ka = nb.to_device(kb), nb.to_device(ka)
        self.cases = list(gc.config5_cases(orc, dnum))
        self.inputs = {}
        for name, level, x, c0, g in self.cases:
            key = (level, x[0, 0], x[-1, -1])
            if key not in self.inputs:
                self.inputs[key] = nb.to_device(x)
        self.c0 = {name: nb.to_device(c0) for name, _, _, c0, _ in self.cases if c0 is not None}

    def dx(self, level, x):
        return self.inputs[(level, x[0, 0], x[-1, -1])]

    def requests(self, orc, seed):
        """(name, request, out_b, out_a, addends) for every case, plus one
        relinearization per level (in place over seeded c0 / c1)."""
        out = []
        n = self.ctx.n
        for name, level, x, c0, g in self.cases:
            ob, oa = nb.empty((level, n)), nb.empty((level, n))
            req = nb.make_request(level, self.dx(level, x), ob, oa, self.kb, self.ka,
                                  c0=self.c0.get(name), automorphism=g)
            out.append((name, req, ob, oa, None))
            if name.endswith("_ks"):
                mods = self.ctx.q[:level]
                r0 = orc.lcg(n, mods, seed + level)
                r1 = orc.lcg(n, mods, seed + level + 1)
                rb, ra = nb.to_device(r0), nb.to_device(r1)
                relin = nb.make_request(level, self.dx(level, x), rb, ra, self.kb, self.ka, add_b=rb, add_a=ra)
                out.append((name, relin, rb, ra, (r0, r1, mods)))
        return out

    def close(self):
        self.g.close()


def _check(d, items):
    """Key switches and rotations against the digests; relinearizations
    against the digest-checked key switch plus their addends."""
    ks = {}
    for name, _, ob, oa, addends in items:
        if addends is None:
            b, a = nb.to_host(ob), nb.to_host(oa)
            assert gc.sha(b) == d[name + "_b"], name
            assert gc.sha(a) == d[name + "_a"], name
            ks[name] = (b, a)
    for name, _, ob, oa, addends in items:
        if addends is not None:
            r0, r1, mods = addends
            b, a = ks[name]
            np.testing.assert_array_equal(nb.to_host(ob), add_mod(b, r0, mods), err_msg=name + " relin b")
            np.testing.assert_array_equal(nb.to_host(oa), add_mod(a, r1, mods), err_msg=name + " relin a")


@pytest.fixture(scope="module")
def shapes(orc):
    import torch
    assert torch.cuda.is_available()
    out = [Shape(orc, dnum) for dnum in gc.CONFIG5_DNUM]
    yield out
    for s in out:
        s.close()


@pytest.mark.parametrize("index", range(len(gc.CONFIG5_DNUM)))
def test_request_table_at_full_size(lib, orc, shapes, index):
    """One ntt_b200_keyswitch_requests call per context: key switch,
    relinearization and four hoisted rotations at L = 32, plus L = 17."""
    import torch
    s = shapes[index]
    items = s.requests(orc, 4000 + s.dnum)
    reqs = [it[1] for it in items]
    s.g.keyswitch_requests(reqs, s.g.requests_workspace(reqs))
    torch.cuda.synchronize()
    assert s.g.device_errors() == 0
    _check(gc.digests(), items)


def test_served_mix_at_full_size_equals_alone(lib, orc, shapes):
    """The three contexts' requests arrive from two host threads into one
    server (4 lanes, waves of up to 16, depth 2, 512 MiB in flight, as the
    bench serves the mixed stream); every result equals the reference's
    result for the request alone."""
    d = gc.digests()
    items = []
    for s in shapes:
        items += [(s, it) for it in s.requests(orc, 5000 + s.dnum)]
    rng = np.random.default_rng(11)
    order = [items[i] for i in rng.permutation(len(items))]
    srv = nb.Server(device=0, lanes=4, max_batch=16, hbm_budget_bytes=8 << 30, depth=2,
                    max_inflight_bytes=512 << 20)
    tickets = []
    lock = threading.Lock()

    def producer(part, delay_s):
        for s, it in part:
            t = srv.submit(s.g, it[1])
            with lock:
                tickets.append(t)
            time.sleep(delay_s)

    threads = [threading.Thread(target=producer, args=(order[i::2], 0.0003 * (i + 1))) for i in range(2)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    infos = [srv.wait(t, timeout_ms=120000) for t in tickets]
    stats = srv.stats()
    srv.close()
    assert all(i.status == nb.OK for i in infos)
    assert stats["completed"] == len(items)
    for s in shapes:
        assert s.g.device_errors() == 0
        _check(d, [it for owner, it in items if owner is s])


def test_sixteen_source_tensor_core_conversion_at_full_size(lib, orc):
    """The dnum = 2 digit conversion (16 sources -> 32 targets) and its ModDown
    conversion (16 -> 32) at N = 65536, on the tensor-core kernel, against the
    oracle's exact approximate-CRT switch."""
    import torch
    ctx = gc.config5_context(orc, 2)
    g = nb.Context.from_oracle(ctx)
    assert nb.tuning_get("conv_tc") == 1
    src_ids, tgt_ids = list(range(16)), list(range(16, 32)) + list(range(32, 48))
    mods = ctx.q + ctx.p
    x = orc.lcg(ctx.n, [mods[i] for i in src_ids], 77)
    out = nb.empty((len(tgt_ids), ctx.n))
    g.switch_basis(out, nb.to_device(x), src_ids, tgt_ids)
    torch.cuda.synchronize()
    assert g.device_errors() == 0
    want = orc.basis_convert(x, [mods[i] for i in src_ids], [mods[i] for i in tgt_ids])
    np.testing.assert_array_equal(nb.to_host(out), want)
    p_ids, q_ids = list(range(32, 48)), list(range(32))
    y = orc.lcg(ctx.n, [mods[i] for i in p_ids], 78)
    out = nb.empty((32, ctx.n))
    g.switch_basis(out, nb.to_device(y), p_ids, q_ids)
    torch.cuda.synchronize()
    want = orc.basis_convert(y, [mods[i] for i in p_ids], [mods[i] for i in q_ids])
    np.testing.assert_array_equal(nb.to_host(out), want)
    g.close()
