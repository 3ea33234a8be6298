"""GPU tests of the evaluation-key cache (ntt_b200_keycache_*) and of the server
taking keys from it by id: least-recently-used eviction within the budget, pins,
stream-ordered release, budget refusal, trim, and exact results when keys are
evicted and uploaded again between waves."""
import ctypes

import numpy as np
import pytest

import ntt_gpu_b200 as nb
from oracle.oracle import synthetic_context
from test_gpu_requests import add_mod, full_keys

pytestmark = pytest.mark.gpu


def _keyswitch_raw(g, level, x, kb_ptr, ka_ptr, c0=None, auto=0):
    """ntt_b200_keyswitch with raw device key pointers from the cache."""
    import torch
    n = g.n
    ob, oa = nb.empty((level, n)), nb.empty((level, n))
    ws = g.workspace(nb.OP_KEYSWITCH, level)
    dx = nb.to_device(x)
    dc0 = nb.to_device(c0) if c0 is not None else None
    rc = nb.load().ntt_b200_keyswitch(g._h, level, ob.data_ptr(), oa.data_ptr(), dx.data_ptr(),
                                      ctypes.c_void_p(kb_ptr), ctypes.c_void_p(ka_ptr),
                                      None if dc0 is None else dc0.data_ptr(), auto, ws.data_ptr(), ws.numel() * 8,
                                      torch.cuda.current_stream().cuda_stream)
    nb._check(rc)
    return nb.to_host(ob), nb.to_host(oa)


def test_cache_lru_pins_budget_and_exact_keys(lib, orc):
    ctx = synthetic_context(orc, 4096, 6, 3, 2)
    g = nb.Context.from_oracle(ctx)
    keys = [full_keys(orc, ctx, 500 + 11 * i) for i in range(4)]
    words = keys[0][0].size
    key_bytes = 2 * 8 * words
    cache = nb.KeyCache(device=0, budget_bytes=int(2.5 * key_bytes))
    for i, (kb, ka) in enumerate(keys):
        cache.insert(g, i, kb, ka)
    with pytest.raises(nb.ContractError):
        cache.insert(g, 0, *keys[0])  # duplicate id
    x = orc.lcg(ctx.n, ctx.q[:6], 42)
    for i in (0, 1, 0, 2, 3, 1):
        b, a = cache.acquire(i)
        got = _keyswitch_raw(g, 6, x, b, a)
        want = orc.keyswitch(ctx, 6, x, keys[i][0], keys[i][1])
        np.testing.assert_array_equal(got[0], want[0])
        np.testing.assert_array_equal(got[1], want[1])
        cache.release(i)
        import torch
        torch.cuda.synchronize()  # the release point has passed: the key is eligible for eviction
    st = cache.stats()
    # 0 miss, 1 miss, 0 hit, 2 miss (evicts 1), 3 miss (evicts 0), 1 miss (evicts 2)
    assert (st["hits"], st["misses"], st["evictions"]) == (1, 5, 3)
    assert st["resident"] == 2 and st["allocated_bytes"] == 2 * key_bytes <= st["budget_bytes"]
    # A pinned key blocks a budget below it. The refused call still evicts the
    # eligible key 1 first (evict eligible entries, then reject); after its
    # release, key 3 is trimmed away.
    cache.acquire(3)
    with pytest.raises(nb.ContractError):
        cache.set_budget(key_bytes // 2)
    assert cache.stats()["evictions"] == 4 and cache.stats()["pinned_bytes"] == key_bytes
    import torch
    cache.release(3)
    torch.cuda.synchronize()
    assert cache.trim() == key_bytes
    cache.set_budget(key_bytes)
    assert cache.stats()["allocated_bytes"] == 0
    with pytest.raises(nb.ContractError):
        cache.release(3)  # not acquired
    cache.close()
    g.close()


def test_server_takes_keys_from_cache_with_eviction(lib, orc):
    """Rotations with 6 keys through a cache that holds 3: keys are evicted and
    uploaded again between waves, and every served result is exact."""
    ctx = synthetic_context(orc, 4096, 6, 3, 2)
    g = nb.Context.from_oracle(ctx)
    keys = [full_keys(orc, ctx, 900 + 13 * i) for i in range(6)]
    key_bytes = 2 * 8 * keys[0][0].size
    cache = nb.KeyCache(device=0, budget_bytes=3 * key_bytes)
    for i, (kb, ka) in enumerate(keys):
        cache.insert(g, 100 + i, kb, ka)
    srv = nb.Server(device=0, lanes=2, max_batch=4, hbm_budget_bytes=1 << 30)
    plain = nb.Server(device=0, lanes=1, max_batch=1, hbm_budget_bytes=1 << 28)
    x = orc.lcg(ctx.n, ctx.q[:6], 7)
    with pytest.raises(nb.ContractError):  # key by id needs an attached cache
        plain.submit(g, nb.make_request(6, nb.to_device(x), nb.empty((6, ctx.n)), nb.empty((6, ctx.n)), key_id=100))
    plain.close()
    srv.attach_keycache(cache)
    rng = np.random.default_rng(3)
    cases = []
    for r in range(32):
        level = int(rng.integers(3, 7))
        k = int(rng.integers(6))
        auto = pow(5, int(rng.integers(1, 30)), 2 * ctx.n)
        x = orc.lcg(ctx.n, ctx.q[:level], 1000 + r)
        c0 = orc.lcg(ctx.n, ctx.q[:level], 2000 + r)
        relin = r % 3 == 0
        dx, dc0 = nb.to_device(x), nb.to_device(c0)
        ob, oa = nb.empty((level, ctx.n)), nb.empty((level, ctx.n))
        if relin:
            c1 = orc.lcg(ctx.n, ctx.q[:level], 3000 + r)
            ob.copy_(dc0)
            oa.copy_(nb.to_device(c1))
            req = nb.make_request(level, dx, ob, oa, add_b=ob, add_a=oa, key_id=100 + k)
        else:
            c1 = None
            req = nb.make_request(level, dx, ob, oa, c0=dc0, automorphism=auto, key_id=100 + k)
        cases.append((level, k, x, c0, c1, auto, relin, dx, dc0, ob, oa, srv.submit(g, req)))
    for case in cases:
        assert srv.wait(case[-1]).status == nb.OK
    srv.close()
    st = cache.stats()
    assert st["misses"] >= 6 and st["evictions"] > 0 and st["allocated_bytes"] <= 3 * key_bytes
    for level, k, x, c0, c1, auto, relin, dx, dc0, ob, oa, _ in cases:
        kb, ka = keys[k]
        if relin:
            wb, wa = orc.keyswitch(ctx, level, x, kb, ka)
            wb, wa = add_mod(wb, c0, ctx.q[:level]), add_mod(wa, c1, ctx.q[:level])
        else:
            wb, wa = orc.keyswitch(ctx, level, x, kb, ka, c0, auto)
        np.testing.assert_array_equal(nb.to_host(ob), wb)
        np.testing.assert_array_equal(nb.to_host(oa), wa)
    cache.close()
    g.close()


def test_cold_key_shared_by_waves_on_several_lanes(lib, orc):
    """A key that is not resident is uploaded on the stream of the first wave
    that needs it; waves on the other lanes that take it while that upload is
    in flight wait for it (every result exact)."""
    ctx = synthetic_context(orc, 16384, 12, 4, 3)
    g = nb.Context.from_oracle(ctx)
    kb, ka = full_keys(orc, ctx, 77)
    cache = nb.KeyCache(device=0, budget_bytes=1 << 30)
    cache.insert(g, 9, kb, ka)
    srv = nb.Server(device=0, lanes=4, max_batch=2, hbm_budget_bytes=2 << 30, depth=2)
    srv.attach_keycache(cache)
    cases = []
    for r in range(16):
        x = orc.lcg(ctx.n, ctx.q, 4100 + r)
        dx = nb.to_device(x)
        ob, oa = nb.empty((12, ctx.n)), nb.empty((12, ctx.n))
        cases.append((x, dx, ob, oa))
    import torch
    torch.cuda.synchronize()
    tickets = [srv.submit(g, nb.make_request(12, dx, ob, oa, key_id=9)) for x, dx, ob, oa in cases]
    infos = [srv.wait(t) for t in tickets]
    srv.close()
    assert all(i.status == nb.OK for i in infos)
    assert len({i.lane for i in infos}) > 1
    st = cache.stats()
    assert st["misses"] == 1 and st["hits"] >= 1
    for x, dx, ob, oa in cases:
        wb, wa = orc.keyswitch(ctx, 12, x, kb, ka)
        np.testing.assert_array_equal(nb.to_host(ob), wb)
        np.testing.assert_array_equal(nb.to_host(oa), wa)
    cache.close()
    g.close()


def test_releases_on_two_streams_both_hold_the_key(lib, orc):
    """A key pinned on two streams and released on both stays resident until
    the work before each release has completed: a release on an idle stream
    after one on a busy stream does not make it evictable."""
    import torch
    ctx = synthetic_context(orc, 65536, 24, 8, 3)
    g = nb.Context.from_oracle(ctx)
    kb, ka = full_keys(orc, ctx, 31)
    key_bytes = 2 * 8 * kb.size
    cache = nb.KeyCache(device=0, budget_bytes=4 * key_bytes)
    cache.insert(g, 1, kb, ka)
    busy, idle = torch.cuda.Stream(), torch.cuda.Stream()
    b, a = cache.acquire(1, stream=busy)
    cache.acquire(1, stream=idle)
    batch, level = 4, 24
    src = nb.to_device(np.stack([orc.lcg(ctx.n, ctx.q, 10 + i) for i in range(batch)]))
    ob, oa = nb.empty((batch, level, ctx.n)), nb.empty((batch, level, ctx.n))
    ws = g.workspace(nb.OP_KEYSWITCH, level, batch)
    busy.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(busy):
        for _ in range(30):  # tens of milliseconds of work that reads the key
            rc = nb.load().ntt_b200_keyswitch_batch(g._h, level, batch, ob.data_ptr(), oa.data_ptr(),
                                                    src.data_ptr(), ctypes.c_void_p(b), ctypes.c_void_p(a), None,
                                                    0, ws.data_ptr(), ws.numel() * 8, busy.cuda_stream)
            nb._check(rc)
    cache.release(1, stream=busy)
    cache.release(1, stream=idle)
    idle.synchronize()
    assert cache.trim() == 0  # the busy stream still reads the key
    busy.synchronize()
    assert cache.trim() == key_bytes
    want = orc.keyswitch(ctx, level, orc.lcg(ctx.n, ctx.q, 10), kb, ka)
    np.testing.assert_array_equal(nb.to_host(ob[0]), want[0])
    np.testing.assert_array_equal(nb.to_host(oa[0]), want[1])
    cache.close()
    g.close()
