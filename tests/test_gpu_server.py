"""GPU tests of the continuous-batching key-switch server (ntt_b200_server_*).

Requests of mixed ring dimension, level, kind (key switch, rotation,
relinearization) and key arrive from several host threads while earlier
waves run; every result must equal the CPU oracle bit for bit (the same
result as the request alone), and admission must respect the HBM budget."""
import threading
import time

import numpy as np
import pytest

import ntt_gpu_b200 as nb
from oracle.oracle import synthetic_context
from test_gpu_requests import Case, _keys

pytestmark = pytest.mark.gpu


def _contexts(orc):
    out = []
    for n, m, k, dnum in ((4096, 8, 3, 3), (8192, 6, 2, 2), (2048, 5, 3, 2)):
        ctx = synthetic_context(orc, n, m, k, dnum)
        g = nb.Context.from_oracle(ctx)
        out.append((ctx, g, [_keys(orc, ctx, 31 * n + i) for i in range(2)]))
    return out


def _random_cases(orc, contexts, count, seed):
    rng = np.random.default_rng(seed)
    kinds = ("switch", "rotate", "relin")
    cases = []
    for i in range(count):
        ctx, g, keysets = contexts[rng.integers(len(contexts))]
        level = int(rng.integers(1, ctx.m + 1))
        kind = kinds[rng.integers(3)]
        step = int(rng.integers(1, 65)) * (1 if rng.integers(2) else -1)
        auto = pow(5, step % (ctx.n // 2), 2 * ctx.n) if kind == "rotate" else 0
        c = Case(orc, ctx, level, seed * 1000 + i, keysets[rng.integers(2)], kind, auto)
        cases.append((ctx, g, c))
    return cases


def _check(orc, cases):
    for ctx, _, c in cases:
        wb, wa = c.expected(orc, ctx)
        np.testing.assert_array_equal(nb.to_host(c.out_b), wb, err_msg=f"{c.kind} N={ctx.n} L={c.level}")
        np.testing.assert_array_equal(nb.to_host(c.out_a), wa, err_msg=f"{c.kind} N={ctx.n} L={c.level}")


# (lanes, depth, max_batch, max_inflight_bytes): a cap of 1 byte lets only one
# wave run at a time (and must never stall); 64 MB admits several small waves.
@pytest.mark.parametrize("lanes,depth,max_batch,cap", [(3, 1, 8, 0), (1, 2, 1, 0), (2, 3, 4, 0), (4, 2, 8, 1),
                                                       (4, 2, 16, 64 << 20)])
def test_served_results_equal_oracle_under_concurrent_arrivals(lib, orc, lanes, depth, max_batch, cap):
    contexts = _contexts(orc)
    cases = _random_cases(orc, contexts, 48, 7 + lanes + cap % 97)
    srv = nb.Server(device=0, lanes=lanes, max_batch=max_batch, hbm_budget_bytes=2 << 30, depth=depth,
                    max_inflight_bytes=cap)
    tickets = {}

    def producer(part, delay_s):
        for ctx, g, c in part:
            tickets[id(c)] = srv.submit(g, c.request())
            time.sleep(delay_s)

    threads = [threading.Thread(target=producer, args=(cases[i::2], 0.0005 * (i + 1))) for i in range(2)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    done = {k: srv.wait(t) for k, t in tickets.items()}
    stats = srv.stats()
    srv.close()
    _check(orc, cases)
    assert stats["completed"] == len(cases)
    assert 0 < stats["p50_ms"] <= stats["p99_ms"] <= stats["max_ms"]
    assert stats["waves"] <= len(cases)
    assert all(i.status == nb.OK and i.latency_us > 0 for i in done.values())


def test_arrivals_during_running_waves_join_later_waves(lib, orc):
    """Continuous batching: more requests than the lanes can hold at once. Later
    requests are admitted into later waves as lanes free up, several requests per
    wave, and a second lane is used only while the first is busy (overlap)."""
    ctx = synthetic_context(orc, 16384, 12, 4, 3)
    g = nb.Context.from_oracle(ctx)
    keys = _keys(orc, ctx, 5)
    first = [Case(orc, ctx, 12, 100 + i, keys, "switch") for i in range(16)]
    later = [Case(orc, ctx, 12, 200 + i, keys, "rotate", 5) for i in range(16)]
    srv = nb.Server(device=0, lanes=2, max_batch=4, hbm_budget_bytes=4 << 30, depth=1, max_inflight_bytes=0)
    t1 = [srv.submit(g, c.request()) for c in first]
    t2 = [srv.submit(g, c.request()) for c in later]
    info = [srv.wait(t) for t in t1 + t2]
    stats = srv.stats()
    srv.close()
    _check(orc, [(ctx, g, c) for c in first + later])
    assert max(i.wave_size for i in info) > 1
    assert len({i.lane for i in info}) == 2
    assert stats["waves"] >= 8  # 32 requests, at most 4 per wave


def test_hbm_budget_admission(lib, orc):
    ctx = synthetic_context(orc, 8192, 6, 3, 2)
    g = nb.Context.from_oracle(ctx)
    keys = _keys(orc, ctx, 8)
    cases = [Case(orc, ctx, 6, 300 + i, keys, "switch") for i in range(6)]
    one = g.requests_workspace_bytes([cases[0].request()])
    two = g.requests_workspace_bytes([cases[0].request(), cases[1].request()])
    assert one < two
    srv = nb.Server(device=0, lanes=4, max_batch=8, hbm_budget_bytes=one)
    tickets = [srv.submit(g, c.request()) for c in cases]
    info = [srv.wait(t) for t in tickets]
    stats = srv.stats()
    srv.close()
    _check(orc, [(ctx, g, c) for c in cases])
    assert all(i.wave_size == 1 for i in info)   # never two requests' workspace at once
    assert stats["peak_bytes"] <= one
    small = nb.Server(device=0, lanes=1, max_batch=1, hbm_budget_bytes=one // 2)
    with pytest.raises(nb.WorkspaceError):
        small.submit(g, cases[0].request())
    small.close()


def test_submission_contract_errors(lib, orc):
    ctx = synthetic_context(orc, 1024, 4, 2, 2)
    g = nb.Context.from_oracle(ctx)
    c = Case(orc, ctx, 4, 1, _keys(orc, ctx, 2), "rotate", 5)
    srv = nb.Server(device=0, lanes=1, max_batch=2, hbm_budget_bytes=1 << 28)
    bad = c.request()
    bad.automorphism = 6
    with pytest.raises(nb.ContractError):
        srv.submit(g, bad)
    t = srv.submit(g, c.request())
    assert srv.wait(t).status == nb.OK
    with pytest.raises(nb.ContractError):
        srv.wait(t)  # already collected
    srv.close()
    _check(orc, [(ctx, g, c)])


def test_reserve_sizes_idle_arenas_within_the_budget(lib, orc):
    ctx = synthetic_context(orc, 8192, 6, 3, 2)
    g = nb.Context.from_oracle(ctx)
    keys = _keys(orc, ctx, 11)
    cases = [Case(orc, ctx, 6, 400 + i, keys, "switch") for i in range(6)]
    one = g.requests_workspace_bytes([cases[0].request()])
    srv = nb.Server(device=0, lanes=3, max_batch=1, hbm_budget_bytes=3 * one, depth=1, max_inflight_bytes=0)
    srv.reserve(one)
    assert srv.stats()["in_flight_bytes"] == 3 * one
    with pytest.raises(nb.ContractError):
        srv.reserve(one + 1)  # three lanes would exceed the budget
    srv.reserve(one)  # already that large: nothing to do
    tickets = [srv.submit(g, c.request()) for c in cases]
    info = [srv.wait(t) for t in tickets]
    stats = srv.stats()
    srv.close()
    _check(orc, [(ctx, g, c) for c in cases])
    assert all(i.status == nb.OK for i in info)
    assert stats["peak_bytes"] == 3 * one  # the reserved arenas carried every wave
