#!/usr/bin/env python
"""Benchmark: batched CKKS Hybrid key switching on B200 (sm_100a).

Workload (one step): a batch of 16 ciphertext components at N = 2^16, L = 24
active Q towers (55-bit), K = 8 P towers (60-bit), dnum = 3 (alpha = 8), one
shared full-context switching key, through ntt_b200_keyswitch_batch. Inputs are
resident in HBM; the working set (~3 GB) is far larger than the 126 MB L2, so
no flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun (N > 1) every rank runs its own replica of the workload on its
own GPU (request-level sharding, no collective on the data path); the timed
region is bracketed by a barrier + synchronize and the MAX over ranks is used.
--impl reference times the reference's own CPU implementation (oracle/_ref,
compiled from its sources) on the host cores instead.

Rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "keyswitch/s N=2^16 L=24 dnum=3 served vs plain, p50/p99 ms; NTT HBM GB/s"
UNIT = "keyswitch/s"
N, LEVEL, K_P, DNUM, BATCH = 65536, 24, 8, 3, 16
E2E_CHUNK = 4  # requests per chunk of the host-buffer pipeline (best of 1, 2, 4 with back-to-back asynchronous calls on a B200)
SEED = 0x7251D9
WORKLOAD = ("batched Hybrid key switch: 16 ciphertext components per GPU at N=2^16, L=24 (55-bit), "
            "K=8 (60-bit), dnum=3 (alpha=8), one shared switching key")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--batch", type=int, default=BATCH)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serving", action="store_true", help="skip the served-vs-plain Poisson legs")
    ap.add_argument("--tune", action="append", default=[], metavar="NAME=VALUE",
                    help="profiling: override a launch tunable (repeatable), e.g. --tune conv_tc=0")
    ap.add_argument("--rotate", action="store_true",
                    help="profiling: every batched request also adds P*c0 and rotates by g = 5 (rotate kernel)")
    ap.add_argument("--e2e-chunk", type=int, default=E2E_CHUNK,
                    help="requests per chunk of the end-to-end host-buffer pipeline")
    ap.add_argument("--kernels-only", action="store_true",
                    help="timed batched steps only (no plain/e2e/CPU legs); for profiler launch lists")
    return ap.parse_args()


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---- clocks during the timed region ------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-i", str(self.device), "-lms", "50"], stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
            return
        # nvidia-smi can take a second to start: the timed region begins after its first sample.
        deadline = time.time() + 10
        while time.time() < deadline and self.proc.poll() is None:
            if os.path.getsize(self.file.name) > 0:
                break
            time.sleep(0.05)

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.1)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.file.flush()
        self.file.seek(0)
        sm, smax, reasons = [], [], set()
        for line in self.file.read().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(self.NAMES, parts[5:9]):
                if flag.lower().startswith("active"):
                    reasons.add(name)
        os.unlink(self.file.name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "samples": len(sm),
                "reasons": sorted(reasons)}


# ---- distributed plumbing -----------------------------------------------------------------
def dist_setup():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(value: float, world: int, device) -> float:
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_teardown(world):
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# ---- CPU side: the reference's own implementation -----------------------------------------
def cpu_context(prm):
    from oracle.oracle import Context as OrcContext
    return OrcContext(prm.n, prm.q, prm.q_psi, prm.p, prm.p_psi, prm.alpha)


def cpu_impl():
    from oracle.oracle import Oracle, Reference
    if Reference.available():
        return Reference(), "reference"
    return Oracle(), "port"


def cpu_inputs(prm, level):
    from ntt_gpu_b200.params import uniform_residues
    x = uniform_residues(prm.n, prm.q[:level], SEED)[0]
    kb = uniform_residues(prm.n, prm.q + prm.p, SEED + 1, polys=prm.full_digits())
    ka = uniform_residues(prm.n, prm.q + prm.p, SEED + 2, polys=prm.full_digits())
    return x, kb, ka


def cpu_baseline_single(prm, samples=3):
    impl, kind = cpu_impl()
    ctx = cpu_context(prm)
    x, kb, ka = cpu_inputs(prm, LEVEL)
    t0 = time.perf_counter()
    for _ in range(samples):
        impl.keyswitch(ctx, LEVEL, x, kb, ka)
    dt = time.perf_counter() - t0
    return {"value": samples / dt, "unit": UNIT, "cores": 1, "kind": kind,
            "sample": f"{samples} sequential key switches (N=2^16, L=24, dnum=3, K=8), one thread, "
                      f"{dt:.1f} s"}


def run_reference(args, rank, world):
    """Reference arm: the reference CPU key switch (Session + HostDriver, compiled from its sources) on the
    host cores, on this arm's workload: each step is the same batch of 16 key switches at N=2^16, L=24,
    dnum=3, K=8, spread over the host threads. Warm-up steps as requested (at most 5); the timed step count
    is bounded so that the run ends within a few minutes."""
    if rank != 0:
        return None
    from concurrent.futures import ThreadPoolExecutor

    from ntt_gpu_b200.params import synthetic_params
    prm = synthetic_params(N, LEVEL, K_P, DNUM)
    impl, kind = cpu_impl()
    ctx = cpu_context(prm)
    x, kb, ka = cpu_inputs(prm, LEVEL)
    threads = min(BATCH, os.cpu_count() or 1)
    try:
        import psutil
        threads = max(1, min(threads, int(psutil.virtual_memory().available // (700 << 20))))
    except Exception:
        pass

    def one(_):
        impl.keyswitch(ctx, LEVEL, x, kb, ka)

    def batch_step(pool):
        list(pool.map(one, range(BATCH)))

    warmup = max(1, min(args.warmup, 5))
    with ThreadPoolExecutor(threads) as pool:
        t0 = time.perf_counter()
        batch_step(pool)
        t_step = time.perf_counter() - t0
        for _ in range(warmup - 1):
            batch_step(pool)
        steps = max(2, min(args.steps, int(120 / max(t_step, 1e-3))))
        t0 = time.perf_counter()
        for _ in range(steps):
            batch_step(pool)
        dt = time.perf_counter() - t0
    value = BATCH * steps / dt
    sample = (f"each step = the batch of {BATCH} key switches at N=2^16, L=24, dnum=3, K=8 (one shared key), "
              f"spread over {threads} host threads; {warmup} warm-up and {steps} timed steps of {args.steps} "
              "requested (bounded to a few minutes)")
    return {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": world,
            "steps": steps, "requested_steps": args.steps, "warmup": warmup, "ms_per_step": dt * 1000 / steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic", "same_config": True,
            "config": {"workload": WORKLOAD, "n": N, "level": LEVEL, "dnum": DNUM, "k": K_P, "batch_per_step": BATCH},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


# ---- GPU side ------------------------------------------------------------------------------------
# ---- configs 1-3: NTT and conversion legs -------------------------------------------------------
def config_legs(nb, device, peak, peak_kind):
    """Config 1 (one 60-bit tower, forward + inverse), config 2 (8 x 32 towers, forward + inverse,
    direct launches and CUDA-graph replay) and config 3 (fused digits and ModDown at L = 24)."""
    import torch

    from ntt_gpu_b200.params import find_primes, find_psi, min_psi, synthetic_params, uniform_residues
    W = 8 * N

    def timed(fn, iters):
        for _ in range(3):
            fn()
        torch.cuda.synchronize(device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(iters):
            fn()
        e1.record()
        torch.cuda.synchronize(device)
        return e0.elapsed_time(e1) / iters

    def leg(ms, nbytes, **extra):
        gbs = nbytes / (ms / 1e3) / 1e9
        return dict({"ms": ms, "algorithmic_bytes": nbytes, "gb_s": gbs, "frac_of_hbm_peak": gbs / peak,
                     "hbm_peak_source": peak_kind}, **extra)

    out = {}
    # config 1: the pinned OpenFHE 60-bit tower (q0, psi from the reference's pinned table).
    q0, psi0 = 1152921504606584833, 18043022392882
    c1 = nb.Context(N, [q0], [psi0], device=device)
    x1 = nb.to_device(uniform_residues(N, [q0], SEED)[0], device)
    y1 = torch.empty_like(x1)
    ms = timed(lambda: (c1.ntt(y1, x1, [0]), c1.ntt(y1, y1, [0], inverse=True)), 200)
    out["config1"] = leg(ms, 4 * W, workload="N=2^16, one 60-bit tower, forward then inverse (latency-bound)")
    c1.close()
    # config 2: 8 polynomials x 32 towers (16 x 50-bit and 16 x 60-bit, interleaved).
    q = [v for pair in zip(find_primes(N, 16, 50), find_primes(N, 16, 60)) for v in pair]
    x2 = nb.to_device(uniform_residues(N, q, SEED, polys=8), device)
    y2 = torch.empty_like(x2)
    ids = list(range(32))
    nbytes = 8 * 32 * 2 * 2 * W

    def config2_run(roots):
        c2 = nb.Context(N, q, roots, device=device)

        def fwd_inv():
            c2.ntt(y2, x2, ids, polys=8, poly_stride=32 * N)
            c2.ntt(y2, y2, ids, polys=8, poly_stride=32 * N, inverse=True)

        direct = timed(fwd_inv, 20)
        graph = torch.cuda.CUDAGraph()
        side = torch.cuda.Stream(device)
        side.wait_stream(torch.cuda.current_stream(device))
        with torch.cuda.stream(side):
            fwd_inv()
        torch.cuda.synchronize(device)
        with torch.cuda.graph(graph):
            fwd_inv()
        replay = timed(graph.replay, 20)
        exact = bool(torch.equal(y2, x2))
        del graph
        c2.close()
        return {"direct": leg(direct, nbytes), "graph_replay": leg(replay, nbytes), "roundtrip_exact": exact}

    out["config2"] = dict({"workload": "N=2^16, 8 polynomials x 32 towers (16 x 50-bit + 16 x 60-bit), forward "
                                       "then inverse; 512 MiB moved, larger than L2"},
                          **config2_run([find_psi(v, N) for v in q]))
    out["config2"]["openfhe_min_roots"] = config2_run([min_psi(v, N) for v in q])
    out["public_call_40x60"] = public_call_leg(nb, device, timed)
    # config 3: fused INTT -> ModUp -> NTT (Hybrid digits) and INTT -> ModDown -> NTT at L = 24.
    prm = synthetic_params(N, LEVEL, K_P, DNUM)
    c3 = nb.Context(prm.n, prm.q, prm.q_psi, prm.p, prm.p_psi, prm.alpha, device)
    c3.prepare(LEVEL)
    T, beta = LEVEL + K_P, prm.digits(LEVEL)
    xq = nb.to_device(uniform_residues(N, prm.q, SEED)[0], device)
    xqp = nb.to_device(uniform_residues(N, prm.q + prm.p, SEED + 1)[0], device)
    digits = torch.empty((beta, T, N), dtype=torch.int64, device=xq.device)
    down = torch.empty((LEVEL, N), dtype=torch.int64, device=xq.device)
    wsd, wsm = c3.workspace(nb.OP_DIGITS, LEVEL), c3.workspace(nb.OP_MOD_DOWN, LEVEL)
    ms_d = timed(lambda: c3.hybrid_digits(LEVEL, digits, xq, wsd), 50)
    ms_m = timed(lambda: c3.mod_down(LEVEL, down, xqp, wsm), 50)
    out["config3"] = {"workload": "N=2^16, L=24 (55-bit), K=8 (60-bit), dnum=3, one polynomial per call",
                      "mod_up_digits": leg(ms_d, W * (LEVEL + beta * T)),
                      "mod_down": leg(ms_m, W * (2 * LEVEL + K_P))}
    # config 4: 16 ciphertexts at uneven levels L = {8, 16, 24}[i mod 3] in one request-table call, one
    # shared key: key switch, relinearization (addends c0, c1) and rotation by one step (g = 5, with c0).
    levels = [(8, 16, 24)[i % 3] for i in range(BATCH)]
    c3.prepare(8)
    c3.prepare(16)
    qp = prm.q + prm.p
    kb = device_residues(N, qp, SEED + 40, prm.full_digits(), device)
    ka = device_residues(N, qp, SEED + 41, prm.full_digits(), device)
    xs = device_residues(N, prm.q, SEED + 42, BATCH, device)
    c0s = device_residues(N, prm.q, SEED + 43, BATCH, device)
    outs = torch.empty((BATCH, 2, LEVEL, N), dtype=torch.int64, device=xs.device)

    def requests(kind):
        reqs = []
        for i, lv in enumerate(levels):
            ob, oa = outs[i, 0, :lv], outs[i, 1, :lv]
            if kind == "rotate":
                reqs.append(nb.make_request(lv, xs[i, :lv], ob, oa, kb, ka, c0=c0s[i, :lv], automorphism=5))
            elif kind == "relinearize":
                reqs.append(nb.make_request(lv, xs[i, :lv], ob, oa, kb, ka, add_b=ob, add_a=oa))
            else:
                reqs.append(nb.make_request(lv, xs[i, :lv], ob, oa, kb, ka))
        return reqs

    batch_bytes = W * (3 * sum(levels) + 2 * prm.digits(LEVEL) * (LEVEL + K_P))
    c4 = {"workload": "N=2^16, K=8, dnum=3 (alpha=8), 16 ciphertexts at L = 8, 16, 24 (6 x 8, 5 x 16, 5 x 24) in "
                      "one ntt_b200_keyswitch_requests call, one shared key; algorithmic bytes = input + 2 outputs "
                      "per request + the key rows touched once",
          "algorithmic_bytes": batch_bytes}
    for kind in ("switch", "relinearize", "rotate"):
        if kind == "relinearize":  # in place: the outputs start as (c0, c1) and receive the switch
            outs[:, 0].copy_(c0s)
            outs[:, 1].copy_(xs)
        reqs = requests(kind)
        ws = c3.requests_workspace(reqs)
        ms = timed(lambda: c3.keyswitch_requests(reqs, ws), 20)
        c4[kind] = dict(leg(ms, batch_bytes), keyswitch_per_s=BATCH / (ms / 1e3))
    out["config4_uneven"] = c4
    c3.close()
    return out


def public_call_leg(nb, device, timed):
    """The reference's published shape (docs/batch40-native-analysis.md:31-34): N=2^16, 40 towers of
    60-bit primes. Resident (device buffers) forward / inverse / pointwise / ring product, and the public
    host-vector calls (ntt_b200_host_transform, the CudaNttTransform forward / inverse /
    pointwise_multiply / multiply) with pageable numpy arrays (the reference's std::vector) and with pinned
    host memory; host validation and both copy directions are inside every public call."""
    import numpy as np
    import torch

    from ntt_gpu_b200.params import find_primes, find_psi, uniform_residues
    q = find_primes(N, 40, 60)
    ctx = nb.Context(N, q, [find_psi(v, N) for v in q], device=device)
    ids = list(range(40))
    a = uniform_residues(N, q, SEED + 70)
    b = uniform_residues(N, q, SEED + 71)
    da, db = nb.to_device(a, device), nb.to_device(b, device)
    y = torch.empty_like(da)

    def resident_multiply():
        ctx.ntt(y, da, ids)
        ctx.ntt(da, da, ids)
        ctx.pointwise(y, y, da, ids)
        ctx.ntt(y, y, ids, inverse=True)

    resident = {"forward_ms": timed(lambda: ctx.ntt(y, da, ids), 50),
                "inverse_ms": timed(lambda: ctx.ntt(y, da, ids, inverse=True), 50),
                "pointwise_ms": timed(lambda: ctx.pointwise(y, da, db, ids), 50)}
    da.copy_(nb.to_device(a, device))
    resident["multiply_ms"] = timed(resident_multiply, 20)
    ws = ctx.host_transform_workspace(nb.HOST_MULTIPLY)
    calls = {}
    for memory in ("pageable", "pinned"):
        if memory == "pageable":
            va, vb = a.copy(), b.copy()
        else:
            va = torch.from_numpy(a.view(np.int64)).pin_memory()
            vb = torch.from_numpy(b.view(np.int64)).pin_memory()
        row = {}
        for name, op, right in (("forward_ms", nb.HOST_FORWARD, None), ("inverse_ms", nb.HOST_INVERSE, None),
                                ("pointwise_ms", nb.HOST_POINTWISE, vb), ("multiply_ms", nb.HOST_MULTIPLY, vb)):
            def call():  # in place; every output is again a canonical input
                ctx.host_transform(op, va, ids, ws, right=right)
            for _ in range(2):
                call()
            t0 = time.perf_counter()
            reps = 10
            for _ in range(reps):
                call()
            row[name] = (time.perf_counter() - t0) * 1e3 / reps
        calls[memory] = row
    ctx.close()
    return {"workload": "N=2^16, 40 towers of 60-bit primes (find_primes), the reference's batch40 shape",
            "resident_device_ms": resident, "public_call_wall_ms": calls,
            "reference_published": {"hardware": "RTX 4080 SUPER (docs/batch40-native-analysis.md:31-34)",
                                    "resident_ms": {"forward": 0.552, "inverse": 0.598, "pointwise": 0.048,
                                                    "multiply": 1.723},
                                    "public_call_ms": {"forward": 8.079, "inverse": 8.045, "pointwise": 11.858,
                                                       "multiply": 12.431}},
            "note": "public calls are synchronous and include host validation of every input residue"}


# ---- serving: seeded Poisson arrivals through the continuous-batching server ---------------------
def device_residues(n, moduli, seed, polys, device):
    """[polys][towers][n] int64 tensor of residues in [0, q_t) from a seeded device generator."""
    import torch
    gen = torch.Generator(device=f"cuda:{device}")
    gen.manual_seed(seed)
    v = torch.randint(0, 1 << 62, (polys, len(moduli), n), generator=gen, dtype=torch.int64,
                      device=f"cuda:{device}")
    q = torch.tensor([int(m) for m in moduli], dtype=torch.int64, device=f"cuda:{device}")
    return v % q[None, :, None]


class Workload:
    """Device-resident inputs, keys and an output ring of one context for served requests."""

    def __init__(self, nb, prm, device, seed, n_inputs=4, n_keys=2, ring=48):
        import torch
        self.prm, self.device = prm, device
        self.ctx = nb.Context(prm.n, prm.q, prm.q_psi, prm.p, prm.p_psi, prm.alpha, device)
        for level in range(1, prm.m + 1):
            self.ctx.prepare(level)
        qp = prm.q + prm.p
        self.inputs = device_residues(prm.n, prm.q, seed, n_inputs, device)
        self.c0 = device_residues(prm.n, prm.q, seed + 1, n_inputs, device)
        self.keys = [(device_residues(prm.n, qp, seed + 10 + 2 * i, prm.full_digits(), device),
                      device_residues(prm.n, qp, seed + 11 + 2 * i, prm.full_digits(), device))
                     for i in range(n_keys)]
        self.out = torch.empty((ring, 2, prm.m, prm.n), dtype=torch.int64, device=f"cuda:{device}")
        self.slot = 0

    def request(self, nb, level, kind, step, i):
        n = self.prm.n
        out = self.out[self.slot % self.out.shape[0]]
        self.slot += 1
        x = self.inputs[i % self.inputs.shape[0]]
        kb, ka = self.keys[i % len(self.keys)]
        ob, oa = out[0, :level], out[1, :level]
        if kind == "rotate":
            g = pow(5, step % (n // 2), 2 * n)
            return nb.make_request(level, x[:level], ob, oa, kb, ka, c0=self.c0[i % self.c0.shape[0]][:level],
                                   automorphism=g)
        if kind == "relin":
            return nb.make_request(level, x[:level], ob, oa, kb, ka, add_b=ob, add_a=oa)
        return nb.make_request(level, x[:level], ob, oa, kb, ka)


def serve_poisson(nb, srv, jobs, rate, seed):
    """Submit jobs [(ctx, request)] at seeded Poisson arrival times of `rate` per second, wait for all."""
    import numpy as np
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, len(jobs))
    srv.stats(reset=True)
    tickets = []
    t_next = time.perf_counter()
    for (ctx, req), gap in zip(jobs, gaps):
        t_next += gap
        while True:
            now = time.perf_counter()
            if now >= t_next:
                break
            if t_next - now > 3e-4:
                time.sleep(t_next - now - 2e-4)
        tickets.append(srv.submit(ctx, req))
    waves = [srv.wait(t).wave_size for t in tickets]
    st = srv.stats(reset=True)
    return {"offered_per_s": rate, "throughput": st["throughput"], "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"],
            "max_ms": st["max_ms"], "mean_queue_ms": st["mean_queue_ms"], "mean_wave": sum(waves) / len(waves),
            "requests": len(jobs)}


def serving_legs(nb, device, batched_value, plain_value, seed=0x5E7E):
    """Served (continuous batching) vs plain (same kernels, one request per wave, one lane)."""
    import numpy as np

    from ntt_gpu_b200.params import synthetic_params
    budget = 40 << 30
    # Served: 4 lanes, 2 waves deep, and a new wave only while the waves in flight hold
    # less than 512 MiB of workspace (about four requests at the headline shape), so
    # small mixed requests run many at a time and large ones gather into full waves.
    served_cfg = {"lanes": 4, "max_batch": BATCH, "depth": 2, "hbm_budget_bytes": budget,
                  "max_inflight_bytes": 512 << 20}
    plain_cfg = {"lanes": 1, "max_batch": 1, "depth": 2, "hbm_budget_bytes": budget, "max_inflight_bytes": 0}
    legs = (("served", served_cfg), ("plain", plain_cfg))
    out = {"served_server": served_cfg,
           "plain_server": dict(plain_cfg, note="same kernels, one request per wave, the next request queued "
                                                "behind the running one on one stream"),
           "arrivals": f"seeded Poisson (numpy default_rng, seed {seed:#x})"}
    # (1) the headline shape: N=2^16, L=24, dnum=3, K=8, key switches.
    prm = synthetic_params(N, LEVEL, K_P, DNUM)
    w = Workload(nb, prm, device, seed)
    head = []
    rates = sorted({round(plain_value * f) for f in (0.5, 0.9, 1.3)} | {round(batched_value * 0.9)})
    # Each lane's arena is sized up front for the largest wave it can carry, so no
    # arena grows (and waits on the driver for memory) while requests are timed.
    wave_bytes = {b: w.ctx.requests_workspace_bytes([w.request(nb, LEVEL, "switch", 0, i) for i in range(b)])
                  for b in (1, BATCH)}
    for rate in rates:
        row = {}
        for name, cfg in legs:
            srv = nb.Server(device=device, **cfg)
            srv.reserve(wave_bytes[cfg["max_batch"]])
            count = max(64, min(400, int(rate * 0.12)))
            jobs = [(w.ctx, w.request(nb, LEVEL, "switch", 0, i)) for i in range(count)]
            # Warm-up: a burst sizes every lane's workspace arena for full waves.
            serve_poisson(nb, srv, jobs[:2 * BATCH * cfg["lanes"]], 1e7, seed + 1)
            row[name] = serve_poisson(nb, srv, jobs, rate, seed)
            srv.close()
        head.append(row)
    out["headline"] = {"workload": "key switches at N=2^16, L=24 (55-bit), K=8 (60-bit), dnum=3",
                       "rates": head}
    w.ctx.close()
    del w
    # (2) the mixed serving workload: N in 2^13..2^16, dnum in {2,3,4}, L in 4..32, K = alpha = ceil(32/dnum),
    #     key switch / relinearize / rotate by +-1..+-64.
    works = {}
    for logn in (13, 14, 15, 16):
        for dnum in (2, 3, 4):
            alpha = -(-32 // dnum)
            works[(logn, dnum)] = Workload(nb, synthetic_params(1 << logn, 32, alpha, dnum), device,
                                           seed + 97 * logn + dnum, ring=80)
    keys = list(works)
    kinds = ("switch", "relin", "rotate")

    def mixed_jobs(count, s):
        r = np.random.default_rng(s)
        jobs = []
        for i in range(count):
            wk = works[keys[r.integers(len(keys))]]
            level = int(r.integers(4, 33))
            kind = kinds[r.integers(3)]
            step = int(r.integers(1, 65)) * (1 if r.integers(2) else -1)
            jobs.append((wk.ctx, wk.request(nb, level, kind, step, i)))
        return jobs

    mixed_bytes = {b: max(wk.ctx.requests_workspace_bytes([wk.request(nb, 32, "rotate", 1, i) for i in range(b)])
                          for wk in works.values()) for b in (1, BATCH)}
    srv = nb.Server(device=device, **served_cfg)
    srv.reserve(mixed_bytes[served_cfg["max_batch"]])
    burst = mixed_jobs(600, seed + 3)
    serve_poisson(nb, srv, burst[:40], 1e6, seed + 4)
    cap = serve_poisson(nb, srv, burst, 1e7, seed + 5)["throughput"]  # saturation: all arrive at once
    srv.close()
    mixed = []
    for frac in (0.5, 0.9):
        rate = cap * frac
        row = {}
        for name, cfg in legs:
            srv = nb.Server(device=device, **cfg)
            srv.reserve(mixed_bytes[cfg["max_batch"]])
            jobs = mixed_jobs(max(100, min(600, int(rate * 0.25))), seed + 7)
            serve_poisson(nb, srv, burst[:2 * BATCH * cfg["lanes"]], 1e7, seed + 6)  # warm-up burst
            row[name] = serve_poisson(nb, srv, jobs, rate, seed + 8)
            srv.close()
        mixed.append(row)
    out["mixed"] = {"workload": "N in {2^13..2^16}, dnum in {2,3,4}, L uniform in 4..32, K = alpha = ceil(32/dnum), "
                                "key switch / relinearize / rotate (steps +-1..+-64), uniform residues, resident "
                                "ciphertexts and keys",
                    "served_saturation_per_s": cap, "rates": mixed}
    for wk in works.values():
        wk.ctx.close()
    return out


def run_ours(args, rank, world, local):
    import torch

    import ntt_gpu_b200 as nb
    from ntt_gpu_b200.params import synthetic_params, uniform_residues

    device = local
    torch.cuda.set_device(device)
    for item in args.tune:
        name, value = item.split("=", 1)
        nb.tuning_set(name, int(value))
    dev = torch.device(f"cuda:{device}")
    B = args.batch
    prm = synthetic_params(N, LEVEL, K_P, DNUM)
    ctx = nb.Context(prm.n, prm.q, prm.q_psi, prm.p, prm.p_psi, prm.alpha, device)
    ctx.prepare(LEVEL)
    T = LEVEL + K_P
    beta = prm.digits(LEVEL)
    x = uniform_residues(N, prm.q, SEED + 1000 * rank, polys=B)
    kb = uniform_residues(N, prm.q + prm.p, SEED + 1, polys=prm.full_digits())
    ka = uniform_residues(N, prm.q + prm.p, SEED + 2, polys=prm.full_digits())
    d_x, d_kb, d_ka = nb.to_device(x, device), nb.to_device(kb, device), nb.to_device(ka, device)
    out_b = torch.empty((B, LEVEL, N), dtype=torch.int64, device=dev)
    out_a = torch.empty_like(out_b)
    ws = ctx.workspace(nb.OP_KEYSWITCH, LEVEL, B)
    stream = torch.cuda.current_stream(dev)

    d_c0 = nb.to_device(uniform_residues(N, prm.q, SEED + 3 + 1000 * rank, polys=B), device) if args.rotate else None

    def step():
        ctx.keyswitch_batch(LEVEL, B, out_b, out_a, d_x, d_kb, d_ka, ws, c0=d_c0,
                            automorphism=5 if args.rotate else 0, stream=stream)

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize(dev)

    # ---- timed region: K batched steps --------------------------------------------------------
    clocks = ClockSampler(device)
    clocks.start()
    barrier(world)
    torch.cuda.synchronize(dev)
    nb.timing_reset()
    nb.timing_enable(True)
    launches0 = nb.kernel_launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    barrier(world)
    launches = nb.kernel_launches() - launches0
    nb.timing_enable(False)
    clock_info = clocks.stop()
    ms = max_over_ranks(e0.elapsed_time(e1), world, dev)
    kernels = {}
    for name in nb.KERNEL_CLASSES:
        count, total = nb.timing_query(name)
        if count:
            kernels[name] = {"launches": count, "total_ms": total, "avg_ms": total / count}
    nb.timing_reset()
    value = B * args.steps * world / (ms / 1000.0)

    # ---- roofline: the dominant kernel class of the step ------------------------------------------------
    # Algorithmic bytes per step and class: each kernel's own input and output words (W = 8N per tower;
    # twiddle, Shoup and CRT tables excluded). A two-pass NTT writes its intermediate in the first pass and
    # reads it in the second, so each pass reads and writes every tower once; the ModDown row pass also reads
    # the epilogue's operand. The fused row pass + key multiplication reads the digits' column-pass outputs,
    # the input's own towers and the shared key rows once, and writes both output channels; on the P towers
    # it also runs the ModDown's inverse row pass before storing (no extra I/O), so the separate inverse row
    # pass then only transforms the inputs. A conversion reads its s sources and writes its t targets.
    W = 8 * N
    fused = "row_mac" in kernels
    p_rows_fused = fused and beta >= 2 and nb.tuning_get("row_mac_inv_rows") != 0
    digit_towers = B * (beta * T - LEVEL)          # digit towers the inputs transform
    fwd_towers_per_step = digit_towers + 2 * B * LEVEL
    inv_towers_per_step = B * (LEVEL + 2 * K_P)
    inv_row_towers_per_step = B * LEVEL + (0 if p_rows_fused else 2 * B * K_P)
    bytes_per_step = {
        "ntt_fwd_col": 2 * fwd_towers_per_step * W,
        "ntt_fwd_row": (3 * 2 * B * LEVEL + (0 if fused else 2 * digit_towers)) * W,
        "ntt_inv_row": 2 * inv_row_towers_per_step * W,
        "ntt_inv_col": 2 * inv_towers_per_step * W,
        "conv": (beta * B * T + 2 * B * (K_P + LEVEL)) * W,
        "row_mac": (digit_towers + B * LEVEL + 2 * beta * T + 2 * B * T) * W,
        "mac": (digit_towers + B * LEVEL + 2 * beta * T + 2 * B * T) * W,
    }
    peak, peak_kind = peaks()
    classes = {}
    for name, nbytes in bytes_per_step.items():
        if name in kernels:
            ms_step = kernels[name]["total_ms"] / args.steps
            gbs = nbytes / (ms_step / 1000.0) / 1e9
            classes[name] = {"algorithmic_bytes_per_step": nbytes, "ms_per_step": ms_step, "achieved_gbs": gbs,
                             "frac_of_hbm_peak": gbs / peak}
    roof = None
    if classes:
        top = max(classes, key=lambda k: classes[k]["ms_per_step"])
        c = classes[top]
        launches_per_step = kernels[top]["launches"] / args.steps
        traffic = None
        tpath = os.path.join(ROOT, "profiles", "dram_traffic.json")
        if os.path.exists(tpath):
            with open(tpath) as f:
                tr = json.load(f).get(top)
            if tr:  # measured DRAM bytes per algorithmic byte (ncu, small case), scaled to this launch
                traffic = tr["dram_per_algorithmic_byte"] * c["algorithmic_bytes_per_step"] / launches_per_step
        roof = {"bound": "hbm", "achieved": c["achieved_gbs"], "peak": peak, "unit": "GB/s",
                "frac": c["frac_of_hbm_peak"], "traffic": traffic, "peak_source": peak_kind, "kernel": top,
                "algorithmic_bytes_per_launch": c["algorithmic_bytes_per_step"] / launches_per_step,
                "units": "W = 524288 B per tower; see classes for every kernel class of the step"}
        # The ceiling that binds the NTT passes: the integer multiply pipe, calibrated on this GPU by
        # register-only mode-2 butterflies (the NTT's own arithmetic, no memory traffic).
        rate = nb.butterfly_rate(device)
        fwd_ms = sum(kernels[k]["total_ms"] for k in ("ntt_fwd_col", "ntt_fwd_row") if k in kernels) / args.steps
        passes_fwd = (fwd_towers_per_step + 2 * B * LEVEL + (0 if fused else digit_towers)) * (N // 2) * 8
        roof["compute"] = {"bound": "integer multiply pipe (mode-2 butterflies)",
                           "kernel": "ntt_fwd_col + ntt_fwd_row (forward NTT passes outside the fused kernel)",
                           "achieved": passes_fwd / (fwd_ms / 1000.0), "peak": rate, "unit": "butterflies/s",
                           "frac": passes_fwd / (fwd_ms / 1000.0) / rate,
                           "peak_source": "ntt_b200_butterfly_rate: register-only mode-2 butterflies, this GPU"}
        roof["classes"] = classes
    total_kernel_ms = sum(k["total_ms"] for k in kernels.values()) or 1.0
    for k in kernels.values():
        k["share"] = k["total_ms"] / total_kernel_ms

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "n": N, "level": LEVEL, "dnum": DNUM, "alpha": prm.alpha, "k": K_P,
                       "batch_per_gpu": B, "global_batch": B * world,
                       "parallelism": f"replicas x{world} (request-level sharding, no collective)",
                       "l2": "inputs, keys, outputs and workspace (~3 GB) exceed the 126 MB L2; no flush"},
            "gpu_launches": launches, "roofline": roof, "clocks": clock_info, "kernels": kernels,
            "ntt_towers_per_step": {"forward": fwd_towers_per_step, "inverse": inv_towers_per_step},
            "key_multiplication": "fused into the digits' forward row pass" if fused else "separate MAC pass"}
    if args.kernels_only:
        ctx.close()
        return line

    # ---- plain path: one request at a time (per-request latency) -------------------------------------
    ws1 = ctx.workspace(nb.OP_KEYSWITCH, LEVEL, 1)
    lat = []
    torch.cuda.synchronize(dev)
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    per = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(B)]
    plain_steps = max(1, min(args.steps, 10))
    p0.record(stream)
    for s in range(plain_steps):
        for r in range(B):
            if s == plain_steps - 1:
                per[r][0].record(stream)
            ctx.keyswitch(LEVEL, out_b[r], out_a[r], d_x[r], d_kb, d_ka, ws1, stream=stream)
            if s == plain_steps - 1:
                per[r][1].record(stream)
    p1.record(stream)
    torch.cuda.synchronize(dev)
    plain_ms = max_over_ranks(p0.elapsed_time(p1), world, dev)
    lat = sorted(a.elapsed_time(b) for a, b in per)
    plain = {"value": B * plain_steps * world / (plain_ms / 1000.0), "unit": UNIT,
             "latency_p50_ms": statistics.median(lat),
             "latency_p99_ms": lat[min(len(lat) - 1, int(round(0.99 * (len(lat) - 1))))],
             "note": "same kernels, one request per call, back to back on one stream"}

    # ---- end to end through the public API with host buffers -----------------------------------------
    # ntt_b200_keyswitch_host_async: pinned host inputs and outputs; each step's batch runs in chunks whose
    # copies to and from the device overlap each other and the kernels, and the next step starts while the
    # last outputs are still leaving; ntt_b200_keyswitch_host_wait joins the caller's stream at the end of
    # the timed region. The timed region holds every step's host->device copy of its inputs and
    # device->host copy of both outputs. The synchronous form (the stream waits for each step's outputs)
    # is timed the same way and reported beside it.
    h_x = torch.from_numpy(x.view("int64")).pin_memory()
    h_b = torch.empty((B, LEVEL, N), dtype=torch.int64).pin_memory()
    h_a = torch.empty_like(h_b).pin_memory()
    e2e_steps = max(3, min(args.steps, 10))
    chunk = args.e2e_chunk
    ws_host = ctx.host_workspace(LEVEL, chunk)

    def e2e_run(steps, wait):
        for _ in range(steps):
            ctx.keyswitch_host(LEVEL, B, chunk, h_x, h_b, h_a, d_kb, d_ka, ws_host, stream=stream, wait=wait)
        ctx.keyswitch_host_wait(stream)

    def e2e_time(wait):
        e2e_run(3, wait)
        barrier(world)
        torch.cuda.synchronize(dev)
        q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        q0.record(stream)
        e2e_run(e2e_steps, wait)
        q1.record(stream)
        torch.cuda.synchronize(dev)
        return max_over_ranks(q0.elapsed_time(q1), world, dev)

    e2e_sync_ms = e2e_time(True)
    e2e_ms = e2e_time(False)
    ref_b = torch.empty_like(out_b)
    ctx.keyswitch_batch(LEVEL, B, ref_b, out_a, d_x, d_kb, d_ka, ws, stream=stream)
    torch.cuda.synchronize(dev)
    e2e_exact = bool(torch.equal(ref_b.cpu(), h_b))
    e2e = {"value": B * e2e_steps * world / (e2e_ms / 1000.0), "unit": UNIT,
           "h2d_bytes_per_step": int(h_x.numel() * 8), "d2h_bytes_per_step": int((h_b.numel() + h_a.numel()) * 8),
           "steps": e2e_steps,
           "api": f"ntt_b200_keyswitch_host_async per step + ntt_b200_keyswitch_host_wait, pinned host buffers, "
                  f"chunks of {chunk}",
           "synchronous_value": B * e2e_steps * world / (e2e_sync_ms / 1000.0),
           "outputs_equal_device_path": e2e_exact}
    # The copy bound of that number: the same step's bytes moved by plain pinned copies alone, the outputs
    # device-to-host while the inputs go host-to-device on another stream (no kernels).
    s_in, s_out = torch.cuda.Stream(dev), torch.cuda.Stream(dev)

    def copies_only():
        with torch.cuda.stream(s_in):
            d_x.copy_(h_x, non_blocking=True)
        with torch.cuda.stream(s_out):
            h_b.copy_(out_b, non_blocking=True)
            h_a.copy_(out_a, non_blocking=True)

    for _ in range(2):
        copies_only()
    torch.cuda.synchronize(dev)
    c0_ = time.perf_counter()
    for _ in range(e2e_steps):
        copies_only()
    torch.cuda.synchronize(dev)
    copy_s = (time.perf_counter() - c0_) / e2e_steps
    e2e["copy_bound"] = {"value": B * world / copy_s, "unit": UNIT, "ms_per_step": copy_s * 1e3,
                         "note": "pinned copies of the step's inputs and outputs only, both directions at once"}
    e2e["frac_of_copy_bound"] = e2e["value"] / e2e["copy_bound"]["value"]

    line["e2e"] = e2e
    line["plain"] = plain
    line["plain_keyswitch_per_s"] = plain["value"]
    line["plain_p50_ms"], line["plain_p99_ms"] = plain["latency_p50_ms"], plain["latency_p99_ms"]
    line["configs"] = config_legs(nb, device, *peaks())
    # the metric's "NTT HBM GB/s": config 2 (8 x 32 towers forward + inverse, CUDA-graph replay), 2W per
    # tower-transform, and its fraction of the HBM peak the line uses
    c2 = line["configs"]["config2"]["graph_replay"]
    line["ntt_hbm_gbs"], line["ntt_hbm_frac"] = c2["gb_s"], c2["frac_of_hbm_peak"]
    if not args.no_serving:
        line["serving"] = serving_legs(nb, device, value, plain["value"])
        # the metric's "served vs plain, p50/p99" at its own shape: the 0.9 x batched-capacity arrival rate
        head = line["serving"]["headline"]["rates"][-1]
        line["served_keyswitch_per_s"] = head["served"]["throughput"]
        line["served_p50_ms"], line["served_p99_ms"] = head["served"]["p50_ms"], head["served"]["p99_ms"]
        line["served_offered_per_s"] = head["served"]["offered_per_s"]
        line["plain_server_keyswitch_per_s"] = head["plain"]["throughput"]
        line["plain_server_p99_ms"] = head["plain"]["p99_ms"]
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_single(prm)
    ctx.close()
    return line


def main():
    args = parse()
    if args.impl == "reference":
        # Rank 0 alone times the CPU reference; other ranks exit without work.
        rank = int(os.environ.get("RANK", "0"))
        line = run_reference(args, rank, int(os.environ.get("WORLD_SIZE", "1")))
    else:
        rank, world, local = dist_setup()
        try:
            line = run_ours(args, rank, world, local)
        finally:
            dist_teardown(world)
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
