"""Autotuner for the launch choices of libntt_b200 (one B200, CUDA events).

Every tunable (ntt_b200_tuning_name) is a launch choice that never changes a
result: the register budget each NTT pass is compiled for (3 or 4 resident
CTAs per SM), whether the row passes stage their twiddles in shared memory, the
conversion kernel (tensor cores, 30-bit limbs or 128-bit accumulators) and its
tiles per CTA, the MAC kernel, and whether the key multiplication runs inside
the digits' row pass (and the ModDown's inverse row pass inside that). The tuner
runs coordinate descent over them on two workloads:

  * ntt:       forward + inverse NTT of 8 polynomials x 32 towers at N = 2^16
               (50/60-bit primes), one launch sequence per direction;
  * keyswitch: batched Hybrid key switch of 16 components at N = 2^16, L = 24,
               K = 8, dnum = 3.

Each candidate is timed with the library's per-kernel CUDA-event timing
(ntt_b200_timing_*), so each choice is measured by the device time of the pass it affects.
The choices and every measurement are written to ntt_gpu_b200/tuning.json,
which ntt_gpu_b200.load() applies.

    python -m ntt_gpu_b200.autotune [--out PATH] [--iters N]
"""
from __future__ import annotations

import argparse
import json
import os

from . import TUNING


def _device_ms(nb, torch, fn, iters, kernels):
    """Summed device milliseconds per call of the given kernel classes."""
    for _ in range(3):
        fn()
    torch.cuda.synchronize()
    nb.timing_reset()
    nb.timing_enable(True)
    for _ in range(iters):
        fn()
    torch.cuda.synchronize()
    nb.timing_enable(False)
    out = {k: nb.timing_query(k)[1] / iters for k in kernels}
    nb.timing_reset()
    return out


def run(out_path: str = TUNING, iters: int = 10) -> dict:
    import torch

    import ntt_gpu_b200 as nb
    from ntt_gpu_b200.params import find_primes, find_psi, synthetic_params, uniform_residues

    nb.load()
    n = 1 << 16
    # ---- workload 1: batched NTT ------------------------------------------------------------
    q = [v for pair in zip(find_primes(n, 16, 50), find_primes(n, 16, 60)) for v in pair]
    tctx = nb.Context(n, q, [find_psi(v, n) for v in q])
    x = nb.to_device(uniform_residues(n, q, 7, polys=8))
    y = nb.empty(tuple(x.shape))
    ids = list(range(32))

    def ntt_step():
        tctx.ntt(y, x, ids, polys=8, poly_stride=32 * n)
        tctx.ntt(y, y, ids, polys=8, poly_stride=32 * n, inverse=True)

    # ---- workload 2: batched key switch -----------------------------------------------------
    prm = synthetic_params(n, 24, 8, 3)
    kctx = nb.Context(prm.n, prm.q, prm.q_psi, prm.p, prm.p_psi, prm.alpha)
    kctx.prepare(24)
    batch = 16
    xs = nb.to_device(uniform_residues(n, prm.q, 9, polys=batch))
    kb = nb.to_device(uniform_residues(n, prm.q + prm.p, 1, polys=prm.full_digits()))
    ka = nb.to_device(uniform_residues(n, prm.q + prm.p, 2, polys=prm.full_digits()))
    ob, oa = nb.empty((batch, 24, n)), nb.empty((batch, 24, n))
    ws = kctx.workspace(nb.OP_KEYSWITCH, 24, batch)

    def ks_step():
        kctx.keyswitch_batch(24, batch, ob, oa, xs, kb, ka, ws)

    # tunable -> (candidates, workload, kernel classes whose device time decides it, tunables pinned
    # while it is measured). The CUDA-core conversion choices serve the plans the tensor-core form
    # does not take (more than 16 sources, moduli outside [2^48, 2^61)), so they are measured with it off.
    cuda_core_conv = {"conv_tc": 0}
    # The separate MAC's choices serve the key switches the fused row pass does not take (mode 0/1
    # contexts, more than 4 digits), so they are measured with it off.
    unfused_mac = {"row_mac": 0}
    plan = [
        ("ntt_minb_fwd_col", (3, 4), ntt_step, ("ntt_fwd_col",), {}),
        ("ntt_minb_fwd_row", (3, 4), ntt_step, ("ntt_fwd_row",), {}),
        ("ntt_minb_inv_row", (3, 4), ntt_step, ("ntt_inv_row",), {}),
        ("ntt_minb_inv_col", (3, 4), ntt_step, ("ntt_inv_col",), {}),
        ("ntt_col_direct", (0, 1), ntt_step, ("ntt_fwd_col", "ntt_inv_col"), {}),
        ("ntt_row_direct", (0, 1), ntt_step, ("ntt_fwd_row", "ntt_inv_row"), {}),
        ("ntt_epi_stage", (0, 1), ks_step, ("ntt_fwd_row",), {}),
        ("intt_unscaled", (0, 1), ks_step, ("ntt_inv_col",), {}),
        ("digits_lazy", (0, 1), ks_step, ("ntt_fwd_row", "mac"), unfused_mac),
        ("ntt_stage_tw_fwd_row", (0, 1), ntt_step, ("ntt_fwd_row",), {}),
        ("ntt_stage_tw_inv_row", (0, 1), ntt_step, ("ntt_inv_row",), {}),
        ("ntt_cluster", (0, 1), ntt_step, ("ntt_fwd_col", "ntt_fwd_row", "ntt_fwd_cluster"), {}),
        ("conv_limbs", (0, 1), ks_step, ("conv",), cuda_core_conv),
        ("conv_blocks_per_sm", (4, 8, 16), ks_step, ("conv",), cuda_core_conv),
        ("mac_limbs", (0, 1), ks_step, ("mac",), unfused_mac),
        ("mac_approx", (0, 1), ks_step, ("mac",), {"mac_limbs": 0, **unfused_mac}),
        ("conv_tc", (0, 1), ks_step, ("conv",), {}),
        ("conv_tc_fixed", (0, 1), ks_step, ("conv",), {"conv_tc": 1}),
        ("conv_tc_tiles", (1, 2, 4, 8), ks_step, ("conv",), {"conv_tc": 1}),
        ("row_mac", (0, 1), ks_step, ("ntt_fwd_row", "mac", "row_mac", "ntt_inv_row"), {}),
        ("row_mac_inv_rows", (0, 1), ks_step, ("row_mac", "ntt_inv_row"), {"row_mac": 1}),
    ]
    measurements, choices = {}, {}
    for name, candidates, step, kernels, pinned in plan:
        saved = {k: nb.tuning_get(k) for k in pinned}
        for k, v in pinned.items():
            nb.tuning_set(k, v)
        times = {}
        for value in candidates:
            nb.tuning_set(name, value)
            times[value] = sum(_device_ms(nb, torch, step, iters, kernels).values())
        best = min(times, key=times.get)
        nb.tuning_set(name, best)
        for k, v in saved.items():
            nb.tuning_set(k, v)
        choices[name] = best
        measurements[name] = {"measured_by": list(kernels), "pinned": dict(pinned),
                              "device_ms_per_call": {str(k): v for k, v in times.items()}}

    def total(step):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for _ in range(3):
            step()
        e0.record()
        for _ in range(iters):
            step()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / iters

    result = {
        "device": torch.cuda.get_device_name(0),
        "sm_count": torch.cuda.get_device_properties(0).multi_processor_count,
        "workloads": {
            "ntt": "forward + inverse NTT, 8 polynomials x 32 towers (16 x 50-bit, 16 x 60-bit), N = 2^16",
            "keyswitch": "batched Hybrid key switch, 16 components, N = 2^16, L = 24, K = 8, dnum = 3",
        },
        "choices": choices,
        "measurements": measurements,
        "tuned_ms_per_call": {"ntt": total(ntt_step), "keyswitch": total(ks_step)},
    }
    tctx.close()
    kctx.close()
    with open(out_path, "w") as f:
        json.dump(result, f, indent=1)
        f.write("\n")
    return result


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=TUNING)
    ap.add_argument("--iters", type=int, default=10)
    args = ap.parse_args()
    res = run(os.path.abspath(args.out), args.iters)
    print(json.dumps(res["choices"]), json.dumps(res["tuned_ms_per_call"]))


if __name__ == "__main__":
    main()
