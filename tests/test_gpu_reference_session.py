"""The drop-in, run: the reference's own resident Session over the B200 driver.

oracle/_ref/libntt_ref_b200.so is minnow54426/ntt-gpu's src/resident.cpp,
compiled unchanged from the reference tree, over this repository's Driver
binding (ntt_gpu_b200/binding/resident_b200.cpp) and libntt_b200.so
(oracle/Makefile, target refb200). Through make_cuda_session the reference's
Session runs mod_up (both domains), mod_down, hybrid_digits,
upload_hybrid_key + hybrid_accumulate + mod_down (key switch),
hybrid_rotate_extended (rotation), multiply, download and close on the B200
kernels; every output must equal the oracle (or, at N = 65536, the digests of
the reference's own CPU chain). Skipped where that library was not built (no
reference tree at build time)."""
import ctypes
import os

import numpy as np
import pytest

import golden_cases as gc
import ntt_gpu_b200 as nb
from oracle.oracle import LCG_SEED, pinned_context, synthetic_context

pytestmark = pytest.mark.gpu

_LIB = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                    "libntt_ref_b200.so")
_U64P = ctypes.POINTER(ctypes.c_uint64)


class _Ctx(ctypes.Structure):
    _fields_ = [("n", ctypes.c_uint64), ("q", _U64P), ("q_psi", _U64P), ("m", ctypes.c_size_t),
                ("p", _U64P), ("p_psi", _U64P), ("k", ctypes.c_size_t), ("alpha", ctypes.c_size_t),
                ("device", ctypes.c_int)]


def _p(a):
    return a.ctypes.data_as(_U64P) if a is not None else None


class RefSession:
    def __init__(self):
        nb.load()  # the binding resolves against this process's libntt_b200.so
        self.lib = ctypes.CDLL(_LIB)
        self.lib.refsess_last_error.restype = ctypes.c_char_p

    def _ctx(self, ctx, device=0):
        self._keep = [np.array(v, dtype=np.uint64) for v in (ctx.q, ctx.q_psi, ctx.p, ctx.p_psi)]
        q, qp, p, pp = self._keep
        return _Ctx(ctx.n, _p(q), _p(qp), len(ctx.q), _p(p), _p(pp), len(ctx.p), ctx.alpha, device)

    def _call(self, name, *args):
        rc = getattr(self.lib, name)(*args)
        if rc != 0:
            raise RuntimeError(self.lib.refsess_last_error().decode())

    def mod_up(self, ctx, level, x, is_eval):
        out = np.zeros((level + ctx.k, ctx.n), dtype=np.uint64)
        c = self._ctx(ctx)
        self._call("refsess_mod_up", ctypes.byref(c), ctypes.c_size_t(level), _p(np.ascontiguousarray(x)),
                   ctypes.c_int(is_eval), _p(out))
        return out

    def mod_down(self, ctx, level, y):
        out = np.zeros((level, ctx.n), dtype=np.uint64)
        c = self._ctx(ctx)
        self._call("refsess_mod_down", ctypes.byref(c), ctypes.c_size_t(level), _p(np.ascontiguousarray(y)), _p(out))
        return out

    def digits(self, ctx, level, x):
        out = np.zeros((ctx.digits(level), level + ctx.k, ctx.n), dtype=np.uint64)
        c = self._ctx(ctx)
        self._call("refsess_digits", ctypes.byref(c), ctypes.c_size_t(level), _p(np.ascontiguousarray(x)), _p(out))
        return out

    def keyswitch(self, ctx, level, x, kb, ka, c0=None, g=0):
        ob, oa = np.zeros((level, ctx.n), dtype=np.uint64), np.zeros((level, ctx.n), dtype=np.uint64)
        ops = ctypes.c_uint64()
        c = self._ctx(ctx)
        self._call("refsess_keyswitch", ctypes.byref(c), ctypes.c_size_t(level), _p(np.ascontiguousarray(x)),
                   _p(np.ascontiguousarray(kb)), _p(np.ascontiguousarray(ka)),
                   _p(None if c0 is None else np.ascontiguousarray(c0)), ctypes.c_uint32(g), _p(ob), _p(oa),
                   ctypes.byref(ops))
        return ob, oa, ops.value

    def multiply(self, ctx, level, a, b):
        out = np.zeros(a.shape, dtype=np.uint64)
        c = self._ctx(ctx)
        self._call("refsess_multiply", ctypes.byref(c), ctypes.c_size_t(level), _p(np.ascontiguousarray(a)),
                   _p(np.ascontiguousarray(b)), _p(out))
        return out

    def open(self, ctx, level, device):
        c = self._ctx(ctx)
        self._call("refsess_open", ctypes.byref(c), ctypes.c_size_t(level), ctypes.c_int(device))


@pytest.fixture(scope="module")
def rs():
    if not os.path.exists(_LIB):
        pytest.skip("the reference Session over the B200 binding was not built (no reference tree)")
    return RefSession()


def _ring_product(orc, mods, psis, a, b):
    fa, fb = orc.ntt(a, mods, psis), orc.ntt(b, mods, psis)
    prod = np.stack([np.array([orc.mul(int(x), int(y), q) for x, y in zip(fa[t], fb[t])], dtype=np.uint64)
                     for t, q in enumerate(mods)])
    return orc.ntt(prod, mods, psis, inverse=True)


@pytest.mark.parametrize("shape", ["pinned", "small"])
def test_reference_session_over_b200_driver(lib, orc, rs, shape):
    ctx = pinned_context() if shape == "pinned" else synthetic_context(orc, 1024, 7, 3, 3)
    kb, ka = gc.full_keys(orc, ctx, 21)
    for level in ((5, 3, 1) if shape == "pinned" else (7, 4)):
        x = orc.lcg(ctx.n, ctx.q[:level], LCG_SEED + level)
        y = orc.lcg(ctx.n, ctx.qp_moduli(level), 77 + level)
        c0 = orc.lcg(ctx.n, ctx.q[:level], 9 + level)
        np.testing.assert_array_equal(rs.mod_up(ctx, level, x, 0), orc.mod_up(ctx, level, x, 0))
        np.testing.assert_array_equal(rs.mod_up(ctx, level, x, 1), orc.mod_up(ctx, level, x, 1))
        np.testing.assert_array_equal(rs.mod_down(ctx, level, y), orc.mod_down(ctx, level, y))
        np.testing.assert_array_equal(rs.digits(ctx, level, x), orc.hybrid_digits(ctx, level, x))
        b, a, ops = rs.keyswitch(ctx, level, x, kb, ka)
        wb, wa = orc.keyswitch(ctx, level, x, kb, ka)
        np.testing.assert_array_equal(b, wb)
        np.testing.assert_array_equal(a, wa)
        assert ops > 0
        b, a, _ = rs.keyswitch(ctx, level, x, kb, ka, c0, 5)
        wb, wa = orc.keyswitch(ctx, level, x, kb, ka, c0, 5)
        np.testing.assert_array_equal(b, wb)
        np.testing.assert_array_equal(a, wa)
    if shape == "small":
        level = 4
        mods = ctx.qp_moduli(level)
        psis = (ctx.q_psi[:level] + ctx.p_psi)
        a_ = orc.lcg(ctx.n, mods, 101)
        b_ = orc.lcg(ctx.n, mods, 102)
        np.testing.assert_array_equal(rs.multiply(ctx, level, a_, b_), _ring_product(orc, mods, psis, a_, b_))


def test_reference_session_full_size_digests(lib, orc, rs):
    """N = 65536, L = 24, dnum = 3: the reference's Session over the B200 driver
    gives the reference CPU chain's key switch and rotation (golden digests)."""
    d = gc.digests()
    for name, ctx, level, x, (kb, ka), c0, g in gc.full_size_cases(orc):
        if not name.startswith("bench_L24"):
            continue
        b, a, _ = rs.keyswitch(ctx, level, x, kb, ka, c0, g)
        assert gc.sha(b) == d[name + "_b"] and gc.sha(a) == d[name + "_a"], name


def test_transport_errors_reach_the_reference_session(lib, orc, rs):
    """A device the transport cannot open fails the session with the library's
    "CUDA: ..." error (the reference's runtime_error convention); nothing runs."""
    ctx = pinned_context()
    with pytest.raises(RuntimeError, match="CUDA"):
        rs.open(ctx, 3, 4096)
    rs.open(ctx, 3, 0)
