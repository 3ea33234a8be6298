"""ctypes binding of the CPU checker libraries (test infrastructure only).

`liboracle.so` is the plain-C restatement of the reference algorithms
(oracle.c); `_ref/libntt_ref.so`, when present, is the reference's own CPU
implementation compiled from its sources (ref_bridge.cpp + src/resident.cpp).
Only tests, the smoke check and the benchmark's CPU baseline import this
module; the product never does.

Arrays are numpy uint64 in limb-major layout: shape (towers, n).
"""
from __future__ import annotations

import ctypes
import os
import shutil
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_U64 = ctypes.c_uint64
_SZ = ctypes.c_size_t
_P = ctypes.c_void_p


def _ptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.uint64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_P)


def build(force: bool = False) -> None:
    """Compile liboracle.so (and oracle/_ref - the reference CPU library, its CUDA path and its
    Session over the B200 binding - when the reference tree exists)."""
    target = os.path.join(HERE, "liboracle.so")
    if force or not os.path.exists(target):
        subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    ref = os.path.join(HERE, "_ref", "libntt_ref.so")
    if force or not os.path.exists(ref):
        subprocess.run(["make", "-s", "-C", HERE, "ref"], check=True)
    # The reference's CUDA resident path (the second GPU comparator) needs nvcc.
    ref_cuda = os.path.join(HERE, "_ref", "libntt_ref_cuda.so")
    if (force or not os.path.exists(ref_cuda)) and shutil.which("nvcc"):
        subprocess.run(["make", "-s", "-C", HERE, "refcuda"], check=True)
    # The reference's own Session over this repository's Driver binding (needs libntt_b200.so).
    ref_b200 = os.path.join(HERE, "_ref", "libntt_ref_b200.so")
    if force or not os.path.exists(ref_b200):
        subprocess.run(["make", "-s", "-C", HERE, "refb200"], check=True)


class _Ctx(ctypes.Structure):
    _fields_ = [("n", _U64), ("m", _SZ), ("k", _SZ), ("alpha", _SZ),
                ("q", _P), ("q_psi", _P), ("p", _P), ("p_psi", _P)]


@dataclass
class Context:
    """Full CKKS context: M Q towers, K P towers, digit width alpha."""
    n: int
    q: list
    q_psi: list
    p: list
    p_psi: list
    alpha: int

    @property
    def m(self) -> int:
        return len(self.q)

    @property
    def k(self) -> int:
        return len(self.p)

    def digits(self, level: int) -> int:
        return 1 + (level - 1) // self.alpha

    def full_digits(self) -> int:
        return 1 + (self.m - 1) // self.alpha

    def qp_moduli(self, level: int) -> list:
        return list(self.q[:level]) + list(self.p)

    def _struct(self):
        arrays = [np.asarray(v, dtype=np.uint64) for v in (self.q, self.q_psi, self.p, self.p_psi)]
        s = _Ctx(self.n, self.m, self.k, self.alpha, *[a.ctypes.data_as(_P) for a in arrays])
        return s, arrays  # keep arrays alive


class Oracle:
    def __init__(self):
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        lib = ctypes.CDLL(path)
        self.lib = lib
        for name in ("orc_add_mod", "orc_sub_mod", "orc_mul_mod", "orc_pow_mod",
                     "orc_shoup_multiply", "orc_bit_reverse", "orc_find_psi", "orc_splitmix",
                     "orc_automorphism_source_index", "orc_barrett_multiply",
                     "orc_barrett_quotient"):
            getattr(lib, name).restype = _U64
        lib.orc_add_mod.argtypes = [_U64] * 3
        lib.orc_sub_mod.argtypes = [_U64] * 3
        lib.orc_mul_mod.argtypes = [_U64] * 3
        lib.orc_pow_mod.argtypes = [_U64] * 3
        lib.orc_inv_mod.argtypes = [_U64, _U64, ctypes.POINTER(_U64)]
        lib.orc_shoup_precompute.argtypes = [_U64, _U64, ctypes.POINTER(_U64)]
        lib.orc_shoup_multiply.argtypes = [_U64] * 4
        lib.orc_barrett_precompute.argtypes = [_U64, ctypes.POINTER(_U64), ctypes.POINTER(_U64)]
        lib.orc_barrett_multiply.argtypes = [_U64] * 5
        lib.orc_barrett_quotient.argtypes = [_U64] * 5
        lib.orc_bit_reverse.argtypes = [_U64, _U64]
        lib.orc_is_prime.argtypes = [_U64]
        lib.orc_find_primes.argtypes = [_U64, _U64, _U64, _P]
        lib.orc_find_psi.argtypes = [_U64, _U64]
        lib.orc_ntt_towers.argtypes = [_P, _U64, _SZ, _P, _P, ctypes.c_int]
        lib.orc_basis_convert.argtypes = [_P, _U64, _P, _SZ, _P, _SZ, _P]
        lib.orc_automorphism_source_index.argtypes = [_U64, _U64, _U64, ctypes.c_uint32]
        cp = ctypes.POINTER(_Ctx)
        lib.orc_context_check.argtypes = [cp, _SZ]
        lib.orc_mod_up.argtypes = [cp, _SZ, _P, ctypes.c_int, _P]
        lib.orc_mod_down.argtypes = [cp, _SZ, _P, _P]
        lib.orc_hybrid_digits.argtypes = [cp, _SZ, _P, _P]
        lib.orc_pack_key.argtypes = [cp, _SZ, _P, _P]
        lib.orc_hybrid_accumulate.argtypes = [cp, _SZ, _P, _P, _P, _P, _P]
        lib.orc_hybrid_rotate_extended.argtypes = [cp, _SZ, _P, _P, _P, ctypes.c_uint32, _P, _P]
        lib.orc_keyswitch.argtypes = [cp, _SZ, _P, _P, _P, _P, ctypes.c_uint32, _P, _P]
        lib.orc_lcg_fill.argtypes = [_P, _U64, _SZ, _P, _U64]
        lib.orc_splitmix.argtypes = [_U64]
        lib.orc_splitmix_fill.argtypes = [_P, _U64, _SZ, _P, _U64]

    # ---- scalar arithmetic -------------------------------------------------
    def add(self, a, b, q): return self.lib.orc_add_mod(a, b, q)
    def sub(self, a, b, q): return self.lib.orc_sub_mod(a, b, q)
    def mul(self, a, b, q): return self.lib.orc_mul_mod(a, b, q)
    def pow(self, a, e, q): return self.lib.orc_pow_mod(a, e, q)

    def inv(self, x, q):
        out = _U64()
        return None if self.lib.orc_inv_mod(x, q, ctypes.byref(out)) else out.value

    def shoup(self, x, w, q):
        wq = _U64()
        if self.lib.orc_shoup_precompute(w, q, ctypes.byref(wq)):
            return None
        return self.lib.orc_shoup_multiply(x, w, wq.value, q)

    def barrett_precompute(self, q):
        lo, hi = _U64(), _U64()
        if self.lib.orc_barrett_precompute(q, ctypes.byref(lo), ctypes.byref(hi)):
            return None
        return lo.value, hi.value

    def barrett(self, a, b, q):
        lohi = self.barrett_precompute(q)
        return None if lohi is None else self.lib.orc_barrett_multiply(a, b, q, *lohi)

    def barrett_estimate(self, a, b, q):
        lo, hi = self.barrett_precompute(q)
        prod = a * b
        return self.lib.orc_barrett_quotient(prod & (2**64 - 1), prod >> 64, q, lo, hi)

    def is_prime(self, n): return bool(self.lib.orc_is_prime(n))

    def find_primes(self, n, count, bits):
        out = np.zeros(count, dtype=np.uint64)
        if self.lib.orc_find_primes(n, count, bits, _ptr(out)):
            raise ValueError("prime search exhausted the bit range")
        return [int(v) for v in out]

    def find_psi(self, q, n): return int(self.lib.orc_find_psi(q, n))

    # ---- array operations ----------------------------------------------------
    def ntt(self, values: np.ndarray, q, psi, inverse=False) -> np.ndarray:
        v = np.ascontiguousarray(values, dtype=np.uint64).copy()
        towers, n = v.shape
        qa = np.asarray(q, dtype=np.uint64)
        pa = np.asarray(psi, dtype=np.uint64)
        if self.lib.orc_ntt_towers(_ptr(v), n, towers, _ptr(qa), _ptr(pa), int(inverse)):
            raise ValueError("invalid NTT parameters")
        return v

    def basis_convert(self, values: np.ndarray, source, target) -> np.ndarray:
        v = np.ascontiguousarray(values, dtype=np.uint64)
        n = v.shape[-1]
        out = np.zeros((len(target), n), dtype=np.uint64)
        s = np.asarray(source, dtype=np.uint64)
        t = np.asarray(target, dtype=np.uint64)
        if self.lib.orc_basis_convert(_ptr(v), n, _ptr(s), len(source), _ptr(t), len(target), _ptr(out)):
            raise ValueError("invalid basis conversion")
        return out

    def automorphism_source_index(self, k, n, g):
        return int(self.lib.orc_automorphism_source_index(k, n, int(n).bit_length() - 1, g))

    def mod_up(self, ctx: Context, level, values, is_eval):
        s, keep = ctx._struct()
        v = np.ascontiguousarray(values, dtype=np.uint64)
        out = np.zeros((level + ctx.k, ctx.n), dtype=np.uint64)
        if self.lib.orc_mod_up(ctypes.byref(s), level, _ptr(v), int(is_eval), _ptr(out)):
            raise ValueError("invalid ModUp")
        return out

    def mod_down(self, ctx: Context, level, values):
        s, keep = ctx._struct()
        v = np.ascontiguousarray(values, dtype=np.uint64)
        out = np.zeros((level, ctx.n), dtype=np.uint64)
        if self.lib.orc_mod_down(ctypes.byref(s), level, _ptr(v), _ptr(out)):
            raise ValueError("invalid ModDown")
        return out

    def hybrid_digits(self, ctx: Context, level, values):
        s, keep = ctx._struct()
        v = np.ascontiguousarray(values, dtype=np.uint64)
        out = np.zeros((ctx.digits(level), level + ctx.k, ctx.n), dtype=np.uint64)
        if self.lib.orc_hybrid_digits(ctypes.byref(s), level, _ptr(v), _ptr(out)):
            raise ValueError("invalid Hybrid digits")
        return out

    def keyswitch(self, ctx: Context, level, values, key_b, key_a, c0=None, automorphism=0):
        s, keep = ctx._struct()
        v = np.ascontiguousarray(values, dtype=np.uint64)
        kb = np.ascontiguousarray(key_b, dtype=np.uint64)
        ka = np.ascontiguousarray(key_a, dtype=np.uint64)
        c = None if c0 is None else np.ascontiguousarray(c0, dtype=np.uint64)
        ob = np.zeros((level, ctx.n), dtype=np.uint64)
        oa = np.zeros((level, ctx.n), dtype=np.uint64)
        if self.lib.orc_keyswitch(ctypes.byref(s), level, _ptr(v), _ptr(kb), _ptr(ka), _ptr(c),
                                  automorphism, _ptr(ob), _ptr(oa)):
            raise ValueError("invalid key switch")
        return ob, oa

    def lcg(self, n, moduli, seed) -> np.ndarray:
        out = np.zeros((len(moduli), n), dtype=np.uint64)
        m = np.asarray(moduli, dtype=np.uint64)
        self.lib.orc_lcg_fill(_ptr(out), n, len(moduli), _ptr(m), seed)
        return out

    def splitmix(self, n, moduli, seed) -> np.ndarray:
        out = np.zeros((len(moduli), n), dtype=np.uint64)
        m = np.asarray(moduli, dtype=np.uint64)
        self.lib.orc_splitmix_fill(_ptr(out), n, len(moduli), _ptr(m), seed)
        return out


class Reference:
    """The reference's own CPU implementation (oracle/_ref), when built."""

    PATH = os.path.join(HERE, "_ref", "libntt_ref.so")

    @classmethod
    def available(cls) -> bool:
        return os.path.exists(cls.PATH)

    def __init__(self):
        lib = ctypes.CDLL(self.PATH)
        self.lib = lib
        lib.ref_last_error.restype = ctypes.c_char_p
        for name in ("ref_add_mod", "ref_sub_mod", "ref_mul_mod", "ref_pow_mod", "ref_find_psi"):
            getattr(lib, name).restype = _U64
        lib.ref_add_mod.argtypes = [_U64] * 3
        lib.ref_sub_mod.argtypes = [_U64] * 3
        lib.ref_mul_mod.argtypes = [_U64] * 3
        lib.ref_pow_mod.argtypes = [_U64] * 3
        lib.ref_inv_mod.argtypes = [_U64, _U64, ctypes.POINTER(_U64)]
        lib.ref_shoup.argtypes = [_U64, _U64, _U64, ctypes.POINTER(_U64)]
        lib.ref_barrett.argtypes = [_U64, _U64, _U64, ctypes.POINTER(_U64)]
        lib.ref_find_primes.argtypes = [_U64, _U64, _U64, _P]
        lib.ref_find_psi.argtypes = [_U64, _U64]
        lib.ref_ntt.argtypes = [_P, _U64, _U64, _U64, ctypes.c_int]
        lib.ref_basis_convert.argtypes = [_P, _U64, _P, _SZ, _P, _SZ, _P]
        ctx = [_U64, _P, _P, _SZ, _P, _P, _SZ, _SZ, _SZ]
        lib.ref_mod_up.argtypes = ctx + [_P, ctypes.c_int, _P]
        lib.ref_mod_down.argtypes = ctx + [_P, _P]
        lib.ref_hybrid_digits.argtypes = ctx + [_P, _P]
        lib.ref_keyswitch.argtypes = ctx + [_P, _P, _P, _P, ctypes.c_uint32, _P, _P]

    def _err(self):
        return RuntimeError(self.lib.ref_last_error().decode())

    def _ctx(self, ctx: Context, level):
        arrays = [np.asarray(v, dtype=np.uint64) for v in (ctx.q, ctx.q_psi, ctx.p, ctx.p_psi)]
        args = [ctx.n, _ptr(arrays[0]), _ptr(arrays[1]), ctx.m, _ptr(arrays[2]), _ptr(arrays[3]),
                ctx.k, ctx.alpha, level]
        return args, arrays

    def ntt(self, values, q, psi, inverse=False):
        v = np.ascontiguousarray(values, dtype=np.uint64).copy()
        for t in range(v.shape[0]):
            row = np.ascontiguousarray(v[t])
            if self.lib.ref_ntt(_ptr(row), v.shape[1], q[t], psi[t], int(inverse)):
                raise self._err()
            v[t] = row
        return v

    def basis_convert(self, values, source, target):
        v = np.ascontiguousarray(values, dtype=np.uint64)
        n = v.shape[-1]
        out = np.zeros((len(target), n), dtype=np.uint64)
        s = np.asarray(source, dtype=np.uint64)
        t = np.asarray(target, dtype=np.uint64)
        if self.lib.ref_basis_convert(_ptr(v), n, _ptr(s), len(source), _ptr(t), len(target), _ptr(out)):
            raise self._err()
        return out

    def mod_up(self, ctx: Context, level, values, is_eval):
        args, keep = self._ctx(ctx, level)
        v = np.ascontiguousarray(values, dtype=np.uint64)
        out = np.zeros((level + ctx.k, ctx.n), dtype=np.uint64)
        if self.lib.ref_mod_up(*args, _ptr(v), int(is_eval), _ptr(out)):
            raise self._err()
        return out

    def mod_down(self, ctx: Context, level, values):
        args, keep = self._ctx(ctx, level)
        v = np.ascontiguousarray(values, dtype=np.uint64)
        out = np.zeros((level, ctx.n), dtype=np.uint64)
        if self.lib.ref_mod_down(*args, _ptr(v), _ptr(out)):
            raise self._err()
        return out

    def hybrid_digits(self, ctx: Context, level, values):
        args, keep = self._ctx(ctx, level)
        v = np.ascontiguousarray(values, dtype=np.uint64)
        out = np.zeros((ctx.digits(level), level + ctx.k, ctx.n), dtype=np.uint64)
        if self.lib.ref_hybrid_digits(*args, _ptr(v), _ptr(out)):
            raise self._err()
        return out

    def keyswitch(self, ctx: Context, level, values, key_b, key_a, c0=None, automorphism=0):
        args, keep = self._ctx(ctx, level)
        v = np.ascontiguousarray(values, dtype=np.uint64)
        kb = np.ascontiguousarray(key_b, dtype=np.uint64)
        ka = np.ascontiguousarray(key_a, dtype=np.uint64)
        c = None if c0 is None else np.ascontiguousarray(c0, dtype=np.uint64)
        ob = np.zeros((level, ctx.n), dtype=np.uint64)
        oa = np.zeros((level, ctx.n), dtype=np.uint64)
        if self.lib.ref_keyswitch(*args, _ptr(v), _ptr(kb), _ptr(ka), _ptr(c), automorphism,
                                  _ptr(ob), _ptr(oa)):
            raise self._err()
        return ob, oa


# The pinned OpenFHE 1.6.1 parameters of the reference's Hybrid fixture
# (tests/openfhe_hybrid_tests.cpp:1050-1055): N = 65536, M = 5 Q towers then
# K = 3 P towers, alpha = 3. The roots are OpenFHE's (minimum primitive 2N-th).
PINNED_N = 65536
PINNED_Q = [1152921504606584833, 1125899902124033, 1125899911168001,
            1125899903827969, 1125899908022273]
PINNED_Q_PSI = [18043022392882, 15995550378, 21670117260, 938640682, 6511788946]
PINNED_P = [1152921504598720513, 1152921504597016577, 1152921504595968001]
PINNED_P_PSI = [800790938143, 17749908910371, 11469071954203]
PINNED_ALPHA = 3

LCG_SEED = 0x7251D9  # include/ntt/benchmark_inputs.hpp:9


def pinned_context() -> Context:
    return Context(PINNED_N, PINNED_Q, PINNED_Q_PSI, PINNED_P, PINNED_P_PSI, PINNED_ALPHA)


def synthetic_context(orc: Oracle, n: int, m: int, k: int, dnum: int,
                      q_bits: int = 55, p_bits: int = 60) -> Context:
    """The benchmark context: find_primes (ascending) Q of q_bits and P of
    p_bits, roots by find_psi, alpha = ceil(M / dnum)."""
    q = orc.find_primes(n, m, q_bits)
    p = orc.find_primes(n, k, p_bits)
    alpha = -(-m // dnum)
    return Context(n, q, [orc.find_psi(v, n) for v in q], p, [orc.find_psi(v, n) for v in p], alpha)
