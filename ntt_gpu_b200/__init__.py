"""B200 (sm_100a) CKKS NTT / ModUp / ModDown / Hybrid key-switch path.

Python access to the C ABI of include/ntt_b200.h (libntt_b200.so, built in
tree by ntt_gpu_b200/build.py). Device buffers are torch CUDA tensors of dtype
int64 holding u64 residues bit-for-bit; streams are torch CUDA streams. The
CUDA library is the only implementation: there is no CPU fallback, and loading
fails loudly when the library is missing.

Errors follow the reference's conventions (include/ntt/backend_contract.hpp:20-26,
src/cuda/ntt_kernels.cu:40-46): invalid arguments raise ContractError (a
ValueError) before anything is enqueued; CUDA failures raise CudaError.
"""
from __future__ import annotations

import ctypes
import os

from .build import LIB

__all__ = ["ContractError", "CudaError", "WorkspaceError", "Context", "KsRequest", "make_request", "Server", "KeyCache",
           "library", "load",
           "kernel_launches", "OP_MOD_UP", "OP_MOD_DOWN", "OP_DIGITS", "OP_KEYSWITCH"]

OK, ERR_CONTRACT, ERR_CUDA, ERR_UNSUPPORTED, ERR_WORKSPACE, ERR_TIMEOUT, NOT_READY = range(7)
OP_MOD_UP, OP_MOD_DOWN, OP_DIGITS, OP_KEYSWITCH = 1, 2, 3, 4


class ContractError(ValueError):
    """Invalid argument or layout; raised before any device work is enqueued."""


class CudaError(RuntimeError):
    """CUDA runtime failure."""


class WorkspaceError(ValueError):
    """Workspace missing or too small."""


class TimeoutError_(RuntimeError):
    """A bounded device wait expired."""


_lib = None
_U64, _SZ, _P, _I = ctypes.c_uint64, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_int

_SIGNATURES = {
    "ntt_b200_last_error": ([], ctypes.c_char_p),
    "ntt_b200_kernel_launches": ([], _U64),
    "ntt_b200_context_create": ([ctypes.POINTER(_P), _I, _U64, _P, _P, _SZ, _P, _P, _SZ, _SZ], _I),
    "ntt_b200_context_destroy": ([_P], _I),
    "ntt_b200_context_table_bytes": ([_P, ctypes.POINTER(_SZ)], _I),
    "ntt_b200_context_prepare": ([_P, _SZ], _I),
    "ntt_b200_ntt": ([_P, _P, _P, _P, _SZ, _SZ, _SZ, _I, _P], _I),
    "ntt_b200_pointwise": ([_P, _P, _P, _P, _P, _SZ, _SZ, _SZ, _P], _I),
    "ntt_b200_switch_basis": ([_P, _P, _P, _P, _SZ, _P, _SZ, _P], _I),
    "ntt_b200_correct": ([_P, _SZ, _P, _P, _P, _P], _I),
    "ntt_b200_hybrid_mac": ([_P, _SZ, _P, _P, _P, _P, _P, _P], _I),
    "ntt_b200_hybrid_rotate": ([_P, _SZ, _P, _P, _P, _P, _P, ctypes.c_uint32, _P], _I),
    "ntt_b200_workspace_bytes": ([_P, _I, _SZ, _SZ, ctypes.POINTER(_SZ)], _I),
    "ntt_b200_mod_up": ([_P, _SZ, _P, _P, _I, _P, _SZ, _P], _I),
    "ntt_b200_mod_down": ([_P, _SZ, _P, _P, _P, _SZ, _P], _I),
    "ntt_b200_hybrid_digits": ([_P, _SZ, _P, _P, _P, _SZ, _P], _I),
    "ntt_b200_keyswitch": ([_P, _SZ, _P, _P, _P, _P, _P, _P, ctypes.c_uint32, _P, _SZ, _P], _I),
    "ntt_b200_keyswitch_batch": ([_P, _SZ, _SZ, _P, _P, _P, _P, _P, _P, ctypes.c_uint32, _P, _SZ, _P], _I),
    "ntt_b200_hybrid_mac_digits": ([_P, _SZ, _P, _P, _P, _P, _P, _SZ, _I, _I, _P], _I),
    "ntt_b200_keyswitch_requests_workspace": ([_P, _P, _SZ, ctypes.POINTER(_SZ)], _I),
    "ntt_b200_keyswitch_requests": ([_P, _P, _SZ, _P, _SZ, _P], _I),
    "ntt_b200_keyswitch_host_workspace": ([_P, _SZ, _SZ, _I, ctypes.POINTER(_SZ)], _I),
    "ntt_b200_keyswitch_host": ([_P, _SZ, _SZ, _SZ, _P, _P, _P, _P, _P, _P, ctypes.c_uint32, _P, _SZ, _P], _I),
    "ntt_b200_keyswitch_host_async": ([_P, _SZ, _SZ, _SZ, _P, _P, _P, _P, _P, _P, ctypes.c_uint32, _P, _SZ, _P], _I),
    "ntt_b200_keyswitch_host_wait": ([_P, _P], _I),
    "ntt_b200_server_last_error": ([], ctypes.c_char_p),
    "ntt_b200_server_create": ([ctypes.POINTER(_P), _P], _I),
    "ntt_b200_server_submit": ([_P, _P, _P, ctypes.POINTER(_U64)], _I),
    "ntt_b200_server_wait": ([_P, _U64, ctypes.c_uint32, _P], _I),
    "ntt_b200_server_drain": ([_P, ctypes.c_uint32], _I),
    "ntt_b200_server_stats": ([_P, _P, _I], _I),
    "ntt_b200_server_destroy": ([_P], _I),
    "ntt_b200_server_attach_keycache": ([_P, _P], _I),
    "ntt_b200_server_reserve": ([_P, _SZ], _I),
    "ntt_b200_context_key_words": ([_P, ctypes.POINTER(_SZ)], _I),
    "ntt_b200_device_errors": ([_P, ctypes.POINTER(_I), _I], _I),
    "ntt_b200_keycache_last_error": ([], ctypes.c_char_p),
    "ntt_b200_keycache_create": ([ctypes.POINTER(_P), _I, _SZ], _I),
    "ntt_b200_keycache_destroy": ([_P], _I),
    "ntt_b200_keycache_insert": ([_P, _P, _U64, _P, _P], _I),
    "ntt_b200_keycache_contains": ([_P, _U64, ctypes.POINTER(_P)], _I),
    "ntt_b200_keycache_acquire": ([_P, _U64, _P, ctypes.POINTER(_P), ctypes.POINTER(_P)], _I),
    "ntt_b200_keycache_release": ([_P, _U64, _P], _I),
    "ntt_b200_keycache_stats": ([_P, _P], _I),
    "ntt_b200_keycache_set_budget": ([_P, _SZ], _I),
    "ntt_b200_keycache_trim": ([_P, ctypes.POINTER(_SZ)], _I),
    "ntt_b200_stream_create": ([_I, ctypes.POINTER(_P)], _I),
    "ntt_b200_stream_destroy": ([_P], _I),
    "ntt_b200_stream_synchronize": ([_P], _I),
    "ntt_b200_alloc": ([_I, _SZ, _P, ctypes.POINTER(_P)], _I),
    "ntt_b200_free": ([_P, _P], _I),
    "ntt_b200_memcpy": ([_P, _P, _SZ, _I, _P], _I),
    "ntt_b200_event_create": ([_I, ctypes.POINTER(_P)], _I),
    "ntt_b200_event_destroy": ([_P], _I),
    "ntt_b200_event_record": ([_P, _P], _I),
    "ntt_b200_event_query": ([_P], _I),
    "ntt_b200_event_synchronize": ([_P], _I),
    "ntt_b200_mod_down_static_max_bytes": ([], _SZ),
    "ntt_b200_mod_down_static": ([_P, _SZ, _P, _P, _P], _I),
    "ntt_b200_tuning_set": ([ctypes.c_char_p, ctypes.c_int64], _I),
    "ntt_b200_tuning_get": ([ctypes.c_char_p, ctypes.POINTER(ctypes.c_int64)], _I),
    "ntt_b200_tuning_name": ([_SZ], ctypes.c_char_p),
    "ntt_b200_timing_enable": ([_I], _I),
    "ntt_b200_timing_reset": ([], _I),
    "ntt_b200_timing_query": ([ctypes.c_char_p, ctypes.POINTER(_U64), ctypes.POINTER(ctypes.c_double)], _I),
    "ntt_b200_butterfly_rate": ([_I, ctypes.POINTER(ctypes.c_double)], _I),
    "ntt_b200_host_transform_workspace": ([_P, _I, ctypes.POINTER(_SZ)], _I),
    "ntt_b200_host_transform": ([_P, _I, _P, _P, _P, _SZ, _P, _SZ, _P], _I),
    "ntt_b200_arith_probe": ([_I, _I, _P, _SZ, _P, _P], _I),
    "ntt_b200_conv_wait_polls": ([_I], _I),
    "ntt_b200_inject_setup_failure": ([_SZ], _I),
    "ntt_b200_setup_operations": ([ctypes.POINTER(_SZ)], _I),
}

HOST_FORWARD, HOST_INVERSE, HOST_POINTWISE, HOST_MULTIPLY = 0, 1, 2, 3


class KsRequest(ctypes.Structure):
    """ntt_b200_ks_request: one key-switch / rotation / relinearization request."""
    _fields_ = [("src", _P), ("out_b", _P), ("out_a", _P), ("key_b", _P), ("key_a", _P), ("c0", _P),
                ("add_b", _P), ("add_a", _P), ("automorphism", ctypes.c_uint32), ("level", ctypes.c_uint32),
                ("key_id", _U64)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("device", _I), ("lanes", _I), ("max_batch", _I), ("depth", _I), ("hbm_budget_bytes", _SZ),
                ("max_inflight_bytes", _SZ)]


class TicketInfo(ctypes.Structure):
    _fields_ = [("status", _I), ("wave_size", ctypes.c_uint32), ("lane", _I), ("reserved", _I),
                ("queue_us", ctypes.c_double), ("latency_us", ctypes.c_double)]


class ServerReport(ctypes.Structure):
    _fields_ = [("completed", _U64), ("waves", _U64), ("mean_wave", ctypes.c_double), ("p50_ms", ctypes.c_double),
                ("p99_ms", ctypes.c_double), ("max_ms", ctypes.c_double), ("throughput", ctypes.c_double),
                ("mean_queue_ms", ctypes.c_double), ("peak_bytes", _SZ), ("in_flight_bytes", _SZ)]


def make_request(level, src, out_b, out_a, key_b=None, key_a=None, c0=None, automorphism=0, add_b=None, add_a=None,
                 key_id=0):
    """A KsRequest from torch CUDA tensors (None for the optional ones). With
    key_b = key_a = None the server takes the key from its key cache by key_id."""
    return KsRequest(_ptr(src), _ptr(out_b), _ptr(out_a), _ptr(key_b), _ptr(key_a), _ptr(c0), _ptr(add_b),
                     _ptr(add_a), int(automorphism), int(level), int(key_id))


class KeyCacheReport(ctypes.Structure):
    _fields_ = [("budget_bytes", _SZ), ("allocated_bytes", _SZ), ("pinned_bytes", _SZ), ("keys", _U64),
                ("resident", _U64), ("hits", _U64), ("misses", _U64), ("evictions", _U64)]


TUNING = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning.json")


def load(path: str = LIB):
    """Load libntt_b200.so, bind every entry point of include/ntt_b200.h and
    apply the autotuner's committed choices (tuning.json) if present."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"libntt_b200.so not built at {path}; run ntt_gpu_b200/build.py")
    lib = ctypes.CDLL(path)
    for name, (args, res) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    if os.path.exists(TUNING):
        import json
        with open(TUNING) as f:
            for name, value in json.load(f).get("choices", {}).items():
                tuning_set(name, value)
    return lib


def tuning_names() -> list:
    lib, out, i = load(), [], 0
    while True:
        name = lib.ntt_b200_tuning_name(i)
        if not name:
            return out
        out.append(name.decode())
        i += 1


def tuning_set(name: str, value: int):
    _check(load().ntt_b200_tuning_set(name.encode(), int(value)))


def tuning_get(name: str) -> int:
    v = ctypes.c_int64()
    _check(load().ntt_b200_tuning_get(name.encode(), ctypes.byref(v)))
    return int(v.value)


def library():
    return load()


def kernel_launches() -> int:
    return int(load().ntt_b200_kernel_launches())


def _check(rc: int, server: bool = False, cache: bool = False):
    if rc == OK:
        return
    lib = load()
    msg = (lib.ntt_b200_server_last_error() if server else
           lib.ntt_b200_keycache_last_error() if cache else lib.ntt_b200_last_error()).decode()
    if rc == ERR_CONTRACT or rc == ERR_UNSUPPORTED:
        raise ContractError(msg)
    if rc == ERR_WORKSPACE:
        raise WorkspaceError(msg)
    if rc == ERR_TIMEOUT:
        raise TimeoutError_(msg)
    raise CudaError(msg)


def _arr(values, ctype=_U64):
    values = [int(v) for v in values]
    return (ctype * max(1, len(values)))(*values)


def _ptr(t) -> int | None:
    """Device address of a torch tensor (or None)."""
    if t is None:
        return None
    assert t.is_cuda and t.is_contiguous(), "expected a contiguous CUDA tensor"
    return t.data_ptr()


def _stream(stream) -> int | None:
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


class Context:
    """One CKKS context (N, M Q towers, K P towers, alpha) with HBM tables.

    Tower ids: Q tower i -> i, P tower j -> M + j.
    """

    def __init__(self, n, q, q_psi, p=(), p_psi=(), alpha=1, device=0):
        lib = load()
        self.n, self.m, self.k, self.alpha, self.device = int(n), len(q), len(p), int(alpha), int(device)
        self.q, self.q_psi, self.p, self.p_psi = list(q), list(q_psi), list(p), list(p_psi)
        handle = _P()
        _check(lib.ntt_b200_context_create(ctypes.byref(handle), self.device, self.n, _arr(q), _arr(q_psi),
                                           self.m, _arr(p), _arr(p_psi), self.k, self.alpha))
        self._h = handle
        self._lib = lib

    @classmethod
    def from_oracle(cls, ctx, device=0):
        return cls(ctx.n, ctx.q, ctx.q_psi, ctx.p, ctx.p_psi, ctx.alpha, device)

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            _check(self._lib.ntt_b200_context_destroy(self._h))
            self._h = _P()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- helpers -----------------------------------------------------------------
    def digits(self, level):
        return 1 + (level - 1) // self.alpha

    def full_digits(self):
        return 1 + (self.m - 1) // self.alpha

    def qp_ids(self, level):
        return list(range(level)) + [self.m + j for j in range(self.k)]

    def device_errors(self, clear=False) -> int:
        """Count of expired bounded waits on the GPU (0 when every kernel completed normally)."""
        out = _I()
        _check(self._lib.ntt_b200_device_errors(self._h, ctypes.byref(out), int(clear)))
        return out.value

    def table_bytes(self) -> int:
        out = _SZ()
        _check(self._lib.ntt_b200_context_table_bytes(self._h, ctypes.byref(out)))
        return out.value

    def prepare(self, level):
        _check(self._lib.ntt_b200_context_prepare(self._h, level))

    def workspace_bytes(self, op, level, batch=1) -> int:
        out = _SZ()
        _check(self._lib.ntt_b200_workspace_bytes(self._h, op, level, batch, ctypes.byref(out)))
        return out.value

    def workspace(self, op, level, batch=1):
        import torch
        nbytes = self.workspace_bytes(op, level, batch)
        return torch.empty(max(1, (nbytes + 7) // 8), dtype=torch.int64, device=f"cuda:{self.device}")

    # ---- primitives ---------------------------------------------------------------
    def ntt(self, dst, src, tower_ids, polys=1, poly_stride=0, inverse=False, stream=None):
        _check(self._lib.ntt_b200_ntt(self._h, _ptr(dst), _ptr(src), _arr(tower_ids, ctypes.c_uint32),
                                      len(tower_ids), polys, poly_stride, int(inverse), _stream(stream)))

    def pointwise(self, dst, left, right, tower_ids, polys=1, poly_stride=0, stream=None):
        _check(self._lib.ntt_b200_pointwise(self._h, _ptr(dst), _ptr(left), _ptr(right),
                                            _arr(tower_ids, ctypes.c_uint32), len(tower_ids), polys,
                                            poly_stride, _stream(stream)))

    def switch_basis(self, dst, src, source_ids, target_ids, stream=None):
        _check(self._lib.ntt_b200_switch_basis(self._h, _ptr(dst), _ptr(src),
                                               _arr(source_ids, ctypes.c_uint32), len(source_ids),
                                               _arr(target_ids, ctypes.c_uint32), len(target_ids),
                                               _stream(stream)))

    def correct(self, level, dst, left, right, stream=None):
        _check(self._lib.ntt_b200_correct(self._h, level, _ptr(dst), _ptr(left), _ptr(right), _stream(stream)))

    def hybrid_mac(self, level, out_b, out_a, digits, key_b, key_a, stream=None):
        _check(self._lib.ntt_b200_hybrid_mac(self._h, level, _ptr(out_b), _ptr(out_a), _ptr(digits),
                                             _ptr(key_b), _ptr(key_a), _stream(stream)))

    def hybrid_mac_digits(self, level, out_b, out_a, digits, keys_b, keys_a, full_key_rows=True,
                          accumulate=False, stream=None):
        """MAC over per-digit buffers (lists of device tensors, one entry per digit).

        full_key_rows: keys are full-context digits (M+K towers) rather than packed
        active QP rows. accumulate: add into out_b/out_a instead of overwriting."""
        count = len(digits)
        if not (len(keys_b) == len(keys_a) == count):
            raise ContractError("one key_b and one key_a buffer per digit")
        vec = ctypes.c_void_p * max(1, count)
        _check(self._lib.ntt_b200_hybrid_mac_digits(
            self._h, level, _ptr(out_b), _ptr(out_a), vec(*[_ptr(d) for d in digits]),
            vec(*[_ptr(k) for k in keys_b]), vec(*[_ptr(k) for k in keys_a]), count, int(full_key_rows),
            int(accumulate), _stream(stream)))

    def hybrid_rotate(self, level, out_b, out_a, ext_b, ext_a, c0, automorphism, stream=None):
        _check(self._lib.ntt_b200_hybrid_rotate(self._h, level, _ptr(out_b), _ptr(out_a), _ptr(ext_b),
                                                _ptr(ext_a), _ptr(c0), automorphism, _stream(stream)))

    # ---- composites -----------------------------------------------------------------
    def mod_up(self, level, dst, src, src_is_eval, workspace, stream=None):
        _check(self._lib.ntt_b200_mod_up(self._h, level, _ptr(dst), _ptr(src), int(src_is_eval),
                                         _ptr(workspace), workspace.numel() * 8, _stream(stream)))

    def mod_down(self, level, dst, src, workspace, stream=None):
        _check(self._lib.ntt_b200_mod_down(self._h, level, _ptr(dst), _ptr(src), _ptr(workspace),
                                           workspace.numel() * 8, _stream(stream)))

    def hybrid_digits(self, level, digits, src, workspace, stream=None):
        _check(self._lib.ntt_b200_hybrid_digits(self._h, level, _ptr(digits), _ptr(src), _ptr(workspace),
                                                workspace.numel() * 8, _stream(stream)))

    def keyswitch_batch(self, level, batch, out_b, out_a, src, key_b, key_a, workspace, c0=None,
                        automorphism=0, stream=None):
        _check(self._lib.ntt_b200_keyswitch_batch(self._h, level, batch, _ptr(out_b), _ptr(out_a), _ptr(src),
                                                  _ptr(key_b), _ptr(key_a), _ptr(c0), automorphism,
                                                  _ptr(workspace), workspace.numel() * 8, _stream(stream)))

    def requests_workspace_bytes(self, reqs) -> int:
        arr = (KsRequest * len(reqs))(*reqs)
        out = _SZ()
        _check(self._lib.ntt_b200_keyswitch_requests_workspace(self._h, arr, len(reqs), ctypes.byref(out)))
        return out.value

    def requests_workspace(self, reqs):
        import torch
        nbytes = self.requests_workspace_bytes(reqs)
        return torch.empty(max(1, (nbytes + 7) // 8), dtype=torch.int64, device=f"cuda:{self.device}")

    def keyswitch_requests(self, reqs, workspace, stream=None):
        arr = (KsRequest * len(reqs))(*reqs)
        _check(self._lib.ntt_b200_keyswitch_requests(self._h, arr, len(reqs), _ptr(workspace),
                                                     workspace.numel() * 8, _stream(stream)))

    def host_workspace(self, level, chunk, rotate=False):
        import torch
        out = _SZ()
        _check(self._lib.ntt_b200_keyswitch_host_workspace(self._h, level, chunk, int(rotate), ctypes.byref(out)))
        return torch.empty(max(1, (out.value + 7) // 8), dtype=torch.int64, device=f"cuda:{self.device}")

    def keyswitch_host(self, level, batch, chunk, h_src, h_out_b, h_out_a, key_b, key_a, workspace, h_c0=None,
                       automorphism=0, stream=None, wait=True):
        """Host tensors (pinned CPU int64) in and out; keys and workspace on the device.
        wait=False: ntt_b200_keyswitch_host_async (join later with keyswitch_host_wait)."""
        def hp(t):
            if t is None:
                return None
            assert not t.is_cuda and t.is_contiguous()
            return t.data_ptr()
        fn = self._lib.ntt_b200_keyswitch_host if wait else self._lib.ntt_b200_keyswitch_host_async
        _check(fn(self._h, level, batch, chunk, hp(h_src), hp(h_out_b), hp(h_out_a), _ptr(key_b), _ptr(key_a),
                  hp(h_c0), automorphism, _ptr(workspace), workspace.numel() * 8, _stream(stream)))

    def keyswitch_host_wait(self, stream=None):
        """Make `stream` wait for the outputs of every host-buffer key switch so far."""
        _check(self._lib.ntt_b200_keyswitch_host_wait(self._h, _stream(stream)))

    def host_transform_workspace(self, op):
        import torch
        out = _SZ()
        _check(self._lib.ntt_b200_host_transform_workspace(self._h, int(op), ctypes.byref(out)))
        return torch.empty(max(1, (out.value + 7) // 8), dtype=torch.int64, device=f"cuda:{self.device}")

    def host_transform(self, op, values, tower_ids, workspace, right=None, stream=None):
        """The reference's CudaNttTransform public calls on host arrays (numpy
        uint64 or CPU int64 tensors, limb-major, contiguous), synchronous and in
        place on `values`: HOST_FORWARD, HOST_INVERSE, HOST_POINTWISE (values *=
        right), HOST_MULTIPLY (ring product)."""
        def hp(a):
            if a is None:
                return None
            if hasattr(a, "ctypes"):
                assert a.dtype.itemsize == 8 and a.flags["C_CONTIGUOUS"]
                return a.ctypes.data
            assert not a.is_cuda and a.is_contiguous()
            return a.data_ptr()
        ids = _arr(tower_ids, ctypes.c_uint32)
        _check(self._lib.ntt_b200_host_transform(self._h, int(op), hp(values), hp(right), ids, len(tower_ids),
                                                 _ptr(workspace), workspace.numel() * 8, _stream(stream)))

    def keyswitch(self, level, out_b, out_a, src, key_b, key_a, workspace, c0=None, automorphism=0,
                  stream=None):
        _check(self._lib.ntt_b200_keyswitch(self._h, level, _ptr(out_b), _ptr(out_a), _ptr(src), _ptr(key_b),
                                            _ptr(key_a), _ptr(c0), automorphism, _ptr(workspace),
                                            workspace.numel() * 8, _stream(stream)))


class Server:
    """Continuous-batching key-switch server (ntt_b200_server_*).

    submit() takes a KsRequest over device-resident buffers (kept alive by the
    caller until wait() returns) and returns a ticket; wait() blocks until the
    request's wave finished on the GPU and returns its TicketInfo.
    """

    # Defaults: the configuration measured best on a B200 over uniform N=2^16
    # batches and a mixed N=2^13..2^16 stream (4 lanes, 2 waves deep, new waves
    # only while less than 512 MiB of workspace is in flight).
    def __init__(self, device=0, lanes=4, max_batch=16, hbm_budget_bytes=8 << 30, depth=2,
                 max_inflight_bytes=512 << 20):
        self._lib = load()
        cfg = ServerConfig(int(device), int(lanes), int(max_batch), int(depth), int(hbm_budget_bytes),
                           int(max_inflight_bytes))
        h = _P()
        _check(self._lib.ntt_b200_server_create(ctypes.byref(h), ctypes.byref(cfg)), server=True)
        self._h = h

    def submit(self, ctx: "Context", req: KsRequest) -> int:
        t = _U64()
        _check(self._lib.ntt_b200_server_submit(self._h, ctx._h, ctypes.byref(req), ctypes.byref(t)), server=True)
        return t.value

    def wait(self, ticket: int, timeout_ms: int = 60000) -> TicketInfo:
        info = TicketInfo()
        _check(self._lib.ntt_b200_server_wait(self._h, ticket, timeout_ms, ctypes.byref(info)), server=True)
        return info

    def reserve(self, bytes_per_lane: int):
        """Grow every idle lane's workspace arena to bytes_per_lane up front."""
        _check(self._lib.ntt_b200_server_reserve(self._h, int(bytes_per_lane)), server=True)

    def attach_keycache(self, cache: "KeyCache"):
        _check(self._lib.ntt_b200_server_attach_keycache(self._h, cache._h), server=True)
        self._cache = cache  # the cache outlives the server

    def drain(self, timeout_ms: int = 120000):
        _check(self._lib.ntt_b200_server_drain(self._h, timeout_ms), server=True)

    def stats(self, reset=False) -> dict:
        st = ServerReport()
        _check(self._lib.ntt_b200_server_stats(self._h, ctypes.byref(st), int(reset)), server=True)
        return {f: getattr(st, f) for f, _ in ServerReport._fields_}

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            _check(self._lib.ntt_b200_server_destroy(self._h), server=True)
            self._h = _P()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class KeyCache:
    """Evaluation-key cache (ntt_b200_keycache_*): host keys made resident in
    HBM on demand within a byte budget, least-recently-used eviction of keys
    that are unpinned and whose last use has completed."""

    def __init__(self, device=0, budget_bytes=8 << 30):
        self._lib = load()
        h = _P()
        _check(self._lib.ntt_b200_keycache_create(ctypes.byref(h), int(device), int(budget_bytes)), cache=True)
        self._h = h

    def insert(self, ctx: "Context", key_id: int, key_b, key_a):
        """key_b / key_a: host numpy uint64 arrays of full-context digits."""
        import numpy as np
        kb = np.ascontiguousarray(key_b, dtype=np.uint64)
        ka = np.ascontiguousarray(key_a, dtype=np.uint64)
        words = _SZ()
        _check(self._lib.ntt_b200_context_key_words(ctx._h, ctypes.byref(words)))
        if kb.size != words.value or ka.size != words.value:
            raise ContractError(f"key must hold {words.value} words per channel")
        _check(self._lib.ntt_b200_keycache_insert(self._h, ctx._h, int(key_id), kb.ctypes.data, ka.ctypes.data),
               cache=True)

    def acquire(self, key_id: int, stream=None):
        """(key_b, key_a) device addresses, pinned until release()."""
        b, a = _P(), _P()
        _check(self._lib.ntt_b200_keycache_acquire(self._h, int(key_id), _stream(stream), ctypes.byref(b),
                                                   ctypes.byref(a)), cache=True)
        return b.value, a.value

    def release(self, key_id: int, stream=None):
        _check(self._lib.ntt_b200_keycache_release(self._h, int(key_id), _stream(stream)), cache=True)

    def stats(self) -> dict:
        st = KeyCacheReport()
        _check(self._lib.ntt_b200_keycache_stats(self._h, ctypes.byref(st)), cache=True)
        return {f: getattr(st, f) for f, _ in KeyCacheReport._fields_}

    def set_budget(self, nbytes: int):
        _check(self._lib.ntt_b200_keycache_set_budget(self._h, int(nbytes)), cache=True)

    def trim(self) -> int:
        freed = _SZ()
        _check(self._lib.ntt_b200_keycache_trim(self._h, ctypes.byref(freed)), cache=True)
        return freed.value

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            _check(self._lib.ntt_b200_keycache_destroy(self._h), cache=True)
            self._h = _P()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


KERNEL_CLASSES = ("ntt_fwd_col", "ntt_fwd_row", "ntt_fwd_cluster", "ntt_inv_row", "ntt_inv_col", "ntt_small",
                  "conv", "mac", "row_mac", "rotate", "correct", "pointwise", "table")


def arith_probe(op: int, queries, device: int = 0):
    """Device arithmetic probe (ntt_b200_arith_probe): queries is a [count][5]
    uint64 numpy array; returns the [count] results computed on the GPU."""
    import numpy as np
    import torch
    q = to_device(np.ascontiguousarray(queries, dtype=np.uint64), device)
    out = torch.empty((q.shape[0],), dtype=torch.int64, device=f"cuda:{device}")
    _check(load().ntt_b200_arith_probe(device, int(op), q.data_ptr(), q.shape[0], out.data_ptr(),
                                       torch.cuda.current_stream(device).cuda_stream))
    return to_host(out)


def butterfly_rate(device: int = 0) -> float:
    """Mode-2 NTT butterflies per second on `device` with operands in registers
    (ntt_b200_butterfly_rate): the multiply-pipe ceiling of the NTT passes."""
    out = ctypes.c_double()
    _check(load().ntt_b200_butterfly_rate(int(device), ctypes.byref(out)))
    return out.value


def timing_enable(on: bool = True):
    _check(load().ntt_b200_timing_enable(int(on)))


def timing_reset():
    _check(load().ntt_b200_timing_reset())


def timing_query(kernel: str):
    """(launches, total device milliseconds) of one kernel class since the last reset."""
    n, ms = _U64(), ctypes.c_double()
    _check(load().ntt_b200_timing_query(kernel.encode(), ctypes.byref(n), ctypes.byref(ms)))
    return int(n.value), float(ms.value)


def to_device(array, device=0):
    """numpy uint64 array -> CUDA int64 tensor with the same bits."""
    import numpy as np
    import torch
    a = np.ascontiguousarray(array, dtype=np.uint64)
    return torch.from_numpy(a.view(np.int64)).to(f"cuda:{device}")


def to_host(tensor):
    """CUDA int64 tensor -> numpy uint64 array with the same bits."""
    import numpy as np
    return tensor.detach().cpu().numpy().view(np.uint64)


def empty(shape, device=0):
    import torch
    return torch.empty(shape, dtype=torch.int64, device=f"cuda:{device}")
