// Exact 64-bit modular arithmetic for sm_100a CUDA cores.
//
// Residues are u64 and every public result is canonical ([0, q)), matching the
// reference contract (docs/modular-arithmetic-contract.md:25-31 in
// minnow54426/ntt-gpu). Internally the NTT uses Harvey's lazy butterflies:
// values live in [0, 4q) between stages, which needs q < 2^62 ("lazy" moduli);
// moduli in [2^62, 2^63) take the strict path where every value stays canonical.
//
// Multiplication by a constant w uses Shoup's precomputed quotient
// w' = floor(w * 2^64 / q) (reference include/ntt/shoup.hpp:7-27): for ANY
// x < 2^64, x*w - hi64(x*w')*q lies in [0, 2q).
#pragma once
#include <cstdint>

namespace b200 {
using u64 = uint64_t;

struct Shoup {
  u64 w, wq;  // constant and floor(w * 2^64 / q)
};

__device__ __forceinline__ u64 mulhi(u64 a, u64 b) { return __umul64hi(a, b); }

// x*w mod q in [0, 2q) for any x < 2^64 (q < 2^63).
__device__ __forceinline__ u64 shoup_lazy(u64 x, u64 w, u64 wq, u64 q) {
  return x * w - mulhi(x, wq) * q;
}
__device__ __forceinline__ u64 csub(u64 x, u64 m) { return x >= m ? x - m : x; }
__device__ __forceinline__ u64 shoup_canon(u64 x, u64 w, u64 wq, u64 q) {
  return csub(shoup_lazy(x, w, wq, q), q);
}
__device__ __forceinline__ u64 add_mod(u64 a, u64 b, u64 q) { return csub(a + b, q); }  // q < 2^63
__device__ __forceinline__ u64 sub_mod(u64 a, u64 b, u64 q) { return a >= b ? a - b : a + (q - b); }

// ---- NTT butterflies --------------------------------------------------------
// Forward Cooley-Tukey (x, y) -> (x + w*y, x - w*y).
// LAZY: inputs and outputs in [0, 4q). Strict: canonical in and out.
template <bool LAZY>
__device__ __forceinline__ void ct_butterfly(u64 &x, u64 &y, u64 w, u64 wq, u64 q, u64 q2) {
  if constexpr (LAZY) {
    const u64 a = csub(x, q2);
    const u64 t = shoup_lazy(y, w, wq, q);
    x = a + t;
    y = a + q2 - t;
  } else {
    const u64 t = shoup_canon(y, w, wq, q);
    const u64 a = x;
    x = add_mod(a, t, q);
    y = sub_mod(a, t, q);
  }
}

// Inverse Gentleman-Sande (x, y) -> (x + y, (x - y) * w).
// LAZY: inputs and outputs in [0, 2q). Strict: canonical.
template <bool LAZY>
__device__ __forceinline__ void gs_butterfly(u64 &x, u64 &y, u64 w, u64 wq, u64 q, u64 q2) {
  if constexpr (LAZY) {
    const u64 s = csub(x + y, q2);
    const u64 d = x + q2 - y;
    y = shoup_lazy(d, w, wq, q);
    x = s;
  } else {
    const u64 s = add_mod(x, y, q);
    const u64 d = sub_mod(x, y, q);
    y = shoup_canon(d, w, wq, q);
    x = s;
  }
}

// Last inverse stage with the N^-1 scale folded in: outputs canonical.
// (x, y) -> ((x + y) * n_inv, (x - y) * w * n_inv); wn = w * n_inv.
template <bool LAZY>
__device__ __forceinline__ void gs_last(u64 &x, u64 &y, Shoup ninv, Shoup wn, u64 q, u64 q2) {
  if constexpr (LAZY) {
    const u64 s = x + y;       // < 4q
    const u64 d = x + q2 - y;  // < 4q
    x = shoup_canon(s, ninv.w, ninv.wq, q);
    y = shoup_canon(d, wn.w, wn.wq, q);
  } else {
    const u64 s = add_mod(x, y, q);
    const u64 d = sub_mod(x, y, q);
    x = shoup_canon(s, ninv.w, ninv.wq, q);
    y = shoup_canon(d, wn.w, wn.wq, q);
  }
}

// [0, 4q) -> [0, q).
__device__ __forceinline__ u64 reduce4(u64 x, u64 q, u64 q2) { return csub(csub(x, q2), q); }

// ---- 128-bit accumulation ------------------------------------------------------
// Exact sums of u64 products for the approximate-CRT basis switch and the Hybrid
// MAC, on the compiler's native 128-bit integers. Acc192 adds a word counting
// carries out of 128 bits (for sums that may reach 2^128).
using u128 = unsigned __int128;
struct Acc128 {
  u128 v = 0;
};
__device__ __forceinline__ void acc_mad(Acc128 &a, u64 x, u64 y) { a.v += (u128)x * y; }
struct Acc192 {
  u128 v = 0;
  u64 top = 0;
};
__device__ __forceinline__ void acc_mad(Acc192 &a, u64 x, u64 y) {
  const u128 before = a.v;
  a.v += (u128)x * y;
  a.top += a.v < before;
}

// Reduction constants of a modulus m (m < 2^63):
//   one = floor(2^64 / m)               (Shoup quotient of w = 1)
//   r64 = 2^64 mod m, r64q its Shoup quotient
//   r128 = 2^128 mod m, r128q its Shoup quotient
struct Reducer {
  u64 m, one, r64, r64q, r128, r128q;
};

// x mod m for any x < 2^64.
__device__ __forceinline__ u64 reduce64(u64 x, const Reducer &r) {
  return csub(x - mulhi(x, r.one) * r.m, r.m);
}
// v mod m in [0, 4m) (m < 2^62): hi * (2^64 mod m) and lo each reduced to [0, 2m).
__device__ __forceinline__ u64 reduce128_lazy(u128 v, const Reducer &r) {
  const u64 hi = (u64)(v >> 64), lo = (u64)v;
  return shoup_lazy(hi, r.r64, r.r64q, r.m) + (lo - mulhi(lo, r.one) * r.m);
}
// (hi * 2^64 + lo) mod m, canonical, for any m < 2^63.
__device__ __forceinline__ u64 reduce128(u64 lo, u64 hi, const Reducer &r) {
  const u64 a = csub(shoup_lazy(hi, r.r64, r.r64q, r.m), r.m);
  const u64 b = reduce64(lo, r);
  return add_mod(a, b, r.m);
}
__device__ __forceinline__ u64 reduce(const Acc128 &a, const Reducer &r) {
  return reduce128((u64)a.v, (u64)(a.v >> 64), r);
}
__device__ __forceinline__ u64 reduce(const Acc192 &a, const Reducer &r) {
  const u64 low = reduce128((u64)a.v, (u64)(a.v >> 64), r);
  const u64 top = csub(shoup_lazy(a.top, r.r128, r.r128q, r.m), r.m);
  return add_mod(low, top, r.m);
}
// Result in [0, 4m) when the sum is below 2^128 and m < 2^62; canonical otherwise.
template <bool LAZY>
__device__ __forceinline__ u64 reduce_out(const Acc128 &a, const Reducer &r) {
  if constexpr (LAZY) return reduce128_lazy(a.v, r);
  else return reduce(a, r);
}
template <bool LAZY>
__device__ __forceinline__ u64 reduce_out(const Acc192 &a, const Reducer &r) {
  return reduce(a, r);
}
// a * b mod m for canonical a, b.
__device__ __forceinline__ u64 mul_mod(u64 a, u64 b, const Reducer &r) {
  return reduce128(a * b, mulhi(a, b), r);
}
}  // namespace b200
