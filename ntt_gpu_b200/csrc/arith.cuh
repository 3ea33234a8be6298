// Exact 64-bit modular arithmetic for sm_100a CUDA cores.
//
// Residues are u64 and every public result is canonical ([0, q)), matching the
// reference contract (docs/modular-arithmetic-contract.md:25-31 in
// minnow54426/ntt-gpu). Internally the NTT keeps lazy ranges between stages
// (the butterfly MODEs below): moduli below 2^61 take the fast path, moduli
// below 2^62 Harvey's lazy butterflies, and moduli in [2^62, 2^63) the strict
// path where every value stays canonical.
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
// MODE selects the value ranges kept between stages:
//   0 strict: canonical in and out (any q < 2^63);
//   1 lazy:   Harvey's butterflies, forward [0, 4q), inverse [0, 2q) (q < 2^62);
//   2 fast:   approximate-quotient Shoup products (below), forward [0, 8q),
//             inverse [0, 4q) (q < 2^61).

// Shoup product with an approximate quotient, for any x < 2^64 and q < 2^62.
// With x = xh:xl and w' = wh:wl (32-bit halves), the quotient estimate is
// xh*wh + hi(xl*wh) + hi(xh*wl): it drops xl*wl and every carry between the
// partial products, so it is at most 2 below floor(x*w'/2^64), which is itself
// at most 1 below floor(x*w/q). Hence x*w - estimate*q lies in [0, 4q); it is
// formed mod 2^64 as x*w + estimate*(2^64 - q). No product needs a carry
// fix-up and no comparison is involved. The estimate's last term is a plain
// 64-bit add, which leaves the multiply pipe (the NTT's bottleneck) to the
// products.
__device__ __forceinline__ u64 shoup_approx(u64 x, u64 w, u64 wq, u64 qneg) {
  const uint32_t xl = (uint32_t)x, xh = (uint32_t)(x >> 32);
  const uint32_t wl = (uint32_t)wq, wh = (uint32_t)(wq >> 32);
  uint32_t h1, h2;
  u64 qh, r;
  asm("mul.hi.u32 %0, %1, %2;" : "=r"(h1) : "r"(xl), "r"(wh));
  asm("mul.hi.u32 %0, %1, %2;" : "=r"(h2) : "r"(xh), "r"(wl));
  asm("mad.wide.u32 %0, %1, %2, %3;" : "=l"(qh) : "r"(xh), "r"(wh), "l"((u64)h1));
  asm("add.u64 %0, %1, %2;" : "=l"(qh) : "l"(qh), "l"((u64)h2));
  asm("mul.lo.u64 %0, %1, %2;" : "=l"(r) : "l"(x), "l"(w));
  asm("mad.lo.u64 %0, %1, %2, %3;" : "=l"(r) : "l"(qh), "l"(qneg), "l"(r));
  return r;
}
// x - m if x >= m, else x; requires x - m in (-2^63, 2^63) (the sign decides).
__device__ __forceinline__ u64 csub_sign(u64 x, u64 m) {
  const u64 d = x - m;
  return (int64_t)d < 0 ? x : d;
}

// Forward Cooley-Tukey (x, y) -> (x + w*y, x - w*y). FRESH (mode 2): x is a
// transform input, already below 4q, so it needs no reduction first.
template <int MODE, bool FRESH = false>
__device__ __forceinline__ void ct_butterfly(u64 &x, u64 &y, u64 w, u64 wq, u64 q, u64 q2) {
  if constexpr (MODE == 2) {
    const u64 q4 = 2 * q2;
    const u64 a = FRESH ? x : csub_sign(x, q4);  // [0, 8q) -> [0, 4q)
    const u64 t = shoup_approx(y, w, wq, 0 - q);
    x = a + t;
    y = a + q4 - t;
  } else if constexpr (MODE == 1) {
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

// Forward butterflies without any reduction, for moduli q < 2^57 (a mode-2
// context's towers below that size; the Q towers of the benchmark contexts
// are 55-bit). With t = the approximate-quotient product in [0, 4q):
//   x' = x + t, y' = x + 4q - t,
// so from inputs in [0, R) both outputs lie in [0, R + 4q): the range grows by
// 4q per stage. A forward transform starts below 4q and runs at most 16
// stages, so every value stays below 68q < 2^64 for q < 2^57 (not always
// below 2^63: 68q passes 2^63 once q > 2^63 / 68). Nothing needs the top bit
// clear: the products accept any 64-bit input, the consumers below reduce
// with reduce64_approx (any word) before any conditional subtraction, and the
// ModDown epilogue's left + 68q - x stays below 69q < 2^64. The per-stage conditional subtraction of
// ct_butterfly (most of its ALU work) disappears; the transform's consumer
// reduces once (reduce_free_final) or takes the lazy values directly.
constexpr u64 kFreeModulusBound = u64(1) << 57;
constexpr int kFreeRangeFactor = 68;  // values stay below 68q
static_assert(kFreeRangeFactor == 4 + 4 * 16, "inputs below 4q, 4q more per stage, at most 16 stages (N <= 2^16)");
static_assert(u64(kFreeRangeFactor + 1) <= ~u64(0) / kFreeModulusBound, "69q (the epilogue's span) fits a word");
template <bool FREE, int MODE, bool FRESH = false>
__device__ __forceinline__ void ct_bf(u64 &x, u64 &y, u64 w, u64 wq, u64 q, u64 q2) {
  if constexpr (FREE) {
    const u64 t = shoup_approx(y, w, wq, 0 - q);
    const u64 a = x;
    x = a + t;
    y = a + 2 * q2 - t;
  } else {
    ct_butterfly<MODE, FRESH>(x, y, w, wq, q, q2);
  }
}

// Inverse Gentleman-Sande (x, y) -> (x + y, (x - y) * w). FRESH (mode 2): x and
// y are canonical transform inputs, so x + y < 2q already lies in [0, 4q).
template <int MODE, bool FRESH = false>
__device__ __forceinline__ void gs_butterfly(u64 &x, u64 &y, u64 w, u64 wq, u64 q, u64 q2) {
  if constexpr (MODE == 2) {
    const u64 q4 = 2 * q2;
    const u64 s = FRESH ? x + y : csub_sign(x + y, q4);
    const u64 d = x + q4 - y;
    y = shoup_approx(d, w, wq, 0 - q);
    x = s;
  } else if constexpr (MODE == 1) {
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
template <int MODE>
__device__ __forceinline__ void gs_last(u64 &x, u64 &y, Shoup ninv, Shoup wn, u64 q, u64 q2) {
  if constexpr (MODE != 0) {
    const u64 span = MODE == 2 ? 2 * q2 : q2;  // inputs in [0, span)
    const u64 s = x + y;
    const u64 d = x + span - y;
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
// A forward transform's stage range -> canonical.
template <int MODE>
__device__ __forceinline__ u64 reduce_final(u64 x, u64 q, u64 q2) {
  if constexpr (MODE == 2) return csub_sign(csub_sign(csub_sign(x, 2 * q2), q2), q);
  else if constexpr (MODE == 1) return reduce4(x, q, q2);
  else return x;
}

// Canonical x mod q from a reduction-free forward transform's values (any
// x < 2^64): reduce64_approx (defined below) brings x into [0, 4q), two
// subtractions finish it.
__device__ __forceinline__ u64 reduce64_approx(u64 x, u64 one, u64 mneg);
__device__ __forceinline__ u64 reduce_free_final(u64 x, u64 q, u64 one) {
  return csub_sign(csub_sign(reduce64_approx(x, one, 0 - q), 2 * q), q);
}

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
// x mod m in [0, 4m) for any x < 2^64 and m < 2^62: shoup_approx with w = 1
// (one = floor(2^64 / m)), so x - e*m lies in [0, 4m) by the same argument.
__device__ __forceinline__ u64 reduce64_approx(u64 x, u64 one, u64 mneg) {
  const uint32_t xl = (uint32_t)x, xh = (uint32_t)(x >> 32);
  const uint32_t ol = (uint32_t)one, oh = (uint32_t)(one >> 32);
  uint32_t h1, h2;
  u64 e, r;
  asm("mul.hi.u32 %0, %1, %2;" : "=r"(h1) : "r"(xl), "r"(oh));
  asm("mul.hi.u32 %0, %1, %2;" : "=r"(h2) : "r"(xh), "r"(ol));
  asm("mad.wide.u32 %0, %1, %2, %3;" : "=l"(e) : "r"(xh), "r"(oh), "l"((u64)h1));
  asm("add.u64 %0, %1, %2;" : "=l"(e) : "l"(e), "l"((u64)h2));
  asm("mad.lo.u64 %0, %1, %2, %3;" : "=l"(r) : "l"(e), "l"(mneg), "l"(x));
  return r;
}
// (hi * 2^64 + lo) mod m, canonical, for m < 2^61: each half reduced into
// [0, 4m) with an approximate quotient, the sum (below 8m) brought to [0, m).
__device__ __forceinline__ u64 reduce128_approx(u64 lo, u64 hi, const Reducer &r) {
  const u64 mneg = 0 - r.m;
  const u64 s = shoup_approx(hi, r.r64, r.r64q, mneg) + reduce64_approx(lo, r.one, mneg);
  return csub_sign(csub_sign(csub_sign(s, 4 * r.m), 2 * r.m), r.m);
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

// ---- Barrett multiplication (include/ntt/barrett.hpp:10-50) ---------------------
// With mu = floor(2^128 / q) (mu_lo + 2^64 mu_hi) and x = a * b < q^2 < 2^126,
// e = floor(x * mu / 2^128) is floor(x / q) or one below it, so x - e q lies in
// [0, 2q) and is exact in its low 64 bits; one conditional subtraction ends it.
// Writing x = xh 2^64 + xl, x * mu / 2^128 = xh mu_hi + (xh mu_lo + xl mu_hi +
// hi(xl mu_lo)) / 2^64 + (a fraction that cannot carry), so e is xh mu_hi plus
// the high words of the two cross products plus the carry out of their low
// words and hi(xl mu_lo). e < q < 2^63 fits one word, so its products wrap.
struct Barrett {
  u64 q, mu_lo, mu_hi;
};
__device__ __forceinline__ u64 barrett_mul(u64 a, u64 b, const Barrett &p) {
  const u64 xl = a * b, xh = mulhi(a, b);
  const u64 c1 = xh * p.mu_lo, c2 = xl * p.mu_hi;  // low words of the cross products
  const u64 t = c1 + c2;
  const u64 u = t + mulhi(xl, p.mu_lo);
  const u64 carry = u64(t < c1) + u64(u < t);
  const u64 e = xh * p.mu_hi + mulhi(xh, p.mu_lo) + mulhi(xl, p.mu_hi) + carry;
  return csub(xl - e * p.q, p.q);
}
}  // namespace b200
