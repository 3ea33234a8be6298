// Element-wise and basis-conversion kernels of the Hybrid key-switch path.
// All are streaming integer kernels over limb-major [tower][N] words.
#pragma once
#include <cstdint>
#include <type_traits>

#include "arith.cuh"
#include "tables.cuh"

namespace b200 {

constexpr int kEwThreads = 256;

// ---- approximate-CRT basis switch ---------------------------------------------
// out[slot[i]][k] = [sum_j y_j[k] * Bhat_j mod m_i]_{m_i},
// y_j[k] = [x_j[k] * Bhat_j^-1]_{b_j}   (include/ntt/basis_conversion.hpp:13-30).
// The sum is exact (128- or 192-bit) and reduced once per output; it is never
// reduced modulo the source product (the approximate lift the reference keeps).
struct ConvArgs {
  const ConvPlan *plan;
  const u64 *src;   // source tower j at src + j * n (+ poly * src_poly_stride)
  u64 *dst;         // target i at dst + slot[i] * n (+ poly * dst_poly_stride)
  u64 src_poly_stride, dst_poly_stride;
  uint16_t slot[kMaxConvTargets];
  int logn;
  int targets_per_block;
};

template <int MAXS, bool WIDE>
__global__ void __launch_bounds__(kEwThreads) conv_kernel(ConvArgs a) {
  __shared__ u64 hat[MAXS * kMaxConvTargets];
  __shared__ Reducer red[kMaxConvTargets];
  __shared__ u64 sq[MAXS];
  __shared__ Shoup sinv[MAXS];
  const ConvPlan &p = *a.plan;
  const int s = p.s;
  const int t0 = blockIdx.y * a.targets_per_block;
  const int t1 = min(p.t, t0 + a.targets_per_block);
  const int nt = t1 - t0;
  for (int i = threadIdx.x; i < s * nt; i += blockDim.x) {
    const int j = i / nt, t = i % nt;
    hat[j * nt + t] = p.hat[j * p.t + t0 + t];
  }
  for (int t = threadIdx.x; t < nt; t += blockDim.x) red[t] = p.tgt[t0 + t];
  for (int j = threadIdx.x; j < s; j += blockDim.x) {
    sq[j] = p.src_q[j];
    sinv[j] = p.src_inv[j];
  }
  __syncthreads();
  const u64 n = u64(1) << a.logn;
  const u64 k = u64(blockIdx.x) * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const u64 *src = a.src + blockIdx.z * a.src_poly_stride;
  u64 *dst = a.dst + blockIdx.z * a.dst_poly_stride;
  u64 y[MAXS];
#pragma unroll
  for (int j = 0; j < MAXS; ++j)
    if (j < s) y[j] = shoup_canon(src[j * n + k], sinv[j].w, sinv[j].wq, sq[j]);
  for (int t = 0; t < nt; ++t) {
    u64 out;
    if constexpr (WIDE) {
      Acc192 acc;
      acc_zero(acc);
#pragma unroll
      for (int j = 0; j < MAXS; ++j)
        if (j < s) acc_mad(acc, y[j], hat[j * nt + t]);
      out = reduce(acc, red[t]);
    } else {
      Acc128 acc{0, 0};
#pragma unroll
      for (int j = 0; j < MAXS; ++j)
        if (j < s) acc_mad(acc, y[j], hat[j * nt + t]);
      out = reduce(acc, red[t]);
    }
    dst[u64(a.slot[t0 + t]) * n + k] = out;
  }
}

// ---- ModDown tail: (l - r) * [P^-1]_q  (resident_conversion.hpp:45-49) ---------
struct CorrectArgs {
  u64 *dst, *dst_odd;  // dst_odd set: polynomial z writes (z odd ? dst_odd : dst) + (z / 2) * stride
  const u64 *left, *right;
  const Shoup *pinv;  // [P^-1]_q by Q tower
  const TowerConsts *tc;
  u64 poly_stride_dst, poly_stride_left, poly_stride_right;
  int towers, logn;
};
__global__ void __launch_bounds__(kEwThreads) correct_kernel(CorrectArgs a) {
  const u64 n = u64(1) << a.logn;
  const u64 i = u64(blockIdx.x) * blockDim.x + threadIdx.x;
  const int t = blockIdx.y;
  if (i >= n) return;
  const u64 q = a.tc[t].q;  // Q tower t has global id t
  const Shoup pinv = a.pinv[t];
  const u64 z = blockIdx.z;
  const u64 l = a.left[z * a.poly_stride_left + t * n + i];
  const u64 r = a.right[z * a.poly_stride_right + t * n + i];
  u64 *dst = a.dst_odd ? ((z & 1) ? a.dst_odd : a.dst) + (z >> 1) * a.poly_stride_dst
                       : a.dst + z * a.poly_stride_dst;
  dst[t * n + i] = shoup_canon(sub_mod(l, r, q), pinv.w, pinv.wq, q);
}

// ---- Hybrid MAC over all digits in one pass --------------------------------------
// Z_b[t] = sum_d D_d[t] * KB_d[row(t)], Z_a likewise (resident.cpp:530-570 with
// hybrid_mac_value, resident_conversion.hpp:50-54). Keys are full-context:
// digit d, row r at key + d * key_digit_stride + r * n; row(t) = t for active Q,
// M + (t - L) for P (key_indices, backend_contract.hpp:112-119).
struct MacArgs {
  u64 *out_b, *out_a;
  const u64 *digits;    // digit d, tower t at digits + d * digit_stride + t * n
  const u64 *input;     // if set: digit d's own Q towers are read from input + t * n
  const u64 *key_b, *key_a;
  const TowerConsts *tc;
  u64 digit_stride, key_digit_stride;
  u64 poly_stride_out, poly_stride_digits, poly_stride_input;
  int level, m, beta, alpha, logn;
};
// Grid: x = coefficient block, y = request, z = QP tower. Requests vary faster
// than towers, so the key rows of one tower stay in L2 while every request of
// the batch streams through them.
template <bool WIDE>
__global__ void __launch_bounds__(kEwThreads) mac_kernel(MacArgs a) {
  const u64 n = u64(1) << a.logn;
  const u64 i = u64(blockIdx.x) * blockDim.x + threadIdx.x;
  const int t = blockIdx.z;
  const u64 z = blockIdx.y;
  if (i >= n) return;
  const int g = t < a.level ? t : a.m + (t - a.level);
  const Reducer red = a.tc[g].red;
  const u64 *d = a.digits + z * a.poly_stride_digits + t * n + i;
  const int own = (a.input && t < a.level) ? t / a.alpha : -1;
  const u64 *kb = a.key_b + u64(g) * n + i;
  const u64 *ka = a.key_a + u64(g) * n + i;
  using Acc = typename std::conditional<WIDE, Acc192, Acc128>::type;
  Acc ab{}, aa{};
  for (int j = 0; j < a.beta; ++j) {
    const u64 x = j == own ? a.input[z * a.poly_stride_input + t * n + i] : d[j * a.digit_stride];
    acc_mad(ab, x, kb[j * a.key_digit_stride]);
    acc_mad(aa, x, ka[j * a.key_digit_stride]);
  }
  const u64 o = z * a.poly_stride_out + t * n + i;
  a.out_b[o] = reduce(ab, red);
  a.out_a[o] = reduce(aa, red);
}

// ---- rotation: automorphism gather plus P*c0 on Q towers ------------------------
// resident_adapter.inc:44-59 semantics with automorphism_source_index and
// rotated_b_value (resident_conversion.hpp:15-29).
__device__ __forceinline__ uint32_t automorphism_source(uint32_t k, int logn, uint32_t g) {
  const uint32_t odd = 2 * (__brev(k) >> (32 - logn)) + 1;
  const uint32_t src = (uint32_t)((u64(odd) * g) & ((u64(2) << logn) - 1));
  return __brev(src >> 1) >> (32 - logn);
}
struct RotateArgs {
  u64 *out_b, *out_a;
  const u64 *ext_b, *ext_a, *c0;
  const DownPlan *plan;
  const TowerConsts *tc;
  u64 poly_stride, c0_poly_stride;
  int level, m, logn;
  uint32_t g;
};
__global__ void __launch_bounds__(kEwThreads) rotate_kernel(RotateArgs a) {
  const u64 n = u64(1) << a.logn;
  const u64 k = u64(blockIdx.x) * blockDim.x + threadIdx.x;
  const int t = blockIdx.y;
  if (k >= n) return;
  const u64 z = blockIdx.z;
  const u64 src = t * n + automorphism_source((uint32_t)k, a.logn, a.g);
  u64 b = a.ext_b[z * a.poly_stride + src];
  if (t < a.level) {
    const u64 q = a.tc[t].q;
    const Shoup pm = a.plan->p_mod[t];
    b = add_mod(b, shoup_canon(a.c0[z * a.c0_poly_stride + src], pm.w, pm.wq, q), q);
  }
  a.out_b[z * a.poly_stride + t * n + k] = b;
  a.out_a[z * a.poly_stride + t * n + k] = a.ext_a[z * a.poly_stride + src];
}

// ---- pointwise product ------------------------------------------------------------
struct PointwiseArgs {
  u64 *dst;
  const u64 *left, *right;
  const TowerConsts *tc;
  u64 poly_stride;
  uint16_t id[kMaxTowers];
  int towers, logn;
};
__global__ void __launch_bounds__(kEwThreads) pointwise_kernel(PointwiseArgs a) {
  const u64 n = u64(1) << a.logn;
  const u64 i = u64(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int t = blockIdx.y;
  const Reducer red = a.tc[a.id[t]].red;
  const u64 o = blockIdx.z * a.poly_stride + t * n + i;
  a.dst[o] = mul_mod(a.left[o], a.right[o], red);
}

}  // namespace b200
