// Device-resident tables of one CKKS context, built once per context and kept
// in HBM for its lifetime (the reference rebuilds and re-uploads conversion
// tables on every Session::switch_basis call, src/resident.cpp:350-365).
//
// Towers are addressed by a global id: Q tower i -> i, P tower j -> M + j.
#pragma once
#include <cstdint>

#include "arith.cuh"

namespace b200 {

struct TowerConsts {
  u64 q, q2;        // modulus and 2q
  Shoup ninv;       // N^-1
  Shoup last_inv;   // psi^-(N/2) * N^-1: the inverse's last butterfly with the scale folded in
  Reducer red;      // generic reduction constants
};

struct DeviceTables {
  const TowerConsts *tc;  // [M + K]
  // (w, w') pairs at index k: w = psi^bitrev(k) (forward) or psi^-bitrev(k)
  // (inverse), k in [1, N); the group-twiddle layout of the reference's
  // transform_twiddles (include/ntt/transform_stage.hpp:19-30).
  const ulonglong2 *fwd;  // [M + K][N]
  const ulonglong2 *inv;  // [M + K][N]
  int logn;
};

// Lane-major order of the row passes' register-bit stages. In a two-pass
// transform (N >= 2^12, R = N / 256 rows, logR = logN - 8) stage s = logR + sp,
// sp = 4..7, gives row `row` the 2^sp entries at 2^s + row * 2^sp, and lane u
// (0..15) of that row reads offsets u * 2^(sp-4) + k, k < 2^(sp-4). The tables
// hold offset u * 2^(sp-4) + k at position 16 k + u, so for a fixed k the 16
// lanes of a row read 16 consecutive entries (256 contiguous bytes) instead of
// entries 2^(sp-4) apart. Stages below logR + 4 keep the plain layout.
__host__ __device__ constexpr uint32_t row_lane_major(uint32_t u, uint32_t k) { return (k << 4) | u; }
constexpr int kLaneMajorMinLogn = 12;

// Approximate-CRT switch from `s` source towers to `t` target towers
// (include/ntt/basis_conversion.hpp:13-30):
//   y_j = [x_j * Bhat_j^-1]_{b_j},  out_i = [sum_j y_j * [Bhat_j]_{m_i}]_{m_i}.
// Plans built with `ninv` fold N^-1 into Bhat_j^-1, for sources that arrive
// straight out of an unscaled inverse NTT (N times the coefficients, lazily
// reduced); y_j, and so every output, is the same as the scaled path's.
constexpr int kMaxConvSources = 40;
constexpr int kMaxConvTargets = 80;
struct ConvPlan {
  int s, t;
  u64 src_q[kMaxConvSources];
  Shoup src_inv[kMaxConvSources];      // Bhat_j^-1 mod b_j
  uint16_t src_id[kMaxConvSources];    // global tower ids
  uint16_t tgt_id[kMaxConvTargets];
  Reducer tgt[kMaxConvTargets];
  u64 hat[kMaxConvSources * kMaxConvTargets];  // [j][i] = Bhat_j mod m_i
  u64 tc_wq32[kMaxConvTargets];                 // floor(2^96 / m_i): Shoup quotient of 2^32 mod m_i (m_i > 2^32)
};

// ModDown tail constants for one level: per Q tower [P^-1]_q and [P]_q.
constexpr int kMaxTowers = 128;
struct DownPlan {
  Shoup p_inv[kMaxTowers];
  Shoup p_mod[kMaxTowers];
};

}  // namespace b200
