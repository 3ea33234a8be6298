// Forward row pass of the Hybrid digits fused with the key multiplication.
//
// The key switch's digits (Session::hybrid_digits, src/resident.cpp:458-491)
// are used once, by the MAC (Session::hybrid_accumulate, src/resident.cpp:
// 530-570, hybrid_mac_value of include/ntt/resident_conversion.hpp:50-54).
// Here one CTA takes one QP tower t, one block of 2 * WARPS rows (256 words
// each) and one distinct input. It runs the forward NTT's row pass (the last
// 8 stages) of every digit that has to be transformed at that tower, keeps the
// transformed rows in shared memory, and then forms, for every request that
// shares the input,
//   Z_b[t] = sum_d D_d[t] * KB_d[row(t)],  Z_a[t] = sum_d D_d[t] * KA_d[row(t)]
// with exact 128-bit sums and one reduction per output; the digit a Q tower
// belongs to is read from the input itself (it is the input's own tower). The
// digits never reach HBM: the separate MAC pass, and its re-read of every
// digit tower, is gone. With ROT, the rotation of the extended result happens
// in the same stores (P * c0 added on b's Q towers, slot i stored at the slot
// the automorphism moves it to; resident_hybrid_rotate_kernel of
// src/cuda/resident_adapter.inc:44-59).
//
// On the P towers the ModDown starts right away (p_inverse_rows): the MAC
// leaves both channels' values in shared memory, over the digit words it has
// just read, and the inverse NTT's row pass (Session::mod_down's transform,
// src/resident.cpp:448-457) runs on them before anything is stored, so the P
// part is written once, as that pass's output, instead of being written by
// the MAC and read and rewritten by a separate row pass. A rotation moves whole
// rows: the automorphism's source slot of destination row r_d lies in one row
// r_s, which depends on r_d only, so the row pass of r_d gathers its 256 words
// from row r_s of the CTA.
//
// Layout: each warp owns two rows through both register phases of every
// digit's row pass and through the MAC, so the CTA never synchronises; its
// dynamic shared memory holds one padded region of 2 * WARPS rows per digit it
// transforms. The Q towers (beta - 1 digits: their own digit is the input) and
// the P towers (beta digits) run as two launches with their own region counts,
// so the common Q towers fit three CTAs per SM at beta = 3.
// Arithmetic: every modulus below 2^61 (butterfly mode 2). Digits stay in the
// butterflies' lazy range: [0, 8q), or [0, 68q) for towers below 2^57 whose
// butterflies skip the per-stage reduction; keys and the input are canonical,
// so with at most 4 digits the sums stay below max(4 * 8q * q, 4 * 68q * q)
// < 2^127 and the approximate-quotient reduction (reduce128_approx) applies.
#pragma once
#include <cstdint>

#include "arith.cuh"
#include "kernels.cuh"
#include "ntt.cuh"
#include "tables.cuh"

namespace b200 {

struct RowMacArgs {
  MacArgs mac;            // outputs, keys, input, request table, rotation (see mac2_kernel)
  const u64 *digits;      // digit d of tower t, distinct input u: digits + u * digit_stride + (d * towers + t) * n
  u64 digit_stride;
  const u64 *groups;      // request-table mode: per distinct input, first request | count << 32
  int towers;             // L + K
  // P towers, beta >= 2, one request per input: the P part of both channels
  // goes through the ModDown's first pass (the inverse NTT's row pass) in
  // shared memory and is stored as that pass's output.
  bool p_inverse_rows;
};

// Shared memory of one launch: Q towers transform beta - 1 digits (their own
// digit is the input), P towers all beta. Regions of 2 * WARPS padded rows.
template <int WARPS>
constexpr int row_mac_smem_bytes(int regions) {
  return regions * 2 * WARPS * kRowPad * int(sizeof(u64));
}
// CTAs per SM that a launch's shared memory allows (228 KiB per SM, 1 KiB of
// it reserved per CTA), at most 3: the register bound of __launch_bounds__, so
// that a launch whose shared memory admits fewer CTAs gets the registers.
template <int WARPS>
constexpr int row_mac_ctas_per_sm(int regions) {
  const int per_cta = row_mac_smem_bytes<WARPS>(regions) + 1024;
  const int fit = (228 * 1024) / per_cta;
  return fit < 1 ? 1 : fit > 3 ? 3 : fit;
}

// 8-byte global -> shared copy that completes asynchronously (cp.async groups).
__device__ __forceinline__ void rm_copy8(u64 *smem, const u64 *gmem) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(smem))),
               "l"(gmem)
               : "memory");
}

// PT: the launch covers the P towers (tower t = L + blockIdx.z), else the Q
// towers (t = blockIdx.z). The digits a CTA transforms run in order through
// shared-memory regions 0, 1, ...; the rows of the next one are copied into
// its region (cp.async) while the current one's butterflies run.
// FREE: reduction-free butterflies (ct_bf) for a tower with q < 2^57; its
// digits then reach the key multiplication below 68q, and the sums stay below
// 4 * 68q * q < 2^123.
template <int LOGN, int BETA, int WARPS, bool ROT, bool PT, bool FREE>
__device__ __forceinline__ void row_mac_body(const RowMacArgs &a, const DeviceTables &T, u64 *rm_digits) {
  constexpr int LR = LOGN - 8;
  constexpr u64 N = u64(1) << LOGN;
  constexpr int kRows = 2 * WARPS;  // rows per CTA
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int h = lane >> 4, u = lane & 15;
  const int L = a.mac.level;
  const int t = PT ? L + int(blockIdx.z) : int(blockIdx.z);
  const int gid = PT ? a.mac.m + int(blockIdx.z) : t;  // global tower id (key_indices, backend_contract.hpp:112-119)
  const TowerConsts *tc = T.tc + gid;
  const u64 q = tc->q, q2 = tc->q2;
  const ulonglong2 *tw = T.fwd + u64(gid) * N;
  const int wrow = blockIdx.x * kRows + 2 * warp;  // the warp's first row
  const int row = wrow + h;
  const u64 input = blockIdx.y;
  const int own = PT ? -1 : t / a.mac.alpha;
  constexpr int kMaxRegions = PT ? BETA : BETA - 1;
  // Digit of region i, and the source rows of a digit.
  auto digit_of = [&](int i) { return PT ? i : (i < own ? i : i + 1); };
  // The copy's addresses are rebuilt from a laundered lane index each time, so
  // none of them stays live across the butterflies of the digit in flight.
  auto stage_rows = [&](int i) {
    uint32_t ln = lane;
    asm volatile("" : "+r"(ln));
    // Word k of the lane: row k / 8 of the warp's two, column ln + 32 (k % 8)
    // (pad_col of it: ln + ln / 16 + 34 (k % 8)).
    const u64 *src =
        a.digits + input * a.digit_stride + (u64(digit_of(i)) * a.towers + t) * N + u64(wrow) * 256 + ln;
    u64 *dst = rm_digits + (i * kRows + 2 * warp) * kRowPad + ln + (ln >> 4);
#pragma unroll 4
    for (int k = 0; k < 16; ++k) rm_copy8(dst + (k >> 3) * kRowPad + 34 * (k & 7), src + (k >> 3) * 256 + 32 * (k & 7));
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  if constexpr (kMaxRegions > 0) stage_rows(0);

  // Row passes (stages logR .. logN-1) of the digits this tower transforms.
#pragma unroll 1
  for (int i = 0; i < kMaxRegions; ++i) {
    if (i + 1 < kMaxRegions) {
      stage_rows(i + 1);
      asm volatile("cp.async.wait_group 1;" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    }
    __syncwarp();
    u64 *my = rm_digits + (i * kRows + 2 * warp + h) * kRowPad;
    u64 x[16];
#pragma unroll
    for (int e = 0; e < 16; ++e) x[e] = my[pad_col(e * 16 + u)];
#pragma unroll
    for (int sp = 0; sp < 4; ++sp) {
      const int s = LR + sp, dd = 8 >> sp;
#pragma unroll
      for (int e = 0; e < 16; ++e) {
        if (e & dd) continue;
        const Shoup w = tw_load(tw + (1 << s) + (row << sp) + (e >> (4 - sp)));
        ct_bf<FREE, 2>(x[e], x[e + dd], w.w, w.wq, q, q2);
      }
    }
    __syncwarp();
#pragma unroll
    for (int e = 0; e < 16; ++e) my[pad_col(e * 16 + u)] = x[e];
    __syncwarp();
#pragma unroll
    for (int e = 0; e < 16; ++e) x[e] = my[pad_col(u * 16 + e)];
#pragma unroll
    for (int sp = 4; sp < 8; ++sp) {
      const int s = LR + sp, dd = 1 << (7 - sp);
#pragma unroll
      for (int e = 0; e < 16; ++e) {
        if (e & dd) continue;
        const Shoup w = tw_load(tw + (1 << s) + (row << sp) + row_lane_major(u, e >> (8 - sp)));
        ct_bf<FREE, 2>(x[e], x[e + dd], w.w, w.wq, q, q2);
      }
    }
    // Each thread overwrites exactly the words it has just read: no barrier.
#pragma unroll
    for (int e = 0; e < 16; ++e) my[pad_col(u * 16 + e)] = x[e];
  }
  __syncwarp();

  // Key multiplication over the warp's two rows: 2 adjacent coefficients per
  // lane and step, 16-byte loads of the input's own tower and of the keys.
  const Reducer red = tc->red;
  // Two digit regions hold the two channels; the host sets p_inverse_rows
  // only when every input serves one request (its digits are then dead).
  const bool inv_rows = PT && BETA >= 2 && a.p_inverse_rows;
  u64 first = input, count = 1;
  if (a.groups) {
    const u64 gw = a.groups[input];
    first = gw & 0xFFFFFFFFu;
    count = gw >> 32;
  }
  for (u64 z = first; z < first + count; ++z) {
    const MacBases mb = mac_bases(a.mac, z);
    const u64 *kb[BETA], *ka[BETA];
#pragma unroll
    for (int d = 0; d < BETA; ++d) {
      kb[d] = (a.mac.req ? mb.kb + d * a.mac.key_digit_stride : a.mac.key_b[d]) + u64(gid) * N;
      ka[d] = (a.mac.req ? mb.ka + d * a.mac.key_digit_stride : a.mac.key_a[d]) + u64(gid) * N;
    }
    const u64 obase = z * a.mac.poly_stride_out + u64(t) * N;
    const uint32_t gi = ROT ? inverse_mod_pow2(mb.g) : 1u;
    Shoup pm{0, 0};
    if (ROT && mb.c0 && !PT) pm = a.mac.plan->p_mod[t];
    // Step `it` of a lane takes row wrow + it / 4, columns c = 2 lane +
    // 64 (it % 4): a per-lane base plus offsets (pad_col(c) = 2 lane +
    // lane / 8 + 68 (it % 4) in shared memory).
    const u64 ibase = u64(wrow) * 256 + 2 * lane;
    const int sbase = 2 * warp * kRowPad + 2 * lane + (lane >> 3);
#pragma unroll 2
    for (int it = 0; it < 8; ++it) {
      const int rr = it >> 2;
      const u64 i = ibase + rr * 256 + 64 * (it & 3);
      const int soff = sbase + rr * kRowPad + 68 * (it & 3);
      Acc128 b0{}, b1{}, a0{}, a1{};
#pragma unroll
      for (int d = 0; d < BETA; ++d) {
        ulonglong2 x;
        if (!PT && d == own) {
          x = *reinterpret_cast<const ulonglong2 *>(mb.input + u64(t) * N + i);
        } else {
          const int region = PT ? d : (d < own ? d : d - 1);
          const u64 *sd = rm_digits + region * kRows * kRowPad + soff;
          x = make_ulonglong2(sd[0], sd[1]);
        }
        const ulonglong2 vb = *reinterpret_cast<const ulonglong2 *>(kb[d] + i);
        const ulonglong2 va = *reinterpret_cast<const ulonglong2 *>(ka[d] + i);
        acc_mad(b0, x.x, vb.x);
        acc_mad(b1, x.y, vb.y);
        acc_mad(a0, x.x, va.x);
        acc_mad(a1, x.y, va.y);
      }
      ulonglong2 rb, ra;
      rb.x = reduce128_approx((u64)b0.v, (u64)(b0.v >> 64), red);
      rb.y = reduce128_approx((u64)b1.v, (u64)(b1.v >> 64), red);
      ra.x = reduce128_approx((u64)a0.v, (u64)(a0.v >> 64), red);
      ra.y = reduce128_approx((u64)a1.v, (u64)(a1.v >> 64), red);
      if (inv_rows) {
        // Channel b over digit 0's words of these two slots, channel a over
        // digit 1's: this lane has read them above and no other lane reads them.
        u64 *sb = rm_digits + soff;
        u64 *sa = sb + kRows * kRowPad;
        sb[0] = rb.x;
        sb[1] = rb.y;
        sa[0] = ra.x;
        sa[1] = ra.y;
        continue;
      }
      if constexpr (ROT) {
        if (!PT && mb.c0) {  // rotated_b_value: b + P * c0 on the Q towers
          const ulonglong2 cc = *reinterpret_cast<const ulonglong2 *>(mb.c0 + u64(t) * N + i);
          rb.x = add_mod(rb.x, shoup_canon(cc.x, pm.w, pm.wq, red.m), red.m);
          rb.y = add_mod(rb.y, shoup_canon(cc.y, pm.w, pm.wq, red.m), red.m);
        }
        const u64 d0 = obase + automorphism_source((uint32_t)i, LOGN, gi);
        const u64 d1 = obase + automorphism_source((uint32_t)i + 1, LOGN, gi);
        a.mac.out_b[d0] = rb.x;
        a.mac.out_b[d1] = rb.y;
        a.mac.out_a[d0] = ra.x;
        a.mac.out_a[d1] = ra.y;
      } else {
        *reinterpret_cast<ulonglong2 *>(a.mac.out_b + obase + i) = rb;
        *reinterpret_cast<ulonglong2 *>(a.mac.out_a + obase + i) = ra;
      }
    }
    if (inv_rows) {
      // The inverse NTT's row pass of the warp's two destination rows per
      // channel, 16 threads per row; with a rotation, destination row rd takes
      // slot automorphism_source(rd * 256 + col, g) of source row `row`.
      __syncwarp();
      // In bit-reversed slot order (br_k: k-bit reversal, R = logN - 8 row bits)
      // the automorphism moves source row `row` to destination row
      //   rd = br_R((((2 br_R(row) + 1) g^-1) >> 1) mod 2^R),
      // and destination word (rd, 16u + e) comes from column
      //   br8((base + 16 * (br4(e) g mod 16)) mod 256) of row `row`, with
      //   base = br4(u) g + (((2 br_R(rd) + 1) g mod 2N) >> (logN - 7))
      // (automorphism_source written out in 32-bit arithmetic).
      int rd = row;
      uint32_t base = 0, g16 = 0;
      if constexpr (ROT) {
        constexpr int R = LOGN - 8;
        const uint32_t rbr = __brev(uint32_t(row)) >> (32 - R);
        rd = int(__brev((((2 * rbr + 1) * gi) >> 1) & ((1u << R) - 1)) >> (32 - R));
        const uint32_t g = mb.g, dbr = __brev(uint32_t(rd)) >> (32 - R);
        const uint32_t carry = (((2 * dbr + 1) * g) & uint32_t(2 * N - 1)) >> (LOGN - 7);
        base = (__brev(uint32_t(u)) >> 28) * g + carry;
        g16 = g & 15u;
      }
      const ulonglong2 *itw = T.inv + u64(gid) * N;
#pragma unroll 1
      for (int ch = 0; ch < 2; ++ch) {
        u64 *my = rm_digits + (ch * kRows + 2 * warp + h) * kRowPad;
        u64 x[16];
#pragma unroll
        for (int e = 0; e < 16; ++e) {
          constexpr uint32_t kBr4[16] = {0, 8, 4, 12, 2, 10, 6, 14, 1, 9, 5, 13, 3, 11, 7, 15};
          const uint32_t cs =
              ROT ? __brev((base + 16 * ((kBr4[e] * g16) & 15u)) & 255u) >> 24 : uint32_t(u * 16 + e);
          x[e] = my[pad_col(int(cs))];
        }
        inv_row_stages<LOGN, 2, FREE>(x, my, itw, rd, u, q, q2);
        u64 *o = (ch == 0 ? a.mac.out_b : a.mac.out_a) + obase + u64(rd) * 256 + u;
#pragma unroll
        for (int e = 0; e < 16; ++e) o[e * 16] = x[e];
      }
    }
  }
}

// The CTA's tower decides the butterflies: reduction-free below 2^57.
template <int LOGN, int BETA, int WARPS, bool ROT, bool PT>
__global__ void __launch_bounds__(WARPS * 32, row_mac_ctas_per_sm<WARPS>(PT ? BETA : BETA - 1))
    ntt_fwd_row_mac(RowMacArgs a, DeviceTables T) {
  extern __shared__ __align__(16) u64 rm_digits[];  // [regions][2 * WARPS rows][kRowPad]
  const int gid = PT ? a.mac.m + int(blockIdx.z) : int(blockIdx.z);
  if (T.tc[gid].q < kFreeModulusBound)
    row_mac_body<LOGN, BETA, WARPS, ROT, PT, true>(a, T, rm_digits);
  else
    row_mac_body<LOGN, BETA, WARPS, ROT, PT, false>(a, T, rm_digits);
}

}  // namespace b200
