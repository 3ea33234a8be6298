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

// LAZY_OUT: outputs in [0, 4m) for a lazy forward NTT that consumes them
// directly (it accepts [0, 4q) inputs); otherwise canonical.
template <int MAXS, bool WIDE, bool LAZY_OUT>
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
  using Acc = typename std::conditional<WIDE, Acc192, Acc128>::type;
  int t = 0;
  for (; t + 1 < nt; t += 2) {
    Acc a0{}, a1{};
#pragma unroll
    for (int j = 0; j < MAXS; ++j)
      if (j < s) {
        acc_mad(a0, y[j], hat[j * nt + t]);
        acc_mad(a1, y[j], hat[j * nt + t + 1]);
      }
    dst[u64(a.slot[t0 + t]) * n + k] = reduce_out<LAZY_OUT>(a0, red[t]);
    dst[u64(a.slot[t0 + t + 1]) * n + k] = reduce_out<LAZY_OUT>(a1, red[t + 1]);
  }
  if (t < nt) {
    Acc a0{};
#pragma unroll
    for (int j = 0; j < MAXS; ++j)
      if (j < s) acc_mad(a0, y[j], hat[j * nt + t]);
    dst[u64(a.slot[t0 + t]) * n + k] = reduce_out<LAZY_OUT>(a0, red[t]);
  }
}

// Same switch when every source and target modulus is below 2^60 and s <= 8:
// with y = y1*2^30 + y0 and Bhat = h1*2^30 + h0 (30-bit limbs), the exact sum
// is H*2^60 + C*2^30 + L with L = sum y0*h0, H = sum y1*h1 and
// C = sum (y0*h1 + y1*h0) = sum (y0+y1)(h0+h1) - L - H. Each term costs three
// 32x32->64 multiply-adds and no carry handling: L, H < 8*2^60 and C < 8*2^61
// fit in 64 bits, and the (y0+y1)(h0+h1) sum may wrap because only its
// difference C is used. The result equals conv_kernel's bit for bit.
template <int MAXS, bool LAZY_OUT>
__global__ void __launch_bounds__(kEwThreads) conv_limb_kernel(ConvArgs a) {
  constexpr uint32_t kMask30 = (1u << 30) - 1;
  __shared__ uint4 hl[MAXS * kMaxConvTargets];  // (h0, h1, h0 + h1, 0) per (source, target)
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
    const u64 h = p.hat[j * p.t + t0 + t];
    const uint32_t lo = (uint32_t)h & kMask30, hi = (uint32_t)(h >> 30);
    hl[j * nt + t] = make_uint4(lo, hi, lo + hi, 0);
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
  uint32_t y0[MAXS], y1[MAXS], ys[MAXS];
#pragma unroll
  for (int j = 0; j < MAXS; ++j) {
    const u64 y = j < s ? shoup_canon(src[j * n + k], sinv[j].w, sinv[j].wq, sq[j]) : 0;
    y0[j] = (uint32_t)y & kMask30;
    y1[j] = (uint32_t)(y >> 30);
    ys[j] = y0[j] + y1[j];
  }
  auto finish = [&](u64 lo, u64 hi, u64 mid, int t) {
    Acc128 v;
    v.v = ((u128)hi << 60) + ((u128)(mid - lo - hi) << 30) + lo;
    dst[u64(a.slot[t0 + t]) * n + k] = reduce_out<LAZY_OUT>(v, red[t]);
  };
  int t = 0;
  for (; t + 1 < nt; t += 2) {
    u64 lo0 = 0, hi0 = 0, mid0 = 0, lo1 = 0, hi1 = 0, mid1 = 0;
#pragma unroll
    for (int j = 0; j < MAXS; ++j) {
      if (j < s) {
        const uint4 h = hl[j * nt + t], g = hl[j * nt + t + 1];
        lo0 += (u64)y0[j] * h.x;
        hi0 += (u64)y1[j] * h.y;
        mid0 += (u64)ys[j] * h.z;
        lo1 += (u64)y0[j] * g.x;
        hi1 += (u64)y1[j] * g.y;
        mid1 += (u64)ys[j] * g.z;
      }
    }
    finish(lo0, hi0, mid0, t);
    finish(lo1, hi1, mid1, t + 1);
  }
  if (t < nt) {
    u64 lo = 0, hi = 0, mid = 0;
#pragma unroll
    for (int j = 0; j < MAXS; ++j) {
      if (j < s) {
        const uint4 h = hl[j * nt + t];
        lo += (u64)y0[j] * h.x;
        hi += (u64)y1[j] * h.y;
        mid += (u64)ys[j] * h.z;
      }
    }
    finish(lo, hi, mid, t);
  }
}

// ---- approximate-CRT switch on the tensor cores (tcgen05, unsigned int8) -----------
// For a target m_t the output only has to be congruent to sum_j y_j * Bhat_jt
// modulo m_t. With y_j = sum_a y_ja 2^(8a) (byte limbs) and the precomputed
// c_jat = [Bhat_jt * 2^(8a)]_{m_t} = sum_b c_jatb 2^(8b):
//   sum_j y_j Bhat_jt == sum_b 2^(8b) S_tb  (mod m_t),  S_tb = sum_{j,a} y_ja c_jatb,
// and every S_tb is a plain dot product of bytes (at most 128 terms of 255^2,
// below 2^23): one [128 coefficients x 8s] x [8s x 8 per target] unsigned int8
// matrix product with int32 accumulators in tensor memory. Each thread folds
// its coefficient's eight S_tb per target into H * 2^32 + L (H, L < 2^47) and
// reduces it with one approximate quotient (tc_fold_reduce) into [0, 3.5m) for
// 2^48 <= m_t < 2^61; the result is left there (lazy output, within [0, 4m))
// or brought to [0, m). It is congruent to conv_kernel's output modulo m_t,
// hence identical once canonical.
//
// Grid: (runs of tiles_per_cta coefficient tiles, part, polynomial), where a
// part is one conversion (plan, source, destination) of the launch.
// CTA = 128 threads = 128 coefficients = the 128 TMEM lanes. A: one row of
// 8s bytes per coefficient. B: groups of 8 targets (64 rows of 8s bytes),
// built on the host per plan. Both use the canonical K-major layout without
// swizzle: core matrices of 8 rows x 16 bytes stored as [k chunk][row group]
// [8 rows][16 B], so SBO = 128 B and LBO = (rows / 8) * 128 B. Targets run in
// groups of 8 through 64 TMEM columns. A CTA runs `tiles_per_cta` consecutive
// 128-coefficient tiles; the next tile's s source rows are copied into shared
// memory (cp.async) while the current tile's products and reductions run.
// Every mbarrier wait is bounded: a timeout is reported through `err` (results
// of that CTA are then invalid), and the CTA waits (bounded) for its own bulk
// copy, matrix product and staged rows before it frees its TMEM and returns.
// Dynamic shared memory: A (128 x kpad), B (groups x 64 x kpad), staging (s KiB).
constexpr int kTcThreads = 128;
constexpr int kTcGroupTargets = 8;
constexpr int kTcGroupRows = 64;  // 8 targets x 8 output bytes
// Conversions of one launch (grid y): the Hybrid digits of one level, which
// all convert alpha sources into the L + K - alpha others, share one launch.
constexpr int kTcMaxParts = 4;
struct ConvTcPart {
  const ConvPlan *plan;
  const uint8_t *bmat;  // [groups][64 rows x kpad] bytes, canonical layout
  const u64 *src;
  u64 *dst;
  uint16_t slot[kMaxConvTargets];
};
struct ConvTcArgs {
  ConvTcPart part[kTcMaxParts];  // same source and target counts (and so kpad, groups) in every part
  u64 src_poly_stride, dst_poly_stride;
  int logn, kpad, groups;
  int tiles_per_cta;  // coefficient tiles per CTA (B, TMEM and barriers set up once per CTA)
  int first_wait_polls;  // poll limit of the first bounded wait (for B); the others use kTcWaitPolls
  int *err;
};

// r == h * 2^32 + l (mod m), r in [0, 3.5m), for h, l < 2^47, 2^48 <= m < 2^61
// and wq = floor(2^96 / m) (< 2^48). The quotient estimate
//   e = hh*wh + floor((hh*wl + hl*wh) / 2^32)    (h = hh:hl, wq = wh:wl)
// drops only hl*wl / 2^64 < 1 and a fraction below 1 from h * wq / 2^64, and
// h * wq / 2^64 is within h / 2^64 < 2^-17 of h * 2^32 / m; so e is the true
// quotient floor(h * 2^32 / m) minus 0, 1 or 2, and h * 2^32 - e m lies in
// [0, 3m). Adding l < 2^47 <= m / 2 keeps the result below 3.5m. As e < 2^32,
// e * m mod 2^64 takes one wide and one low 32-bit product, and h * 2^32 mod
// 2^64 is hl in the high word. mneg = 2^64 - m.
__device__ __forceinline__ u64 tc_fold_reduce(u64 h, u64 l, u64 mneg, u64 wq) {
  const uint32_t hl = uint32_t(h), hh = uint32_t(h >> 32);
  const uint32_t wl = uint32_t(wq), wh = uint32_t(wq >> 32);
  const u64 mid = u64(hh) * wl + u64(hl) * wh;      // < 2^49
  const uint32_t e = hh * wh + uint32_t(mid >> 32);  // < 2^32
  const u64 base = l + (u64(hl) << 32);              // h * 2^32 + l mod 2^64
  return base + u64(e) * uint32_t(mneg) + (u64(e * uint32_t(mneg >> 32)) << 32);
}

__host__ __device__ __forceinline__ int tc_canon(int r, int k, int rows) {
  return ((k >> 4) * (rows >> 3) + (r >> 3)) * 128 + (r & 7) * 16 + (k & 15);
}
__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
// Bounded wait for the completion of the mbarrier phase with the given parity:
// at most `polls` polls (0 gives up at once).
constexpr int kTcWaitPolls = 1 << 20;
__device__ __forceinline__ bool tc_wait(uint32_t bar, uint32_t parity, int polls = kTcWaitPolls) {
  uint32_t got = 0;
  for (int it = 0; it < polls && !got; ++it)
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(got)
        : "r"(bar), "r"(parity));
  return got != 0;
}
// 16-byte global -> shared copy that completes asynchronously (cp.async.wait_group).
__device__ __forceinline__ void tc_copy16(void *smem, const void *gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_addr(smem)), "l"(gmem) : "memory");
}
// Shared-memory matrix descriptor: SWIZZLE_NONE, Blackwell version 1.
__device__ __forceinline__ u64 tc_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return u64((addr >> 4) & 0x3FFF) | (u64((lbo >> 4) & 0x3FFF) << 16) | (u64((sbo >> 4) & 0x3FFF) << 32) |
         (u64(1) << 46);
}

// FS, FT: when nonzero, the plan's source and target counts as compile-time
// constants (the plan must have exactly FS sources and FT targets), so the
// per-tile loops unroll; zero takes them from the plan at run time.
template <bool LAZY_OUT, int FS = 0, int FT = 0>
__global__ void __launch_bounds__(kTcThreads) conv_tc_kernel(const __grid_constant__ ConvTcArgs a) {
  extern __shared__ __align__(1024) uint8_t tc_smem[];
  __shared__ __align__(8) u64 mbar, bbar;
  __shared__ uint32_t tmem_base;
  __shared__ u64 tm[kMaxConvTargets], twq[kMaxConvTargets];
  __shared__ u64 sq[kMaxConvSources];
  __shared__ Shoup sinv[kMaxConvSources];
  const ConvTcPart &part = a.part[blockIdx.y];
  const ConvPlan &p = *part.plan;
  const int s = FS ? FS : p.s, t_count = FT ? FT : p.t;
  const int kpad = FS ? (8 * FS + 31) / 32 * 32 : a.kpad;
  const int groups = FT ? (FT + kTcGroupTargets - 1) / kTcGroupTargets : a.groups;
  const int tid = threadIdx.x, warp = tid >> 5;
  uint8_t *sa = tc_smem;                      // 128 x kpad
  uint8_t *sb = tc_smem + kTcThreads * kpad;  // groups x 64 x kpad
  const uint32_t bbytes = uint32_t(groups * kTcGroupRows * kpad);
  uint8_t *stage = sb + bbytes;                // s x 128 words: the next tile's source rows
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&mbar)), "r"(1));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&bbar)), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;");
    // B (built on the host in canonical order) arrives by one bulk copy while
    // the first tile's A rows are computed; 16-byte aligned, size a multiple of 16.
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(&bbar)), "r"(bbytes));
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(sb)),
        "l"(part.bmat), "r"(bbytes), "r"(smem_addr(&bbar))
        : "memory");
  }
  for (int t = tid; t < t_count; t += kTcThreads) {
    tm[t] = p.tgt[t].m;
    twq[t] = p.tc_wq32[t];
  }
  for (int j = tid; j < s; j += kTcThreads) {
    sq[j] = p.src_q[j];
    sinv[j] = p.src_inv[j];
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_base)),
                 "r"(kTcGroupRows));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  __syncthreads();
  const uint32_t tmem = tmem_base;
  const u64 n = u64(1) << a.logn;
  const u64 *src = part.src + blockIdx.z * a.src_poly_stride;
  u64 *dst = part.dst + blockIdx.z * a.dst_poly_stride;
  // idesc: S32 accumulate, unsigned 8-bit A and B, K-major, N = 64, M = 128.
  const uint32_t idesc = (2u << 4) | (uint32_t(kTcGroupRows >> 3) << 17) | (uint32_t(kTcThreads >> 4) << 24);
  const uint32_t tiles = uint32_t(n / kTcThreads);
  // The s source rows of a tile (128 words each) are copied into `stage` while
  // the previous tile's matrix products and reductions run.
  auto stage_tile = [&](uint32_t tile) {
    const u64 *rows = src + u64(tile) * kTcThreads;
    // Each pass of the CTA copies two source rows: row j, words w and w + 1.
    const int w = (tid & (kTcThreads / 2 - 1)) * 2;
#pragma unroll(FS ? 8 : 1)
    for (int j = tid / (kTcThreads / 2); j < s; j += 2)
      tc_copy16(stage + (j * kTcThreads + w) * sizeof(u64), rows + (u64(j) << a.logn) + w);
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  const uint32_t first = blockIdx.x * uint32_t(a.tiles_per_cta);
  if (first < tiles) stage_tile(first);
  bool ok = true, b_pending = true, mma_pending = false;
  uint32_t phase = 0;  // completed MMA groups so far (mbarrier phase parity)
  for (int ti = 0; ti < a.tiles_per_cta && ok; ++ti) {
    const uint32_t tile = first + ti;
    if (tile >= tiles) break;  // uniform across the CTA
    const u64 k = u64(tile) * kTcThreads + tid;
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncthreads();
    const u64 *rows = reinterpret_cast<const u64 *>(stage);
    // A row of this thread's coefficient: the byte limbs of y_j, zero-padded.
#pragma unroll(FS ? 16 : 1)
    for (int j = 0; j < kpad / 8; ++j) {
      const u64 y = j < s ? shoup_canon(rows[j * kTcThreads + tid], sinv[j].w, sinv[j].wq, sq[j]) : 0;
      *reinterpret_cast<u64 *>(sa + tc_canon(tid, j * 8, kTcThreads)) = y;  // little-endian bytes = limbs
    }
    asm volatile("fence.proxy.async.shared::cta;");
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    // Every thread has read the staged rows: bring in the next tile's.
    if (ti + 1 < a.tiles_per_cta && tile + 1 < tiles) stage_tile(tile + 1);
    if (ti == 0) {  // B must have landed before the first MMA reads it
      if (!__syncthreads_and(tc_wait(smem_addr(&bbar), 0, a.first_wait_polls))) {
        ok = false;
        break;
      }
      b_pending = false;
    }
#pragma unroll(FT ? 10 : 1)
    for (int g = 0; g < groups; ++g) {
      if (tid == 0) {
        for (int i = 0; i < kpad / 32; ++i) {
          const u64 da = tc_desc(smem_addr(sa) + i * 2 * (kTcThreads / 8) * 128, (kTcThreads / 8) * 128, 128);
          const u64 db = tc_desc(smem_addr(sb + g * kTcGroupRows * kpad) + i * 2 * (kTcGroupRows / 8) * 128,
                                 (kTcGroupRows / 8) * 128, 128);
          const uint32_t acc = i > 0;
          asm volatile(
              "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
              "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
              "l"(da), "l"(db), "r"(idesc), "r"(acc));
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
            smem_addr(&mbar)));
      }
      // One decision for the whole CTA: every thread leaves together on a timeout.
      const bool all_done = __syncthreads_and(tc_wait(smem_addr(&mbar), phase & 1));
      asm volatile("tcgen05.fence::after_thread_sync;");
      if (!all_done) {
        ok = false;
        mma_pending = true;
        break;
      }
      ++phase;
      const int tl_end = min(kTcGroupTargets, t_count - g * kTcGroupTargets);
      // Four targets' 8 columns per load, one wait per load.
#pragma unroll
      for (int tq = 0; tq < kTcGroupTargets; tq += 4) {
        if (tq >= tl_end) break;
        uint32_t v[32];
        const uint32_t addr = tmem + (uint32_t(warp * 32) << 16) + uint32_t(tq * 8);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
            "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
              "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
              "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]),
              "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]),
              "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
            : "r"(addr));
        asm volatile("tcgen05.wait::ld.sync.aligned;");
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int tl = tq + u;
          if (tl >= tl_end) break;
          const uint32_t *w = v + 8 * u;
          // Each sum is below 2^23, so w0 + w1 * 2^8 and w2 + w3 * 2^8 fit in 32 bits.
          const u64 lo4 = u64(w[0] + (w[1] << 8)) + (u64(w[2] + (w[3] << 8)) << 16);
          const u64 hi4 = u64(w[4] + (w[5] << 8)) + (u64(w[6] + (w[7] << 8)) << 16);
          const int t = g * kTcGroupTargets + tl;
          const u64 m = tm[t];
          u64 r = tc_fold_reduce(hi4, lo4, 0 - m, twq[t]);  // [0, 3.5m)
          if constexpr (!LAZY_OUT) r = csub_sign(csub_sign(r, 2 * m), m);
          dst[(u64(part.slot[t]) << a.logn) + k] = r;  // slot * n (n = 2^logn)
        }
      }
      // Every lane's loads are done before the next MMA reuses the columns.
      asm volatile("tcgen05.fence::before_thread_sync;");
      __syncthreads();
      asm volatile("tcgen05.fence::after_thread_sync;");
    }
  }
  if (!ok && tid == 0) atomicExch(a.err, 1);
  // Nothing may still write this CTA's shared memory or TMEM once it leaves:
  // B, a timed-out matrix product and any staged rows are waited for (bounded).
  if (b_pending) tc_wait(smem_addr(&bbar), 0);
  if (mma_pending) tc_wait(smem_addr(&mbar), phase & 1);
  asm volatile("cp.async.wait_all;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcGroupRows));
}

// ---- ModDown tail: (l - r) * [P^-1]_q  (resident_conversion.hpp:45-49) ---------
struct CorrectArgs {
  u64 *dst, *dst_odd;  // dst_odd set: polynomial z writes (z odd ? dst_odd : dst) + (z / 2) * stride
  u64 *const *dst_list;        // optional: polynomial z writes dst_list[z]
  const u64 *const *add_list;  // optional: add_list[z] (if not null) is added to the result
  const u64 *left, *right;
  const Shoup *pinv;  // [P^-1]_q by Q tower
  const TowerConsts *tc;
  u64 poly_stride_dst, poly_stride_left, poly_stride_right;
  int towers, logn;
};
static __global__ void __launch_bounds__(kEwThreads) correct_kernel(CorrectArgs a) {
  const u64 n = u64(1) << a.logn;
  const u64 i = u64(blockIdx.x) * blockDim.x + threadIdx.x;
  const int t = blockIdx.y;
  if (i >= n) return;
  const u64 q = a.tc[t].q;  // Q tower t has global id t
  const Shoup pinv = a.pinv[t];
  const u64 z = blockIdx.z;
  const u64 l = a.left[z * a.poly_stride_left + t * n + i];
  const u64 r = a.right[z * a.poly_stride_right + t * n + i];
  u64 *dst = a.dst_list ? a.dst_list[z]
             : a.dst_odd ? ((z & 1) ? a.dst_odd : a.dst) + (z >> 1) * a.poly_stride_dst
                         : a.dst + z * a.poly_stride_dst;
  u64 o = shoup_canon(sub_mod(l, r, q), pinv.w, pinv.wq, q);
  const u64 *add = a.add_list ? a.add_list[z] : nullptr;
  if (add) o = add_mod(o, add[t * n + i], q);
  dst[t * n + i] = o;
}

// ---- Hybrid MAC over all digits in one pass --------------------------------------
// Z_b[t] = sum_d D_d[t] * KB_d[row(t)], Z_a likewise (resident.cpp:530-570 with
// hybrid_mac_value, resident_conversion.hpp:50-54). Keys are either full-context
// rows (row(t) = t for active Q, M + (t - L) for P: key_indices,
// backend_contract.hpp:112-119) or already packed active rows (row(t) = t).
// With accumulate set, the result is added to the existing outputs (the
// reference's per-digit primitive for digits after the first).
constexpr int kMaxDigits = 40;

// One key-switch request of a request-table launch (a device-resident table
// written by put_words before the pipeline runs).
// Evaluation-domain automorphism X -> X^g on the bit-reversed layout: output
// slot k takes input slot automorphism_source(k) (automorphism_source_index of
// include/ntt/resident_conversion.hpp:15-29; resident_adapter.inc:44-59).
__device__ __forceinline__ uint32_t automorphism_source(uint32_t k, int logn, uint32_t g) {
  const uint32_t odd = 2 * (__brev(k) >> (32 - logn)) + 1;
  const uint32_t src = (uint32_t)((u64(odd) * g) & ((u64(2) << logn) - 1));
  return __brev(src >> 1) >> (32 - logn);
}
// g^-1 mod 2^32 for odd g by Newton's iteration x <- x(2 - gx), which doubles
// the correct low bits (g*g = 1 mod 8 gives 3 to start: 6, 12, 24, 48). Input
// slot i of the automorphism by g lands in output slot automorphism_source(i)
// of g^-1, since (2 bitrev(i) + 1) g^-1 undoes the multiplication by g.
__device__ __forceinline__ uint32_t inverse_mod_pow2(uint32_t g) {
  uint32_t x = g;
#pragma unroll
  for (int r = 0; r < 4; ++r) x *= 2u - g * x;
  return x;
}

struct ReqDesc {
  const u64 *src;            // evaluation Q_L component being switched ([L][N])
  const u64 *key_b, *key_a;  // full-context key: digit d at key + d * key_digit_stride
  const u64 *c0;             // rotation: first component ([L][N]); null: no rotation
  uint32_t g;                // automorphism index (1 = identity)
  uint32_t dslot;            // digit slot; requests that share an input share its digits
  u64 pad;
};
static_assert(sizeof(ReqDesc) == 48, "ReqDesc is uploaded as 6 words");

struct MacArgs {
  u64 *out_b, *out_a;
  const u64 *digit[kMaxDigits];  // digit d, tower t at digit[d] + z * poly_stride_digits + t * n
  const u64 *key_b[kMaxDigits], *key_a[kMaxDigits];
  const u64 *input;              // if set: digit d's own Q towers are read from input + t * n
  const TowerConsts *tc;
  const ReqDesc *req;            // if set: per-request input, keys and digit slot (full-context keys)
  u64 key_digit_stride;          // words between key digits (request-table mode)
  u64 poly_stride_out, poly_stride_digits, poly_stride_input;
  int level, m, beta, alpha, logn;
  bool full_key_rows, accumulate;
  // Rotation fused into the MAC (mac2_kernel<..., ROT>): request z adds P * c0
  // on its Q towers of the b channel and writes slot i to automorphism slot
  // automorphism_source(i, g^-1). Request-table mode takes c0 and g from req[z].
  const u64 *c0;
  u64 c0_poly_stride;
  const DownPlan *plan;  // the level's P mod q_i
  uint32_t g;
};

// Per-request bases of a MAC thread: request z's digit slot, input and keys.
struct MacBases {
  u64 dz;
  const u64 *input;
  const u64 *kb, *ka;  // request-table mode: digit 0 of the request's key
  const u64 *c0;       // rotation: the request's c0 (null: none)
  uint32_t g;          // rotation: the request's automorphism (1: identity)
};
__device__ __forceinline__ MacBases mac_bases(const MacArgs &a, u64 z) {
  MacBases m;
  if (a.req) {
    const ReqDesc r = a.req[z];
    m.dz = r.dslot;
    m.input = r.src;
    m.kb = r.key_b;
    m.ka = r.key_a;
    m.c0 = r.c0;
    m.g = r.g;
  } else {
    m.dz = z;
    m.input = a.input ? a.input + z * a.poly_stride_input : nullptr;
    m.kb = m.ka = nullptr;
    m.c0 = a.c0 ? a.c0 + z * a.c0_poly_stride : nullptr;
    m.g = a.g;
  }
  return m;
}
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
  const u64 row = (a.full_key_rows || a.req) ? u64(g) : u64(t);
  const MacBases mb = mac_bases(a, z);
  const int own = (mb.input && t < a.level) ? t / a.alpha : -1;
  const u64 doff = mb.dz * a.poly_stride_digits + t * n + i;
  using Acc = typename std::conditional<WIDE, Acc192, Acc128>::type;
  Acc ab{}, aa{};
#pragma unroll 4
  for (int j = 0; j < a.beta; ++j) {
    const u64 x = j == own ? mb.input[t * n + i] : a.digit[j][doff];
    const u64 *kb = a.req ? mb.kb + j * a.key_digit_stride : a.key_b[j];
    const u64 *ka = a.req ? mb.ka + j * a.key_digit_stride : a.key_a[j];
    acc_mad(ab, x, kb[row * n + i]);
    acc_mad(aa, x, ka[row * n + i]);
  }
  const u64 o = z * a.poly_stride_out + t * n + i;
  u64 rb = reduce(ab, red), ra = reduce(aa, red);
  if (a.accumulate) {
    rb = add_mod(rb, a.out_b[o], red.m);
    ra = add_mod(ra, a.out_a[o], red.m);
  }
  a.out_b[o] = rb;
  a.out_a[o] = ra;
}

// Same MAC with a compile-time digit count and two adjacent coefficients per
// thread (16-byte loads of every digit and key row).
// APPROX (every modulus below 2^61, sums below 2^128): the final reductions
// take approximate quotients (reduce128_approx); results are identical.
// ROT: the rotation of the extended result (rotate_kernel) happens here: the
// sums at slot i, plus P * c0[i] on the b channel's Q towers, are stored at
// the slot that the automorphism moves i to. That saves the rotation's full
// read and write of both QP channels; the stores are 8-byte scattered ones
// within a tower, which L2 merges before they reach HBM. Not with accumulate.
// Resident CTAs per SM: 5 (48 registers), 6 with the rotation (40). The MAC
// waits mostly on its loads, and the extra warps cut its time by 5% and 10%
// on a B200 (16 requests at L = 24) against the unconstrained 52 registers,
// despite a few bytes of spills.
template <int BETA, bool WIDE, bool APPROX = false, bool ROT = false>
__global__ void __launch_bounds__(kEwThreads, ROT ? 6 : 5) mac2_kernel(MacArgs a) {
  static_assert(!(WIDE && APPROX), "approximate reduction needs sums below 2^128");
  const u64 n = u64(1) << a.logn;
  const u64 i = (u64(blockIdx.x) * blockDim.x + threadIdx.x) * 2;
  const int t = blockIdx.z;
  const u64 z = blockIdx.y;
  if (i >= n) return;
  const int g = t < a.level ? t : a.m + (t - a.level);
  const Reducer red = a.tc[g].red;
  const u64 row = (a.full_key_rows || a.req) ? u64(g) : u64(t);
  const MacBases mb = mac_bases(a, z);
  const int own = (mb.input && t < a.level) ? t / a.alpha : -1;
  const u64 doff = mb.dz * a.poly_stride_digits + t * n + i;
  using Acc = typename std::conditional<WIDE, Acc192, Acc128>::type;
  Acc b0{}, b1{}, a0{}, a1{};
#pragma unroll
  for (int j = 0; j < BETA; ++j) {
    const ulonglong2 x = j == own ? *reinterpret_cast<const ulonglong2 *>(mb.input + t * n + i)
                                  : *reinterpret_cast<const ulonglong2 *>(a.digit[j] + doff);
    const u64 *kbp = a.req ? mb.kb + j * a.key_digit_stride : a.key_b[j];
    const u64 *kap = a.req ? mb.ka + j * a.key_digit_stride : a.key_a[j];
    const ulonglong2 kb = *reinterpret_cast<const ulonglong2 *>(kbp + row * n + i);
    const ulonglong2 ka = *reinterpret_cast<const ulonglong2 *>(kap + row * n + i);
    acc_mad(b0, x.x, kb.x);
    acc_mad(b1, x.y, kb.y);
    acc_mad(a0, x.x, ka.x);
    acc_mad(a1, x.y, ka.y);
  }
  const u64 o = z * a.poly_stride_out + t * n + i;
  ulonglong2 rb, ra;
  if constexpr (APPROX) {
    rb.x = reduce128_approx((u64)b0.v, (u64)(b0.v >> 64), red);
    rb.y = reduce128_approx((u64)b1.v, (u64)(b1.v >> 64), red);
    ra.x = reduce128_approx((u64)a0.v, (u64)(a0.v >> 64), red);
    ra.y = reduce128_approx((u64)a1.v, (u64)(a1.v >> 64), red);
  } else {
    rb.x = reduce(b0, red);
    rb.y = reduce(b1, red);
    ra.x = reduce(a0, red);
    ra.y = reduce(a1, red);
  }
  if constexpr (ROT) {
    if (mb.c0 && t < a.level) {  // rotated_b_value: b + P * c0 on the Q towers
      const Shoup pm = a.plan->p_mod[t];
      const ulonglong2 c = *reinterpret_cast<const ulonglong2 *>(mb.c0 + t * n + i);
      rb.x = add_mod(rb.x, shoup_canon(c.x, pm.w, pm.wq, red.m), red.m);
      rb.y = add_mod(rb.y, shoup_canon(c.y, pm.w, pm.wq, red.m), red.m);
    }
    const uint32_t gi = inverse_mod_pow2(mb.g);
    const u64 base = o - i;
    const u64 d0 = base + automorphism_source((uint32_t)i, a.logn, gi);
    const u64 d1 = base + automorphism_source((uint32_t)i + 1, a.logn, gi);
    a.out_b[d0] = rb.x;
    a.out_b[d1] = rb.y;
    a.out_a[d0] = ra.x;
    a.out_a[d1] = ra.y;
    return;
  }
  if (a.accumulate) {
    const ulonglong2 ob = *reinterpret_cast<const ulonglong2 *>(a.out_b + o);
    const ulonglong2 oa = *reinterpret_cast<const ulonglong2 *>(a.out_a + o);
    rb.x = add_mod(rb.x, ob.x, red.m);
    rb.y = add_mod(rb.y, ob.y, red.m);
    ra.x = add_mod(ra.x, oa.x, red.m);
    ra.y = add_mod(ra.y, oa.y, red.m);
  }
  *reinterpret_cast<ulonglong2 *>(a.out_b + o) = rb;
  *reinterpret_cast<ulonglong2 *>(a.out_a + o) = ra;
}

// Same MAC with 30-bit limbs, when every QP modulus is below 2^60 and
// BETA <= 8: each product x * k = (x1*2^30 + x0)(k1*2^30 + k0) accumulates
// into L += x0*k0, H += x1*k1 and M += (x0+x1)(k0+k1); the exact sum is
// H*2^60 + (M - L - H)*2^30 + L (conv_limb_kernel's scheme: three multiply-adds
// per product and no carry handling). Results equal mac2_kernel's bit for bit.
template <int BETA>
__global__ void __launch_bounds__(kEwThreads) mac2_limb_kernel(MacArgs a) {
  constexpr u64 kMask30 = (u64(1) << 30) - 1;
  const u64 n = u64(1) << a.logn;
  const u64 i = (u64(blockIdx.x) * blockDim.x + threadIdx.x) * 2;
  const int t = blockIdx.z;
  const u64 z = blockIdx.y;
  if (i >= n) return;
  const int g = t < a.level ? t : a.m + (t - a.level);
  const Reducer red = a.tc[g].red;
  const u64 row = (a.full_key_rows || a.req) ? u64(g) : u64(t);
  const MacBases mb = mac_bases(a, z);
  const int own = (mb.input && t < a.level) ? t / a.alpha : -1;
  const u64 doff = mb.dz * a.poly_stride_digits + t * n + i;
  // accumulators by (channel, coefficient): b.x, b.y, a.x, a.y
  u64 lo[4] = {0, 0, 0, 0}, hi[4] = {0, 0, 0, 0}, mid[4] = {0, 0, 0, 0};
  auto mad = [&](int s, u64 x0, u64 x1, u64 xs, u64 k) {
    const u64 k0 = k & kMask30, k1 = k >> 30;
    lo[s] += (u64)(uint32_t)x0 * (uint32_t)k0;
    hi[s] += (u64)(uint32_t)x1 * (uint32_t)k1;
    mid[s] += (u64)(uint32_t)xs * (uint32_t)(k0 + k1);
  };
#pragma unroll
  for (int j = 0; j < BETA; ++j) {
    const ulonglong2 x = j == own ? *reinterpret_cast<const ulonglong2 *>(mb.input + t * n + i)
                                  : *reinterpret_cast<const ulonglong2 *>(a.digit[j] + doff);
    const u64 *kbp = a.req ? mb.kb + j * a.key_digit_stride : a.key_b[j];
    const u64 *kap = a.req ? mb.ka + j * a.key_digit_stride : a.key_a[j];
    const ulonglong2 kb = *reinterpret_cast<const ulonglong2 *>(kbp + row * n + i);
    const ulonglong2 ka = *reinterpret_cast<const ulonglong2 *>(kap + row * n + i);
    const u64 p0 = x.x & kMask30, p1 = x.x >> 30, q0 = x.y & kMask30, q1 = x.y >> 30;
    mad(0, p0, p1, p0 + p1, kb.x);
    mad(1, q0, q1, q0 + q1, kb.y);
    mad(2, p0, p1, p0 + p1, ka.x);
    mad(3, q0, q1, q0 + q1, ka.y);
  }
  u64 r[4];
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    Acc128 v;
    v.v = ((u128)hi[s] << 60) + ((u128)(mid[s] - lo[s] - hi[s]) << 30) + lo[s];
    r[s] = reduce(v, red);
  }
  const u64 o = z * a.poly_stride_out + t * n + i;
  ulonglong2 rb = make_ulonglong2(r[0], r[1]), ra = make_ulonglong2(r[2], r[3]);
  if (a.accumulate) {
    const ulonglong2 ob = *reinterpret_cast<const ulonglong2 *>(a.out_b + o);
    const ulonglong2 oa = *reinterpret_cast<const ulonglong2 *>(a.out_a + o);
    rb.x = add_mod(rb.x, ob.x, red.m);
    rb.y = add_mod(rb.y, ob.y, red.m);
    ra.x = add_mod(ra.x, oa.x, red.m);
    ra.y = add_mod(ra.y, oa.y, red.m);
  }
  *reinterpret_cast<ulonglong2 *>(a.out_b + o) = rb;
  *reinterpret_cast<ulonglong2 *>(a.out_a + o) = ra;
}

// ---- rotation: automorphism gather plus P*c0 on Q towers ------------------------
// With a request table, request z rotates by req[z].g and adds P * req[z].c0
// (a request without c0 and g = 1 passes through unchanged).
struct RotateArgs {
  u64 *out_b, *out_a;
  const u64 *ext_b, *ext_a, *c0;
  const DownPlan *plan;
  const TowerConsts *tc;
  const ReqDesc *req;
  u64 poly_stride, c0_poly_stride;
  int level, m, logn;
  uint32_t g;
};
static __global__ void __launch_bounds__(kEwThreads) rotate_kernel(RotateArgs a) {
  const u64 n = u64(1) << a.logn;
  const u64 k = u64(blockIdx.x) * blockDim.x + threadIdx.x;
  const int t = blockIdx.y;
  if (k >= n) return;
  const u64 z = blockIdx.z;
  uint32_t g = a.g;
  const u64 *c0 = a.c0 ? a.c0 + z * a.c0_poly_stride : nullptr;
  if (a.req) {
    g = a.req[z].g;
    c0 = a.req[z].c0;
  }
  const u64 src = t * n + automorphism_source((uint32_t)k, a.logn, g);
  u64 b = a.ext_b[z * a.poly_stride + src];
  if (c0 && t < a.level) {
    const u64 q = a.tc[t].q;
    const Shoup pm = a.plan->p_mod[t];
    b = add_mod(b, shoup_canon(c0[src], pm.w, pm.wq, q), q);
  }
  a.out_b[z * a.poly_stride + t * n + k] = b;
  a.out_a[z * a.poly_stride + t * n + k] = a.ext_a[z * a.poly_stride + src];
}

// ---- request-table upload ------------------------------------------------------------
// Copies a small table from the launch's parameter space into device memory,
// so a host-built table reaches the GPU in stream order without a host staging
// buffer.
template <int WORDS>
struct Words {
  uint32_t count;
  u64 w[WORDS];
};
template <int WORDS>
__global__ void put_words(Words<WORDS> p, u64 *dst) {
  for (uint32_t i = threadIdx.x; i < p.count; i += blockDim.x) dst[i] = p.w[i];
}

// ---- device arithmetic probes ------------------------------------------------------
// One query per thread (5 words each), as the reference probes its device
// arithmetic against host 128-bit arithmetic (tests/basis_cuda.cu:49-65):
//   op 0: (x, w, w', q)          -> x * w mod q, Shoup, canonical;
//   op 1: (a, b, q, mu_lo, mu_hi) -> a * b mod q, Barrett with mu = floor(2^128 / q);
//   op 2: (x, w, w', q)          -> the NTT's approximate-quotient Shoup product, in [0, 4q).
static __global__ void __launch_bounds__(kEwThreads) arith_probe_kernel(int op, const u64 *queries, u64 count, u64 *out) {
  const u64 i = u64(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const u64 *qr = queries + 5 * i;
  if (op == 0) {
    out[i] = shoup_canon(qr[0], qr[1], qr[2], qr[3]);
  } else if (op == 1) {
    out[i] = barrett_mul(qr[0], qr[1], Barrett{qr[2], qr[3], qr[4]});
  } else {
    out[i] = shoup_approx(qr[0], qr[1], qr[2], 0 - qr[3]);
  }
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
static __global__ void __launch_bounds__(kEwThreads) pointwise_kernel(PointwiseArgs a) {
  const u64 n = u64(1) << a.logn;
  const u64 i = u64(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int t = blockIdx.y;
  const Reducer red = a.tc[a.id[t]].red;
  const u64 o = blockIdx.z * a.poly_stride + t * n + i;
  a.dst[o] = mul_mod(a.left[o], a.right[o], red);
}

}  // namespace b200
