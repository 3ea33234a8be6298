// Negacyclic NTT kernels for sm_100a.
//
// Transform (identical outputs to the reference NegacyclicNtt,
// include/ntt/ntt.hpp:96-158): forward maps natural coefficients to evaluations
// at psi^(2j+1) stored in bit-reversed order; inverse maps them back and scales
// by N^-1. The schedule is the group-twiddle Cooley-Tukey / Gentleman-Sande
// pair of the reference's CUDA path (include/ntt/transform_stage.hpp:40-80):
// stage s (m = 2^s groups) pairs j with j + N/2^(s+1) and uses twiddle
// T[2^s + (j >> (logN - s))].
//
// B200 schedule. N = R x 256 (R = 2^(logN-8), 16 <= R <= 256) is split in two
// passes over 4096-word (32 KiB) tiles, one CTA of 256 threads each:
//   column pass: stages 0 .. logR-1 over R rows x (4096/R) columns,
//   row pass:    stages logR .. logN-1 over 16 contiguous rows of 256 words.
// Each thread keeps 16 words in registers and runs up to 4 stages there
// (radix-16), exchanging through shared memory between register phases.
// Global traffic is staged through shared memory so every load and store is a
// coalesced 16-byte vector access. Forward = column pass then row pass; inverse
// = row pass then column pass with N^-1 folded into its last butterfly.
// Small transforms (N <= 2048) run one CTA per tower entirely in shared memory.
#pragma once
#include <cooperative_groups.h>
#include <cstdint>

#include "arith.cuh"
#include "tables.cuh"

namespace b200 {

constexpr int kNttThreads = 256;
constexpr int kTileWords = 4096;
constexpr int kRowPad = 272;  // 256 words + one pad word per 16

// A batch of tower transforms: slot y (blockIdx.z) of polynomial z
// (blockIdx.y) is read at src + z * src_stride + off[y] * N, written at
// dst + z * dst_stride + off[y] * N, and uses the tables of global tower id[y].
// Polynomials vary faster than slots, so the CTAs that read one tower's
// twiddle table run back to back and find it in L2.
// Optional destination split: with dst_odd set, polynomial z is written at
// (z odd ? dst_odd : dst) + (z / 2) * dst_stride (the b and a channels of a
// key switch land in separate caller buffers).
// Optional forward epilogue (ModDown tail, include/ntt/resident_conversion.hpp:45-49):
// with epi_left set, the last forward pass writes (left - ntt(x)) * pinv[id].
// Optional per-polynomial pointer lists (device arrays indexed by z) replace
// the strided bases: src_list[z] / dst_list[z] are polynomial z's source and
// destination, and add_list[z] (entries may be null) is added to the ModDown
// epilogue's output (relinearization: c0 + b, c1 + a).
constexpr int kMaxSlots = 128;
struct NttBatch {
  u64 *dst;
  const u64 *src;
  u64 src_stride, dst_stride;
  u64 *dst_odd;
  const u64 *const *src_list;
  u64 *const *dst_list;
  const u64 *const *add_list;
  const u64 *epi_left;
  u64 epi_left_stride;
  const Shoup *epi_pinv;
  uint32_t off[kMaxSlots];
  uint16_t id[kMaxSlots];
  bool unscaled;  // host side: inverse without N^-1 (selects the UNSCALED column pass)
  bool lazy_out;  // forward: leave the outputs in the butterflies' range ([0, 8q) in mode 2)
};

__device__ __forceinline__ const u64 *poly_src(const NttBatch &b, u64 z) {
  return b.src_list ? b.src_list[z] : b.src + z * b.src_stride;
}
__device__ __forceinline__ u64 *poly_dst(const NttBatch &b, u64 z) {
  if (b.dst_list) return b.dst_list[z];
  return b.dst_odd ? ((z & 1) ? b.dst_odd : b.dst) + (z >> 1) * b.dst_stride : b.dst + z * b.dst_stride;
}
__device__ __forceinline__ const u64 *poly_add(const NttBatch &b, u64 z) {
  return b.add_list ? b.add_list[z] : nullptr;
}

// MINB: minimum resident CTAs per SM the compiler must allow (register cap
// 65536 / (256 * MINB)); 4 gives 32 warps per SM at 64 registers, 3 gives 24
// warps at 85 registers. The autotuner picks it per pass.

struct TowerView {
  const TowerConsts *c;
  const ulonglong2 *tw;
  const u64 *src;
  u64 *dst;
};

__device__ __forceinline__ TowerView tower_view(const NttBatch &b, const DeviceTables &T, bool inv) {
  const uint32_t slot = blockIdx.z;
  const uint32_t g = b.id[slot];
  const u64 n = u64(1) << T.logn;
  const u64 offset = u64(b.off[slot]) * n;
  TowerView v;
  v.c = T.tc + g;
  v.tw = (inv ? T.inv : T.fwd) + g * n;
  const u64 z = blockIdx.y;
  v.src = poly_src(b, z) + offset;
  v.dst = poly_dst(b, z) + offset;
  return v;
}

// Block indices passed through an empty asm, so that addresses recomputed from
// them at the end of a kernel are not merged with the copies computed at its
// start (which would keep those alive, in registers or spilled, across the
// butterflies).
struct BlockIds {
  uint32_t x, slot, poly;
};
__device__ __forceinline__ BlockIds fresh_block_ids() {
  BlockIds i{blockIdx.x, blockIdx.z, blockIdx.y};
  asm volatile("" : "+r"(i.x), "+r"(i.slot), "+r"(i.poly));
  return i;
}
// Offset of the slot's tower inside a polynomial, and that tower's destination.
__device__ __forceinline__ u64 tower_offset(const NttBatch &b, const DeviceTables &T, const BlockIds &i) {
  return u64(b.off[i.slot]) * (u64(1) << T.logn);
}
__device__ __forceinline__ u64 *tower_dst(const NttBatch &b, const DeviceTables &T, const BlockIds &i) {
  return poly_dst(b, i.poly) + tower_offset(b, T, i);
}

// Hint: bring [p, p + bytes) into L2 (p 16-byte aligned, bytes a multiple of 16).
__device__ __forceinline__ void prefetch_l2(const void *p, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

__device__ __forceinline__ Shoup tw_load(const ulonglong2 *p) {
  const ulonglong2 v = __ldg(p);
  return Shoup{v.x, v.y};
}

// Gentleman-Sande stages that skip the sums' conditional subtraction (mode 2,
// towers below 2^57): STAGES stages on 16 registers, register distances 1, 2,
// 4, 8 in that order, registers entering below F * q. Each register's bound
// after each stage is known at compile time (gs_bound): the sum of a pair
// doubles the pair's bound, the difference side restarts below 4q (the
// approximate-quotient product takes any word below 2^64), so the difference
// is formed as x + bound(y) - y. From 4q the largest bound is 64q after four
// stages, below 2^63. At the end every register takes exactly the conditional
// subtractions that bring it below 4q: log2(bound / 4q) of them, 15 per thread
// for four stages from 4q instead of one per butterfly (32).
// tw_of(j, e): the Shoup twiddle of pair (e, e + 2^j) in stage j.
__host__ __device__ constexpr int gs_bound(int f, int e, int j) {
  int last = -1;  // the last stage (register bit) in which e was the difference side
  for (int i = 0; i < j; ++i)
    if ((e >> i) & 1) last = i;
  return last < 0 ? f << j : 4 << (j - 1 - last);
}
// Compile-time proof of gs_bound for F and STAGES, by the stage-by-stage
// propagation it summarises: bounds in units of q, registers entering below F;
// in each pair the sum's bound is the sum of both, the difference side leaves
// the product below 4. It also checks what the butterflies rely on: both
// registers of a pair share a bound B (so x + Bq - y never underflows), the
// product's input x + Bq - y < 2Bq and every bound stay at or below 64
// (64q < 2^63 for q < 2^57: no wrap, and csub_sign's sign test holds), and
// the halving ladder at the end (32q, 16q, 8q, 4q) reaches 4q from any bound
// up to 64.
__host__ __device__ constexpr bool gs_bound_holds(int f, int stages) {
  int b[16] = {};
  for (int e = 0; e < 16; ++e) b[e] = f;
  for (int j = 0; j < stages; ++j) {
    const int d = 1 << j;
    for (int e = 0; e < 16; ++e) {
      if (e & d) continue;
      if (b[e] != gs_bound(f, e, j) || b[e + d] != b[e] || 2 * b[e] > 64) return false;
      b[e] += b[e + d];
      b[e + d] = 4;
    }
  }
  for (int e = 0; e < 16; ++e)
    if (b[e] != gs_bound(f, e, stages) || b[e] > 64) return false;
  return true;
}
template <int F, int STAGES, typename TwOf>
__device__ __forceinline__ void gs_stages_light(u64 (&x)[16], TwOf tw_of, u64 q) {
  const u64 qneg = 0 - q;
#pragma unroll
  for (int j = 0; j < STAGES; ++j) {
    const int d = 1 << j;
#pragma unroll
    for (int e = 0; e < 16; ++e) {
      if (e & d) continue;
      const Shoup w = tw_of(j, e);
      const u64 s = x[e] + x[e + d];
      x[e + d] = shoup_approx(x[e] + u64(gs_bound(F, e, j)) * q - x[e + d], w.w, w.wq, qneg);
      x[e] = s;
    }
  }
  static_assert(F <= 4 && STAGES <= 4, "bounds stay at or below 64q");
  static_assert(gs_bound_holds(F, STAGES), "gs_bound disagrees with the stage-by-stage bounds");
  const u64 q4 = 4 * q, q8 = 8 * q, q16 = 16 * q, q32 = 32 * q;
#pragma unroll
  for (int e = 0; e < 16; ++e) {
    const int f = gs_bound(F, e, STAGES);  // x[e] < f q; each step halves the bound
    if (f > 32) x[e] = csub_sign(x[e], q32);
    if (f > 16) x[e] = csub_sign(x[e], q16);
    if (f > 8) x[e] = csub_sign(x[e], q8);
    if (f > 4) x[e] = csub_sign(x[e], q4);
  }
}

// Coalesced copy of a [rows x width] global block (row stride `stride` words)
// into shared memory with the given padded row pitch. width is a multiple of 2.
template <int ROWS, int WIDTH, int PITCH, bool PAD16>
__device__ __forceinline__ void load_block(u64 *smem, const u64 *g, u64 stride) {
  constexpr int CHUNKS = ROWS * WIDTH / 2;
  for (int j = threadIdx.x; j < CHUNKS; j += kNttThreads) {
    const int r = j / (WIDTH / 2), c = (j % (WIDTH / 2)) * 2;
    const ulonglong2 v = *reinterpret_cast<const ulonglong2 *>(g + r * stride + c);
    const int s = r * PITCH + c + (PAD16 ? (c >> 4) : 0);
    if constexpr (PAD16) {  // padded rows: s may be odd, so two 8-byte stores
      smem[s] = v.x;
      smem[s + 1] = v.y;
    } else {  // one 16-byte store (no bank conflict)
      *reinterpret_cast<ulonglong2 *>(smem + s) = v;
    }
  }
}
template <int ROWS, int WIDTH, int PITCH, bool PAD16>
__device__ __forceinline__ void store_block(u64 *g, const u64 *smem, u64 stride) {
  constexpr int CHUNKS = ROWS * WIDTH / 2;
  for (int j = threadIdx.x; j < CHUNKS; j += kNttThreads) {
    const int r = j / (WIDTH / 2), c = (j % (WIDTH / 2)) * 2;
    const int s = r * PITCH + c + (PAD16 ? (c >> 4) : 0);
    ulonglong2 v;
    if constexpr (PAD16) {
      v.x = smem[s];
      v.y = smem[s + 1];
    } else {
      v = *reinterpret_cast<const ulonglong2 *>(smem + s);
    }
    *reinterpret_cast<ulonglong2 *>(g + r * stride + c) = v;
  }
}

// ---- column pass -------------------------------------------------------------
// Tile: R rows x COLS columns starting at column blockIdx.x * COLS.
// Thread (c, u): c = tid % COLS, u = tid / COLS in [0, R/16).
// Mapping A: element e is row e * (R/16) + u     (varies the top 4 row bits).
// Mapping B: element e is row (u * 2^(8-logR) + (e >> (logR-4))) * (R/16) + (e & (R/16-1))
//            (varies the low logR-4 row bits).
template <int LOGN>
struct ColGeom {
  static constexpr int LR = LOGN - 8, R = 1 << LR, COLS = kTileWords / R, TPC = R / 16;
  static constexpr int LO_BITS = LR - 4;
  __device__ static int row_a(int e, int u) { return e * TPC + u; }
  __device__ static int row_b(int e, int u) {
    return ((u << (8 - LR)) + (e >> LO_BITS)) * TPC + (e & (TPC - 1));
  }
};

// DIRECT: the half-warps of both mappings read and write 16 or more
// consecutive words of one row, so with DIRECT set the passes load their
// inputs and store their outputs straight between registers and global memory
// (coalesced 8-byte accesses) and use shared memory only for the exchange
// between the two register phases.
// FREE: the reduction-free butterflies (ct_bf) for a tower with q < 2^57; the
// pass then leaves its values below 4q + 4q * logR.
template <int LOGN, int MODE, bool DIRECT, bool FREE>
__device__ __forceinline__ void fwd_col_body(const NttBatch &b, const DeviceTables &T, u64 *tile, ulonglong2 *tw) {
  using G = ColGeom<LOGN>;
  constexpr int N = 1 << LOGN;
  constexpr u64 kStride = N >> G::LR;
  const TowerView v = tower_view(b, T, false);
  const u64 q = v.c->q, q2 = v.c->q2;
  const int col0 = blockIdx.x * G::COLS;
  const int c = threadIdx.x % G::COLS, u = threadIdx.x / G::COLS;
  u64 x[16];
  if constexpr (DIRECT) {
#pragma unroll
    for (int e = 0; e < 16; ++e) x[e] = v.src[G::row_a(e, u) * kStride + col0 + c];
  }
  for (int i = threadIdx.x; i < G::R; i += kNttThreads) tw[i] = v.tw[i];
  if constexpr (!DIRECT) load_block<G::R, G::COLS, G::COLS, false>(tile, v.src + col0, kStride);
  __syncthreads();
  if constexpr (!DIRECT) {
#pragma unroll
    for (int e = 0; e < 16; ++e) x[e] = tile[G::row_a(e, u) * G::COLS + c];
  }
  // Stages 0..3: row bit logR-1-s == register bit 3-s; group = e >> (4-s).
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    const int d = 8 >> s;
#pragma unroll
    for (int e = 0; e < 16; ++e) {
      if (e & d) continue;
      const ulonglong2 w = tw[(1 << s) + (e >> (4 - s))];
      // Stage 0 reads the transform's inputs, below 4q (canonical, or a
      // basis switch's lazy output), so mode 2 skips their first reduction.
      if (s == 0)
        ct_bf<FREE, MODE, true>(x[e], x[e + d], w.x, w.y, q, q2);
      else
        ct_bf<FREE, MODE>(x[e], x[e + d], w.x, w.y, q, q2);
    }
  }
  if constexpr (G::LR > 4) {
    if constexpr (!DIRECT) __syncthreads();  // every thread has read its inputs from the tile
#pragma unroll
    for (int e = 0; e < 16; ++e) tile[G::row_a(e, u) * G::COLS + c] = x[e];
    __syncthreads();
#pragma unroll
    for (int e = 0; e < 16; ++e) x[e] = tile[G::row_b(e, u) * G::COLS + c];
    // Stages 4..logR-1: row bit logR-1-s == register bit logR-1-s. With
    // row_b(e, u) = 16u + e and k = logR - s <= 4 the twiddle is entry
    // (1 << s) + (u << (4 - k)) + (e >> k): one base per stage.
#pragma unroll
    for (int s = 4; s < G::LR; ++s) {
      const int d = 1 << (G::LR - 1 - s), k = G::LR - s;
      const ulonglong2 *tws = tw + (1 << s) + (u << (4 - k));
#pragma unroll
      for (int e = 0; e < 16; ++e) {
        if (e & d) continue;
        const ulonglong2 w = tws[e >> k];
        ct_bf<FREE, MODE>(x[e], x[e + d], w.x, w.y, q, q2);
      }
    }
    if constexpr (DIRECT) {
      u64 *const dst = tower_dst(b, T, fresh_block_ids()) + col0 + c;
#pragma unroll
      for (int e = 0; e < 16; ++e) dst[G::row_b(e, u) * kStride] = x[e];
      return;
    }
    __syncthreads();
#pragma unroll
    for (int e = 0; e < 16; ++e) tile[G::row_b(e, u) * G::COLS + c] = x[e];
  } else {
    if constexpr (DIRECT) {
      u64 *const dst = tower_dst(b, T, fresh_block_ids()) + col0 + c;
#pragma unroll
      for (int e = 0; e < 16; ++e) dst[G::row_a(e, u) * kStride] = x[e];
      return;
    }
    __syncthreads();
#pragma unroll
    for (int e = 0; e < 16; ++e) tile[G::row_a(e, u) * G::COLS + c] = x[e];
  }
  __syncthreads();
  store_block<G::R, G::COLS, G::COLS, false>(tower_dst(b, T, fresh_block_ids()) + col0, tile, kStride);
}

// The CTA's tower decides the butterflies: reduction-free below 2^57 (mode 2).
template <int LOGN, int MODE, int MINB, bool DIRECT>
__global__ void __launch_bounds__(kNttThreads, MINB) ntt_fwd_col(NttBatch b, DeviceTables T) {
  __shared__ __align__(16) u64 tile[kTileWords];
  __shared__ ulonglong2 tw[ColGeom<LOGN>::R];
  if (MODE == 2 && T.tc[b.id[blockIdx.z]].q < kFreeModulusBound)
    fwd_col_body<LOGN, MODE, DIRECT, MODE == 2>(b, T, tile, tw);
  else
    fwd_col_body<LOGN, MODE, DIRECT, false>(b, T, tile, tw);
}

// LIGHT (mode 2, q < 2^57): the stages before the last skip the sums'
// reduction (gs_stages_light; each register phase ends below 4q), and the
// last stage, with or without N^-1, runs as usual.
template <int LOGN, int MODE, bool DIRECT, bool UNSCALED, bool LIGHT>
__device__ __forceinline__ void inv_col_body(const NttBatch &b, const DeviceTables &T, u64 *tile, ulonglong2 *tw) {
  using G = ColGeom<LOGN>;
  constexpr int N = 1 << LOGN;
  constexpr u64 kStride = N >> G::LR;
  const TowerView v = tower_view(b, T, true);
  const u64 q = v.c->q, q2 = v.c->q2;
  const int col0 = blockIdx.x * G::COLS;
  const int c = threadIdx.x % G::COLS, u = threadIdx.x / G::COLS;
  u64 x[16];
  if constexpr (DIRECT) {
#pragma unroll
    for (int e = 0; e < 16; ++e)
      x[e] = v.src[(G::LR > 4 ? G::row_b(e, u) : G::row_a(e, u)) * kStride + col0 + c];
  }
  for (int i = threadIdx.x; i < G::R; i += kNttThreads) tw[i] = v.tw[i];
  if constexpr (!DIRECT) load_block<G::R, G::COLS, G::COLS, false>(tile, v.src + col0, kStride);
  __syncthreads();
  if constexpr (G::LR > 4) {
    if constexpr (!DIRECT) {
#pragma unroll
      for (int e = 0; e < 16; ++e) x[e] = tile[G::row_b(e, u) * G::COLS + c];
    }
    // Stages logR-1 .. 4: row bit logR-1-s == register bit logR-1-s.
    if constexpr (LIGHT) {
      gs_stages_light<4, G::LR - 4>(
          x,
          [&](int j, int e) {
            const int s = G::LR - 1 - j, k = G::LR - s;  // row_b(e, u) >> k = (u << (4 - k)) + (e >> k)
            const ulonglong2 w = tw[(1 << s) + (u << (4 - k)) + (e >> k)];
            return Shoup{w.x, w.y};
          },
          q);
    } else {
#pragma unroll
      for (int s = G::LR - 1; s >= 4; --s) {
        const int d = 1 << (G::LR - 1 - s), k = G::LR - s;
        const ulonglong2 *tws = tw + (1 << s) + (u << (4 - k));  // as in the forward pass
#pragma unroll
        for (int e = 0; e < 16; ++e) {
          if (e & d) continue;
          const ulonglong2 w = tws[e >> k];
          gs_butterfly<MODE>(x[e], x[e + d], w.x, w.y, q, q2);
        }
      }
    }
    if constexpr (!DIRECT) __syncthreads();  // every thread has read its inputs from the tile
#pragma unroll
    for (int e = 0; e < 16; ++e) tile[G::row_b(e, u) * G::COLS + c] = x[e];
    __syncthreads();
#pragma unroll
    for (int e = 0; e < 16; ++e) x[e] = tile[G::row_a(e, u) * G::COLS + c];
  } else if constexpr (!DIRECT) {
#pragma unroll
    for (int e = 0; e < 16; ++e) x[e] = tile[G::row_a(e, u) * G::COLS + c];
  }
  // Stages 3..1, then stage 0 with N^-1 folded in.
  if constexpr (LIGHT) {
    gs_stages_light<4, 3>(
        x,
        [&](int j, int e) {
          const int s = 3 - j;
          const ulonglong2 w = tw[(1 << s) + (e >> (4 - s))];
          return Shoup{w.x, w.y};
        },
        q);
  } else {
#pragma unroll
    for (int s = 3; s >= 1; --s) {
      const int d = 8 >> s;
#pragma unroll
      for (int e = 0; e < 16; ++e) {
        if (e & d) continue;
        const ulonglong2 w = tw[(1 << s) + (e >> (4 - s))];
        gs_butterfly<MODE>(x[e], x[e + d], w.x, w.y, q, q2);
      }
    }
  }
  if constexpr (UNSCALED) {
    const ulonglong2 w = tw[1];  // stage 0: every pair (e, e + 8) uses T[1]
#pragma unroll
    for (int e = 0; e < 8; ++e) gs_butterfly<MODE>(x[e], x[e + 8], w.x, w.y, q, q2);
  } else {
    const Shoup ninv = v.c->ninv, last = v.c->last_inv;
#pragma unroll
    for (int e = 0; e < 8; ++e) gs_last<MODE>(x[e], x[e + 8], ninv, last, q, q2);
  }
  if constexpr (DIRECT) {
    u64 *const dst = tower_dst(b, T, fresh_block_ids()) + col0 + c;
#pragma unroll
    for (int e = 0; e < 16; ++e) dst[G::row_a(e, u) * kStride] = x[e];
    return;
  }
  __syncthreads();
#pragma unroll
  for (int e = 0; e < 16; ++e) tile[G::row_a(e, u) * G::COLS + c] = x[e];
  __syncthreads();
  store_block<G::R, G::COLS, G::COLS, false>(tower_dst(b, T, fresh_block_ids()) + col0, tile, kStride);
}

// UNSCALED: the last stage is a plain Gentleman-Sande butterfly (no N^-1) and
// the outputs stay lazily reduced: N times the coefficients, in [0, 4q) for
// mode 2 and [0, 2q) for mode 1. For a basis switch that folds N^-1 into its
// constants (conv_plan with ninv), which reduces its inputs itself.
// The CTA's tower decides the butterflies: reduction-light below 2^57 (mode 2).
template <int LOGN, int MODE, int MINB, bool DIRECT, bool UNSCALED = false>
__global__ void __launch_bounds__(kNttThreads, MINB) ntt_inv_col(NttBatch b, DeviceTables T) {
  __shared__ __align__(16) u64 tile[kTileWords];
  __shared__ ulonglong2 tw[ColGeom<LOGN>::R];
  if (MODE == 2 && T.tc[b.id[blockIdx.z]].q < kFreeModulusBound)
    inv_col_body<LOGN, MODE, DIRECT, UNSCALED, MODE == 2>(b, T, tile, tw);
  else
    inv_col_body<LOGN, MODE, DIRECT, UNSCALED, false>(b, T, tile, tw);
}

// ---- row pass ----------------------------------------------------------------
// Tile: 16 rows x 256 words starting at row blockIdx.x * 16; thread (r, u),
// r = tid / 16, u = tid % 16. Mapping A: element e is column e*16 + u.
// Mapping B: element e is column u*16 + e. Shared rows are padded to 272 words
// (one pad word per 16) so both mappings are bank-conflict free.
__device__ __forceinline__ int pad_col(int col) { return col + (col >> 4); }

// Warp-local copies between global memory and a warp's two padded tile rows
// (rows 2w and 2w+1 of the tile belong to warp w in both row passes): 16-byte
// coalesced chunks and no CTA-wide barrier, so the warps of a CTA run their
// load, butterfly and store phases independently and overlap one another.
// Step `it` (0..7) of lane l copies columns c = 2l + 64 (it % 4) of row
// 2w + it / 4: a per-lane base plus constants (pad_col(c) = 2l + l / 8 +
// 68 (it % 4)).
__device__ __forceinline__ void load_rows_warp(u64 *tile, const u64 *g) {
  const int lane = threadIdx.x & 31, r0 = (threadIdx.x >> 5) * 2;
  const u64 *gb = g + r0 * 256 + 2 * lane;
  u64 *tb = tile + r0 * kRowPad + 2 * lane + (lane >> 3);
#pragma unroll
  for (int it = 0; it < 8; ++it) {
    const ulonglong2 v = *reinterpret_cast<const ulonglong2 *>(gb + (it >> 2) * 256 + 64 * (it & 3));
    u64 *t = tb + (it >> 2) * kRowPad + 68 * (it & 3);
    t[0] = v.x;
    t[1] = v.y;
  }
}
__device__ __forceinline__ void store_rows_warp(u64 *g, const u64 *tile) {
  const int lane = threadIdx.x & 31, r0 = (threadIdx.x >> 5) * 2;
  u64 *gb = g + r0 * 256 + 2 * lane;
  const u64 *tb = tile + r0 * kRowPad + 2 * lane + (lane >> 3);
#pragma unroll
  for (int it = 0; it < 8; ++it) {
    const u64 *t = tb + (it >> 2) * kRowPad + 68 * (it & 3);
    *reinterpret_cast<ulonglong2 *>(gb + (it >> 2) * 256 + 64 * (it & 3)) = make_ulonglong2(t[0], t[1]);
  }
}

// Twiddles of the row passes' register-bit stages (s' = 4..7): lane u of row r
// needs T[2^s + (row << s') + (16u + e) >> (8 - s')], which the tables hold in
// lane-major order (row_lane_major), so the 16 lanes of a row read 16
// consecutive entries. With STW set, the CTA first copies the stage's 16 * 2^s'
// twiddles, contiguous in the table, into shared memory with coalesced 16-byte
// loads, entry k at 16-byte slot k + k/8; the data tile's buffer (free while the
// values sit in registers) holds the largest stage (2048 entries, 36 KiB).
constexpr int kRowStwWords = 2 * (2048 + 2048 / 8);
__device__ __forceinline__ void stage_twiddles(ulonglong2 *st, const ulonglong2 *tw, int s, int sp, int row0) {
  const ulonglong2 *src = tw + (1 << s) + (row0 << sp);
  const int count = 16 << sp;
  for (int k = threadIdx.x; k < count; k += kNttThreads) st[k + (k >> 3)] = __ldg(src + k);
}
__device__ __forceinline__ Shoup staged_twiddle(const ulonglong2 *st, int k) {
  const ulonglong2 v = st[k + (k >> 3)];
  return Shoup{v.x, v.y};
}

// DIRECT (without STW): in mapping A the 16 lanes of a row read 16
// consecutive words, so the forward row pass loads its inputs, and the inverse
// row pass stores its outputs, straight between registers and global memory;
// the other side stays staged through the warp's tile rows (mapping B puts the
// lanes 128 bytes apart).
// EPI_SMEM (ModDown launches of the direct form, b.epi_left set): each warp
// copies its two rows of the epilogue's `left` operand into dynamic shared
// memory (kEpiSmemBytes per CTA, rows of 256 words) with cp.async at kernel
// start, so the epilogue reads them from shared memory after the butterflies.
constexpr int kEpiSmemBytes = 16 * 256 * sizeof(u64);
__device__ __forceinline__ void ntt_copy16(void *smem, const void *gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(smem))),
               "l"(gmem)
               : "memory");
}

// FREE: the reduction-free butterflies for a tower with q < 2^57, continuing
// from the column pass's values below 4q + 4q * logR; the outputs are then
// reduced once (canonical, or [0, 4q) for the ModDown epilogue) or left below
// 68q (lazy_out).
template <int LOGN, int MODE, bool STW, bool DIRECT, bool EPI_SMEM, bool FREE>
__device__ __forceinline__ void fwd_row_body(const NttBatch &b, const DeviceTables &T, u64 *tile, u64 *epi_rows) {
  constexpr int LR = LOGN - 8;
  const TowerView v = tower_view(b, T, false);
  const u64 q = v.c->q, q2 = v.c->q2;
  const int row0 = blockIdx.x * 16;
  if (b.epi_left != nullptr) {
    // The ModDown epilogue reads its operands only after the butterflies:
    // start moving this warp's two rows of them (4 KiB per operand) now.
    const u64 off = u64(b.off[blockIdx.z]) * (u64(1) << T.logn) + (row0 + 2 * (threadIdx.x >> 5)) * 256;
    const u64 *lrows = b.epi_left + blockIdx.y * b.epi_left_stride + off;
    if constexpr (EPI_SMEM) {
      u64 *dst = epi_rows + 2 * (threadIdx.x >> 5) * 256;
      for (int j = threadIdx.x & 31; j < 256; j += 32) ntt_copy16(dst + 2 * j, lrows + 2 * j);
      asm volatile("cp.async.commit_group;" ::: "memory");
    } else if ((threadIdx.x & 31) == 0) {
      prefetch_l2(lrows, 2 * 256 * sizeof(u64));
    }
    const u64 *add = poly_add(b, blockIdx.y);
    if (add && (threadIdx.x & 31) == 0) prefetch_l2(add + off, 2 * 256 * sizeof(u64));
  }
  const int r = threadIdx.x / 16, u = threadIdx.x % 16;
  const int row = row0 + r;
  u64 *my = tile + r * kRowPad;
  u64 x[16];
  if constexpr (DIRECT) {
    const u64 *in = v.src + row * 256 + u;
#pragma unroll
    for (int e = 0; e < 16; ++e) x[e] = in[e * 16];
  } else {
    if constexpr (STW) {
      load_block<16, 256, kRowPad, true>(tile, v.src + row0 * 256, 256);
      __syncthreads();
    } else {
      load_rows_warp(tile, v.src + row0 * 256);
      __syncwarp();
    }
#pragma unroll
    for (int e = 0; e < 16; ++e) x[e] = my[pad_col(e * 16 + u)];
  }
  // Stages LR + s', s' = 0..3: column bit 7-s' == register bit 3-s'.
#pragma unroll
  for (int sp = 0; sp < 4; ++sp) {
    const int s = LR + sp, d = 8 >> sp;
#pragma unroll
    for (int e = 0; e < 16; ++e) {
      if (e & d) continue;
      const Shoup w = tw_load(v.tw + (1 << s) + (row << sp) + (e >> (4 - sp)));
      ct_bf<FREE, MODE>(x[e], x[e + d], w.w, w.wq, q, q2);
    }
  }
  __syncwarp();
#pragma unroll
  for (int e = 0; e < 16; ++e) my[pad_col(e * 16 + u)] = x[e];
  __syncwarp();
#pragma unroll
  for (int e = 0; e < 16; ++e) x[e] = my[pad_col(u * 16 + e)];
  // Stages LR + s', s' = 4..7: column bit 7-s' == register bit 7-s'.
  if constexpr (STW) {
    ulonglong2 *st = reinterpret_cast<ulonglong2 *>(tile);
#pragma unroll
    for (int sp = 4; sp < 8; ++sp) {
      const int s = LR + sp, d = 1 << (7 - sp);
      __syncthreads();  // the tile (data, or the previous stage's twiddles) is no longer read
      stage_twiddles(st, v.tw, s, sp, row0);
      __syncthreads();
#pragma unroll
      for (int e = 0; e < 16; ++e) {
        if (e & d) continue;
        const Shoup w = staged_twiddle(st, (r << sp) + row_lane_major(u, e >> (8 - sp)));
        ct_bf<FREE, MODE>(x[e], x[e + d], w.w, w.wq, q, q2);
      }
    }
    __syncthreads();  // staged twiddles read by every warp before the data returns
  } else {
#pragma unroll
    for (int sp = 4; sp < 8; ++sp) {
      const int s = LR + sp, d = 1 << (7 - sp);
#pragma unroll
      for (int e = 0; e < 16; ++e) {
        if (e & d) continue;
        const Shoup w = tw_load(v.tw + (1 << s) + (row << sp) + row_lane_major(u, e >> (8 - sp)));
        ct_bf<FREE, MODE>(x[e], x[e + d], w.w, w.wq, q, q2);
      }
    }
  }
  // Mode 2 with the ModDown epilogue: the values only need to reach [0, 4q)
  // (or stay below 68q after reduction-free butterflies), since the epilogue
  // forms (left + span - x) * P^-1 and reduces that itself.
  const bool epi4 = MODE == 2 && b.epi_left != nullptr;
  const bool canonical = !b.lazy_out && !epi4;
  const u64 one = v.c->red.one;
#pragma unroll
  for (int e = 0; e < 16; ++e) {
    if constexpr (FREE) {
      if (canonical) x[e] = reduce_free_final(x[e], q, one);
      // the ModDown epilogue takes x below 68q directly (below)
    } else {
      if (canonical) x[e] = reduce_final<MODE>(x[e], q, q2);
      else if (epi4) x[e] = csub_sign(x[e], 2 * q2);
    }
    my[pad_col(u * 16 + e)] = x[e];
  }
  if constexpr (STW) {
    __syncthreads();
  } else {
    __syncwarp();
  }
  const BlockIds ids = fresh_block_ids();
  const u64 rows_off = tower_offset(b, T, ids) + ids.x * 16 * 256;
  u64 *out = poly_dst(b, ids.poly) + rows_off;
  if (b.epi_left == nullptr) {
    if constexpr (STW)
      store_block<16, 256, kRowPad, true>(out, tile, 256);
    else
      store_rows_warp(out, tile);
    return;
  }
  const u64 *left = b.epi_left + ids.poly * b.epi_left_stride + rows_off;
  const Shoup pinv = b.epi_pinv[b.id[ids.slot]];
  const u64 *add = poly_add(b, ids.poly);
  if (add) add += rows_off;
  // Epilogue over the rows this thread's group owns: every row with STW (the
  // CTA synchronised above), the warp's own two rows otherwise.
  // Either way each thread handles 8 chunks of 2 words; the fixed trip count
  // lets every chunk's loads be in flight together.
  const int j0 = STW ? int(threadIdx.x) : int(threadIdx.x & 31) + (int(threadIdx.x >> 5) * 2) * 128;
  constexpr int kJStep = STW ? kNttThreads : 32;
  static_assert(8 * kJStep * (STW ? 1 : 8) == 16 * 128, "8 chunks per thread cover the CTA's 16 rows");
  if constexpr (EPI_SMEM) {  // this warp's own copies of its two rows
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncwarp();
  }
  // Without STW, chunk `it` of lane l in warp w is row 2w + it / 4, columns
  // c = 2l + 64 (it % 4): a per-thread base plus constants (pad_col(c) =
  // 2l + l / 8 + 68 (it % 4)), so no chunk recomputes its address.
  const int lane = threadIdx.x & 31;
  const int gbase = int(threadIdx.x >> 5) * 512 + 2 * lane;
  const int sbase = int(threadIdx.x >> 5) * 2 * kRowPad + 2 * lane + (lane >> 3);
#pragma unroll
  for (int it = 0; it < 8; ++it) {
    int goff, sidx;
    if constexpr (STW) {
      const int j = j0 + it * kJStep;
      const int rr = j >> 7, c = (j & 127) * 2;
      goff = rr * 256 + c;
      sidx = rr * kRowPad + pad_col(c);
    } else {
      goff = gbase + (it >> 2) * 256 + 64 * (it & 3);
      sidx = sbase + (it >> 2) * kRowPad + 68 * (it & 3);
    }
    const ulonglong2 l = EPI_SMEM ? *reinterpret_cast<const ulonglong2 *>(epi_rows + goff)
                                  : *reinterpret_cast<const ulonglong2 *>(left + goff);
    ulonglong2 o;
    if constexpr (MODE == 2) {
      // left < q and x < 4q: left + 4q - x lies in (0, 5q), below 2^64 for q < 2^61;
      // the approximate-quotient product lands in [0, 4q), two subtractions finish it.
      // x < 4q, or x < 68q after reduction-free butterflies: left + span - x
      // lies in (0, span + q), below 2^64, and the product accepts any word.
      const u64 span = FREE ? u64(kFreeRangeFactor) * q : 2 * q2, qneg = 0 - q;
      o.x = csub_sign(csub_sign(shoup_approx(l.x + span - tile[sidx], pinv.w, pinv.wq, qneg), q2), q);
      o.y = csub_sign(csub_sign(shoup_approx(l.y + span - tile[sidx + 1], pinv.w, pinv.wq, qneg), q2), q);
    } else {
      o.x = shoup_canon(sub_mod(l.x, tile[sidx], q), pinv.w, pinv.wq, q);
      o.y = shoup_canon(sub_mod(l.y, tile[sidx + 1], q), pinv.w, pinv.wq, q);
    }
    if (add) {
      const ulonglong2 e = *reinterpret_cast<const ulonglong2 *>(add + goff);
      o.x = add_mod(o.x, e.x, q);
      o.y = add_mod(o.y, e.y, q);
    }
    *reinterpret_cast<ulonglong2 *>(out + goff) = o;
  }
}

// The CTA's tower decides the butterflies: reduction-free below 2^57 (mode 2).
template <int LOGN, int MODE, int MINB, bool STW, bool DIRECT, bool EPI_SMEM = false>
__global__ void __launch_bounds__(kNttThreads, MINB) ntt_fwd_row(NttBatch b, DeviceTables T) {
  static_assert(!(STW && DIRECT), "the staged-twiddle form has no direct variant");
  static_assert(!EPI_SMEM || DIRECT, "the staged epilogue operand goes with the direct form");
  __shared__ __align__(16) u64 tile[STW ? kRowStwWords : 16 * kRowPad];
  extern __shared__ __align__(16) u64 epi_rows[];  // EPI_SMEM: 16 x 256 words of `left`
  if (MODE == 2 && T.tc[b.id[blockIdx.z]].q < kFreeModulusBound)
    fwd_row_body<LOGN, MODE, STW, DIRECT, EPI_SMEM, MODE == 2>(b, T, tile, epi_rows);
  else
    fwd_row_body<LOGN, MODE, STW, DIRECT, EPI_SMEM, false>(b, T, tile, epi_rows);
}

// ---- single-pass forward transform over a thread-block cluster (N = 2^16) -------
// One cluster of 8 CTAs (512 threads each) per tower and polynomial; CTA k of
// the cluster:
//   1. runs the column pass (stages 0..7) on columns 32k .. 32k + 31, reading
//      its inputs from global memory, and keeps the results in its shared
//      memory as [256 rows][32 columns];
//   2. after a cluster barrier, gathers rows 32k .. 32k + 31 (word e * 16 + u
//      of a row lies in CTA e / 2, column (e % 2) * 16 + u) from the 8 CTAs'
//      shared memory into registers;
//   3. after a second barrier (every CTA has read what it needs from the
//      others, so its shared memory is free), runs the row pass (stages
//      8..15) on its 32 rows and stores them.
// The tower crosses HBM once each way (2W) instead of twice (4W). Every thread
// of every CTA of a cluster takes the same path to both barriers (the tower,
// and so the butterflies, are the same for the whole cluster).
constexpr int kClusterCtas = 8, kClusterThreads = 512;
constexpr int kClusterSmemBytes = 32 * kRowPad * int(sizeof(u64));  // 32 padded rows >= 256 x 32 words

template <int MODE, bool FREE>
__device__ __forceinline__ void fwd_cluster_body(const NttBatch &b, const DeviceTables &T, u64 *sm, ulonglong2 *tw) {
  namespace cg = cooperative_groups;
  constexpr int LR = 8;
  cg::cluster_group cluster = cg::this_cluster();
  const int k = int(cluster.block_rank());
  const TowerView v = tower_view(b, T, false);
  const u64 q = v.c->q, q2 = v.c->q2;
  u64 x[16];
  {
    // Column pass: thread (c, u), column 32k + c; mapping A holds rows
    // e * 16 + u (stages 0..3), mapping B rows u * 16 + e (stages 4..7).
    const int c = threadIdx.x % 32, u = threadIdx.x / 32;
    const u64 *in = v.src + 32 * k + c;
#pragma unroll
    for (int e = 0; e < 16; ++e) x[e] = in[(e * 16 + u) * 256];
    for (int i = threadIdx.x; i < 256; i += kClusterThreads) tw[i] = v.tw[i];
    __syncthreads();
#pragma unroll
    for (int st = 0; st < 4; ++st) {
      const int d = 8 >> st;
#pragma unroll
      for (int e = 0; e < 16; ++e) {
        if (e & d) continue;
        const ulonglong2 w = tw[(1 << st) + (e >> (4 - st))];
        if (st == 0)
          ct_bf<FREE, MODE, true>(x[e], x[e + d], w.x, w.y, q, q2);
        else
          ct_bf<FREE, MODE>(x[e], x[e + d], w.x, w.y, q, q2);
      }
    }
#pragma unroll
    for (int e = 0; e < 16; ++e) sm[(e * 16 + u) * 32 + c] = x[e];
    __syncthreads();
#pragma unroll
    for (int e = 0; e < 16; ++e) x[e] = sm[(u * 16 + e) * 32 + c];
#pragma unroll
    for (int st = 4; st < LR; ++st) {
      const int d = 1 << (LR - 1 - st);
#pragma unroll
      for (int e = 0; e < 16; ++e) {
        if (e & d) continue;
        const ulonglong2 w = tw[(1 << st) + ((u * 16 + e) >> (LR - st))];
        ct_bf<FREE, MODE>(x[e], x[e + d], w.x, w.y, q, q2);
      }
    }
    // Each word of mapping B is read and rewritten by the same thread.
#pragma unroll
    for (int e = 0; e < 16; ++e) sm[(u * 16 + e) * 32 + c] = x[e];
  }
  cluster.sync();  // every CTA's column results are complete and visible to the cluster
  // Row pass: thread (r, u), row 32k + r; warp w owns rows 2w and 2w + 1.
  const int r = threadIdx.x / 16, u = threadIdx.x % 16;
  const int row = 32 * k + r;
#pragma unroll
  for (int e = 0; e < 16; ++e) {
    const u64 *owner = cluster.map_shared_rank(sm, unsigned(e >> 1));
    x[e] = owner[row * 32 + (e & 1) * 16 + u];
  }
  cluster.sync();  // every CTA has read its rows from the others: shared memory is free
  u64 *my = sm + r * kRowPad;
#pragma unroll
  for (int sp = 0; sp < 4; ++sp) {
    const int st = LR + sp, d = 8 >> sp;
#pragma unroll
    for (int e = 0; e < 16; ++e) {
      if (e & d) continue;
      const Shoup w = tw_load(v.tw + (1 << st) + (row << sp) + (e >> (4 - sp)));
      ct_bf<FREE, MODE>(x[e], x[e + d], w.w, w.wq, q, q2);
    }
  }
#pragma unroll
  for (int e = 0; e < 16; ++e) my[pad_col(e * 16 + u)] = x[e];
  __syncwarp();
#pragma unroll
  for (int e = 0; e < 16; ++e) x[e] = my[pad_col(u * 16 + e)];
#pragma unroll
  for (int sp = 4; sp < 8; ++sp) {
    const int st = LR + sp, d = 1 << (7 - sp);
#pragma unroll
    for (int e = 0; e < 16; ++e) {
      if (e & d) continue;
      const Shoup w = tw_load(v.tw + (1 << st) + (row << sp) + row_lane_major(u, e >> (8 - sp)));
      ct_bf<FREE, MODE>(x[e], x[e + d], w.w, w.wq, q, q2);
    }
  }
  const u64 one = v.c->red.one;
#pragma unroll
  for (int e = 0; e < 16; ++e) {
    if constexpr (FREE)
      x[e] = reduce_free_final(x[e], q, one);
    else
      x[e] = reduce_final<MODE>(x[e], q, q2);
    my[pad_col(u * 16 + e)] = x[e];
  }
  __syncwarp();
  store_rows_warp(tower_dst(b, T, fresh_block_ids()) + u64(32 * k) * 256, sm);
}

// The cluster's tower decides the butterflies: reduction-free below 2^57.
static __global__ void __cluster_dims__(kClusterCtas, 1, 1) __launch_bounds__(kClusterThreads, 2)
    ntt_fwd_cluster16(NttBatch b, DeviceTables T) {
  extern __shared__ __align__(16) u64 sm[];
  __shared__ ulonglong2 tw[256];
  if (T.tc[b.id[blockIdx.z]].q < kFreeModulusBound)
    fwd_cluster_body<2, true>(b, T, sm, tw);
  else
    fwd_cluster_body<2, false>(b, T, sm, tw);
}

// The inverse row pass's butterflies (stages logR + 7 .. logR, Gentleman-Sande)
// on row `row` of a tower, by the 16 threads u = 0..15 of that row, with every
// twiddle read from global memory. On entry x[e] holds the row's word u*16 + e
// (canonical: the first stage adds without reducing); on exit x[e] holds its
// word e*16 + u. `my` is the row's padded shared-memory buffer, used for the
// exchange between the two register phases; the row's threads may still be
// reading it on entry (the exchange starts with __syncwarp).
// LIGHT (mode 2, q < 2^57): the stages skip the sums' reduction
// (gs_stages_light); either way the outputs lie below 4q.
template <int LOGN, int MODE, bool LIGHT = false>
__device__ __forceinline__ void inv_row_stages(u64 (&x)[16], u64 *my, const ulonglong2 *tw, int row, int u, u64 q,
                                               u64 q2) {
  constexpr int LR = LOGN - 8;
  if constexpr (LIGHT) {
    static_assert(MODE == 2, "reduction-light butterflies are mode 2");
    // Stages LR + 7 - j, j = 0..3, then LR + 3 - j: canonical inputs (F = 1).
    gs_stages_light<1, 4>(
        x,
        [&](int j, int e) {
          const int sp = 7 - j;
          return tw_load(tw + (1 << (LR + sp)) + (row << sp) + row_lane_major(u, e >> (8 - sp)));
        },
        q);
    __syncwarp();
#pragma unroll
    for (int e = 0; e < 16; ++e) my[pad_col(u * 16 + e)] = x[e];
    __syncwarp();
#pragma unroll
    for (int e = 0; e < 16; ++e) x[e] = my[pad_col(e * 16 + u)];
    gs_stages_light<4, 4>(
        x,
        [&](int j, int e) {
          const int sp = 3 - j;
          return tw_load(tw + (1 << (LR + sp)) + (row << sp) + (e >> (4 - sp)));
        },
        q);
  } else {
    // Stages LR + s', s' = 7..4: column bit 7-s' == register bit 7-s'.
#pragma unroll
    for (int sp = 7; sp >= 4; --sp) {
      const int s = LR + sp, d = 1 << (7 - sp);
#pragma unroll
      for (int e = 0; e < 16; ++e) {
        if (e & d) continue;
        const Shoup w = tw_load(tw + (1 << s) + (row << sp) + row_lane_major(u, e >> (8 - sp)));
        if (sp == 7)
          gs_butterfly<MODE, true>(x[e], x[e + d], w.w, w.wq, q, q2);
        else
          gs_butterfly<MODE>(x[e], x[e + d], w.w, w.wq, q, q2);
      }
    }
    __syncwarp();
#pragma unroll
    for (int e = 0; e < 16; ++e) my[pad_col(u * 16 + e)] = x[e];
    __syncwarp();
#pragma unroll
    for (int e = 0; e < 16; ++e) x[e] = my[pad_col(e * 16 + u)];
    // Stages LR + s', s' = 3..0: column bit 7-s' == register bit 3-s'.
#pragma unroll
    for (int sp = 3; sp >= 0; --sp) {
      const int s = LR + sp, d = 8 >> sp;
#pragma unroll
      for (int e = 0; e < 16; ++e) {
        if (e & d) continue;
        const Shoup w = tw_load(tw + (1 << s) + (row << sp) + (e >> (4 - sp)));
        gs_butterfly<MODE>(x[e], x[e + d], w.w, w.wq, q, q2);
      }
    }
  }
}

template <int LOGN, int MODE, int MINB, bool STW, bool DIRECT>
__global__ void __launch_bounds__(kNttThreads, MINB) ntt_inv_row(NttBatch b, DeviceTables T) {
  static_assert(!(STW && DIRECT), "the staged-twiddle form has no direct variant");
  constexpr int LR = LOGN - 8;
  __shared__ __align__(16) u64 tile[STW ? kRowStwWords : 16 * kRowPad];
  const TowerView v = tower_view(b, T, true);
  const u64 q = v.c->q, q2 = v.c->q2;
  const int row0 = blockIdx.x * 16;
  if constexpr (STW) {
    load_block<16, 256, kRowPad, true>(tile, v.src + row0 * 256, 256);
    __syncthreads();
  } else {
    load_rows_warp(tile, v.src + row0 * 256);
    __syncwarp();
  }
  const int r = threadIdx.x / 16, u = threadIdx.x % 16;
  const int row = row0 + r;
  u64 *my = tile + r * kRowPad;
  u64 x[16];
#pragma unroll
  for (int e = 0; e < 16; ++e) x[e] = my[pad_col(u * 16 + e)];
  if constexpr (STW) {
    // Stages LR + s', s' = 7..4, twiddles staged in shared memory per stage.
    ulonglong2 *st = reinterpret_cast<ulonglong2 *>(tile);
#pragma unroll
    for (int sp = 7; sp >= 4; --sp) {
      const int s = LR + sp, d = 1 << (7 - sp);
      __syncthreads();  // the tile (data, or the previous stage's twiddles) is no longer read
      stage_twiddles(st, v.tw, s, sp, row0);
      __syncthreads();
#pragma unroll
      for (int e = 0; e < 16; ++e) {
        if (e & d) continue;
        const Shoup w = staged_twiddle(st, (r << sp) + row_lane_major(u, e >> (8 - sp)));
        gs_butterfly<MODE>(x[e], x[e + d], w.w, w.wq, q, q2);
      }
    }
    __syncthreads();  // staged twiddles read by every warp before the data returns
    __syncwarp();
#pragma unroll
    for (int e = 0; e < 16; ++e) my[pad_col(u * 16 + e)] = x[e];
    __syncwarp();
#pragma unroll
    for (int e = 0; e < 16; ++e) x[e] = my[pad_col(e * 16 + u)];
#pragma unroll
    for (int sp = 3; sp >= 0; --sp) {
      const int s = LR + sp, d = 8 >> sp;
#pragma unroll
      for (int e = 0; e < 16; ++e) {
        if (e & d) continue;
        const Shoup w = tw_load(v.tw + (1 << s) + (row << sp) + (e >> (4 - sp)));
        gs_butterfly<MODE>(x[e], x[e + d], w.w, w.wq, q, q2);
      }
    }
  } else if (MODE == 2 && q < kFreeModulusBound) {
    inv_row_stages<LOGN, MODE, MODE == 2>(x, my, v.tw, row, u, q, q2);
  } else {
    inv_row_stages<LOGN, MODE>(x, my, v.tw, row, u, q, q2);
  }
  if constexpr (DIRECT) {
    u64 *const out = tower_dst(b, T, fresh_block_ids()) + row * 256 + u;
#pragma unroll
    for (int e = 0; e < 16; ++e) out[e * 16] = x[e];
  } else {
#pragma unroll
    for (int e = 0; e < 16; ++e) my[pad_col(e * 16 + u)] = x[e];
    if constexpr (STW) {
      __syncthreads();
      store_block<16, 256, kRowPad, true>(tower_dst(b, T, fresh_block_ids()) + row0 * 256, tile, 256);
    } else {
      __syncwarp();
      store_rows_warp(tower_dst(b, T, fresh_block_ids()) + row0 * 256, tile);
    }
  }
}

// ---- small transforms (N <= 2048): one CTA per tower, strict arithmetic -------
template <bool INV>
__global__ void __launch_bounds__(kNttThreads) ntt_small(NttBatch b, DeviceTables T) {
  __shared__ u64 a[2048];
  const TowerView v = tower_view(b, T, INV);
  const int logn = T.logn, n = 1 << logn;
  const u64 q = v.c->q;
  for (int i = threadIdx.x; i < n; i += blockDim.x) a[i] = v.src[i];
  __syncthreads();
  if (!INV) {
    for (int s = 0; s < logn; ++s) {
      const int lt = logn - 1 - s;  // pair distance 2^lt
      for (int p = threadIdx.x; p < n / 2; p += blockDim.x) {
        const int grp = p >> lt, j = (grp << (lt + 1)) + (p & ((1 << lt) - 1));
        const Shoup w = tw_load(v.tw + (1 << s) + grp);
        const u64 t = shoup_canon(a[j + (1 << lt)], w.w, w.wq, q);
        const u64 x = a[j];
        a[j] = add_mod(x, t, q);
        a[j + (1 << lt)] = sub_mod(x, t, q);
      }
      __syncthreads();
    }
  } else {
    for (int s = logn - 1; s >= 0; --s) {
      const int lt = logn - 1 - s;
      for (int p = threadIdx.x; p < n / 2; p += blockDim.x) {
        const int grp = p >> lt, j = (grp << (lt + 1)) + (p & ((1 << lt) - 1));
        const u64 x = a[j], y = a[j + (1 << lt)];
        if (s == 0) {
          a[j] = shoup_canon(add_mod(x, y, q), v.c->ninv.w, v.c->ninv.wq, q);
          a[j + (1 << lt)] = shoup_canon(sub_mod(x, y, q), v.c->last_inv.w, v.c->last_inv.wq, q);
        } else {
          const Shoup w = tw_load(v.tw + (1 << s) + grp);
          a[j] = add_mod(x, y, q);
          a[j + (1 << lt)] = shoup_canon(sub_mod(x, y, q), w.w, w.wq, q);
        }
      }
      __syncthreads();
    }
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) v.dst[i] = a[i];
}

// ---- butterfly-rate calibration ------------------------------------------------
// The forward NTT's arithmetic alone: each thread keeps 16 values in registers
// and runs `rounds` radix-16 rounds (4 stages x 8 mode-2 Cooley-Tukey
// butterflies) with twiddles held in registers, with no memory traffic. The
// values stay in [0, 8q); they are folded into one word that is stored only
// if it equals a fixed constant, so the work cannot be dropped. This measures
// the multiply-pipe ceiling that bounds the NTT passes on the running GPU.
static __global__ void __launch_bounds__(kNttThreads, 4)
    butterfly_rate_kernel(u64 *sink, u64 q, Shoup w0, Shoup w1, Shoup w2, Shoup w3, int rounds) {
  const u64 q2 = 2 * q;
  u64 x[16];
#pragma unroll
  for (int e = 0; e < 16; ++e) x[e] = (u64(blockIdx.x) * 4096 + threadIdx.x * 16 + e) % q;
  for (int r = 0; r < rounds; ++r) {
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      const int d = 8 >> s;
      const Shoup w = s == 0 ? w0 : s == 1 ? w1 : s == 2 ? w2 : w3;
#pragma unroll
      for (int e = 0; e < 16; ++e) {
        if (e & d) continue;
        ct_butterfly<2>(x[e], x[e + d], w.w, w.wq, q, q2);
      }
    }
  }
  u64 fold = 0;
#pragma unroll
  for (int e = 0; e < 16; ++e) fold ^= x[e];
  if (fold == 0x9E3779B97F4A7C15ull) sink[0] = fold;
}

}  // namespace b200
