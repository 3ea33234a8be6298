// Persistent, double-buffered versions of the two NTT passes (N = 2^12 .. 2^16).
//
// Same transform, schedule and register mappings as ntt.cuh; the difference is
// the data movement. Each CTA walks a strided list of 4096-word tiles and, while
// it computes tile i out of one shared buffer, the next tile (and, in the column
// pass, its 2^logR column twiddles) streams into the other buffer with 16-byte
// cp.async copies. The copy engine's latency therefore overlaps the butterflies
// instead of stalling every CTA at the start of its tile.
//
// Row-pass tiles are 16 dense rows of 256 words whose 16-byte chunks are XOR
// swizzled inside each 128-byte segment (chunk c lives at c ^ ((c >> 3) & 7)):
// mapping A (8-byte accesses, lane = column) and mapping B (16-byte accesses,
// lane = 16-column group) are then both bank-conflict free, and every chunk stays
// 16-byte aligned for cp.async.
#pragma once
#include <cstdint>

#include "ntt.cuh"

namespace b200 {

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int PENDING>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(PENDING) : "memory");
}

// Work item w of a persistent launch: tile x of slot y of polynomial z.
struct TileCoord {
  uint32_t x, slot, z;
};
__device__ __forceinline__ TileCoord tile_coord(uint32_t w, uint32_t tiles_per_tower, uint32_t slots) {
  TileCoord c;
  c.x = w % tiles_per_tower;
  const uint32_t rest = w / tiles_per_tower;
  c.slot = rest % slots;
  c.z = rest / slots;
  return c;
}
__device__ __forceinline__ TowerView view_at(const NttBatch &b, const DeviceTables &T, bool inv, uint32_t slot,
                                             u64 z) {
  const uint32_t g = b.id[slot];
  const u64 n = u64(1) << T.logn;
  const u64 offset = u64(b.off[slot]) * n;
  TowerView v;
  v.c = T.tc + g;
  v.tw = (inv ? T.inv : T.fwd) + g * n;
  v.src = poly_src(b, z) + offset;
  v.dst = poly_dst(b, z) + offset;
  return v;
}

// ---- column pass ---------------------------------------------------------------------
template <int LOGN>
constexpr int col_smem_bytes() {
  return 2 * kTileWords * 8 + 2 * (1 << (LOGN - 8)) * 16;
}

template <int LOGN, int MODE, bool INV>
__global__ void __launch_bounds__(kNttThreads, 3) ntt_col_ps(NttBatch b, DeviceTables T, uint32_t slots,
                                                             uint32_t total) {
  using G = ColGeom<LOGN>;
  constexpr int N = 1 << LOGN;
  constexpr uint32_t TPT = N / kTileWords;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  u64 *data = reinterpret_cast<u64 *>(smem_raw);                              // [2][4096]
  ulonglong2 *tws = reinterpret_cast<ulonglong2 *>(data + 2 * kTileWords);  // [2][R]

  auto prefetch = [&](uint32_t w, int buf) {
    const TileCoord tc = tile_coord(w, TPT, slots);
    const TowerView v = view_at(b, T, INV, tc.slot, tc.z);
    const u64 *src = v.src + tc.x * G::COLS;
    u64 *d = data + buf * kTileWords;
    constexpr int CHUNKS = G::R * G::COLS / 2;
    for (int j = threadIdx.x; j < CHUNKS; j += kNttThreads) {
      const int r = j / (G::COLS / 2), c = (j % (G::COLS / 2)) * 2;
      cp_async16(d + r * G::COLS + c, src + r * (N >> G::LR) + c);
    }
    for (int j = threadIdx.x; j < G::R; j += kNttThreads) cp_async16(tws + buf * G::R + j, v.tw + j);
    cp_async_commit();
  };

  uint32_t w = blockIdx.x;
  if (w < total) prefetch(w, 0);
  const int c = threadIdx.x % G::COLS, u = threadIdx.x / G::COLS;
  for (int buf = 0; w < total; w += gridDim.x, buf ^= 1) {
    const uint32_t next = w + gridDim.x;
    if (next < total) {
      prefetch(next, buf ^ 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const TileCoord tc = tile_coord(w, TPT, slots);
    const TowerView v = view_at(b, T, INV, tc.slot, tc.z);
    const u64 q = v.c->q, q2 = v.c->q2;
    u64 *tile = data + buf * kTileWords;
    const ulonglong2 *tw = tws + buf * G::R;
    u64 x[16];
    if constexpr (!INV) {
#pragma unroll
      for (int e = 0; e < 16; ++e) x[e] = tile[G::row_a(e, u) * G::COLS + c];
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        const int d = 8 >> s;
#pragma unroll
        for (int e = 0; e < 16; ++e) {
          if (e & d) continue;
          const ulonglong2 t = tw[(1 << s) + (e >> (4 - s))];
          ct_butterfly<MODE>(x[e], x[e + d], t.x, t.y, q, q2);
        }
      }
      if constexpr (G::LR > 4) {
        __syncthreads();
#pragma unroll
        for (int e = 0; e < 16; ++e) tile[G::row_a(e, u) * G::COLS + c] = x[e];
        __syncthreads();
#pragma unroll
        for (int e = 0; e < 16; ++e) x[e] = tile[G::row_b(e, u) * G::COLS + c];
#pragma unroll
        for (int s = 4; s < G::LR; ++s) {
          const int d = 1 << (G::LR - 1 - s);
#pragma unroll
          for (int e = 0; e < 16; ++e) {
            if (e & d) continue;
            const ulonglong2 t = tw[(1 << s) + (G::row_b(e, u) >> (G::LR - s))];
            ct_butterfly<MODE>(x[e], x[e + d], t.x, t.y, q, q2);
          }
        }
        __syncthreads();
#pragma unroll
        for (int e = 0; e < 16; ++e) tile[G::row_b(e, u) * G::COLS + c] = x[e];
      } else {
        __syncthreads();
#pragma unroll
        for (int e = 0; e < 16; ++e) tile[G::row_a(e, u) * G::COLS + c] = x[e];
      }
    } else {
      if constexpr (G::LR > 4) {
#pragma unroll
        for (int e = 0; e < 16; ++e) x[e] = tile[G::row_b(e, u) * G::COLS + c];
#pragma unroll
        for (int s = G::LR - 1; s >= 4; --s) {
          const int d = 1 << (G::LR - 1 - s);
#pragma unroll
          for (int e = 0; e < 16; ++e) {
            if (e & d) continue;
            const ulonglong2 t = tw[(1 << s) + (G::row_b(e, u) >> (G::LR - s))];
            gs_butterfly<MODE>(x[e], x[e + d], t.x, t.y, q, q2);
          }
        }
        __syncthreads();
#pragma unroll
        for (int e = 0; e < 16; ++e) tile[G::row_b(e, u) * G::COLS + c] = x[e];
        __syncthreads();
      }
#pragma unroll
      for (int e = 0; e < 16; ++e) x[e] = tile[G::row_a(e, u) * G::COLS + c];
#pragma unroll
      for (int s = 3; s >= 1; --s) {
        const int d = 8 >> s;
#pragma unroll
        for (int e = 0; e < 16; ++e) {
          if (e & d) continue;
          const ulonglong2 t = tw[(1 << s) + (e >> (4 - s))];
          gs_butterfly<MODE>(x[e], x[e + d], t.x, t.y, q, q2);
        }
      }
      const Shoup ninv = v.c->ninv, last = v.c->last_inv;
#pragma unroll
      for (int e = 0; e < 8; ++e) gs_last<MODE>(x[e], x[e + 8], ninv, last, q, q2);
      __syncthreads();
#pragma unroll
      for (int e = 0; e < 16; ++e) tile[G::row_a(e, u) * G::COLS + c] = x[e];
    }
    __syncthreads();
    u64 *dst = v.dst + tc.x * G::COLS;
    constexpr int CHUNKS = G::R * G::COLS / 2;
    for (int j = threadIdx.x; j < CHUNKS; j += kNttThreads) {
      const int r = j / (G::COLS / 2), cc = (j % (G::COLS / 2)) * 2;
      *reinterpret_cast<ulonglong2 *>(dst + r * (N >> G::LR) + cc) =
          *reinterpret_cast<const ulonglong2 *>(tile + r * G::COLS + cc);
    }
    __syncthreads();
  }
}

// ---- row pass ----------------------------------------------------------------------------
__device__ __forceinline__ int swz_chunk(int chunk) { return chunk ^ ((chunk >> 3) & 7); }
// Word position of column col inside a swizzled 256-word row.
__device__ __forceinline__ int swz_word(int col) { return (swz_chunk(col >> 1) << 1) | (col & 1); }

constexpr int kRowPsSmem = 2 * kTileWords * 8;

template <int LOGN, int MODE, bool INV>
__global__ void __launch_bounds__(kNttThreads, 3) ntt_row_ps(NttBatch b, DeviceTables T, uint32_t slots,
                                                             uint32_t total) {
  constexpr int LR = LOGN - 8;
  constexpr int N = 1 << LOGN;
  constexpr uint32_t TPT = N / kTileWords;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  u64 *data = reinterpret_cast<u64 *>(smem_raw);  // [2][16][256], swizzled

  auto prefetch = [&](uint32_t w, int buf) {
    const TileCoord tc = tile_coord(w, TPT, slots);
    const TowerView v = view_at(b, T, INV, tc.slot, tc.z);
    const u64 *src = v.src + u64(tc.x) * kTileWords;
    u64 *d = data + buf * kTileWords;
    for (int j = threadIdx.x; j < kTileWords / 2; j += kNttThreads) {
      const int r = j >> 7, chunk = j & 127;
      cp_async16(d + r * 256 + swz_chunk(chunk) * 2, src + r * 256 + chunk * 2);
    }
    cp_async_commit();
  };

  uint32_t w = blockIdx.x;
  if (w < total) prefetch(w, 0);
  const int r = threadIdx.x / 16, u = threadIdx.x % 16;
  for (int buf = 0; w < total; w += gridDim.x, buf ^= 1) {
    const uint32_t next = w + gridDim.x;
    if (next < total) {
      prefetch(next, buf ^ 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const TileCoord tc = tile_coord(w, TPT, slots);
    const TowerView v = view_at(b, T, INV, tc.slot, tc.z);
    const u64 q = v.c->q, q2 = v.c->q2;
    const int row = tc.x * 16 + r;
    u64 *my = data + buf * kTileWords + r * 256;
    u64 x[16];
    if constexpr (!INV) {
#pragma unroll
      for (int e = 0; e < 16; ++e) x[e] = my[swz_word(e * 16 + u)];
#pragma unroll
      for (int sp = 0; sp < 4; ++sp) {
        const int s = LR + sp, d = 8 >> sp;
#pragma unroll
        for (int e = 0; e < 16; ++e) {
          if (e & d) continue;
          const Shoup t = tw_load(v.tw + (1 << s) + (row << sp) + (e >> (4 - sp)));
          ct_butterfly<MODE>(x[e], x[e + d], t.w, t.wq, q, q2);
        }
      }
      __syncwarp();
#pragma unroll
      for (int e = 0; e < 16; ++e) my[swz_word(e * 16 + u)] = x[e];
      __syncwarp();
#pragma unroll
      for (int e = 0; e < 16; e += 2) {
        const ulonglong2 p = *reinterpret_cast<const ulonglong2 *>(my + swz_chunk(u * 8 + e / 2) * 2);
        x[e] = p.x;
        x[e + 1] = p.y;
      }
#pragma unroll
      for (int sp = 4; sp < 8; ++sp) {
        const int s = LR + sp, d = 1 << (7 - sp);
#pragma unroll
        for (int e = 0; e < 16; ++e) {
          if (e & d) continue;
          const Shoup t = tw_load(v.tw + (1 << s) + (row << sp) + row_lane_major(u, e >> (8 - sp)));
          ct_butterfly<MODE>(x[e], x[e + d], t.w, t.wq, q, q2);
        }
      }
#pragma unroll
      for (int e = 0; e < 16; e += 2) {
        ulonglong2 p;
        p.x = reduce_final<MODE>(x[e], q, q2);
        p.y = reduce_final<MODE>(x[e + 1], q, q2);
        *reinterpret_cast<ulonglong2 *>(my + swz_chunk(u * 8 + e / 2) * 2) = p;
      }
    } else {
#pragma unroll
      for (int e = 0; e < 16; e += 2) {
        const ulonglong2 p = *reinterpret_cast<const ulonglong2 *>(my + swz_chunk(u * 8 + e / 2) * 2);
        x[e] = p.x;
        x[e + 1] = p.y;
      }
#pragma unroll
      for (int sp = 7; sp >= 4; --sp) {
        const int s = LR + sp, d = 1 << (7 - sp);
#pragma unroll
        for (int e = 0; e < 16; ++e) {
          if (e & d) continue;
          const Shoup t = tw_load(v.tw + (1 << s) + (row << sp) + row_lane_major(u, e >> (8 - sp)));
          gs_butterfly<MODE>(x[e], x[e + d], t.w, t.wq, q, q2);
        }
      }
      __syncwarp();
#pragma unroll
      for (int e = 0; e < 16; e += 2) {
        ulonglong2 p;
        p.x = x[e];
        p.y = x[e + 1];
        *reinterpret_cast<ulonglong2 *>(my + swz_chunk(u * 8 + e / 2) * 2) = p;
      }
      __syncwarp();
#pragma unroll
      for (int e = 0; e < 16; ++e) x[e] = my[swz_word(e * 16 + u)];
#pragma unroll
      for (int sp = 3; sp >= 0; --sp) {
        const int s = LR + sp, d = 8 >> sp;
#pragma unroll
        for (int e = 0; e < 16; ++e) {
          if (e & d) continue;
          const Shoup t = tw_load(v.tw + (1 << s) + (row << sp) + (e >> (4 - sp)));
          gs_butterfly<MODE>(x[e], x[e + d], t.w, t.wq, q, q2);
        }
      }
#pragma unroll
      for (int e = 0; e < 16; ++e) my[swz_word(e * 16 + u)] = x[e];
    }
    __syncthreads();
    const u64 *tile = data + buf * kTileWords;
    u64 *out = v.dst + u64(tc.x) * kTileWords;
    if (INV || b.epi_left == nullptr) {
      for (int j = threadIdx.x; j < kTileWords / 2; j += kNttThreads) {
        const int rr = j >> 7, chunk = j & 127;
        *reinterpret_cast<ulonglong2 *>(out + rr * 256 + chunk * 2) =
            *reinterpret_cast<const ulonglong2 *>(tile + rr * 256 + swz_chunk(chunk) * 2);
      }
    } else {
      // ModDown tail: (left - ntt(x)) * [P^-1]_q.
      const u64 *left = b.epi_left + u64(tc.z) * b.epi_left_stride + u64(b.off[tc.slot]) * N + u64(tc.x) * kTileWords;
      const Shoup pinv = b.epi_pinv[b.id[tc.slot]];
      const u64 *add = poly_add(b, tc.z);
      if (add) add += u64(b.off[tc.slot]) * N + u64(tc.x) * kTileWords;
      for (int j = threadIdx.x; j < kTileWords / 2; j += kNttThreads) {
        const int rr = j >> 7, chunk = j & 127;
        const ulonglong2 t = *reinterpret_cast<const ulonglong2 *>(tile + rr * 256 + swz_chunk(chunk) * 2);
        const ulonglong2 l = *reinterpret_cast<const ulonglong2 *>(left + rr * 256 + chunk * 2);
        ulonglong2 o;
        o.x = shoup_canon(sub_mod(l.x, t.x, q), pinv.w, pinv.wq, q);
        o.y = shoup_canon(sub_mod(l.y, t.y, q), pinv.w, pinv.wq, q);
        if (add) {
          const ulonglong2 e = *reinterpret_cast<const ulonglong2 *>(add + rr * 256 + chunk * 2);
          o.x = add_mod(o.x, e.x, q);
          o.y = add_mod(o.y, e.y, q);
        }
        *reinterpret_cast<ulonglong2 *>(out + rr * 256 + chunk * 2) = o;
      }
    }
    __syncthreads();
  }
}

}  // namespace b200
