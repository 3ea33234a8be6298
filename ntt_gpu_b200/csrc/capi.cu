// C ABI of the B200 CKKS key-switch path (declarations in include/ntt_b200.h).
// Host side: parameter validation, HBM-resident tables, plan caches and kernel
// launches. Composite operations (ModUp, ModDown, Hybrid digits, key switch)
// run on the caller's stream with a caller-provided workspace.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <initializer_list>
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

#include "../../include/ntt_b200.h"
#include "arith.cuh"
#include "kernels.cuh"
#include "ntt.cuh"
#include "rowmac.cuh"
#include "rowmac.h"
#include "tables.cuh"

using b200::u64;
using u128 = unsigned __int128;

namespace {
thread_local std::string g_last_error;
std::atomic<uint64_t> g_launches{0};
// Test hooks, off by default: the poll limit of the tensor-core conversion's
// first bounded wait, and a context-setup operation to fail (0 = none).
std::atomic<int> g_conv_first_wait{1 << 20};
std::atomic<size_t> g_setup_fail_at{0};
std::atomic<size_t> g_setup_operations{0};

struct ContractError : std::invalid_argument {
  using std::invalid_argument::invalid_argument;
};
struct WorkspaceError : std::invalid_argument {
  using std::invalid_argument::invalid_argument;
};
struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};
void require(bool ok, const char *why) {
  if (!ok) throw ContractError(why);
}
// A failed runtime call also leaves its (non-sticky) error as the thread's
// last error; it is cleared here so that a later, unrelated launch check does
// not report it again.
void check_cuda(cudaError_t e, const char *call) {
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    throw CudaError(std::string("CUDA: ") + call + ": " + cudaGetErrorString(e));
  }
}
#define CUDA_CHECK(x) check_cuda((x), #x)

template <class F> int guarded(F f) {
  try {
    f();
    return NTT_B200_OK;
  } catch (const WorkspaceError &e) {
    g_last_error = e.what();
    return NTT_B200_ERR_WORKSPACE;
  } catch (const ContractError &e) {
    g_last_error = e.what();
    return NTT_B200_ERR_CONTRACT;
  } catch (const CudaError &e) {
    g_last_error = e.what();
    return NTT_B200_ERR_CUDA;
  } catch (const std::exception &e) {
    g_last_error = e.what();
    return NTT_B200_ERR_CUDA;
  }
}

// ---- host integer arithmetic -------------------------------------------------
u64 h_mul(u64 a, u64 b, u64 q) { return (u64)(((u128)a * b) % q); }
u64 h_pow(u64 a, u64 e, u64 q) {
  u64 r = 1 % q, b = a % q;
  for (; e; e >>= 1) {
    if (e & 1) r = h_mul(r, b, q);
    b = h_mul(b, b, q);
  }
  return r;
}
u64 h_inv(u64 x, u64 q) {
  require(x % q != 0, "inverse of zero");
  return h_pow(x, q - 2, q);
}
u64 h_shoup(u64 w, u64 q) { return (u64)(((u128)w << 64) / q); }
b200::Shoup h_shoup_pair(u64 w, u64 q) { return {w, h_shoup(w, q)}; }
bool h_is_prime(u64 n) {
  static const u64 bases[12] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
  if (n < 2) return false;
  for (u64 p : bases)
    if (n % p == 0) return n == p;
  u64 d = n - 1, s = 0;
  while (!(d & 1)) d >>= 1, ++s;
  for (u64 a : bases) {
    u64 x = h_pow(a, d, n);
    if (x == 1 || x == n - 1) continue;
    bool composite = true;
    for (u64 r = 1; r < s; ++r) {
      x = h_mul(x, x, n);
      if (x == n - 1) {
        composite = false;
        break;
      }
    }
    if (composite) return false;
  }
  return true;
}
uint32_t h_bitrev(uint32_t x, int bits) {
  uint32_t r = 0;
  for (int i = 0; i < bits; ++i) r = (r << 1) | ((x >> i) & 1);
  return r;
}
// Reorders one tower's twiddle table (bit-reversed group layout) into the
// row passes' lane-major order for stages logN-4 .. logN-1 (b200::row_lane_major).
void lane_major_rows(ulonglong2 *tw, int logn) {
  const int lr = logn - 8;
  std::vector<ulonglong2> block;
  for (int sp = 4; sp < 8; ++sp) {
    const uint32_t s = lr + sp, width = 1u << sp, lanes_k = 1u << (sp - 4);
    for (uint32_t row = 0; row < (1u << lr); ++row) {
      ulonglong2 *b = tw + (1u << s) + row * width;
      block.assign(b, b + width);
      for (uint32_t u = 0; u < 16; ++u)
        for (uint32_t k = 0; k < lanes_k; ++k) b[b200::row_lane_major(u, k)] = block[u * lanes_k + k];
    }
  }
}
b200::Reducer h_reducer(u64 m) {
  b200::Reducer r;
  r.m = m;
  r.one = h_shoup(1, m);
  r.r64 = (u64)(((u128)1 << 64) % m);
  r.r64q = h_shoup(r.r64, m);
  r.r128 = h_mul(r.r64, r.r64, m);
  r.r128q = h_shoup(r.r128, m);
  return r;
}

// Dynamic shared memory limit of every tensor-core conversion kernel, raised
// once per device when its first plan is built (so launches, also inside a
// graph capture, make no attribute calls).
void ensure_conv_tc_attributes(int device) {
  static std::mutex mu;
  static bool done[64] = {};
  std::lock_guard<std::mutex> lock(mu);
  if (device < 0 || device >= 64 || done[device]) return;
  const int bytes = 160 * 1024;
  CUDA_CHECK(cudaFuncSetAttribute(b200::conv_tc_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  CUDA_CHECK(cudaFuncSetAttribute(b200::conv_tc_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  CUDA_CHECK(cudaFuncSetAttribute(b200::conv_tc_kernel<false, 8, 24>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  CUDA_CHECK(cudaFuncSetAttribute(b200::conv_tc_kernel<true, 8, 24>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  CUDA_CHECK(cudaFuncSetAttribute(b200::conv_tc_kernel<false, 8, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  CUDA_CHECK(cudaFuncSetAttribute(b200::conv_tc_kernel<true, 8, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  CUDA_CHECK(cudaFuncSetAttribute(b200::conv_tc_kernel<false, 8, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  CUDA_CHECK(cudaFuncSetAttribute(b200::conv_tc_kernel<true, 8, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  done[device] = true;
}

struct DeviceGuard {
  int previous = -1;
  explicit DeviceGuard(int device) {
    CUDA_CHECK(cudaGetDevice(&previous));
    if (previous != device) CUDA_CHECK(cudaSetDevice(device));
  }
  ~DeviceGuard() {
    int now = -1;
    if (cudaGetDevice(&now) == cudaSuccess && now != previous) cudaSetDevice(previous);
  }
};

struct HostConvPlan {
  b200::ConvPlan *device = nullptr;
  int s = 0, t = 0;
  bool wide = false;
  bool limb = false;  // all moduli < 2^60 and s <= 8: the 30-bit-limb kernel applies
  // Tensor-core form (s <= 16): byte limbs of [Bhat_jt * 2^(8a)]_{m_t} in the
  // canonical K-major layout, groups of 8 targets x 8 output bytes.
  uint8_t *tc_b = nullptr;
  int tc_kpad = 0, tc_groups = 0;
};
}  // namespace

// Streams a request-list call spreads its level groups over: the caller's
// stream plus kChunkLanes - 1 side streams forked from it and joined back.
constexpr size_t kChunkLanes = 4;

struct ntt_b200_context_s {
  int device = 0;
  u64 n = 0;
  int logn = 0;
  size_t m = 0, k = 0, alpha = 0;
  int mode = 2;  // NTT butterfly mode: 2 all moduli < 2^61, 1 all < 2^62, 0 otherwise
  std::vector<u64> mod, psi;  // [M + K] by global id
  b200::TowerConsts *d_tc = nullptr;
  int *d_err = nullptr;  // set by kernels whose bounded waits expired (read by ntt_b200_device_errors)
  ulonglong2 *d_fwd = nullptr, *d_inv = nullptr;
  b200::DeviceTables tables{};
  size_t table_bytes = 0;
  std::mutex mu;
  // (sources, targets, N^-1 folded into Bhat_j^-1) -> plan
  std::map<std::tuple<std::vector<uint16_t>, std::vector<uint16_t>, bool>, HostConvPlan> conv;
  std::map<size_t, b200::DownPlan *> down;
  // Host-buffer pipeline (ntt_b200_keyswitch_host): two copy streams and the
  // per-slot events that hand the two device staging slots between them and
  // the compute stream. Created on first use.
  cudaStream_t copy_in = nullptr, copy_out = nullptr;
  cudaEvent_t ev_in[2] = {nullptr, nullptr}, ev_comp[2] = {nullptr, nullptr}, ev_out[2] = {nullptr, nullptr};
  cudaEvent_t ev_start = nullptr;
  std::mutex pipe_mu;
  // Request lists whose requests span several levels run one level group per
  // stream: side streams forked from the caller's stream by ev_fork and joined
  // back by ev_join. Created by ntt_b200_context_prepare (so capture never
  // creates them) or on first use; chunk_mu keeps each call's event records
  // and waits paired when several host threads share the context.
  cudaStream_t side[kChunkLanes - 1] = {};
  cudaEvent_t ev_fork = nullptr, ev_join[kChunkLanes - 1] = {};
  std::mutex chunk_mu;

  size_t towers() const { return m + k; }

  ~ntt_b200_context_s() {
    // Destruction requires quiescence: the caller has synchronised every stream
    // that used this context (the reference frees tables only after proven
    // quiescence, src/cuda/resident_adapter.inc:107-115).
    for (auto &kv : conv) {
      cudaFree(kv.second.device);
      if (kv.second.tc_b) cudaFree(kv.second.tc_b);
    }
    if (d_err) cudaFree(d_err);
    for (auto &kv : down) cudaFree(kv.second);
    if (copy_in) cudaStreamDestroy(copy_in);
    if (copy_out) cudaStreamDestroy(copy_out);
    for (cudaEvent_t e : {ev_in[0], ev_in[1], ev_comp[0], ev_comp[1], ev_out[0], ev_out[1], ev_start})
      if (e) cudaEventDestroy(e);
    for (cudaStream_t s : side)
      if (s) cudaStreamDestroy(s);
    for (cudaEvent_t e : ev_join)
      if (e) cudaEventDestroy(e);
    if (ev_fork) cudaEventDestroy(ev_fork);
    cudaFree(d_tc);
    cudaFree(d_fwd);
    cudaFree(d_inv);
  }

  // ninv: the plan expects its sources straight out of an unscaled inverse NTT
  // (N times the coefficients, lazily reduced) and folds N^-1 into Bhat_j^-1,
  // so y_j = [x_j * Bhat_j^-1 * N^-1]_{b_j} and every output is unchanged.
  const HostConvPlan &conv_plan(const std::vector<uint16_t> &src, const std::vector<uint16_t> &tgt,
                                bool ninv = false) {
    std::lock_guard<std::mutex> lock(mu);
    auto key = std::make_tuple(src, tgt, ninv);
    auto it = conv.find(key);
    if (it != conv.end()) return it->second;
    require(!src.empty() && src.size() <= (size_t)b200::kMaxConvSources, "basis switch requires 1..40 source towers");
    require(!tgt.empty() && tgt.size() <= (size_t)b200::kMaxConvTargets, "basis switch requires 1..80 target towers");
    std::vector<uint16_t> all(src);
    all.insert(all.end(), tgt.begin(), tgt.end());
    for (auto id : all) require(id < towers(), "tower id out of range");
    std::sort(all.begin(), all.end());
    require(std::adjacent_find(all.begin(), all.end()) == all.end(), "basis switch requires distinct disjoint towers");
    auto plan = std::make_unique<b200::ConvPlan>();
    std::memset(plan.get(), 0, sizeof(b200::ConvPlan));
    const int s = (int)src.size(), t = (int)tgt.size();
    plan->s = s;
    plan->t = t;
    u64 max_src = 0, max_tgt = 0;
    for (int j = 0; j < s; ++j) {
      const u64 b = mod[src[j]];
      u64 hat = 1;
      for (int o = 0; o < s; ++o)
        if (o != j) hat = h_mul(hat, mod[src[o]] % b, b);
      plan->src_q[j] = b;
      const u64 hat_inv = h_inv(hat, b);
      plan->src_inv[j] = h_shoup_pair(ninv ? h_mul(hat_inv, h_inv(n % b, b), b) : hat_inv, b);
      plan->src_id[j] = src[j];
      max_src = std::max(max_src, b);
      for (int i = 0; i < t; ++i) {
        const u64 m_i = mod[tgt[i]];
        u64 h = 1;
        for (int o = 0; o < s; ++o)
          if (o != j) h = h_mul(h, mod[src[o]] % m_i, m_i);
        plan->hat[j * t + i] = h;
      }
    }
    for (int i = 0; i < t; ++i) {
      plan->tgt_id[i] = tgt[i];
      plan->tgt[i] = h_reducer(mod[tgt[i]]);
      plan->tc_wq32[i] = (u64)((((u128)1) << 96) / mod[tgt[i]]);  // fits: m_i > 2^32
      max_tgt = std::max(max_tgt, mod[tgt[i]]);
    }
    HostConvPlan hp;
    hp.s = s;
    hp.t = t;
    const u128 prod = (u128)(max_src - 1) * (max_tgt - 1);
    hp.wide = prod > (~(u128)0) / (u128)s;
    hp.limb = s <= 8 && max_src < (u64(1) << 60) && max_tgt < (u64(1) << 60);
    DeviceGuard guard(device);
    CUDA_CHECK(cudaMalloc(&hp.device, sizeof(b200::ConvPlan)));
    CUDA_CHECK(cudaMemcpy(hp.device, plan.get(), sizeof(b200::ConvPlan), cudaMemcpyHostToDevice));
    // The tensor-core form's reduction needs 2^48 <= m_t < 2^61 (see conv_tc_kernel).
    u64 min_tgt = ~u64(0);
    for (int i = 0; i < t; ++i) min_tgt = std::min(min_tgt, mod[tgt[i]]);
    if (s <= 16 && n >= (u64)b200::kTcThreads && min_tgt >= (u64(1) << 48) && max_tgt < (u64(1) << 61)) {
      // B rows n' = 8 * (target within its group) + output byte b, columns
      // k' = 8 * source + input byte a: byte b of [Bhat_jt * 2^(8a)]_{m_t}.
      hp.tc_kpad = (8 * s + 31) / 32 * 32;
      hp.tc_groups = (t + b200::kTcGroupTargets - 1) / b200::kTcGroupTargets;
      const int rows = b200::kTcGroupRows, kpad = hp.tc_kpad;
      std::vector<uint8_t> bm((size_t)hp.tc_groups * rows * kpad, 0);
      for (int i = 0; i < t; ++i) {
        const u64 m_i = mod[tgt[i]];
        const int g = i / b200::kTcGroupTargets, tl = i % b200::kTcGroupTargets;
        for (int j = 0; j < s; ++j) {
          u64 c = plan->hat[j * t + i] % m_i;  // [Bhat_jt]_{m_t} * 2^(8a), a = 0..7
          for (int a = 0; a < 8; ++a) {
            for (int b = 0; b < 8; ++b)
              bm[(size_t)g * rows * kpad + b200::tc_canon(tl * 8 + b, j * 8 + a, rows)] = (uint8_t)(c >> (8 * b));
            c = h_mul(c, 256 % m_i, m_i);
          }
        }
      }
      CUDA_CHECK(cudaMalloc(&hp.tc_b, bm.size()));
      CUDA_CHECK(cudaMemcpy(hp.tc_b, bm.data(), bm.size(), cudaMemcpyHostToDevice));
      ensure_conv_tc_attributes(device);
    }
    return conv.emplace(key, hp).first->second;
  }

  // Lookups that never build or upload a plan (nullptr when absent).
  const HostConvPlan *find_conv_plan(const std::vector<uint16_t> &src, const std::vector<uint16_t> &tgt,
                                     bool ninv = false) {
    std::lock_guard<std::mutex> lock(mu);
    auto it = conv.find(std::make_tuple(src, tgt, ninv));
    return it == conv.end() ? nullptr : &it->second;
  }
  b200::DownPlan *find_down_plan(size_t level) {
    std::lock_guard<std::mutex> lock(mu);
    auto it = down.find(level);
    return it == down.end() ? nullptr : it->second;
  }

  b200::DownPlan *down_plan(size_t level) {
    std::lock_guard<std::mutex> lock(mu);
    auto it = down.find(level);
    if (it != down.end()) return it->second;
    b200::DownPlan host{};
    for (size_t t = 0; t < level; ++t) {
      const u64 q = mod[t];
      u64 prod = 1;
      for (size_t j = 0; j < k; ++j) prod = h_mul(prod, mod[m + j] % q, q);
      host.p_inv[t] = h_shoup_pair(h_inv(prod, q), q);
      host.p_mod[t] = h_shoup_pair(prod, q);
    }
    b200::DownPlan *d = nullptr;
    DeviceGuard guard(device);
    CUDA_CHECK(cudaMalloc(&d, sizeof(b200::DownPlan)));
    CUDA_CHECK(cudaMemcpy(d, &host, sizeof(b200::DownPlan), cudaMemcpyHostToDevice));
    return down.emplace(level, d).first->second;
  }
};

namespace {
using Ctx = ntt_b200_context_s;

void require_ctx(const Ctx *c) { require(c != nullptr, "null context"); }
void require_level(const Ctx *c, size_t level, bool need_p = true) {
  require(level >= 1 && level <= c->m, "invalid active Q count");
  require(!need_p || c->k > 0, "QP requires P towers");
  require(level <= 40 && c->k <= 40, "conversion requires 1..40 active Q and P towers");
}
cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }
// Kernels move tower data with 16-byte vector accesses.
void require_aligned(std::initializer_list<const void *> ptrs) {
  for (const void *p : ptrs)
    require(p == nullptr || (reinterpret_cast<uintptr_t>(p) & 15) == 0,
            "device pointers must be 16-byte aligned");
}

// ---- per-kernel CUDA-event timing (opt-in) ------------------------------------------
// When enabled, every launch is bracketed by two events on its own stream; the
// query sums cudaEventElapsedTime per kernel class (the external-clock protocol
// of the reference's collect_elapsed, include/ntt/measurement.hpp:41-58).
struct TimerRecord {
  const char *name;
  cudaEvent_t start, stop;
};
struct TimerRegistry {
  std::mutex mu;
  std::atomic<bool> enabled{false};
  std::vector<TimerRecord> records;
  std::vector<cudaEvent_t> pool;
  cudaEvent_t take() {
    if (!pool.empty()) {
      cudaEvent_t e = pool.back();
      pool.pop_back();
      return e;
    }
    cudaEvent_t e = nullptr;
    CUDA_CHECK(cudaEventCreate(&e));
    return e;
  }
} g_timer;

struct Timed {
  const char *name;
  cudaStream_t st;
  cudaEvent_t start = nullptr;
  Timed(const char *kernel, cudaStream_t stream) : name(kernel), st(stream) {
    if (!g_timer.enabled.load()) return;
    std::lock_guard<std::mutex> lock(g_timer.mu);
    start = g_timer.take();
    CUDA_CHECK(cudaEventRecord(start, st));
  }
  // kernels: launches the record covers (the fused row pass + key
  // multiplication is two: the Q towers, then the P towers).
  void done(int kernels = 1) {
    CUDA_CHECK(cudaGetLastError());
    g_launches += kernels;
    if (!start) return;
    std::lock_guard<std::mutex> lock(g_timer.mu);
    cudaEvent_t stop = g_timer.take();
    CUDA_CHECK(cudaEventRecord(stop, st));
    g_timer.records.push_back({name, start, stop});
  }
};

// ---- NTT launches ----------------------------------------------------------------
struct Slot {
  uint32_t off;
  uint16_t id;
};

// Where the second pass of a forward transform writes, when it differs from
// the first pass's output: a split (b/a) destination and the ModDown epilogue.
struct NttFinal {
  u64 *dst = nullptr, *dst_odd = nullptr;
  u64 stride = 0;
  u64 *const *dst_list = nullptr;        // per-polynomial destinations (device array)
  const u64 *const *add_list = nullptr;  // per-polynomial addends (device array; entries may be null)
  const u64 *epi_left = nullptr;
  u64 epi_left_stride = 0;
  const b200::Shoup *epi_pinv = nullptr;
};

// ---- tuning -------------------------------------------------------------------------
// Launch choices that do not change any result, set by name through
// ntt_b200_tuning_set (ntt_gpu_b200/autotune.py measures them on the device and
// commits its choices to ntt_gpu_b200/tuning.json, which the loader applies).
struct Tunable {
  const char *name;
  std::atomic<int64_t> value;
  int64_t lo, hi;
};
Tunable g_tuning[] = {
    {"ntt_minb_fwd_col", {4}, 3, 4},   // CTAs per SM the forward column pass is compiled for
    {"ntt_minb_fwd_row", {4}, 3, 4},
    {"ntt_minb_inv_row", {4}, 3, 4},
    {"ntt_minb_inv_col", {4}, 3, 4},
    {"ntt_col_direct", {1}, 0, 1},     // column passes load and store between registers and global memory
    {"ntt_row_direct", {1}, 0, 1},     // row passes load (forward) / store (inverse) mapping A directly
    {"intt_unscaled", {1}, 0, 1},      // inverse NTTs feeding a basis switch leave N^-1 to the switch
    {"digits_lazy", {1}, 0, 1},        // Hybrid digits feeding the fused MAC skip their final reduction
    {"ntt_epi_stage", {0}, 0, 1},      // ModDown row pass stages its `left` rows in shared memory (measured slower)
    {"ntt_stage_tw_fwd_row", {0}, 0, 1},  // row passes stage their register-stage twiddles in shared memory
    {"ntt_stage_tw_inv_row", {0}, 0, 1},
    {"conv_limbs", {1}, 0, 1},         // 30-bit-limb conversion kernel where it applies
    {"mac_approx", {1}, 0, 1},         // MAC reductions with approximate quotients (moduli below 2^61)
    {"mac_limbs", {0}, 0, 1},          // 30-bit-limb MAC kernel where it applies (slower on B200: off)
    {"mac_rotate", {1}, 0, 1},         // key-switch rotations fused into the MAC's stores (else a gather pass)
    {"conv_tc", {1}, 0, 1},            // tensor-core (tcgen05, int8 limbs) conversion where it applies
    {"conv_blocks_per_sm", {8}, 1, 64}, // target conversion blocks per SM when splitting targets
    {"conv_tc_tiles", {4}, 1, 16},     // 128-coefficient tiles per tensor-core conversion CTA
    {"conv_tc_fixed", {1}, 0, 1},      // tensor-core conversion kernels compiled for 8 -> 24/16/8 towers
    {"row_mac", {1}, 0, 1},            // key multiplication fused into the digits' forward row pass
    {"row_mac_max_beta", {4}, 1, 4},   // largest digit count the fused row pass takes (shared memory per CTA grows with it)
    {"row_mac_inv_rows", {1}, 0, 1},   // its P towers run the ModDown's inverse row pass before they are stored
    {"host_chunk_towers", {4}, 1, 128}, // towers the host-array transforms check and copy per step
    {"ntt_cluster", {0}, 0, 1},        // plain N = 2^16 forward transforms in one pass over an 8-CTA cluster
};
Tunable *find_tunable(const char *name) {
  for (auto &t : g_tuning)
    if (name && std::strcmp(t.name, name) == 0) return &t;
  return nullptr;
}
int64_t tuned(const char *name) { return find_tunable(name)->value.load(std::memory_order_relaxed); }

// SM count of a device (cached).
int device_sms(int device) {
  static int sms[64] = {0};
  if (device < 0 || device >= 64) throw ContractError("device ordinal out of range");
  if (!sms[device]) CUDA_CHECK(cudaDeviceGetAttribute(&sms[device], cudaDevAttrMultiProcessorCount, device));
  return sms[device];
}
// An inverse NTT that only feeds a basis switch skips N^-1 (folded into the
// switch's plan) when the two-pass kernels run it.
bool intt_unscaled(const Ctx &c) { return c.logn >= 12 && tuned("intt_unscaled") != 0; }
// Hybrid digits that only feed the fused MAC stay in the forward NTT's lazy
// range: [0, 8q), or [0, 68q) for towers below 2^57 (reduction-free forward
// butterflies). With every modulus below 2^61 and at most 4 digits, the MAC's
// 128-bit sums stay below 2^127 and its reductions give canonical results. The
// 30-bit-limb MAC needs inputs below 2^60, so it rules this out.
bool digits_lazy(const Ctx &c, size_t beta) {
  return c.mode == 2 && beta <= 4 && c.logn >= 12 && tuned("digits_lazy") != 0 &&
         tuned("mac_limbs") == 0;
}

// The forward row pass of a ModDown launch with its `left` operand staged in
// dynamic shared memory (the direct form).
template <int LOGN, int MODE, int MINB>
void launch_fwd_row_epi(const Ctx &c, const b200::NttBatch &b, dim3 grid, cudaStream_t st) {
  static int attr_set[64] = {};
  auto kernel = b200::ntt_fwd_row<LOGN, MODE, MINB, false, true, true>;
  if (!attr_set[c.device]) {
    CUDA_CHECK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, b200::kEpiSmemBytes));
    attr_set[c.device] = 1;
  }
  kernel<<<grid, b200::kNttThreads, b200::kEpiSmemBytes, st>>>(b, c.tables);
}

// row_done (inverse): the row pass has run already (inside the fused row pass +
// key multiplication), so the column pass reads the source directly.
template <int LOGN, int MODE>
void launch_ntt_2pass(const Ctx &c, const b200::NttBatch &b, const NttFinal *fin, int slots, int polys,
                      bool inverse, cudaStream_t st, bool col_only, bool row_done) {
  const dim3 grid((1u << LOGN) / b200::kTileWords, polys, slots);
  b200::NttBatch second = b;
  if (!row_done) {
    second.src = b.dst;
    second.src_stride = b.dst_stride;
    second.src_list = nullptr;
  }
  if (fin) {
    second.dst = fin->dst;
    second.dst_odd = fin->dst_odd;
    second.dst_stride = fin->stride;
    second.dst_list = fin->dst_list;
    second.add_list = fin->add_list;
    second.epi_left = fin->epi_left;
    second.epi_left_stride = fin->epi_left_stride;
    second.epi_pinv = fin->epi_pinv;
  }
#define NTT_LAUNCH(kernel, batch, ...)                                                        \
  do {                                                                                        \
    if (tuned("ntt_minb_" #kernel) == 3)                                                      \
      b200::ntt_##kernel<LOGN, MODE, 3, ##__VA_ARGS__><<<grid, b200::kNttThreads, 0, st>>>(batch, c.tables); \
    else                                                                                      \
      b200::ntt_##kernel<LOGN, MODE, 4, ##__VA_ARGS__><<<grid, b200::kNttThreads, 0, st>>>(batch, c.tables); \
  } while (0)
  if (!inverse) {
    if constexpr (LOGN == 16 && MODE == 2) {
      // A plain forward transform (canonical outputs, no ModDown epilogue)
      // in one pass over a thread-block cluster per tower (ntt_fwd_cluster16).
      if (!fin && !col_only && !b.lazy_out && tuned("ntt_cluster")) {
        static int attr_set[64] = {};
        if (!attr_set[c.device]) {
          CUDA_CHECK(cudaFuncSetAttribute(b200::ntt_fwd_cluster16, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          b200::kClusterSmemBytes));
          attr_set[c.device] = 1;
        }
        Timed t("ntt_fwd_cluster", st);
        b200::ntt_fwd_cluster16<<<dim3(b200::kClusterCtas, polys, slots), b200::kClusterThreads,
                                   b200::kClusterSmemBytes, st>>>(b, c.tables);
        t.done();
        return;
      }
    }
    Timed t1("ntt_fwd_col", st);
    if (tuned("ntt_col_direct"))
      NTT_LAUNCH(fwd_col, b, true);
    else
      NTT_LAUNCH(fwd_col, b, false);
    t1.done();
    if (col_only) return;  // the fused row pass + key multiplication finishes the transform
    Timed t2("ntt_fwd_row", st);
    if (tuned("ntt_stage_tw_fwd_row"))
      NTT_LAUNCH(fwd_row, second, true, false);
    else if (tuned("ntt_row_direct") && second.epi_left && tuned("ntt_epi_stage")) {
      if (tuned("ntt_minb_fwd_row") == 3)
        launch_fwd_row_epi<LOGN, MODE, 3>(c, second, grid, st);
      else
        launch_fwd_row_epi<LOGN, MODE, 4>(c, second, grid, st);
    } else if (tuned("ntt_row_direct"))
      NTT_LAUNCH(fwd_row, second, false, true);
    else
      NTT_LAUNCH(fwd_row, second, false, false);
    t2.done();
  } else {
    if (!row_done) {
      Timed t1("ntt_inv_row", st);
      if (tuned("ntt_stage_tw_inv_row"))
        NTT_LAUNCH(inv_row, b, true, false);
      else if (tuned("ntt_row_direct"))
        NTT_LAUNCH(inv_row, b, false, true);
      else
        NTT_LAUNCH(inv_row, b, false, false);
      t1.done();
    }
    Timed t2("ntt_inv_col", st);
    if (second.unscaled) {
      if (tuned("ntt_col_direct"))
        NTT_LAUNCH(inv_col, second, true, true);
      else
        NTT_LAUNCH(inv_col, second, false, true);
    } else if (tuned("ntt_col_direct")) {
      NTT_LAUNCH(inv_col, second, true);
    } else {
      NTT_LAUNCH(inv_col, second, false);
    }
    t2.done();
  }
#undef NTT_LAUNCH
}

template <int MODE>
void launch_ntt_chunk(const Ctx &c, const b200::NttBatch &b, const NttFinal *fin, int slots, int polys,
                      bool inverse, cudaStream_t st, bool col_only, bool row_done) {
  switch (c.logn) {
    case 12: launch_ntt_2pass<12, MODE>(c, b, fin, slots, polys, inverse, st, col_only, row_done); break;
    case 13: launch_ntt_2pass<13, MODE>(c, b, fin, slots, polys, inverse, st, col_only, row_done); break;
    case 14: launch_ntt_2pass<14, MODE>(c, b, fin, slots, polys, inverse, st, col_only, row_done); break;
    case 15: launch_ntt_2pass<15, MODE>(c, b, fin, slots, polys, inverse, st, col_only, row_done); break;
    case 16: launch_ntt_2pass<16, MODE>(c, b, fin, slots, polys, inverse, st, col_only, row_done); break;
    default: throw ContractError("unsupported ring dimension");
  }
}

dim3 ew_grid(const Ctx &c, size_t towers, size_t polys) {
  return dim3((unsigned)((c.n + b200::kEwThreads - 1) / b200::kEwThreads), (unsigned)towers,
              (unsigned)polys);
}

// NTT of a list of slots (tower offset from the base, global id) over `polys`
// polynomials with separate source and destination strides (words). `fin`
// (forward only) redirects the final pass: split destination and/or the ModDown
// epilogue (left - x) * P^-1; small transforms run it as a separate kernel.
// src_list (device array, one entry per polynomial) replaces src / src_stride.
// col_only (two-pass forward transforms, mode 2): run the column pass alone;
// the fused row pass + key multiplication (ntt_fwd_row_mac) finishes it.
// row_done (two-pass inverse transforms, mode 2): src has been through the
// row pass already (the fused kernel's P towers); run the column pass alone.
void run_ntt(const Ctx &c, u64 *dst, const u64 *src, const std::vector<Slot> &slots_in, size_t polys,
             u64 src_stride, u64 dst_stride, bool inverse, cudaStream_t st, const NttFinal *fin = nullptr,
             const u64 *const *src_list = nullptr, bool unscaled = false, bool lazy_out = false,
             bool col_only = false, bool row_done = false) {
  require(polys >= 1 && polys <= 65535, "polynomial batch out of range");
  require(!col_only || (!inverse && !fin && c.logn >= 12 && c.mode == 2),
          "a column pass alone is a two-pass mode-2 forward transform");
  require(!row_done || (inverse && !src_list && c.logn >= 12 && c.mode == 2),
          "a transform from its column pass is a two-pass mode-2 inverse");
  require(!fin || !inverse, "final-pass redirection is forward only");
  require(!unscaled || (inverse && c.logn >= 12), "unscaled transforms are two-pass inverses only");
  require(!lazy_out || (!inverse && !fin && c.logn >= 12), "lazy outputs are two-pass forward transforms only");
  // Slots of one tower (e.g. the same target tower of several Hybrid digits)
  // run back to back, so its twiddle table is read from HBM once per launch.
  // Every slot carries its own offset and tower id, so the order changes no
  // result; ascending Q-slot layouts keep their order.
  std::vector<Slot> slots(slots_in);
  std::stable_sort(slots.begin(), slots.end(), [](const Slot &a, const Slot &b) { return a.id < b.id; });
  for (size_t first = 0; first < slots.size(); first += b200::kMaxSlots) {
    const size_t count = std::min<size_t>(b200::kMaxSlots, slots.size() - first);
    b200::NttBatch b{};
    b.src_stride = src_stride;
    b.dst_stride = dst_stride;
    for (size_t i = 0; i < count; ++i) {
      b.off[i] = slots[first + i].off;
      b.id[i] = slots[first + i].id;
    }
    b.src = src;
    b.dst = dst;
    b.src_list = src_list;
    b.unscaled = unscaled;
    b.lazy_out = lazy_out;
    if (c.logn <= 11) {
      const dim3 grid(1, (unsigned)polys, (unsigned)count);
      const int threads = std::min<int>(b200::kNttThreads, std::max<int>(32, (int)(c.n / 2)));
      {
        Timed t("ntt_small", st);
        if (inverse)
          b200::ntt_small<true><<<grid, threads, 0, st>>>(b, c.tables);
        else
          b200::ntt_small<false><<<grid, threads, 0, st>>>(b, c.tables);
        t.done();
      }
      if (fin) {
        // Separate tail: only contiguous Q-slot layouts (slot i = Q tower i) reach here.
        b200::CorrectArgs a{};
        a.dst = fin->dst;
        a.dst_odd = fin->dst_odd;
        a.dst_list = fin->dst_list;
        a.add_list = fin->add_list;
        a.left = fin->epi_left;
        a.right = dst;
        a.pinv = fin->epi_pinv;
        a.tc = c.d_tc;
        a.poly_stride_dst = fin->stride;
        a.poly_stride_left = fin->epi_left_stride;
        a.poly_stride_right = dst_stride;
        a.towers = (int)count;
        a.logn = c.logn;
        Timed t("correct", st);
        b200::correct_kernel<<<ew_grid(c, count, polys), b200::kEwThreads, 0, st>>>(a);
        t.done();
      }
    } else if (c.mode == 2) {
      launch_ntt_chunk<2>(c, b, fin, (int)count, (int)polys, inverse, st, col_only, row_done);
    } else if (c.mode == 1) {
      launch_ntt_chunk<1>(c, b, fin, (int)count, (int)polys, inverse, st, false, false);
    } else {
      launch_ntt_chunk<0>(c, b, fin, (int)count, (int)polys, inverse, st, false, false);
    }
  }
}

std::vector<Slot> contiguous_slots(const std::vector<uint16_t> &ids, uint32_t first_off = 0) {
  std::vector<Slot> s;
  for (size_t i = 0; i < ids.size(); ++i) s.push_back({first_off + (uint32_t)i, ids[i]});
  return s;
}
std::vector<uint16_t> range_ids(size_t begin, size_t end) {
  std::vector<uint16_t> v;
  for (size_t i = begin; i < end; ++i) v.push_back((uint16_t)i);
  return v;
}
std::vector<uint16_t> qp_ids(const Ctx &c, size_t level) {
  auto v = range_ids(0, level);
  for (size_t j = 0; j < c.k; ++j) v.push_back((uint16_t)(c.m + j));
  return v;
}

// ---- conversion launches ---------------------------------------------------------
// The "conv_limbs" tunable selects between the limb kernel and the 128-bit-
// accumulator kernel where both apply (identical results).
bool conv_limbs_enabled() { return tuned("conv_limbs") != 0; }
template <int MAXS>
void launch_conv_t(const HostConvPlan &p, const b200::ConvArgs &a, dim3 grid, bool lazy_out, cudaStream_t st) {
  if constexpr (MAXS <= 8) {
    if (p.limb && conv_limbs_enabled()) {
      if (lazy_out)
        b200::conv_limb_kernel<MAXS, true><<<grid, b200::kEwThreads, 0, st>>>(a);
      else
        b200::conv_limb_kernel<MAXS, false><<<grid, b200::kEwThreads, 0, st>>>(a);
      return;
    }
  }
  if (p.wide)
    b200::conv_kernel<MAXS, true, false><<<grid, b200::kEwThreads, 0, st>>>(a);
  else if (lazy_out)
    b200::conv_kernel<MAXS, false, true><<<grid, b200::kEwThreads, 0, st>>>(a);
  else
    b200::conv_kernel<MAXS, false, false><<<grid, b200::kEwThreads, 0, st>>>(a);
}
// One conversion of a tensor-core launch: plan, source and destination (the
// polynomial strides are shared by the launch) and the targets' slots.
struct ConvPart {
  const HostConvPlan *plan;
  u64 *dst;
  const u64 *src;
  std::vector<uint16_t> slots;
};
// Parts of one launch convert the same numbers of sources and targets.
void run_conv_tc(const Ctx &c, const std::vector<ConvPart> &parts, size_t polys, u64 src_stride, u64 dst_stride,
                 cudaStream_t st, bool lazy_out) {
  require(!parts.empty() && parts.size() <= (size_t)b200::kTcMaxParts, "conversion parts out of range");
  const HostConvPlan &p = *parts[0].plan;
  b200::ConvTcArgs a{};
  for (size_t i = 0; i < parts.size(); ++i) {
    const HostConvPlan &q = *parts[i].plan;
    require(q.s == p.s && q.t == p.t && q.tc_kpad == p.tc_kpad && q.tc_groups == p.tc_groups && q.tc_b,
            "conversions of one launch differ in shape");
    a.part[i].plan = q.device;
    a.part[i].bmat = q.tc_b;
    a.part[i].src = parts[i].src;
    a.part[i].dst = parts[i].dst;
    for (size_t j = 0; j < parts[i].slots.size(); ++j) a.part[i].slot[j] = parts[i].slots[j];
  }
  a.src_poly_stride = src_stride;
  a.dst_poly_stride = dst_stride;
  a.logn = c.logn;
  a.kpad = p.tc_kpad;
  a.groups = p.tc_groups;
  a.first_wait_polls = g_conv_first_wait.load(std::memory_order_relaxed);
  a.err = c.d_err;
  const int smem = b200::kTcThreads * p.tc_kpad + p.tc_groups * b200::kTcGroupRows * p.tc_kpad +
                   p.s * b200::kTcThreads * (int)sizeof(u64);
  ensure_conv_tc_attributes(c.device);
  const size_t units = polys * parts.size();
  auto launch = [&](auto kernel) {
    const size_t tiles = c.n / b200::kTcThreads;
    // The tuned tiles per CTA, halved while the grid would cover fewer than 4
    // CTAs per SM (small batches: one request's switch is only 512 tiles).
    size_t per_cta = (size_t)tuned("conv_tc_tiles");
    const size_t want = 4 * (size_t)device_sms(c.device);
    while (per_cta > 1 && ((tiles + per_cta - 1) / per_cta) * units < want) per_cta = (per_cta + 1) / 2;
    a.tiles_per_cta = (int)per_cta;
    const dim3 grid((unsigned)((tiles + per_cta - 1) / per_cta), (unsigned)parts.size(), (unsigned)polys);
    Timed t("conv", st);
    kernel<<<grid, b200::kTcThreads, smem, st>>>(a);
    t.done();
  };
  // The key switch's conversions (8 sources to 24, 16 or 8 targets: ModUp digits
  // and ModDown with alpha = K = 8) run kernels compiled for their shape.
  const int shape = tuned("conv_tc_fixed") && p.s == 8 ? (p.t == 24 ? 1 : p.t == 16 ? 2 : p.t == 8 ? 3 : 0) : 0;
  switch (2 * shape + (lazy_out ? 1 : 0)) {
    case 0: launch(b200::conv_tc_kernel<false>); break;
    case 1: launch(b200::conv_tc_kernel<true>); break;
    case 2: launch(b200::conv_tc_kernel<false, 8, 24>); break;
    case 3: launch(b200::conv_tc_kernel<true, 8, 24>); break;
    case 4: launch(b200::conv_tc_kernel<false, 8, 16>); break;
    case 5: launch(b200::conv_tc_kernel<true, 8, 16>); break;
    case 6: launch(b200::conv_tc_kernel<false, 8, 8>); break;
    default: launch(b200::conv_tc_kernel<true, 8, 8>); break;
  }
}

// lazy_out: outputs in [0, 4m), only for a lazy forward NTT that consumes them.
void run_conv(const Ctx &c, const HostConvPlan &p, u64 *dst, const u64 *src,
              const std::vector<uint16_t> &slots, size_t polys, u64 src_stride, u64 dst_stride,
              cudaStream_t st, bool lazy_out = false) {
  lazy_out = lazy_out && c.mode >= 1 && c.logn >= 12;
  require(polys >= 1 && polys <= 65535, "polynomial batch out of range");
  if (p.tc_b && tuned("conv_tc") != 0) {
    run_conv_tc(c, {ConvPart{&p, dst, src, slots}}, polys, src_stride, dst_stride, st, lazy_out);
    return;
  }
  b200::ConvArgs a{};
  a.plan = p.device;
  a.src = src;
  a.dst = dst;
  a.src_poly_stride = src_stride;
  a.dst_poly_stride = dst_stride;
  for (size_t i = 0; i < slots.size(); ++i) a.slot[i] = slots[i];
  a.logn = c.logn;
  // All targets per block when the batch alone fills the GPU (the scaled
  // inputs y_j are then computed once per coefficient); otherwise split the
  // targets across blocks for parallelism.
  const size_t base_blocks = ((c.n + b200::kEwThreads - 1) / b200::kEwThreads) * polys;
  const size_t want_blocks = (size_t)device_sms(c.device) * (size_t)tuned("conv_blocks_per_sm");
  int tpb = p.t;
  if (base_blocks < want_blocks) tpb = std::max<int>(4, (int)((p.t * base_blocks + want_blocks - 1) / want_blocks));
  a.targets_per_block = std::min(tpb, p.t);
  const dim3 grid((unsigned)((c.n + b200::kEwThreads - 1) / b200::kEwThreads),
                  (unsigned)((p.t + a.targets_per_block - 1) / a.targets_per_block), (unsigned)polys);
  Timed t("conv", st);
  if (p.s <= 4) launch_conv_t<4>(p, a, grid, lazy_out, st);
  else if (p.s <= 8) launch_conv_t<8>(p, a, grid, lazy_out, st);
  else if (p.s <= 16) launch_conv_t<16>(p, a, grid, lazy_out, st);
  else launch_conv_t<40>(p, a, grid, lazy_out, st);
  t.done();
}

// Conversions of several parts over the same polynomials and strides:
// tensor-core parts of one shape share launches (up to kTcMaxParts each), the
// others run one by one.
void run_convs(const Ctx &c, const std::vector<ConvPart> &parts, size_t polys, u64 src_stride, u64 dst_stride,
               cudaStream_t st, bool lazy_out = false) {
  require(polys >= 1 && polys <= 65535, "polynomial batch out of range");
  const bool lazy_tc = lazy_out && c.mode >= 1 && c.logn >= 12;
  std::vector<ConvPart> batch;
  auto flush = [&] {
    if (!batch.empty()) run_conv_tc(c, batch, polys, src_stride, dst_stride, st, lazy_tc);
    batch.clear();
  };
  for (const ConvPart &part : parts) {
    const HostConvPlan &p = *part.plan;
    if (!p.tc_b || tuned("conv_tc") == 0) {
      flush();
      run_conv(c, p, part.dst, part.src, part.slots, polys, src_stride, dst_stride, st, lazy_out);
      continue;
    }
    if (!batch.empty() && (batch[0].plan->s != p.s || batch[0].plan->t != p.t ||
                           batch.size() == (size_t)b200::kTcMaxParts))
      flush();
    batch.push_back(part);
  }
  flush();
}

// ---- workspace carving -----------------------------------------------------------
size_t aligned_bytes(size_t words) { return ((words * sizeof(u64)) + 255) / 256 * 256; }
struct Carver {
  char *base;
  size_t size, used = 0;
  u64 *take(size_t words) {
    const size_t bytes = aligned_bytes(words);
    if (used + bytes > size) throw WorkspaceError("workspace too small");
    u64 *p = reinterpret_cast<u64 *>(base + used);
    used += bytes;
    return p;
  }
};

size_t workspace_bytes(const Ctx &c, int op, size_t level, size_t batch) {
  const size_t n = c.n, L = level, K = c.k, T = L + K, B = batch;
  const size_t beta = 1 + (L - 1) / c.alpha;
  switch (op) {
    case NTT_B200_OP_MOD_UP: return aligned_bytes(B * L * n);
    case NTT_B200_OP_MOD_DOWN: return aligned_bytes(B * K * n) + aligned_bytes(B * L * n);
    case NTT_B200_OP_DIGITS: return aligned_bytes(B * L * n);
    case NTT_B200_OP_KEYSWITCH:
      return aligned_bytes(B * beta * T * n) + aligned_bytes(B * L * n) + 2 * aligned_bytes(2 * B * T * n) +
             aligned_bytes(2 * B * K * n) + aligned_bytes(2 * B * L * n);
    default: throw ContractError("unknown workspace operation");
  }
}

Carver carve(const Ctx &c, void *ws, size_t bytes, int op, size_t level, size_t batch) {
  const size_t need = workspace_bytes(c, op, level, batch);
  if (need && (!ws || bytes < need)) throw WorkspaceError("workspace missing or too small");
  return Carver{reinterpret_cast<char *>(ws), bytes};
}

// ---- composite operations over a batch of polynomials ----------------------------------
// ModDown of `polys` evaluation-QP polynomials (stride src_stride) into
// evaluation Q_L (stride dst_stride, or split even/odd destinations).
// dst_list / add_list (device arrays, one entry per polynomial) optionally
// redirect each output and add a per-polynomial addend.
// p_rows_done: the P towers of src have been through the inverse NTT's row
// pass already (the fused row pass + key multiplication ran it).
void do_mod_down(Ctx &c, size_t L, size_t polys, u64 *dst, u64 *dst_odd, u64 dst_stride, const u64 *src,
                 u64 src_stride, Carver &ws, cudaStream_t st, u64 *const *dst_list = nullptr,
                 const u64 *const *add_list = nullptr, bool p_rows_done = false) {
  const size_t n = c.n, K = c.k;
  u64 *p_coeff = ws.take(polys * K * n);
  u64 *corr = ws.take(polys * L * n);
  const bool unscaled = intt_unscaled(c);
  run_ntt(c, p_coeff, src + L * n, contiguous_slots(range_ids(c.m, c.m + K)), polys, src_stride, K * n,
          true, st, nullptr, nullptr, unscaled, false, false, p_rows_done);
  const auto &plan = c.conv_plan(range_ids(c.m, c.m + K), range_ids(0, L), unscaled);
  std::vector<uint16_t> slots;
  for (size_t i = 0; i < L; ++i) slots.push_back((uint16_t)i);
  run_conv(c, plan, corr, p_coeff, slots, polys, K * n, L * n, st, true);
  NttFinal fin;
  fin.dst = dst;
  fin.dst_odd = dst_odd;
  fin.stride = dst_stride;
  fin.dst_list = dst_list;
  fin.add_list = add_list;
  fin.epi_left = src;
  fin.epi_left_stride = src_stride;
  fin.epi_pinv = c.down_plan(L)->p_inv;
  run_ntt(c, corr, corr, contiguous_slots(range_ids(0, L)), polys, L * n, L * n, false, st, &fin);
}

// Hybrid digits of `polys` evaluation-Q_L inputs (stride L*n) into digits
// (stride beta*T*n). copy_own = false leaves each digit's own towers unwritten
// (the fused MAC reads them from the input).
// src_list (device array, one input per polynomial) replaces the strided src.
// col_only: the digits' forward transforms stop after their column pass (for
// the fused row pass + key multiplication).
void do_digits(Ctx &c, size_t L, size_t polys, u64 *digits, const u64 *src, Carver &ws, bool copy_own,
               cudaStream_t st, const u64 *const *src_list = nullptr, bool lazy_out = false,
               bool col_only = false) {
  const size_t n = c.n, K = c.k, T = L + K;
  const size_t beta = 1 + (L - 1) / c.alpha;
  const u64 dstride = beta * T * n;
  require(!(copy_own && src_list), "own-tower copies need a strided source");
  u64 *coeff = ws.take(polys * L * n);
  const bool unscaled = intt_unscaled(c);
  run_ntt(c, coeff, src, contiguous_slots(range_ids(0, L)), polys, L * n, L * n, true, st, nullptr, src_list,
          unscaled);
  const auto all = qp_ids(c, L);
  std::vector<Slot> fwd;
  std::vector<ConvPart> convs;  // the digits' conversions: one launch where their shapes agree
  size_t digit = 0;
  for (size_t first = 0; first < L; first += c.alpha, ++digit) {
    const size_t count = std::min(c.alpha, L - first);
    u64 *out = digits + digit * T * n;
    if (copy_own)
      CUDA_CHECK(cudaMemcpy2DAsync(out + first * n, dstride * sizeof(u64), src + first * n,
                                   L * n * sizeof(u64), count * n * sizeof(u64), polys,
                                   cudaMemcpyDeviceToDevice, st));
    std::vector<uint16_t> tgt, slots;
    for (size_t t = 0; t < T; ++t)
      if (t < first || t >= first + count) {
        tgt.push_back(all[t]);
        slots.push_back((uint16_t)t);
        fwd.push_back({(uint32_t)(digit * T + t), all[t]});
      }
    convs.push_back({&c.conv_plan(range_ids(first, first + count), tgt, unscaled), out, coeff + first * n,
                     std::move(slots)});
  }
  run_convs(c, convs, polys, L * n, dstride, st, true);
  run_ntt(c, digits, digits, fwd, polys, dstride, dstride, false, st, nullptr, nullptr, false, lazy_out && !col_only,
          col_only);
}

// MAC of `polys` requests: out_b/out_a of request z at out + z * out_stride;
// digit d of request z at digits[d] + z * digit_poly_stride.
bool mac_limbs_apply(const Ctx &c) {
  u64 max_q = 0;
  for (auto q : c.mod) max_q = std::max(max_q, q);
  return max_q < (u64(1) << 60) && tuned("mac_limbs") != 0;
}

// Whether a key switch at level L rotates inside the MAC (mac2_kernel's ROT
// form: two coefficients per thread, at most 4 digits) instead of a separate
// rotate_kernel pass over the extended result.
bool mac_fuses_rotation(const Ctx &c, size_t L) {
  const size_t beta = 1 + (L - 1) / c.alpha;
  return tuned("mac_rotate") != 0 && c.n >= 2 * (u64)b200::kEwThreads && beta <= 4 && !mac_limbs_apply(c);
}

// Rotation fused into the MAC: c0 of request z at c0 + z * c0_stride (request
// tables carry their own c0 and automorphism).
struct MacRotation {
  bool on = false;
  const u64 *c0 = nullptr;
  u64 c0_stride = 0;
  uint32_t g = 1;
};

// MAC launch arguments: `beta` digits (digit pointers optional: the fused row
// pass reads its digits from its own arguments), keys, outputs and rotation.
b200::MacArgs mac_args(Ctx &c, size_t L, size_t beta, u64 *out_b, u64 *out_a, u64 out_stride,
                       const std::vector<const u64 *> &digits, u64 digit_poly_stride, const u64 *input,
                       const std::vector<const u64 *> &key_b, const std::vector<const u64 *> &key_a,
                       bool full_key_rows, bool accumulate, const b200::ReqDesc *req, const MacRotation &rot) {
  const size_t n = c.n;
  require(beta >= 1 && beta <= (size_t)b200::kMaxDigits &&
              (req || (key_b.size() == beta && key_a.size() == beta)),
          "MAC digit count out of range");
  require(req || !rot.on || ((rot.g & 1) && rot.g < 2 * c.n), "invalid negacyclic automorphism index");
  b200::MacArgs a{};
  a.out_b = out_b;
  a.out_a = out_a;
  for (size_t d = 0; d < beta; ++d) {
    if (d < digits.size()) a.digit[d] = digits[d];
    if (!req) {
      a.key_b[d] = key_b[d];
      a.key_a[d] = key_a[d];
    }
  }
  a.input = input;
  a.tc = c.d_tc;
  a.req = req;
  a.key_digit_stride = c.towers() * n;
  a.poly_stride_out = out_stride;
  a.poly_stride_digits = digit_poly_stride;
  a.poly_stride_input = L * n;
  a.level = (int)L;
  a.m = (int)c.m;
  a.beta = (int)beta;
  a.alpha = (int)c.alpha;
  a.logn = c.logn;
  a.full_key_rows = full_key_rows;
  a.accumulate = accumulate;
  if (rot.on) {
    a.c0 = rot.c0;
    a.c0_poly_stride = rot.c0_stride;
    a.g = rot.g;
    a.plan = c.down_plan(L);
  }
  return a;
}

void do_mac(Ctx &c, size_t L, size_t polys, u64 *out_b, u64 *out_a, u64 out_stride,
            const std::vector<const u64 *> &digits, u64 digit_poly_stride, const u64 *input,
            const std::vector<const u64 *> &key_b, const std::vector<const u64 *> &key_a, bool full_key_rows,
            bool accumulate, cudaStream_t st, const b200::ReqDesc *req = nullptr, bool lazy_digits = false,
            const MacRotation &rot = {}) {
  const size_t n = c.n, T = L + c.k;
  const size_t beta = digits.size();
  require(!rot.on || (mac_fuses_rotation(c, L) && beta == 1 + (L - 1) / c.alpha && !accumulate),
          "rotation fused into the MAC needs its two-coefficient form and no accumulation");
  const b200::MacArgs a = mac_args(c, L, beta, out_b, out_a, out_stride, digits, digit_poly_stride, input, key_b,
                                   key_a, full_key_rows, accumulate, req, rot);
  // Lazy digits lie in [0, 8q), or [0, 68q) for towers below 2^57 (reduction-free
  // forward butterflies); the largest product of a digit and a key word decides
  // whether beta of them can overflow 128 bits.
  u128 prod = 0;
  for (auto q : c.mod) {
    const u64 range = !lazy_digits ? q : (q < b200::kFreeModulusBound ? b200::kFreeRangeFactor : 8) * q;
    prod = std::max(prod, (u128)(range - 1) * (q - 1));
  }
  const bool wide = prod > (~(u128)0) / (u128)beta;
  const bool limbs = mac_limbs_apply(c);
  require(!lazy_digits || (!limbs && beta <= 4 && n >= 2 * b200::kEwThreads), "lazy digits need the 2-coefficient MAC");
  Timed t("mac", st);
  if (n >= 2 * b200::kEwThreads && beta <= 4 && limbs) {
    const dim3 grid2((unsigned)(n / (2 * b200::kEwThreads)), (unsigned)polys, (unsigned)T);
    switch (beta) {
      case 1: b200::mac2_limb_kernel<1><<<grid2, b200::kEwThreads, 0, st>>>(a); break;
      case 2: b200::mac2_limb_kernel<2><<<grid2, b200::kEwThreads, 0, st>>>(a); break;
      case 3: b200::mac2_limb_kernel<3><<<grid2, b200::kEwThreads, 0, st>>>(a); break;
      default: b200::mac2_limb_kernel<4><<<grid2, b200::kEwThreads, 0, st>>>(a); break;
    }
  } else if (n >= 2 * b200::kEwThreads && beta <= 4) {
    const dim3 grid2((unsigned)(n / (2 * b200::kEwThreads)), (unsigned)polys, (unsigned)T);
    auto launch = [&](auto beta_tag) {
      constexpr int B = decltype(beta_tag)::value;
      const bool approx = !wide && c.mode == 2 && tuned("mac_approx");  // every modulus below 2^61
      if (rot.on) {
        if (wide)
          b200::mac2_kernel<B, true, false, true><<<grid2, b200::kEwThreads, 0, st>>>(a);
        else if (approx)
          b200::mac2_kernel<B, false, true, true><<<grid2, b200::kEwThreads, 0, st>>>(a);
        else
          b200::mac2_kernel<B, false, false, true><<<grid2, b200::kEwThreads, 0, st>>>(a);
      } else if (wide) {
        b200::mac2_kernel<B, true><<<grid2, b200::kEwThreads, 0, st>>>(a);
      } else if (approx) {
        b200::mac2_kernel<B, false, true><<<grid2, b200::kEwThreads, 0, st>>>(a);
      } else {
        b200::mac2_kernel<B, false><<<grid2, b200::kEwThreads, 0, st>>>(a);
      }
    };
    switch (beta) {
      case 1: launch(std::integral_constant<int, 1>{}); break;
      case 2: launch(std::integral_constant<int, 2>{}); break;
      case 3: launch(std::integral_constant<int, 3>{}); break;
      default: launch(std::integral_constant<int, 4>{}); break;
    }
  } else {
    const dim3 grid((unsigned)((n + b200::kEwThreads - 1) / b200::kEwThreads), (unsigned)polys, (unsigned)T);
    if (wide)
      b200::mac_kernel<true><<<grid, b200::kEwThreads, 0, st>>>(a);
    else
      b200::mac_kernel<false><<<grid, b200::kEwThreads, 0, st>>>(a);
  }
  t.done();
}

// Full-context key digits d at key + d * (M + K) * N.
std::vector<const u64 *> key_digits(const Ctx &c, const u64 *key, size_t beta) {
  std::vector<const u64 *> v;
  for (size_t d = 0; d < beta; ++d) v.push_back(key + d * c.towers() * c.n);
  return v;
}

// Whether a key switch at level L runs its digits' forward row pass fused with
// the key multiplication (ntt_fwd_row_mac): every modulus below 2^61, a
// two-pass ring size, and at most row_mac_max_beta digits.
bool row_mac_applies(const Ctx &c, size_t L) {
  const size_t beta = 1 + (L - 1) / c.alpha;
  return tuned("row_mac") != 0 && c.mode == 2 && c.logn >= 12 &&
         beta <= (size_t)std::min<int64_t>(tuned("row_mac_max_beta"), b200::kRowMacMaxBeta);
}

// Whether the fused kernel's P towers also run the ModDown's inverse row pass:
// two digits or more (their regions hold the two channels) and one request per
// input (hoisted requests still need the digits after the first request).
bool row_mac_inv_rows_applies(const Ctx &c, size_t L, bool one_request_per_input) {
  const size_t beta = 1 + (L - 1) / c.alpha;
  return one_request_per_input && beta >= 2 && tuned("row_mac_inv_rows") != 0;
}

// The fused row pass + key multiplication over `inputs` distinct inputs whose
// digits have been through their forward column pass (digits + u * beta*T*N).
// Strided mode (req == nullptr): request u is input u, with the shared
// full-context key and, with rot.on, c0 + u * rot.c0_stride. Request-table
// mode: input u serves requests [first, first + count) of `groups`.
// p_inverse_rows: the P towers' outputs leave through the ModDown's inverse row
// pass (row_mac_inv_rows applies).
void do_row_mac(Ctx &c, size_t L, size_t inputs, u64 *out_b, u64 *out_a, u64 out_stride, const u64 *digits,
                const u64 *input, const u64 *key_b, const u64 *key_a, const b200::ReqDesc *req, const u64 *groups,
                const MacRotation &rot, cudaStream_t st, bool p_inverse_rows = false) {
  const size_t n = c.n, T = L + c.k, beta = 1 + (L - 1) / c.alpha;
  require(inputs >= 1 && inputs <= 65535, "request batch out of range");
  std::vector<const u64 *> kb, ka;
  if (!req) {
    kb = key_digits(c, key_b, beta);
    ka = key_digits(c, key_a, beta);
  }
  b200::RowMacArgs a{};
  a.mac = mac_args(c, L, beta, out_b, out_a, out_stride, {}, beta * T * n, input, kb, ka, true, false, req, rot);
  a.digits = digits;
  a.digit_stride = beta * T * n;
  a.groups = groups;
  a.towers = (int)T;
  a.p_inverse_rows = p_inverse_rows;
  Timed t("row_mac", st);
  CUDA_CHECK(b200::row_mac_launch(a, c.tables, c.logn, (int)beta, rot.on, (unsigned)inputs, (unsigned)T, st));
  t.done(T > L ? 2 : 1);
}

void do_rotate(Ctx &c, size_t L, size_t polys, u64 *out_b, u64 *out_a, const u64 *ext_b, const u64 *ext_a,
               u64 stride, const u64 *c0, u64 c0_stride, uint32_t g, cudaStream_t st,
               const b200::ReqDesc *req = nullptr) {
  require(req || ((g & 1) && g < 2 * c.n), "invalid negacyclic automorphism index");
  b200::RotateArgs a{};
  a.out_b = out_b;
  a.out_a = out_a;
  a.ext_b = ext_b;
  a.ext_a = ext_a;
  a.c0 = c0;
  a.plan = c.down_plan(L);
  a.tc = c.d_tc;
  a.req = req;
  a.poly_stride = stride;
  a.c0_poly_stride = c0_stride;
  a.level = (int)L;
  a.m = (int)c.m;
  a.logn = c.logn;
  a.g = g;
  Timed t("rotate", st);
  b200::rotate_kernel<<<ew_grid(c, L + c.k, polys), b200::kEwThreads, 0, st>>>(a);
  t.done();
}

// The Hybrid key switch of `batch` requests at one level with one shared key:
// src/out_b/out_a/c0 are [batch][L][N].
void do_keyswitch(Ctx &c, size_t L, size_t batch, u64 *out_b, u64 *out_a, const u64 *src, const u64 *key_b,
                  const u64 *key_a, const u64 *c0, uint32_t g, Carver &ws, cudaStream_t st) {
  const size_t n = c.n, T = L + c.k;
  const size_t beta = 1 + (L - 1) / c.alpha;
  u64 *digits = ws.take(batch * beta * T * n);
  u64 *acc = ws.take(2 * batch * T * n);  // [batch][b|a][T][N]
  u64 *rot = ws.take(2 * batch * T * n);
  if (c0) require((g & 1) && g < 2 * c.n, "invalid negacyclic automorphism index");
  if (row_mac_applies(c, L)) {
    const bool inv_rows = row_mac_inv_rows_applies(c, L, true);
    do_digits(c, L, batch, digits, src, ws, false, st, nullptr, true, true);
    do_row_mac(c, L, batch, acc, acc + T * n, 2 * T * n, digits, src, key_b, key_a, nullptr, nullptr,
               MacRotation{c0 != nullptr, c0, L * n, g}, st, inv_rows);
    do_mod_down(c, L, 2 * batch, out_b, out_a, L * n, acc, T * n, ws, st, nullptr, nullptr, inv_rows);
    return;
  }
  const bool lazy = digits_lazy(c, beta);
  const bool fused = c0 && mac_fuses_rotation(c, L);
  do_digits(c, L, batch, digits, src, ws, false, st, nullptr, lazy);
  std::vector<const u64 *> dptr;
  for (size_t d = 0; d < beta; ++d) dptr.push_back(digits + d * T * n);
  do_mac(c, L, batch, acc, acc + T * n, 2 * T * n, dptr, beta * T * n, src, key_digits(c, key_b, beta),
         key_digits(c, key_a, beta), true, false, st, nullptr, lazy, MacRotation{fused, c0, L * n, g});
  const u64 *ext = acc;
  if (c0 && !fused) {
    do_rotate(c, L, batch, rot, rot + T * n, acc, acc + T * n, 2 * T * n, c0, L * n, g, st);
    ext = rot;
  }
  do_mod_down(c, L, 2 * batch, out_b, out_a, L * n, ext, T * n, ws, st);
}

// ---- request-table key switch --------------------------------------------------------
// Requests of one call are grouped by level (a shape class) and cut into chunks
// of at most kMaxGroup. Each chunk is one pass of the fused pipeline; every
// kernel reads its request's pointers from a small device table, so a chunk
// mixes keys, rotations, relinearization addends and callers' buffers freely.
// Requests of a chunk that share an input share its digits (the hoisted
// decomposition of the reference's hybrid_rotate_many,
// include/ntt/openfhe_hybrid_adapter.hpp:309-361).
constexpr size_t kMaxGroup = 128;

struct Chunk {
  size_t level = 0;
  std::vector<size_t> idx;          // request indices, call order
  std::vector<const u64 *> usrc;    // unique inputs, first-seen order
  std::vector<uint32_t> dslot;      // per request: index into usrc
  bool rotate = false, add = false;
};

std::vector<Chunk> plan_chunks(const ntt_b200_ks_request *reqs, size_t count) {
  std::vector<size_t> levels;
  for (size_t i = 0; i < count; ++i)
    if (std::find(levels.begin(), levels.end(), (size_t)reqs[i].level) == levels.end())
      levels.push_back(reqs[i].level);
  std::vector<Chunk> out;
  for (size_t L : levels) {
    Chunk cur;
    // Requests that share an input are made adjacent (stable by digit slot),
    // so the fused row pass finds each input's requests as one range.
    auto flush = [&] {
      if (!cur.idx.empty()) {
        std::vector<size_t> order(cur.idx.size());
        for (size_t j = 0; j < order.size(); ++j) order[j] = j;
        std::stable_sort(order.begin(), order.end(),
                         [&](size_t a, size_t b) { return cur.dslot[a] < cur.dslot[b]; });
        Chunk sorted = cur;
        for (size_t j = 0; j < order.size(); ++j) {
          sorted.idx[j] = cur.idx[order[j]];
          sorted.dslot[j] = cur.dslot[order[j]];
        }
        out.push_back(std::move(sorted));
      }
      cur = Chunk{};
    };
    for (size_t i = 0; i < count; ++i) {
      if ((size_t)reqs[i].level != L) continue;
      if (cur.idx.size() == kMaxGroup) flush();
      cur.level = L;
      const u64 *src = reqs[i].src;
      auto it = std::find(cur.usrc.begin(), cur.usrc.end(), src);
      uint32_t slot = (uint32_t)(it - cur.usrc.begin());
      if (it == cur.usrc.end()) cur.usrc.push_back(src);
      cur.idx.push_back(i);
      cur.dslot.push_back(slot);
      cur.rotate = cur.rotate || reqs[i].c0 != nullptr;
      cur.add = cur.add || reqs[i].add_b != nullptr || reqs[i].add_a != nullptr;
    }
    flush();
  }
  return out;
}

// Words of a chunk's device table: ReqDesc[r] | usrc[u] | dst_list[2r] |
// add_list[2r] | groups[u] (input u's requests: first | count << 32).
constexpr size_t table_words(size_t r, size_t u) { return 6 * r + u + 4 * r + u; }
// A full chunk (every request with its own input) fits put_table's largest form.
static_assert(table_words(kMaxGroup, kMaxGroup) <= 2048, "request table of a full chunk exceeds put_words");

size_t chunk_bytes(const Ctx &c, const Chunk &ch) {
  const size_t n = c.n, L = ch.level, K = c.k, T = L + K, r = ch.idx.size(), u = ch.usrc.size();
  const size_t beta = 1 + (L - 1) / c.alpha;
  const bool rot_pass = ch.rotate && !row_mac_applies(c, L) && !mac_fuses_rotation(c, L);
  return aligned_bytes(table_words(r, u)) + aligned_bytes(u * beta * T * n) + aligned_bytes(u * L * n) +
         aligned_bytes(2 * r * T * n) + (rot_pass ? aligned_bytes(2 * r * T * n) : 0) +
         aligned_bytes(2 * r * K * n) + aligned_bytes(2 * r * L * n);
}

template <int W>
void put_table_t(const std::vector<u64> &words, u64 *dst, cudaStream_t st) {
  b200::Words<W> p;
  p.count = (uint32_t)words.size();
  std::memcpy(p.w, words.data(), words.size() * sizeof(u64));
  Timed t("table", st);
  b200::put_words<W><<<1, 256, 0, st>>>(p, dst);
  t.done();
}
void put_table(const std::vector<u64> &words, u64 *dst, cudaStream_t st) {
  if (words.size() <= 256) put_table_t<256>(words, dst, st);
  else if (words.size() <= 1024) put_table_t<1024>(words, dst, st);
  else if (words.size() <= 2048) put_table_t<2048>(words, dst, st);
  else throw ContractError("request table too large");
}

u64 as_word(const void *p) { return (u64)reinterpret_cast<uintptr_t>(p); }

void run_chunk(Ctx &c, const ntt_b200_ks_request *reqs, const Chunk &ch, Carver &ws, cudaStream_t st) {
  const size_t n = c.n, L = ch.level, T = L + c.k, r = ch.idx.size(), u = ch.usrc.size();
  const size_t beta = 1 + (L - 1) / c.alpha;
  u64 *table = ws.take(table_words(r, u));
  std::vector<u64> words;
  words.reserve(table_words(r, u));
  for (size_t j = 0; j < r; ++j) {
    const ntt_b200_ks_request &q = reqs[ch.idx[j]];
    words.push_back(as_word(q.src));
    words.push_back(as_word(q.key_b));
    words.push_back(as_word(q.key_a));
    words.push_back(as_word(q.c0));
    words.push_back((u64)(q.c0 ? q.automorphism : 1u) | ((u64)ch.dslot[j] << 32));
    words.push_back(0);
  }
  for (const u64 *p : ch.usrc) words.push_back(as_word(p));
  for (size_t j = 0; j < r; ++j) {
    words.push_back(as_word(reqs[ch.idx[j]].out_b));
    words.push_back(as_word(reqs[ch.idx[j]].out_a));
  }
  for (size_t j = 0; j < r; ++j) {
    words.push_back(as_word(reqs[ch.idx[j]].add_b));
    words.push_back(as_word(reqs[ch.idx[j]].add_a));
  }
  for (size_t v = 0, j = 0; v < u; ++v) {  // requests are sorted by digit slot
    const size_t first = j;
    while (j < r && ch.dslot[j] == v) ++j;
    words.push_back((u64)first | ((u64)(j - first) << 32));
  }
  put_table(words, table, st);
  const auto *desc = reinterpret_cast<const b200::ReqDesc *>(table);
  const auto *usrc = reinterpret_cast<const u64 *const *>(table + 6 * r);
  auto *dst_list = reinterpret_cast<u64 *const *>(table + 6 * r + u);
  const auto *add_list = reinterpret_cast<const u64 *const *>(table + 6 * r + u + 2 * r);
  const u64 *groups = table + 6 * r + u + 4 * r;

  u64 *digits = ws.take(u * beta * T * n);
  u64 *acc = ws.take(2 * r * T * n);  // [request][b|a][T][N]
  if (row_mac_applies(c, L)) {
    const bool inv_rows = row_mac_inv_rows_applies(c, L, u == r);
    do_digits(c, L, u, digits, nullptr, ws, false, st, usrc, true, true);
    do_row_mac(c, L, u, acc, acc + T * n, 2 * T * n, digits, nullptr, nullptr, nullptr, desc, groups,
               MacRotation{ch.rotate}, st, inv_rows);
    do_mod_down(c, L, 2 * r, nullptr, nullptr, 0, acc, T * n, ws, st, dst_list, ch.add ? add_list : nullptr,
                inv_rows);
    return;
  }
  const bool fused = ch.rotate && mac_fuses_rotation(c, L);
  u64 *rot = ch.rotate && !fused ? ws.take(2 * r * T * n) : nullptr;
  const bool lazy = digits_lazy(c, beta);
  do_digits(c, L, u, digits, nullptr, ws, false, st, usrc, lazy);
  std::vector<const u64 *> dptr;
  for (size_t d = 0; d < beta; ++d) dptr.push_back(digits + d * T * n);
  do_mac(c, L, r, acc, acc + T * n, 2 * T * n, dptr, beta * T * n, nullptr, {}, {}, true, false, st, desc, lazy,
         MacRotation{fused});
  const u64 *ext = acc;
  if (ch.rotate && !fused) {
    do_rotate(c, L, r, rot, rot + T * n, acc, acc + T * n, 2 * T * n, nullptr, 0, 1, st, desc);
    ext = rot;
  }
  do_mod_down(c, L, 2 * r, nullptr, nullptr, 0, ext, T * n, ws, st, dst_list, ch.add ? add_list : nullptr);
}

// Host-side checks of a request list, all before anything is enqueued.
void validate_requests(const Ctx &c, const ntt_b200_ks_request *reqs, size_t count) {
  require(reqs != nullptr && count >= 1, "empty request list");
  require(c.k > 0, "QP requires P towers");
  require(c.k <= 40, "conversion requires 1..40 active Q and P towers");
  struct Span {
    uintptr_t lo, hi;
    size_t req;
    int role;  // 0 input, 1 out_b, 2 out_a, 3 add_b, 4 add_a
  };
  std::vector<Span> spans;
  const size_t key_words = (1 + (c.m - 1) / c.alpha) * c.towers() * c.n;
  for (size_t i = 0; i < count; ++i) {
    const ntt_b200_ks_request &q = reqs[i];
    require(q.level >= 1 && q.level <= c.m && q.level <= 40, "invalid active Q count");
    require(q.src && q.out_b && q.out_a && q.key_b && q.key_a, "null pointer");
    require_aligned({q.src, q.out_b, q.out_a, q.key_b, q.key_a, q.c0, q.add_b, q.add_a});
    if (q.c0) require((q.automorphism & 1) && q.automorphism < 2 * c.n, "invalid negacyclic automorphism index");
    const size_t poly = q.level * c.n * sizeof(u64);
    auto add = [&](const void *p, size_t bytes, int role) {
      if (p) spans.push_back({reinterpret_cast<uintptr_t>(p), reinterpret_cast<uintptr_t>(p) + bytes, i, role});
    };
    add(q.src, poly, 0);
    add(q.c0, poly, 0);
    add(q.key_b, key_words * sizeof(u64), 0);
    add(q.key_a, key_words * sizeof(u64), 0);
    add(q.out_b, poly, 1);
    add(q.out_a, poly, 2);
    add(q.add_b, poly, 3);
    add(q.add_a, poly, 4);
  }
  // Outputs overlap nothing, except a request's own addend at the same address
  // (in-place relinearization).
  for (const Span &o : spans) {
    if (o.role != 1 && o.role != 2) continue;
    for (const Span &x : spans) {
      if (&x == &o || x.hi <= o.lo || o.hi <= x.lo) continue;
      const bool own_addend = x.req == o.req && x.role == o.role + 2 && x.lo == o.lo && x.hi == o.hi;
      require(own_addend, "a request output overlaps another buffer of the call");
    }
  }
}

// Streams for a call's chunks. Chunks of one level stay on one stream, in call
// order, and share its workspace region; the level groups are spread over up
// to kChunkLanes streams, largest first onto the least-loaded stream, so small
// groups fill the GPU beside large ones instead of running one after another.
// Region l is the largest chunk of lane l; the regions lie back to back.
struct LanePlan {
  std::vector<std::vector<size_t>> lanes;  // chunk indices per stream, lane 0 = the caller's
  std::vector<size_t> region;              // workspace bytes per stream
};

LanePlan plan_lanes(const Ctx &c, const std::vector<Chunk> &chunks) {
  std::vector<size_t> levels;
  std::vector<std::vector<size_t>> groups;
  for (size_t i = 0; i < chunks.size(); ++i) {
    const auto it = std::find(levels.begin(), levels.end(), chunks[i].level);
    if (it == levels.end()) {
      levels.push_back(chunks[i].level);
      groups.push_back({i});
    } else {
      groups[size_t(it - levels.begin())].push_back(i);
    }
  }
  std::vector<size_t> work(groups.size(), 0), order(groups.size());
  for (size_t g = 0; g < groups.size(); ++g) {
    for (size_t i : groups[g]) work[g] += chunk_bytes(c, chunks[i]);
    order[g] = g;
  }
  std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return work[a] > work[b]; });
  LanePlan p;
  const size_t nl = std::min(groups.size(), kChunkLanes);
  p.lanes.resize(nl);
  p.region.assign(nl, 0);
  std::vector<size_t> load(nl, 0);
  for (size_t g : order) {
    const size_t l = size_t(std::min_element(load.begin(), load.end()) - load.begin());
    load[l] += work[g];
    for (size_t i : groups[g]) {
      p.lanes[l].push_back(i);
      p.region[l] = std::max(p.region[l], chunk_bytes(c, chunks[i]));
    }
  }
  for (auto &lane : p.lanes) std::sort(lane.begin(), lane.end());
  return p;
}

size_t requests_bytes(const Ctx &c, const std::vector<Chunk> &chunks) {
  size_t need = 0;
  for (size_t r : plan_lanes(c, chunks).region) need += r;
  return need;
}

// Side streams and fork/join events of the request-list path (chunk_mu held).
void ensure_chunk_lanes(Ctx &c) {
  if (c.ev_fork) return;
  DeviceGuard guard(c.device);
  for (auto &s : c.side) CUDA_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  for (auto &e : c.ev_join) CUDA_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  CUDA_CHECK(cudaEventCreateWithFlags(&c.ev_fork, cudaEventDisableTiming));
}
}  // namespace

// =====================================================================================
extern "C" {

const char *ntt_b200_last_error(void) { return g_last_error.c_str(); }
uint64_t ntt_b200_kernel_launches(void) { return g_launches.load(); }

int ntt_b200_butterfly_rate(int device, double *butterflies_per_second) {
  return guarded([&] {
    require(butterflies_per_second != nullptr, "null output");
    DeviceGuard guard(device);
    const u64 q = 1152921504606584833ull;  // a 60-bit NTT prime (mode-2 range)
    const b200::Shoup w[4] = {h_shoup_pair(18043022392882ull % q, q), h_shoup_pair(123456789012345ull, q),
                              h_shoup_pair(q / 3, q), h_shoup_pair(q - 5, q)};
    const unsigned grid = (unsigned)(4 * device_sms(device));
    u64 *sink = nullptr;
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CUDA_CHECK(cudaMalloc(&sink, sizeof(u64)));
    auto cleanup = [&] {
      if (e0) cudaEventDestroy(e0);
      if (e1) cudaEventDestroy(e1);
      if (st) cudaStreamDestroy(st);
      cudaFree(sink);
    };
    try {
      CUDA_CHECK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
      CUDA_CHECK(cudaEventCreate(&e0));
      CUDA_CHECK(cudaEventCreate(&e1));
      auto timed_run = [&](int rounds) {
        CUDA_CHECK(cudaEventRecord(e0, st));
        b200::butterfly_rate_kernel<<<grid, b200::kNttThreads, 0, st>>>(sink, q, w[0], w[1], w[2], w[3], rounds);
        CUDA_CHECK(cudaGetLastError());
        CUDA_CHECK(cudaEventRecord(e1, st));
        CUDA_CHECK(cudaEventSynchronize(e1));
        float ms = 0;
        CUDA_CHECK(cudaEventElapsedTime(&ms, e0, e1));
        return (double)ms;
      };
      timed_run(16);  // warm-up
      const double probe = timed_run(64);
      const int rounds = (int)std::max(64.0, std::min(1e6, 64.0 * 10.0 / std::max(probe, 1e-3)));
      const double ms = timed_run(rounds);
      *butterflies_per_second = double(grid) * b200::kNttThreads * rounds * 32.0 / (ms * 1e-3);
    } catch (...) {
      cleanup();
      throw;
    }
    cleanup();
  });
}

int ntt_b200_tuning_set(const char *name, int64_t value) {
  return guarded([&] {
    Tunable *t = find_tunable(name);
    require(t != nullptr, "unknown tunable");
    require(value >= t->lo && value <= t->hi, "tunable value out of range");
    t->value.store(value);
  });
}

int ntt_b200_tuning_get(const char *name, int64_t *value) {
  return guarded([&] {
    Tunable *t = find_tunable(name);
    require(t != nullptr && value != nullptr, "unknown tunable");
    *value = t->value.load();
  });
}

const char *ntt_b200_tuning_name(size_t index) {
  return index < sizeof(g_tuning) / sizeof(g_tuning[0]) ? g_tuning[index].name : nullptr;
}

int ntt_b200_timing_enable(int on) {
  return guarded([&] { g_timer.enabled = on != 0; });
}

int ntt_b200_timing_reset(void) {
  return guarded([&] {
    std::lock_guard<std::mutex> lock(g_timer.mu);
    for (auto &r : g_timer.records) {
      g_timer.pool.push_back(r.start);
      g_timer.pool.push_back(r.stop);
    }
    g_timer.records.clear();
  });
}

int ntt_b200_timing_query(const char *kernel, uint64_t *launches, double *total_ms) {
  return guarded([&] {
    require(kernel && launches && total_ms, "null argument");
    std::lock_guard<std::mutex> lock(g_timer.mu);
    uint64_t count = 0;
    double ms = 0;
    for (auto &r : g_timer.records) {
      if (std::strcmp(r.name, kernel) != 0) continue;
      CUDA_CHECK(cudaEventSynchronize(r.stop));
      float e = 0;
      CUDA_CHECK(cudaEventElapsedTime(&e, r.start, r.stop));
      ms += e;
      ++count;
    }
    *launches = count;
    *total_ms = ms;
  });
}

int ntt_b200_context_create(ntt_b200_context *out, int device, uint64_t n, const uint64_t *q,
                            const uint64_t *q_psi, size_t m, const uint64_t *p,
                            const uint64_t *p_psi, size_t k, size_t alpha) {
  return guarded([&] {
    require(out != nullptr, "null output handle");
    *out = nullptr;
    require(n >= 2 && (n & (n - 1)) == 0 && n <= 65536, "ring dimension must be a power of two in [2, 65536]");
    require(m >= 1 && q && q_psi, "missing Q towers");
    require(alpha >= 1 && alpha <= m, "invalid Q/digit geometry");
    require(k == 0 || (p && p_psi), "missing P towers");
    require(m + k <= (size_t)b200::kMaxTowers, "at most 128 towers per context");
    require(device >= 0, "invalid device ordinal");
    auto c = std::make_unique<Ctx>();
    c->device = device;
    c->n = n;
    while ((u64(1) << c->logn) < n) ++c->logn;
    c->m = m;
    c->k = k;
    c->alpha = alpha;
    for (size_t i = 0; i < m + k; ++i) {
      const u64 mq = i < m ? q[i] : p[i - m];
      const u64 ps = i < m ? q_psi[i] : p_psi[i - m];
      require(mq > n && mq < (u64(1) << 63) && mq % (2 * n) == 1, "invalid modulus shape");
      require(h_is_prime(mq), "composite modulus");
      require(ps > 0 && ps < mq && h_pow(ps, n, mq) == mq - 1, "invalid primitive root");
      require(std::find(c->mod.begin(), c->mod.end(), mq) == c->mod.end(), "duplicate Q/P modulus");
      c->mod.push_back(mq);
      c->psi.push_back(ps);
      if (mq >= (u64(1) << 61)) c->mode = std::min(c->mode, 1);
      if (mq >= (u64(1) << 62)) c->mode = 0;
    }
    const size_t T = m + k;
    std::vector<b200::TowerConsts> tc(T);
    std::vector<ulonglong2> fwd(T * n), inv(T * n);
    std::vector<u64> pw(n);
    for (size_t g = 0; g < T; ++g) {
      const u64 mq = c->mod[g];
      const u64 root = c->psi[g], root_inv = h_inv(root, mq);
      for (int pass = 0; pass < 2; ++pass) {
        const u64 r = pass ? root_inv : root;
        u64 acc = 1;
        for (u64 e = 0; e < n; ++e) {
          pw[e] = acc;
          acc = h_mul(acc, r, mq);
        }
        ulonglong2 *dst = (pass ? inv.data() : fwd.data()) + g * n;
        for (u64 e = 0; e < n; ++e) {
          const u64 w = pw[e];
          const uint32_t idx = h_bitrev((uint32_t)e, c->logn);
          dst[idx] = make_ulonglong2(w, h_shoup(w, mq));
        }
        if (c->logn >= b200::kLaneMajorMinLogn) lane_major_rows(dst, c->logn);
      }
      const u64 ninv = h_inv(n % mq, mq);
      tc[g].q = mq;
      tc[g].q2 = 2 * mq;
      tc[g].ninv = h_shoup_pair(ninv, mq);
      tc[g].last_inv = h_shoup_pair(h_mul(inv[g * n + 1].x, ninv, mq), mq);
      tc[g].red = h_reducer(mq);
    }
    DeviceGuard guard(device);
    // Every device allocation and upload of the setup is one operation; an
    // injected failure (ntt_b200_inject_setup_failure) throws before the
    // chosen one, and the partly built context unwinds through its destructor
    // (the reference's SetupResources, include/ntt/setup_resources.hpp:19-60).
    const size_t fail_at = g_setup_fail_at.exchange(0);
    size_t ops = 0;
    auto step = [&] {
      if (++ops == fail_at) throw CudaError("CUDA: injected failure before setup operation " + std::to_string(ops));
    };
    step();
    CUDA_CHECK(cudaMalloc(&c->d_tc, T * sizeof(b200::TowerConsts)));
    step();
    CUDA_CHECK(cudaMalloc(&c->d_err, sizeof(int)));
    step();
    CUDA_CHECK(cudaMemset(c->d_err, 0, sizeof(int)));
    step();
    CUDA_CHECK(cudaMalloc(&c->d_fwd, T * n * sizeof(ulonglong2)));
    step();
    CUDA_CHECK(cudaMalloc(&c->d_inv, T * n * sizeof(ulonglong2)));
    step();
    CUDA_CHECK(cudaMemcpy(c->d_tc, tc.data(), T * sizeof(b200::TowerConsts), cudaMemcpyHostToDevice));
    step();
    CUDA_CHECK(cudaMemcpy(c->d_fwd, fwd.data(), T * n * sizeof(ulonglong2), cudaMemcpyHostToDevice));
    step();
    CUDA_CHECK(cudaMemcpy(c->d_inv, inv.data(), T * n * sizeof(ulonglong2), cudaMemcpyHostToDevice));
    g_setup_operations = ops;
    c->tables = b200::DeviceTables{c->d_tc, c->d_fwd, c->d_inv, c->logn};
    CUDA_CHECK(b200::row_mac_prepare(device));
    c->table_bytes = T * sizeof(b200::TowerConsts) + 2 * T * n * sizeof(ulonglong2);
    *out = c.release();
  });
}

int ntt_b200_context_destroy(ntt_b200_context ctx) {
  return guarded([&] {
    if (!ctx) return;
    DeviceGuard guard(ctx->device);
    delete ctx;
  });
}

int ntt_b200_context_table_bytes(ntt_b200_context ctx, size_t *out) {
  return guarded([&] {
    require_ctx(ctx);
    require(out != nullptr, "null output");
    *out = ctx->table_bytes;
  });
}

int ntt_b200_device_errors(ntt_b200_context ctx, int *count, int clear) {
  return guarded([&] {
    require_ctx(ctx);
    require(count != nullptr, "null output");
    DeviceGuard guard(ctx->device);
    CUDA_CHECK(cudaMemcpy(count, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (clear) CUDA_CHECK(cudaMemset(ctx->d_err, 0, sizeof(int)));
  });
}

int ntt_b200_context_key_words(ntt_b200_context ctx, size_t *words) {
  return guarded([&] {
    require_ctx(ctx);
    require(words != nullptr, "null output");
    *words = (1 + (ctx->m - 1) / ctx->alpha) * ctx->towers() * ctx->n;
  });
}

int ntt_b200_context_prepare(ntt_b200_context ctx, size_t level) {
  return guarded([&] {
    require_ctx(ctx);
    require_level(ctx, level);
    Ctx &c = *ctx;
    const size_t L = level, K = c.k;
    c.conv_plan(range_ids(0, L), range_ids(c.m, c.m + K));
    // Both forms of the ModDown and digit plans: scaled (exact inverse NTT)
    // and with N^-1 folded in (unscaled inverse NTT), whichever the tuning picks.
    for (const bool ninv : {false, true}) c.conv_plan(range_ids(c.m, c.m + K), range_ids(0, L), ninv);
    c.down_plan(L);
    const auto all = qp_ids(c, L);
    for (size_t first = 0; first < L; first += c.alpha) {
      const size_t count = std::min(c.alpha, L - first);
      std::vector<uint16_t> tgt;
      for (size_t t = 0; t < L + K; ++t)
        if (t < first || t >= first + count) tgt.push_back(all[t]);
      for (const bool ninv : {false, true}) c.conv_plan(range_ids(first, first + count), tgt, ninv);
    }
    std::lock_guard<std::mutex> lock(c.chunk_mu);
    ensure_chunk_lanes(c);
  });
}

int ntt_b200_ntt(ntt_b200_context ctx, uint64_t *dst, const uint64_t *src, const uint32_t *tower_ids,
                 size_t towers, size_t polys, size_t poly_stride, int inverse, void *stream) {
  return guarded([&] {
    require_ctx(ctx);
    require(dst && src && tower_ids, "null pointer");
    require_aligned({dst, src});
    require(poly_stride % 2 == 0, "polynomial stride must be even");
    require(towers >= 1 && polys >= 1, "empty transform batch");
    require(polys == 1 || poly_stride >= towers * ctx->n, "overlapping polynomial stride");
    std::vector<Slot> slots;
    for (size_t i = 0; i < towers; ++i) {
      require(tower_ids[i] < ctx->towers(), "tower id out of range");
      slots.push_back({(uint32_t)i, (uint16_t)tower_ids[i]});
    }
    DeviceGuard guard(ctx->device);
    run_ntt(*ctx, dst, src, slots, polys, poly_stride, poly_stride, inverse != 0, as_stream(stream));
  });
}

int ntt_b200_pointwise(ntt_b200_context ctx, uint64_t *dst, const uint64_t *left,
                       const uint64_t *right, const uint32_t *tower_ids, size_t towers,
                       size_t polys, size_t poly_stride, void *stream) {
  return guarded([&] {
    require_ctx(ctx);
    require(dst && left && right && tower_ids, "null pointer");
    require_aligned({dst, left, right});
    require(poly_stride % 2 == 0, "polynomial stride must be even");
    require(towers >= 1 && towers <= (size_t)b200::kMaxTowers && polys >= 1 && polys <= 65535,
            "pointwise batch out of range");
    require(polys == 1 || poly_stride >= towers * ctx->n, "overlapping polynomial stride");
    b200::PointwiseArgs a{};
    a.dst = dst;
    a.left = left;
    a.right = right;
    a.tc = ctx->d_tc;
    a.poly_stride = poly_stride;
    for (size_t i = 0; i < towers; ++i) {
      require(tower_ids[i] < ctx->towers(), "tower id out of range");
      a.id[i] = (uint16_t)tower_ids[i];
    }
    a.towers = (int)towers;
    a.logn = ctx->logn;
    DeviceGuard guard(ctx->device);
    const cudaStream_t st = as_stream(stream);
    Timed t("pointwise", st);
    b200::pointwise_kernel<<<ew_grid(*ctx, towers, polys), b200::kEwThreads, 0, st>>>(a);
    t.done();
  });
}

int ntt_b200_switch_basis(ntt_b200_context ctx, uint64_t *dst, const uint64_t *src,
                          const uint32_t *source_ids, size_t s, const uint32_t *target_ids,
                          size_t t, void *stream) {
  return guarded([&] {
    require_ctx(ctx);
    require(dst && src && source_ids && target_ids, "null pointer");
    require_aligned({dst, src});
    require(s >= 1 && s <= 40 && t >= 1 && t <= 40, "basis switch requires 1..40 source and target towers");
    std::vector<uint16_t> sv, tv, slots;
    for (size_t i = 0; i < s; ++i) {
      require(source_ids[i] < ctx->towers(), "tower id out of range");
      sv.push_back((uint16_t)source_ids[i]);
    }
    for (size_t i = 0; i < t; ++i) {
      require(target_ids[i] < ctx->towers(), "tower id out of range");
      tv.push_back((uint16_t)target_ids[i]);
      slots.push_back((uint16_t)i);
    }
    DeviceGuard guard(ctx->device);
    const auto &plan = ctx->conv_plan(sv, tv);
    run_conv(*ctx, plan, dst, src, slots, 1, 0, 0, as_stream(stream));
  });
}

int ntt_b200_correct(ntt_b200_context ctx, size_t level, uint64_t *dst, const uint64_t *left,
                     const uint64_t *right, void *stream) {
  return guarded([&] {
    require_ctx(ctx);
    require_level(ctx, level);
    require(dst && left && right, "null pointer");
    require_aligned({dst, left, right});
    DeviceGuard guard(ctx->device);
    b200::CorrectArgs a{};
    a.dst = dst;
    a.left = left;
    a.right = right;
    a.pinv = ctx->down_plan(level)->p_inv;
    a.tc = ctx->d_tc;
    a.towers = (int)level;
    a.logn = ctx->logn;
    const cudaStream_t st = as_stream(stream);
    Timed t("correct", st);
    b200::correct_kernel<<<ew_grid(*ctx, level, 1), b200::kEwThreads, 0, st>>>(a);
    t.done();
  });
}

int ntt_b200_hybrid_mac(ntt_b200_context ctx, size_t level, uint64_t *out_b, uint64_t *out_a,
                        const uint64_t *digits, const uint64_t *key_b, const uint64_t *key_a,
                        void *stream) {
  return guarded([&] {
    require_ctx(ctx);
    require_level(ctx, level);
    require(out_b && out_a && digits && key_b && key_a, "null pointer");
    require_aligned({out_b, out_a, digits, key_b, key_a});
    DeviceGuard guard(ctx->device);
    const size_t beta = 1 + (level - 1) / ctx->alpha, T = level + ctx->k;
    std::vector<const u64 *> dptr;
    for (size_t d = 0; d < beta; ++d) dptr.push_back(digits + d * T * ctx->n);
    do_mac(*ctx, level, 1, out_b, out_a, 0, dptr, 0, nullptr, key_digits(*ctx, key_b, beta),
           key_digits(*ctx, key_a, beta), true, false, as_stream(stream));
  });
}

int ntt_b200_hybrid_rotate(ntt_b200_context ctx, size_t level, uint64_t *out_b, uint64_t *out_a,
                           const uint64_t *ext_b, const uint64_t *ext_a, const uint64_t *c0,
                           uint32_t automorphism, void *stream) {
  return guarded([&] {
    require_ctx(ctx);
    require_level(ctx, level);
    require(out_b && out_a && ext_b && ext_a && c0, "null pointer");
    require_aligned({out_b, out_a, ext_b, ext_a, c0});
    DeviceGuard guard(ctx->device);
    do_rotate(*ctx, level, 1, out_b, out_a, ext_b, ext_a, 0, c0, 0, automorphism, as_stream(stream));
  });
}

int ntt_b200_workspace_bytes(ntt_b200_context ctx, int op, size_t level, size_t batch, size_t *out) {
  return guarded([&] {
    require_ctx(ctx);
    require_level(ctx, level);
    require(out != nullptr && batch >= 1 && batch <= 65535 / 2, "invalid workspace query");
    *out = workspace_bytes(*ctx, op, level, batch);
  });
}

int ntt_b200_mod_up(ntt_b200_context ctx, size_t level, uint64_t *dst, const uint64_t *src,
                    int src_is_eval, void *workspace, size_t workspace_bytes, void *stream) {
  return guarded([&] {
    require_ctx(ctx);
    require_level(ctx, level);
    require(dst && src, "null pointer");
    require_aligned({dst, src, workspace});
    Ctx &c = *ctx;
    Carver ws = carve(c, workspace, workspace_bytes, NTT_B200_OP_MOD_UP, level, 1);
    DeviceGuard guard(c.device);
    const cudaStream_t st = as_stream(stream);
    const size_t n = c.n, L = level, K = c.k;
    const u64 *coeff = src;
    if (src_is_eval) {
      u64 *tmp = ws.take(L * n);
      run_ntt(c, tmp, src, contiguous_slots(range_ids(0, L)), 1, 0, 0, true, st);
      CUDA_CHECK(cudaMemcpyAsync(dst, src, L * n * sizeof(u64), cudaMemcpyDeviceToDevice, st));
      coeff = tmp;
    } else {
      run_ntt(c, dst, src, contiguous_slots(range_ids(0, L)), 1, 0, 0, false, st);
    }
    const auto &plan = c.conv_plan(range_ids(0, L), range_ids(c.m, c.m + K));
    std::vector<uint16_t> slots;
    for (size_t i = 0; i < K; ++i) slots.push_back((uint16_t)(L + i));
    run_conv(c, plan, dst, coeff, slots, 1, 0, 0, st, true);
    run_ntt(c, dst, dst, contiguous_slots(range_ids(c.m, c.m + K), (uint32_t)L), 1, 0, 0, false, st);
  });
}

int ntt_b200_mod_down(ntt_b200_context ctx, size_t level, uint64_t *dst, const uint64_t *src,
                      void *workspace, size_t workspace_bytes, void *stream) {
  return guarded([&] {
    require_ctx(ctx);
    require_level(ctx, level);
    require(dst && src, "null pointer");
    require_aligned({dst, src, workspace});
    Carver ws = carve(*ctx, workspace, workspace_bytes, NTT_B200_OP_MOD_DOWN, level, 1);
    DeviceGuard guard(ctx->device);
    do_mod_down(*ctx, level, 1, dst, nullptr, 0, src, 0, ws, as_stream(stream));
  });
}

int ntt_b200_hybrid_digits(ntt_b200_context ctx, size_t level, uint64_t *digits, const uint64_t *src,
                           void *workspace, size_t workspace_bytes, void *stream) {
  return guarded([&] {
    require_ctx(ctx);
    require_level(ctx, level);
    require(digits && src, "null pointer");
    require_aligned({digits, src, workspace});
    Carver ws = carve(*ctx, workspace, workspace_bytes, NTT_B200_OP_DIGITS, level, 1);
    DeviceGuard guard(ctx->device);
    do_digits(*ctx, level, 1, digits, src, ws, true, as_stream(stream));
  });
}

int ntt_b200_keyswitch(ntt_b200_context ctx, size_t level, uint64_t *out_b, uint64_t *out_a,
                       const uint64_t *src, const uint64_t *key_b, const uint64_t *key_a,
                       const uint64_t *c0, uint32_t automorphism, void *workspace,
                       size_t workspace_bytes, void *stream) {
  return ntt_b200_keyswitch_batch(ctx, level, 1, out_b, out_a, src, key_b, key_a, c0, automorphism,
                                  workspace, workspace_bytes, stream);
}

int ntt_b200_keyswitch_batch(ntt_b200_context ctx, size_t level, size_t batch, uint64_t *out_b,
                             uint64_t *out_a, const uint64_t *src, const uint64_t *key_b,
                             const uint64_t *key_a, const uint64_t *c0, uint32_t automorphism,
                             void *workspace, size_t workspace_bytes, void *stream) {
  return guarded([&] {
    require_ctx(ctx);
    require_level(ctx, level);
    require(batch >= 1 && batch <= 65535 / 2, "key-switch batch out of range");
    require(out_b && out_a && src && key_b && key_a, "null pointer");
    require_aligned({out_b, out_a, src, key_b, key_a, c0, workspace});
    Ctx &c = *ctx;
    if (c0) require((automorphism & 1) && automorphism < 2 * c.n, "invalid negacyclic automorphism index");
    Carver ws = carve(c, workspace, workspace_bytes, NTT_B200_OP_KEYSWITCH, level, batch);
    DeviceGuard guard(c.device);
    do_keyswitch(c, level, batch, out_b, out_a, src, key_b, key_a, c0, automorphism, ws, as_stream(stream));
  });
}

int ntt_b200_keyswitch_requests_workspace(ntt_b200_context ctx, const ntt_b200_ks_request *reqs,
                                          size_t count, size_t *bytes) {
  return guarded([&] {
    require_ctx(ctx);
    require(bytes != nullptr, "null output");
    validate_requests(*ctx, reqs, count);
    *bytes = requests_bytes(*ctx, plan_chunks(reqs, count));
  });
}

int ntt_b200_keyswitch_requests(ntt_b200_context ctx, const ntt_b200_ks_request *reqs, size_t count,
                                void *workspace, size_t workspace_bytes, void *stream) {
  return guarded([&] {
    require_ctx(ctx);
    Ctx &c = *ctx;
    validate_requests(c, reqs, count);
    require_aligned({workspace});
    const auto chunks = plan_chunks(reqs, count);
    const size_t need = requests_bytes(c, chunks);
    if (!workspace || workspace_bytes < need) throw WorkspaceError("workspace missing or too small");
    DeviceGuard guard(c.device);
    for (const Chunk &ch : chunks) {
      c.conv_plan(range_ids(c.m, c.m + c.k), range_ids(0, ch.level), intt_unscaled(c));
      c.down_plan(ch.level);
    }
    const cudaStream_t st = as_stream(stream);
    const LanePlan plan = plan_lanes(c, chunks);
    char *const base = reinterpret_cast<char *>(workspace);
    if (plan.lanes.size() == 1) {
      for (size_t i : plan.lanes[0]) {
        // Chunks run in stream order, so each reuses the same workspace.
        Carver ws{base, plan.region[0]};
        run_chunk(c, reqs, chunks[i], ws, st);
      }
      return;
    }
    std::lock_guard<std::mutex> lock(c.chunk_mu);
    ensure_chunk_lanes(c);
    CUDA_CHECK(cudaEventRecord(c.ev_fork, st));
    // Every forked stream is joined back into the caller's stream, also when an
    // enqueue fails part way, so no side-stream work outlives the call's stream.
    struct Join {
      Ctx &c;
      cudaStream_t st;
      size_t forked = 0;
      ~Join() {
        for (size_t l = 0; l < forked; ++l) {
          cudaEventRecord(c.ev_join[l], c.side[l]);
          cudaStreamWaitEvent(st, c.ev_join[l], 0);
        }
      }
    } join{c, st};
    size_t off = 0;
    for (size_t l = 0; l < plan.lanes.size(); ++l) {
      const cudaStream_t ls = l == 0 ? st : c.side[l - 1];
      if (l > 0) {
        CUDA_CHECK(cudaStreamWaitEvent(ls, c.ev_fork, 0));
        join.forked = l;
      }
      for (size_t i : plan.lanes[l]) {
        Carver ws{base + off, plan.region[l]};
        run_chunk(c, reqs, chunks[i], ws, ls);
      }
      off += plan.region[l];
    }
  });
}

// ---- host-buffer key switch with overlapped copies ------------------------------------
namespace {
// Copy streams and slot events of the host-buffer pipelines (pipe_mu held).
void ensure_copy_pipeline(Ctx &c) {
  if (c.copy_in) return;
  DeviceGuard guard(c.device);
  CUDA_CHECK(cudaStreamCreateWithFlags(&c.copy_in, cudaStreamNonBlocking));
  CUDA_CHECK(cudaStreamCreateWithFlags(&c.copy_out, cudaStreamNonBlocking));
  for (int i = 0; i < 2; ++i) {
    CUDA_CHECK(cudaEventCreateWithFlags(&c.ev_in[i], cudaEventDisableTiming));
    CUDA_CHECK(cudaEventCreateWithFlags(&c.ev_comp[i], cudaEventDisableTiming));
    CUDA_CHECK(cudaEventCreateWithFlags(&c.ev_out[i], cudaEventDisableTiming));
  }
  CUDA_CHECK(cudaEventCreateWithFlags(&c.ev_start, cudaEventDisableTiming));
}
}  // namespace

size_t host_slot_words(const Ctx &c, size_t level, size_t chunk, bool rotate) {
  return chunk * level * c.n * (rotate ? 4 : 3);  // src (+ c0) in, out_b + out_a
}

int ntt_b200_keyswitch_host_workspace(ntt_b200_context ctx, size_t level, size_t chunk, int rotate,
                                      size_t *bytes) {
  return guarded([&] {
    require_ctx(ctx);
    require_level(ctx, level);
    require(bytes != nullptr && chunk >= 1 && chunk <= 65535 / 2, "invalid host pipeline query");
    *bytes = 2 * aligned_bytes(host_slot_words(*ctx, level, chunk, rotate != 0)) +
             workspace_bytes(*ctx, NTT_B200_OP_KEYSWITCH, level, chunk);
  });
}

namespace {
// The host-buffer pipeline; `join` makes the caller's stream wait for the
// outputs' copies at the end (ntt_b200_keyswitch_host), else the caller joins
// later (ntt_b200_keyswitch_host_async + ntt_b200_keyswitch_host_wait).
int keyswitch_host(ntt_b200_context ctx, size_t level, size_t batch, size_t chunk, const uint64_t *h_src,
                   uint64_t *h_out_b, uint64_t *h_out_a, const uint64_t *key_b, const uint64_t *key_a,
                   const uint64_t *h_c0, uint32_t automorphism, void *workspace, size_t ws_size, void *stream,
                   bool join) {
  return guarded([&] {
    require_ctx(ctx);
    require_level(ctx, level);
    Ctx &c = *ctx;
    require(batch >= 1 && chunk >= 1 && chunk <= 65535 / 2, "invalid batch or chunk");
    require(h_src && h_out_b && h_out_a && key_b && key_a, "null pointer");
    require_aligned({key_b, key_a, workspace});
    const bool rotate = h_c0 != nullptr;
    if (rotate) require((automorphism & 1) && automorphism < 2 * c.n, "invalid negacyclic automorphism index");
    const size_t slot_words = host_slot_words(c, level, chunk, rotate);
    const size_t need = 2 * aligned_bytes(slot_words) + workspace_bytes(c, NTT_B200_OP_KEYSWITCH, level, chunk);
    if (!workspace || ws_size < need) throw WorkspaceError("workspace missing or too small");
    DeviceGuard guard(c.device);
    c.conv_plan(range_ids(c.m, c.m + c.k), range_ids(0, level), intt_unscaled(c));
    c.down_plan(level);
    std::lock_guard<std::mutex> lock(c.pipe_mu);
    ensure_copy_pipeline(c);
    const cudaStream_t st = as_stream(stream);
    char *base = reinterpret_cast<char *>(workspace);
    u64 *slot[2] = {reinterpret_cast<u64 *>(base), reinterpret_cast<u64 *>(base + aligned_bytes(slot_words))};
    char *ks_ws = base + 2 * aligned_bytes(slot_words);
    const size_t ks_bytes = ws_size - 2 * aligned_bytes(slot_words);
    const size_t poly = level * c.n;  // words per request and component
    // The copy streams start after everything already on the caller's stream.
    CUDA_CHECK(cudaEventRecord(c.ev_start, st));
    CUDA_CHECK(cudaStreamWaitEvent(c.copy_in, c.ev_start, 0));
    CUDA_CHECK(cudaStreamWaitEvent(c.copy_out, c.ev_start, 0));
    for (size_t first = 0, k = 0; first < batch; first += chunk, ++k) {
      const size_t r = std::min(chunk, batch - first);
      const int sl = (int)(k & 1);
      u64 *d_src = slot[sl], *d_b = d_src + chunk * poly, *d_a = d_b + chunk * poly;
      u64 *d_c0 = rotate ? d_a + chunk * poly : nullptr;
      // host -> device, once the compute two chunks back has read this slot
      CUDA_CHECK(cudaStreamWaitEvent(c.copy_in, c.ev_comp[sl], 0));
      CUDA_CHECK(cudaMemcpyAsync(d_src, h_src + first * poly, r * poly * sizeof(u64), cudaMemcpyHostToDevice,
                                 c.copy_in));
      if (rotate)
        CUDA_CHECK(cudaMemcpyAsync(d_c0, h_c0 + first * poly, r * poly * sizeof(u64), cudaMemcpyHostToDevice,
                                   c.copy_in));
      CUDA_CHECK(cudaEventRecord(c.ev_in[sl], c.copy_in));
      // compute on the caller's stream, once the inputs are in and the outputs
      // of two chunks back have left for the host
      CUDA_CHECK(cudaStreamWaitEvent(st, c.ev_in[sl], 0));
      CUDA_CHECK(cudaStreamWaitEvent(st, c.ev_out[sl], 0));
      Carver ws{ks_ws, ks_bytes};
      do_keyswitch(c, level, r, d_b, d_a, d_src, key_b, key_a, d_c0, automorphism, ws, st);
      CUDA_CHECK(cudaEventRecord(c.ev_comp[sl], st));
      // device -> host
      CUDA_CHECK(cudaStreamWaitEvent(c.copy_out, c.ev_comp[sl], 0));
      CUDA_CHECK(cudaMemcpyAsync(h_out_b + first * poly, d_b, r * poly * sizeof(u64), cudaMemcpyDeviceToHost,
                                 c.copy_out));
      CUDA_CHECK(cudaMemcpyAsync(h_out_a + first * poly, d_a, r * poly * sizeof(u64), cudaMemcpyDeviceToHost,
                                 c.copy_out));
      CUDA_CHECK(cudaEventRecord(c.ev_out[sl], c.copy_out));
    }
    // The caller's stream continues once every output has reached the host.
    if (join) {
      CUDA_CHECK(cudaStreamWaitEvent(st, c.ev_out[0], 0));
      CUDA_CHECK(cudaStreamWaitEvent(st, c.ev_out[1], 0));
    }
  });
}
}  // namespace

int ntt_b200_keyswitch_host(ntt_b200_context ctx, size_t level, size_t batch, size_t chunk, const uint64_t *h_src,
                            uint64_t *h_out_b, uint64_t *h_out_a, const uint64_t *key_b, const uint64_t *key_a,
                            const uint64_t *h_c0, uint32_t automorphism, void *workspace, size_t ws_size,
                            void *stream) {
  return keyswitch_host(ctx, level, batch, chunk, h_src, h_out_b, h_out_a, key_b, key_a, h_c0, automorphism,
                        workspace, ws_size, stream, true);
}

int ntt_b200_keyswitch_host_async(ntt_b200_context ctx, size_t level, size_t batch, size_t chunk,
                                  const uint64_t *h_src, uint64_t *h_out_b, uint64_t *h_out_a,
                                  const uint64_t *key_b, const uint64_t *key_a, const uint64_t *h_c0,
                                  uint32_t automorphism, void *workspace, size_t ws_size, void *stream) {
  return keyswitch_host(ctx, level, batch, chunk, h_src, h_out_b, h_out_a, key_b, key_a, h_c0, automorphism,
                        workspace, ws_size, stream, false);
}

int ntt_b200_keyswitch_host_wait(ntt_b200_context ctx, void *stream) {
  return guarded([&] {
    require_ctx(ctx);
    Ctx &c = *ctx;
    DeviceGuard guard(c.device);
    std::lock_guard<std::mutex> lock(c.pipe_mu);
    if (!c.copy_in) return;  // no host-buffer call has run on this context
    // The copies to the host run in order on one stream, so its latest two
    // records (one per staging slot) cover every earlier one.
    const cudaStream_t st = as_stream(stream);
    CUDA_CHECK(cudaStreamWaitEvent(st, c.ev_out[0], 0));
    CUDA_CHECK(cudaStreamWaitEvent(st, c.ev_out[1], 0));
  });
}

int ntt_b200_hybrid_mac_digits(ntt_b200_context ctx, size_t level, uint64_t *out_b, uint64_t *out_a,
                               const uint64_t *const *digits, const uint64_t *const *key_b,
                               const uint64_t *const *key_a, size_t count, int full_key_rows, int accumulate,
                               void *stream) {
  return guarded([&] {
    require_ctx(ctx);
    require_level(ctx, level);
    require(out_b && out_a && digits && key_b && key_a, "null pointer");
    require(count >= 1 && count <= (size_t)b200::kMaxDigits, "MAC digit count out of range");
    std::vector<const u64 *> d, kb, ka;
    for (size_t i = 0; i < count; ++i) {
      require(digits[i] && key_b[i] && key_a[i], "null digit or key pointer");
      require_aligned({digits[i], key_b[i], key_a[i]});
      d.push_back(digits[i]);
      kb.push_back(key_b[i]);
      ka.push_back(key_a[i]);
    }
    require_aligned({out_b, out_a});
    DeviceGuard guard(ctx->device);
    do_mac(*ctx, level, 1, out_b, out_a, 0, d, 0, nullptr, kb, ka, full_key_rows != 0, accumulate != 0,
           as_stream(stream));
  });
}

// ---- transport -----------------------------------------------------------------------
int ntt_b200_stream_create(int device, void **stream) {
  return guarded([&] {
    require(stream != nullptr && device >= 0, "invalid stream request");
    DeviceGuard guard(device);
    cudaMemPool_t pool;
    CUDA_CHECK(cudaDeviceGetDefaultMemPool(&pool, device));
    uint64_t keep = UINT64_MAX;  // keep freed blocks cached in the pool
    CUDA_CHECK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    cudaStream_t s = nullptr;
    CUDA_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    *stream = s;
  });
}

int ntt_b200_stream_destroy(void *stream) {
  return guarded([&] {
    if (stream) CUDA_CHECK(cudaStreamDestroy(as_stream(stream)));
  });
}

int ntt_b200_stream_synchronize(void *stream) {
  return guarded([&] { CUDA_CHECK(cudaStreamSynchronize(as_stream(stream))); });
}

int ntt_b200_alloc(int device, size_t bytes, void *stream, void **ptr) {
  return guarded([&] {
    require(ptr != nullptr && device >= 0, "invalid allocation request");
    *ptr = nullptr;
    DeviceGuard guard(device);
    CUDA_CHECK(cudaMallocAsync(ptr, std::max<size_t>(bytes, 256), as_stream(stream)));
  });
}

int ntt_b200_free(void *ptr, void *stream) {
  return guarded([&] {
    if (ptr) CUDA_CHECK(cudaFreeAsync(ptr, as_stream(stream)));
  });
}

int ntt_b200_memcpy(void *dst, const void *src, size_t bytes, int kind, void *stream) {
  return guarded([&] {
    require(dst && src, "null pointer");
    require(kind >= 1 && kind <= 3, "copy kind must be 1 (to device), 2 (to host) or 3 (device to device)");
    const cudaMemcpyKind k = kind == 1 ? cudaMemcpyHostToDevice
                             : kind == 2 ? cudaMemcpyDeviceToHost
                                         : cudaMemcpyDeviceToDevice;
    if (bytes) CUDA_CHECK(cudaMemcpyAsync(dst, src, bytes, k, as_stream(stream)));
  });
}

int ntt_b200_event_create(int device, void **event) {
  return guarded([&] {
    require(event != nullptr && device >= 0, "invalid event request");
    DeviceGuard guard(device);
    cudaEvent_t e = nullptr;
    CUDA_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    *event = e;
  });
}

int ntt_b200_event_destroy(void *event) {
  return guarded([&] {
    if (event) CUDA_CHECK(cudaEventDestroy(reinterpret_cast<cudaEvent_t>(event)));
  });
}

int ntt_b200_event_record(void *event, void *stream) {
  return guarded([&] {
    require(event != nullptr, "null event");
    CUDA_CHECK(cudaEventRecord(reinterpret_cast<cudaEvent_t>(event), as_stream(stream)));
  });
}

int ntt_b200_event_query(void *event) {
  if (!event) {
    g_last_error = "null event";
    return NTT_B200_ERR_CONTRACT;
  }
  const cudaError_t e = cudaEventQuery(reinterpret_cast<cudaEvent_t>(event));
  if (e == cudaSuccess) return NTT_B200_OK;
  if (e == cudaErrorNotReady) {
    (void)cudaGetLastError();
    return NTT_B200_NOT_READY;
  }
  g_last_error = std::string("CUDA: cudaEventQuery: ") + cudaGetErrorString(e);
  return NTT_B200_ERR_CUDA;
}

int ntt_b200_event_synchronize(void *event) {
  return guarded([&] {
    require(event != nullptr, "null event");
    CUDA_CHECK(cudaEventSynchronize(reinterpret_cast<cudaEvent_t>(event)));
  });
}

}  // extern "C"

// ---- allocation-free ModDown ------------------------------------------------------------
// Scratch of ntt_b200_mod_down_static: a file-scope device array every GPU that
// loads this library holds until process exit. Host code never uses the
// symbol's host-side name as a device address: the address comes from
// cudaGetSymbolAddress, once per device, with that device current.
constexpr size_t kStaticScratchWords = size_t(1) << 20;  // 8 MiB
static __device__ __align__(256) uint64_t g_static_scratch[kStaticScratchWords];

namespace {
std::mutex g_static_mu;
uint64_t *g_static_ptr[64] = {nullptr};

uint64_t *static_scratch(int device) {
  require(device >= 0 && device < 64, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_static_mu);
  if (!g_static_ptr[device]) {
    DeviceGuard guard(device);
    void *ptr = nullptr;
    CUDA_CHECK(cudaGetSymbolAddress(&ptr, g_static_scratch));
    g_static_ptr[device] = static_cast<uint64_t *>(ptr);
  }
  return g_static_ptr[device];
}
}  // namespace

extern "C" {
size_t ntt_b200_mod_down_static_max_bytes(void) { return kStaticScratchWords * sizeof(uint64_t); }

int ntt_b200_mod_down_static(ntt_b200_context ctx, size_t level, uint64_t *dst, const uint64_t *src,
                             void *stream) {
  return guarded([&] {
    require_ctx(ctx);
    require_level(ctx, level);
    require(dst && src, "null pointer");
    require_aligned({dst, src});
    Ctx &c = *ctx;
    const size_t need = workspace_bytes(c, NTT_B200_OP_MOD_DOWN, level, 1);
    if (need > kStaticScratchWords * sizeof(uint64_t))
      throw ContractError("ModDown scratch exceeds the 8 MiB static maximum of ntt_b200_mod_down_static "
                          "(needs (K + L) * N * 8 bytes); use ntt_b200_mod_down with a workspace");
    require(c.find_conv_plan(range_ids(c.m, c.m + c.k), range_ids(0, level), intt_unscaled(c)) &&
                c.find_down_plan(level),
            "ntt_b200_mod_down_static needs the level's tables: call ntt_b200_context_prepare(level) first");
    uint64_t *scratch = static_scratch(c.device);
    DeviceGuard guard(c.device);
    Carver ws{reinterpret_cast<char *>(scratch), kStaticScratchWords * sizeof(uint64_t)};
    do_mod_down(c, level, 1, dst, nullptr, 0, src, 0, ws, as_stream(stream));
  });
}
}  // extern "C"

// ---- host-buffer transforms (the reference's CudaNttTransform public calls) ---------------
namespace {
// Towers the host-array transforms check and copy per step (tunable
// host_chunk_towers): a checked chunk is copied while the next is checked.
size_t host_chunk_towers() { return (size_t)tuned("host_chunk_towers"); }

// Device words of a host-array transform's workspace: every tower of the
// context, once per operand.
size_t host_transform_words(const Ctx &c, int op) {
  return (op >= NTT_B200_HOST_POINTWISE ? 2 : 1) * c.towers() * c.n;
}

// Whether towers [first, first + count) of a host array (its tower i at
// v + i * N) are canonical residues of their moduli (the reference's
// validate_values). With q < 2^63, x < q exactly when neither x nor
// (q - 1 - x) mod 2^64 has its top bit set, so one OR over the towers decides
// it without a branch per word.
bool host_values_canonical(const Ctx &c, const u64 *v, const std::vector<uint16_t> &ids, size_t first,
                           size_t count) {
  const size_t n = c.n;
  u64 flags = 0;
  for (size_t t = first; t < first + count; ++t) {
    const u64 qm1 = c.mod[ids[t]] - 1;
    const u64 *p = v + t * n;
    for (size_t i = 0; i < n; ++i) flags |= (qm1 - p[i]) | p[i];
  }
  return (flags >> 63) == 0;
}

void launch_pointwise(const Ctx &c, u64 *dst, const u64 *left, const u64 *right, const std::vector<Slot> &slots,
                      cudaStream_t st) {
  b200::PointwiseArgs a{};
  a.dst = dst;
  a.left = left;
  a.right = right;
  a.tc = c.d_tc;
  a.poly_stride = 0;
  for (size_t i = 0; i < slots.size(); ++i) a.id[i] = slots[i].id;
  a.towers = (int)slots.size();
  a.logn = c.logn;
  Timed t("pointwise", st);
  b200::pointwise_kernel<<<ew_grid(c, slots.size(), 1), b200::kEwThreads, 0, st>>>(a);
  t.done();
}
}  // namespace

extern "C" {
int ntt_b200_host_transform_workspace(ntt_b200_context ctx, int op, size_t *bytes) {
  return guarded([&] {
    require_ctx(ctx);
    require(bytes != nullptr && op >= NTT_B200_HOST_FORWARD && op <= NTT_B200_HOST_MULTIPLY,
            "invalid host transform query");
    *bytes = aligned_bytes(host_transform_words(*ctx, op));
  });
}

int ntt_b200_host_transform(ntt_b200_context ctx, int op, uint64_t *values, const uint64_t *right,
                            const uint32_t *tower_ids, size_t towers, void *workspace, size_t ws_size,
                            void *stream) {
  return guarded([&] {
    require_ctx(ctx);
    Ctx &c = *ctx;
    require(op >= NTT_B200_HOST_FORWARD && op <= NTT_B200_HOST_MULTIPLY, "unknown host transform");
    require(values && tower_ids, "null pointer");
    const bool two = op >= NTT_B200_HOST_POINTWISE;
    require(!two || right, "the product needs a right operand");
    require(towers >= 1 && towers <= (size_t)b200::kMaxTowers, "host transform tower count out of range");
    std::vector<uint16_t> ids(towers);
    for (size_t i = 0; i < towers; ++i) {
      require(tower_ids[i] < c.towers(), "tower id out of range");
      ids[i] = (uint16_t)tower_ids[i];
    }
    require_aligned({workspace});
    // Every tower of this call, once per operand (tower ids may repeat, so this
    // can exceed the size the workspace query reports for the context).
    if (!workspace || ws_size < aligned_bytes((two ? 2 : 1) * towers * c.n))
      throw WorkspaceError("workspace missing or too small");
    DeviceGuard guard(c.device);
    std::lock_guard<std::mutex> lock(c.pipe_mu);
    ensure_copy_pipeline(c);
    const cudaStream_t st = as_stream(stream);
    const size_t n = c.n;
    u64 *d_l = reinterpret_cast<u64 *>(workspace), *d_r = d_l + towers * n;
    // The copies start after the work already on the caller's stream. Each
    // chunk is checked on this thread and then copied while the next one is
    // checked; nothing is computed or written back before every residue passed.
    CUDA_CHECK(cudaEventRecord(c.ev_start, st));
    CUDA_CHECK(cudaStreamWaitEvent(c.copy_in, c.ev_start, 0));
    const size_t chunk = host_chunk_towers();
    bool ok = true;
    for (size_t first = 0; first < towers && ok; first += chunk) {
      const size_t r = std::min(chunk, towers - first);
      ok = host_values_canonical(c, values, ids, first, r) && (!two || host_values_canonical(c, right, ids, first, r));
      if (!ok) break;
      CUDA_CHECK(cudaMemcpyAsync(d_l + first * n, values + first * n, r * n * sizeof(u64), cudaMemcpyHostToDevice,
                                 c.copy_in));
      if (two)
        CUDA_CHECK(cudaMemcpyAsync(d_r + first * n, right + first * n, r * n * sizeof(u64),
                                   cudaMemcpyHostToDevice, c.copy_in));
    }
    if (!ok) {
      // The copies already started read the caller's arrays: finish them
      // before returning, so the caller may release the arrays at once.
      CUDA_CHECK(cudaStreamSynchronize(c.copy_in));
      throw ContractError("host values must be canonical residues of their towers");
    }
    CUDA_CHECK(cudaEventRecord(c.ev_in[0], c.copy_in));
    CUDA_CHECK(cudaStreamWaitEvent(st, c.ev_in[0], 0));
    std::vector<Slot> slots;
    for (size_t i = 0; i < towers; ++i) slots.push_back({(uint32_t)i, ids[i]});
    const u64 stride = towers * n;
    switch (op) {
      case NTT_B200_HOST_FORWARD: run_ntt(c, d_l, d_l, slots, 1, stride, stride, false, st); break;
      case NTT_B200_HOST_INVERSE: run_ntt(c, d_l, d_l, slots, 1, stride, stride, true, st); break;
      case NTT_B200_HOST_POINTWISE: launch_pointwise(c, d_l, d_l, d_r, slots, st); break;
      default:  // the ring product: forward both, pointwise, inverse
        run_ntt(c, d_l, d_l, slots, 1, stride, stride, false, st);
        run_ntt(c, d_r, d_r, slots, 1, stride, stride, false, st);
        launch_pointwise(c, d_l, d_l, d_r, slots, st);
        run_ntt(c, d_l, d_l, slots, 1, stride, stride, true, st);
        break;
    }
    CUDA_CHECK(cudaMemcpyAsync(values, d_l, towers * n * sizeof(u64), cudaMemcpyDeviceToHost, st));
    CUDA_CHECK(cudaStreamSynchronize(st));  // synchronous, as the reference's public calls are
  });
}

// ---- device arithmetic probes and test hooks -----------------------------------------------
int ntt_b200_arith_probe(int device, int op, const uint64_t *queries, size_t count, uint64_t *out, void *stream) {
  return guarded([&] {
    require(op >= 0 && op <= 2, "unknown arithmetic probe");
    require(queries && out && device >= 0, "null pointer");
    require(count >= 1 && count <= (size_t(1) << 30), "probe count out of range");
    DeviceGuard guard(device);
    const cudaStream_t st = as_stream(stream);
    Timed t("probe", st);
    b200::arith_probe_kernel<<<(unsigned)((count + b200::kEwThreads - 1) / b200::kEwThreads), b200::kEwThreads, 0,
                               st>>>(op, queries, count, out);
    t.done();
  });
}

int ntt_b200_conv_wait_polls(int polls) {
  return guarded([&] {
    require(polls >= 0 && polls <= (1 << 20), "poll limit out of range");
    g_conv_first_wait = polls;
  });
}

int ntt_b200_inject_setup_failure(size_t operation) {
  g_setup_fail_at = operation;
  return NTT_B200_OK;
}

int ntt_b200_setup_operations(size_t *count) {
  return guarded([&] {
    require(count != nullptr, "null output");
    *count = g_setup_operations.load();
  });
}
}  // extern "C"
