// Instantiations and launches of the fused digit row pass + key
// multiplication (rowmac.cuh).
#include "rowmac.h"
#include "rowmac.cuh"

#include <mutex>

namespace b200 {
namespace {
constexpr int kWarps = 8;

template <int LOGN, int BETA, bool ROT>
cudaError_t set_attr() {
  cudaError_t e = cudaFuncSetAttribute(ntt_fwd_row_mac<LOGN, BETA, kWarps, ROT, false>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       row_mac_smem_bytes<kWarps>(BETA - 1));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(ntt_fwd_row_mac<LOGN, BETA, kWarps, ROT, true>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, row_mac_smem_bytes<kWarps>(BETA));
  return e;
}

template <int LOGN>
cudaError_t set_attrs_logn() {
  cudaError_t e = cudaSuccess;
  auto keep = [&](cudaError_t r) {
    if (e == cudaSuccess) e = r;
  };
  keep(set_attr<LOGN, 1, false>());
  keep(set_attr<LOGN, 2, false>());
  keep(set_attr<LOGN, 3, false>());
  keep(set_attr<LOGN, 4, false>());
  keep(set_attr<LOGN, 1, true>());
  keep(set_attr<LOGN, 2, true>());
  keep(set_attr<LOGN, 3, true>());
  keep(set_attr<LOGN, 4, true>());
  return e;
}

// Two launches on one stream: the level's Q towers, then the P towers.
template <int LOGN, int BETA, bool ROT>
void launch_t(const RowMacArgs &a, const DeviceTables &T, unsigned inputs, unsigned towers, cudaStream_t st) {
  const unsigned rows = (1u << LOGN) / 256 / (2 * kWarps);
  const unsigned q_towers = (unsigned)a.mac.level, p_towers = towers - q_towers;
  ntt_fwd_row_mac<LOGN, BETA, kWarps, ROT, false>
      <<<dim3(rows, inputs, q_towers), kWarps * 32, row_mac_smem_bytes<kWarps>(BETA - 1), st>>>(a, T);
  if (p_towers)
    ntt_fwd_row_mac<LOGN, BETA, kWarps, ROT, true>
        <<<dim3(rows, inputs, p_towers), kWarps * 32, row_mac_smem_bytes<kWarps>(BETA), st>>>(a, T);
}

template <int LOGN>
void launch_logn(const RowMacArgs &a, const DeviceTables &T, int beta, bool rot, unsigned inputs, unsigned towers,
                 cudaStream_t st) {
  switch (beta * 2 + (rot ? 1 : 0)) {
    case 2: launch_t<LOGN, 1, false>(a, T, inputs, towers, st); break;
    case 3: launch_t<LOGN, 1, true>(a, T, inputs, towers, st); break;
    case 4: launch_t<LOGN, 2, false>(a, T, inputs, towers, st); break;
    case 5: launch_t<LOGN, 2, true>(a, T, inputs, towers, st); break;
    case 6: launch_t<LOGN, 3, false>(a, T, inputs, towers, st); break;
    case 7: launch_t<LOGN, 3, true>(a, T, inputs, towers, st); break;
    case 8: launch_t<LOGN, 4, false>(a, T, inputs, towers, st); break;
    default: launch_t<LOGN, 4, true>(a, T, inputs, towers, st); break;
  }
}
}  // namespace

int row_mac_smem(int beta) { return row_mac_smem_bytes<kWarps>(beta); }  // the P towers' launch

cudaError_t row_mac_prepare(int device) {
  static std::mutex mu;
  static bool done[64] = {};
  if (device < 0 || device >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(mu);
  if (done[device]) return cudaSuccess;
  cudaError_t e = set_attrs_logn<12>();
  if (e == cudaSuccess) e = set_attrs_logn<13>();
  if (e == cudaSuccess) e = set_attrs_logn<14>();
  if (e == cudaSuccess) e = set_attrs_logn<15>();
  if (e == cudaSuccess) e = set_attrs_logn<16>();
  done[device] = e == cudaSuccess;
  return e;
}

cudaError_t row_mac_launch(const RowMacArgs &a, const DeviceTables &T, int logn, int beta, bool rotate,
                           unsigned inputs, unsigned towers, cudaStream_t st) {
  if (beta < 1 || beta > kRowMacMaxBeta) return cudaErrorInvalidValue;
  switch (logn) {
    case 12: launch_logn<12>(a, T, beta, rotate, inputs, towers, st); break;
    case 13: launch_logn<13>(a, T, beta, rotate, inputs, towers, st); break;
    case 14: launch_logn<14>(a, T, beta, rotate, inputs, towers, st); break;
    case 15: launch_logn<15>(a, T, beta, rotate, inputs, towers, st); break;
    case 16: launch_logn<16>(a, T, beta, rotate, inputs, towers, st); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}
}  // namespace b200
