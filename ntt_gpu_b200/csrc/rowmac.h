// Host-side launcher of the fused digit row pass + key multiplication
// (ntt_fwd_row_mac, rowmac.cuh), compiled in its own translation unit
// (rowmac.cu) so that its instantiations build in parallel with capi.cu.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace b200 {
struct RowMacArgs;
struct DeviceTables;

constexpr int kRowMacMaxBeta = 4;

// Dynamic shared memory of the fused kernel for `beta` digits (bytes).
int row_mac_smem(int beta);
// Raises the dynamic shared-memory limit of every instantiation on `device`
// (once per device), so that launches - also inside a stream capture - make no
// attribute calls. Returns the first CUDA error.
cudaError_t row_mac_prepare(int device);
// Grid: (N / 256 / rows per CTA, inputs, towers). logn in 12..16, beta 1..4.
cudaError_t row_mac_launch(const RowMacArgs &a, const DeviceTables &T, int logn, int beta, bool rotate,
                           unsigned inputs, unsigned towers, cudaStream_t st);
}  // namespace b200
