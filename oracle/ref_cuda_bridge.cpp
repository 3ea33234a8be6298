// C bridge over minnow54426/ntt-gpu's own CUDA resident path (measurement
// infrastructure only: the reference's GPU key switch, timed as a second GPU
// comparator). oracle/Makefile compiles this file with nvcc together with the
// reference's src/cuda/ntt_kernels.cu (which includes its resident_adapter.inc)
// and src/resident.cpp, in place under the reference tree, into
// oracle/_ref/libntt_ref_cuda.so. Nothing of the reference is copied: this file
// only calls its public API,
//   - ntt::resident::make_cuda_session (include/ntt/resident.hpp:142-143),
//   - ntt::resident::Session upload_hybrid_key / hybrid_digits /
//     hybrid_accumulate / mod_down / download (include/ntt/resident.hpp:93-141),
// composed exactly as run_hybrid_core does
// (include/ntt/openfhe_hybrid_adapter.hpp:163-181).
#include <chrono>
#include <cstring>
#include <memory>
#include <span>
#include <string>
#include <vector>

#include "ntt/resident.hpp"

namespace {
thread_local std::string last_error;

template <class F> int guarded(F f) {
  try {
    f();
    return 0;
  } catch (const std::exception &e) {
    last_error = e.what();
    return -1;
  }
}

using namespace ntt::proposal;
}  // namespace

extern "C" {
const char *refcuda_last_error() { return last_error.c_str(); }

// `warmup` untimed and then `count` timed key switches of one input component
// at `level` through one CUDA session of the reference on `device`, the
// full-context key uploaded once. Each key switch is the reference's public
// path: upload the input, Hybrid digits, MAC, ModDown of both channels,
// download both outputs and wait for them. *ms_per_keyswitch is the wall time
// per timed key switch; the last outputs land in out_b / out_a.
int refcuda_keyswitch(uint64_t n, const uint64_t *q, const uint64_t *q_psi, size_t m, const uint64_t *p,
                      const uint64_t *p_psi, size_t k, size_t alpha, size_t level, const uint64_t *input,
                      const uint64_t *key_b, const uint64_t *key_a, int device, int warmup, int count,
                      double *ms_per_keyswitch, uint64_t *out_b, uint64_t *out_a) {
  return guarded([&] {
    std::vector<Tower> qs, ps;
    for (size_t i = 0; i < m; ++i) qs.push_back({q[i], q_psi[i]});
    for (size_t i = 0; i < k; ++i) ps.push_back({p[i], p_psi[i]});
    const ParameterHandle prm = Parameters::create(n, qs, ps, alpha);
    const PolynomialLayout base{prm, level, qp_basis(*prm, level), Domain::Coefficient, Order::Natural};
    const PolynomialLayout source{prm, level, q_prefix(*prm, level), Domain::Evaluation, Order::BitReversed};
    const PolynomialLayout full_key{prm, m, qp_basis(*prm, m), Domain::Evaluation, Order::BitReversed};
    const size_t full_digits = 1 + (m - 1) / alpha, full_block = (m + k) * n;
    std::vector<ntt::resident::HybridKeyDigit> rows;
    for (size_t d = 0; d < full_digits; ++d)
      rows.push_back({std::span<const uint64_t>(key_b + d * full_block, full_block),
                      std::span<const uint64_t>(key_a + d * full_block, full_block)});
    const ntt::resident::Limits limits{size_t{1} << 40, size_t{1} << 40, 1u << 20};
    auto session = ntt::resident::make_cuda_session(base, device, limits);
    const auto key = session.upload_hybrid_key(full_key, rows);
    auto one = [&] {
      const auto digits = session.hybrid_digits(session.upload(source, std::span<const uint64_t>(input, level * n)));
      const auto extended = session.hybrid_accumulate(digits, key);
      const auto reduced_b = session.mod_down(extended.b);
      const auto reduced_a = session.mod_down(extended.a);
      const auto download_b = session.download(reduced_b);
      const auto download_a = session.download(reduced_a);
      const auto vb = download_b.wait_values();
      const auto va = download_a.wait_values();
      std::memcpy(out_b, vb.data(), vb.size_bytes());
      std::memcpy(out_a, va.data(), va.size_bytes());
    };
    for (int i = 0; i < warmup; ++i) one();
    const auto t0 = std::chrono::steady_clock::now();
    for (int i = 0; i < count; ++i) one();
    const auto t1 = std::chrono::steady_clock::now();
    *ms_per_keyswitch = std::chrono::duration<double, std::milli>(t1 - t0).count() / (count > 0 ? count : 1);
    session.close();
  });
}
}  // extern "C"
