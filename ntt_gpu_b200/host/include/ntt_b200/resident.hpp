#pragma once
// Resident CKKS session: immutable polynomial handles on one ordered device
// stream, with budgets, an operation journal and poison-on-failure. The public
// surface is the reference's resident API (minnow54426/ntt-gpu
// include/ntt/resident.hpp:20-143) so existing callers - the OpenFHE Hybrid
// adapters among them - switch to the B200 path by linking this library and
// calling make_cuda_session. Every method validates before it enqueues.
#include <exception>
#include <memory>
#include <span>
#include <vector>

#include "ntt_b200/contract.hpp"

namespace ntt::resident {
using proposal::CompletionRecord;
using proposal::Device;
using proposal::Outcome;
using proposal::PolynomialLayout;
using proposal::View;
namespace detail {
struct State;
struct Allocation;
struct Operation;
struct HostStorage;
class Driver;
}  // namespace detail

struct Limits {
  size_t device_bytes = 256 * 1024 * 1024;
  size_t host_bytes = 128 * 1024 * 1024;
  size_t operations = 1024;
};
struct Stats {
  size_t submitted, pending, device_bytes, host_bytes;
  size_t uploads, downloads, device_copies;
  size_t parameter_uploads;
  bool closed, poisoned, quiescent;
};

class Completion {
  std::shared_ptr<detail::State> state_;
  std::shared_ptr<detail::Operation> operation_;
  Completion(std::shared_ptr<detail::State>, std::shared_ptr<detail::Operation>);
  friend class Session;
  friend class Polynomial;
  friend class Download;
  friend struct detail::State;

 public:
  Completion() = default;
  CompletionRecord query() const;
  void wait() const;
};

class Polynomial {
  std::shared_ptr<detail::State> state_;
  std::shared_ptr<detail::Allocation> allocation_;
  std::shared_ptr<detail::Operation> producer_;
  PolynomialLayout layout_{};
  View view_{};
  Polynomial(std::shared_ptr<detail::State>, std::shared_ptr<detail::Allocation>,
             std::shared_ptr<detail::Operation>, PolynomialLayout, View);
  friend class Session;
  friend struct detail::State;

 public:
  Polynomial() = default;
  const PolynomialLayout &layout() const;
  View view() const;
  Completion readiness() const;
};

class Download {
  std::shared_ptr<detail::State> state_;
  std::shared_ptr<detail::Operation> operation_;
  std::shared_ptr<detail::HostStorage> storage_;
  PolynomialLayout layout_{};
  mutable bool validated_ = false;
  Download(std::shared_ptr<detail::State>, std::shared_ptr<detail::Operation>,
           std::shared_ptr<detail::HostStorage>, PolynomialLayout);
  friend class Session;

 public:
  Download() = default;
  Completion completion() const;
  // Host values become visible only after completion and canonical validation.
  std::span<const uint64_t> wait_values() const;
};

struct HybridKeyDigit {
  std::span<const uint64_t> b, a;
};
class HybridKey {
  std::vector<Polynomial> b_, a_;
  friend class Session;
};
struct HybridContributions {
  Polynomial b, a;
};

class Session {
  std::shared_ptr<detail::State> state_;
  detail::State &open_state();
  Polynomial upload_checked(const PolynomialLayout &, std::span<const uint64_t>, std::span<const Completion>);
  Polynomial transform(const Polynomial &, bool inverse, std::span<const Completion>);
  Polynomial join(std::span<const Polynomial>);
  Polynomial correct(const Polynomial &, const Polynomial &);

 public:
  // The driver is the transport seam: make_cuda_session installs the B200
  // driver; tests may inject a CPU transport. There is no automatic fallback.
  explicit Session(std::shared_ptr<detail::Driver>, Limits = {});
  ~Session() noexcept;
  Session(const Session &) = delete;
  Session &operator=(const Session &) = delete;
  Session(Session &&) noexcept = default;
  Session &operator=(Session &&) = delete;
  Device device() const;
  Stats stats() const;
  std::vector<CompletionRecord> history() const;
  Polynomial upload(std::span<const uint64_t>, std::span<const Completion> waits = {});
  Polynomial upload(const PolynomialLayout &, std::span<const uint64_t>, std::span<const Completion> waits = {});
  Polynomial upload_evaluation(std::span<const uint64_t>, std::span<const Completion> waits = {});
  Polynomial forward(const Polynomial &, std::span<const Completion> waits = {});
  Polynomial inverse(const Polynomial &, std::span<const Completion> waits = {});
  Polynomial pointwise(const Polynomial &, const Polynomial &, std::span<const Completion> waits = {});
  // Coefficient-domain unreduced approximate CRT between disjoint bases.
  Polynomial switch_basis(const Polynomial &, const PolynomialLayout &target, std::span<const Completion> waits = {});
  // The session basis must be active Q followed by P (CKKS, reduced noise off).
  // ModUp: coefficient or evaluation Q -> evaluation QP. ModDown: evaluation QP -> evaluation Q.
  Polynomial mod_up(const Polynomial &, std::span<const Completion> waits = {});
  Polynomial mod_down(const Polynomial &, std::span<const Completion> waits = {});
  // Hybrid digits of a complete evaluation Q input, each an evaluation QP polynomial.
  std::vector<Polynomial> hybrid_digits(const Polynomial &, std::span<const Completion> waits = {});
  // Snapshot the active rows of a full-context evaluation QP key.
  HybridKey upload_hybrid_key(const PolynomialLayout &full_key_layout, std::span<const HybridKeyDigit>);
  // Accumulate both channels in evaluation QP (before ModDown).
  HybridContributions hybrid_accumulate(std::span<const Polynomial> digits, const HybridKey &,
                                        std::span<const Completion> waits = {});
  // Add P*c0 on the Q towers, then apply the automorphism to both channels.
  HybridContributions hybrid_rotate_extended(const HybridContributions &, const Polynomial &c0, uint32_t automorphism);
  Polynomial subview(const Polynomial &, size_t first_tower, size_t count, size_t active_q);
  Download download(const Polynomial &, std::span<const Completion> waits = {});
  Download multiply(std::span<const uint64_t>, std::span<const uint64_t>);
  // Stops admission and drains; rethrows the first failure.
  void close();
};

// The B200 session: one non-blocking stream on `device`, tables resident in HBM,
// buffers from a stream-ordered pool.
Session make_cuda_session(const PolynomialLayout &coefficient_layout, int device = 0, Limits = {});
}  // namespace ntt::resident
