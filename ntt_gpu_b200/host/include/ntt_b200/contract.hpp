#pragma once
// Host-side metadata contract of the resident CKKS path: parameter snapshots,
// tower layouts, views and completion records. Same names, meanings and
// validation rules as the reference's proposal contract
// (minnow54426/ntt-gpu include/ntt/backend_contract.hpp:19-311), because the
// Session API and its callers are written against them. Pure host code: no CUDA.
#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <limits>
#include <memory>
#include <span>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace ntt {
namespace arith {
using u128 = unsigned __int128;
inline uint64_t mul_mod(uint64_t a, uint64_t b, uint64_t q) { return uint64_t((u128)a * b % q); }
inline uint64_t pow_mod(uint64_t a, uint64_t e, uint64_t q) {
  uint64_t r = 1 % q, base = a % q;
  for (; e; e >>= 1) {
    if (e & 1) r = mul_mod(r, base, q);
    base = mul_mod(base, base, q);
  }
  return r;
}
inline bool is_prime(uint64_t n) {
  static constexpr uint64_t bases[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
  if (n < 2) return false;
  for (uint64_t p : bases)
    if (n % p == 0) return n == p;
  uint64_t d = n - 1, s = 0;
  while (!(d & 1)) d >>= 1, ++s;
  for (uint64_t a : bases) {
    uint64_t x = pow_mod(a, d, n);
    if (x == 1 || x == n - 1) continue;
    bool witness = true;
    for (uint64_t r = 1; r < s && witness; ++r) {
      x = mul_mod(x, x, n);
      witness = x != n - 1;
    }
    if (witness) return false;
  }
  return true;
}
}  // namespace arith

namespace proposal {
// Invalid arguments; thrown before any device work is enqueued.
struct ContractError : std::invalid_argument {
  using std::invalid_argument::invalid_argument;
};
inline void require(bool ok, const char *why) {
  if (!ok) throw ContractError(why);
}
inline size_t checked_product(size_t a, size_t b) {
  require(a == 0 || b <= std::numeric_limits<size_t>::max() / a, "size overflow");
  return a * b;
}

struct Tower {
  uint64_t q, psi;
  bool operator==(const Tower &) const = default;
};
enum class Family { Q, P };
struct TowerRef {
  Family family;
  size_t index;
  bool operator==(const TowerRef &) const = default;
};

// Immutable deep snapshot of a CKKS context: N, Q towers, P towers and the
// full-context digit width alpha.
class Parameters final {
  uint64_t n_;
  std::vector<Tower> q_, p_;
  size_t alpha_;
  Parameters(uint64_t n, std::vector<Tower> q, std::vector<Tower> p, size_t alpha)
      : n_(n), q_(std::move(q)), p_(std::move(p)), alpha_(alpha) {
    require(n >= 2 && (n & (n - 1)) == 0 && n <= std::numeric_limits<uint32_t>::max() / 2,
            "invalid ring dimension");
    require(!q_.empty() && alpha_ > 0 && alpha_ <= q_.size(), "invalid Q/digit geometry");
    std::vector<uint64_t> seen;
    for (const auto *basis : {&q_, &p_})
      for (const Tower &t : *basis) {
        require(t.q > n && t.q < (uint64_t{1} << 63) && t.q % (2 * n) == 1, "invalid modulus shape");
        require(arith::is_prime(t.q), "composite modulus");
        require(t.psi > 0 && t.psi < t.q && arith::pow_mod(t.psi, n, t.q) == t.q - 1,
                "invalid primitive root");
        require(std::find(seen.begin(), seen.end(), t.q) == seen.end(), "duplicate Q/P modulus");
        seen.push_back(t.q);
      }
  }

 public:
  Parameters &operator=(const Parameters &) = delete;
  static std::shared_ptr<const Parameters> create(uint64_t n, std::vector<Tower> q, std::vector<Tower> p,
                                                  size_t alpha) {
    return std::shared_ptr<const Parameters>(new Parameters(n, std::move(q), std::move(p), alpha));
  }
  uint64_t n() const { return n_; }
  const std::vector<Tower> &q() const { return q_; }
  const std::vector<Tower> &p() const { return p_; }
  size_t alpha() const { return alpha_; }
  bool operator==(const Parameters &o) const {
    return n_ == o.n_ && q_ == o.q_ && p_ == o.p_ && alpha_ == o.alpha_;
  }
  const Tower &tower(TowerRef ref) const {
    require(ref.family == Family::Q || ref.family == Family::P, "invalid basis family");
    const auto &basis = ref.family == Family::Q ? q_ : p_;
    require(ref.index < basis.size(), "tower index out of range");
    return basis[ref.index];
  }
};
using ParameterHandle = std::shared_ptr<const Parameters>;

inline std::vector<TowerRef> q_prefix(const Parameters &p, size_t level) {
  require(level > 0 && level <= p.q().size(), "invalid active Q count");
  std::vector<TowerRef> out(level);
  for (size_t i = 0; i < level; ++i) out[i] = {Family::Q, i};
  return out;
}
inline std::vector<TowerRef> qp_basis(const Parameters &p, size_t level) {
  auto out = q_prefix(p, level);
  require(!p.p().empty(), "QP requires P towers");
  for (size_t j = 0; j < p.p().size(); ++j) out.push_back({Family::P, j});
  return out;
}
// Row of each active QP tower inside a full-context QP key: Q tower i keeps
// row i, P tower j is row M + j.
inline std::vector<size_t> key_indices(const Parameters &p, size_t level) {
  const auto active = qp_basis(p, level);
  std::vector<size_t> out;
  for (const TowerRef &ref : active) out.push_back(ref.family == Family::Q ? ref.index : p.q().size() + ref.index);
  return out;
}

enum class Domain { Coefficient, Evaluation };
enum class Order { Natural, BitReversed };
enum class Encoding { CanonicalU64, MontgomeryU64, LazyU64 };
struct PolynomialLayout {
  ParameterHandle parameters;
  size_t active_q;
  std::vector<TowerRef> towers;
  Domain domain;
  Order order;
  Encoding encoding = Encoding::CanonicalU64;
};

inline void validate(const PolynomialLayout &p) {
  require(bool(p.parameters), "missing parameters");
  require(p.active_q > 0 && p.active_q <= p.parameters->q().size(), "invalid active Q count");
  require(!p.towers.empty(), "empty basis");
  require(p.encoding == Encoding::CanonicalU64, "unsupported residue encoding");
  require((p.domain == Domain::Coefficient && p.order == Order::Natural) ||
              (p.domain == Domain::Evaluation && p.order == Order::BitReversed),
          "domain/order mismatch");
  for (size_t i = 0; i < p.towers.size(); ++i) {
    const TowerRef ref = p.towers[i];
    p.parameters->tower(ref);
    require(ref.family != Family::Q || ref.index < p.active_q, "inactive Q tower");
    require(std::find(p.towers.begin(), p.towers.begin() + i, ref) == p.towers.begin() + i,
            "duplicate view tower");
  }
  checked_product(checked_product(size_t(p.parameters->n()), p.towers.size()), sizeof(uint64_t));
}
inline size_t bytes(const PolynomialLayout &p) {
  validate(p);
  return checked_product(checked_product(size_t(p.parameters->n()), p.towers.size()), sizeof(uint64_t));
}
inline void validate_host_values(const PolynomialLayout &p, std::span<const uint64_t> values) {
  require(values.size() == bytes(p) / sizeof(uint64_t), "host length mismatch");
  const size_t n = p.parameters->n();
  for (size_t t = 0; t < p.towers.size(); ++t) {
    const uint64_t q = p.parameters->tower(p.towers[t]).q;
    const uint64_t *row = values.data() + t * n;
    require(std::all_of(row, row + n, [q](uint64_t v) { return v < q; }), "noncanonical host residue");
  }
}

struct Device {
  int ordinal;
  uint64_t session;
  bool operator==(const Device &) const = default;
};
struct Token {
  uint64_t id, generation;
  bool operator==(const Token &) const = default;
};
struct Stream {
  Device device;
  Token token;
  bool operator==(const Stream &) const = default;
};
inline void validate(Device d) { require(d.ordinal >= 0 && d.session != 0, "invalid device/session"); }
inline void validate(Token t) { require(t.id != 0 && t.generation != 0, "invalid token"); }
inline void validate(Stream s) {
  validate(s.device);
  validate(s.token);
}

struct AllocationRecord {
  Token token;
  Device device;
  size_t capacity_bytes;
  PolynomialLayout layout;
  bool live = true;
};
// Whole contiguous towers of one allocation.
struct View {
  Token allocation;
  size_t first_tower, tower_count, active_q;
};
inline PolynomialLayout validate_view(const View &v, const AllocationRecord &record, Device expected) {
  validate(record.token);
  validate(record.device);
  validate(expected);
  validate(v.allocation);
  require(record.live && v.allocation == record.token, "stale allocation/generation");
  require(record.device == expected, "device/session mismatch");
  require(record.capacity_bytes >= bytes(record.layout), "allocation too short");
  require(v.active_q > 0 && v.active_q <= record.layout.active_q, "view cannot add active Q towers");
  require(v.tower_count > 0 && v.first_tower <= record.layout.towers.size() &&
              v.tower_count <= record.layout.towers.size() - v.first_tower,
          "view extent out of range");
  PolynomialLayout out = record.layout;
  out.active_q = v.active_q;
  out.towers.assign(record.layout.towers.begin() + v.first_tower,
                    record.layout.towers.begin() + v.first_tower + v.tower_count);
  validate(out);
  return out;
}
inline size_t byte_offset(const View &v, const AllocationRecord &record) {
  validate_view(v, record, record.device);
  return checked_product(checked_product(v.first_tower, size_t(record.layout.parameters->n())), sizeof(uint64_t));
}
inline void require_layout(const PolynomialLayout &actual, const PolynomialLayout &expected) {
  validate(actual);
  validate(expected);
  require(*actual.parameters == *expected.parameters && actual.active_q == expected.active_q &&
              actual.towers == expected.towers && actual.domain == expected.domain &&
              actual.order == expected.order && actual.encoding == expected.encoding,
          "operation layout mismatch");
}
inline PolynomialLayout transform_layout(const PolynomialLayout &input, bool inverse) {
  validate(input);
  require(input.domain == (inverse ? Domain::Evaluation : Domain::Coefficient), "wrong transform input domain");
  PolynomialLayout out = input;
  out.domain = inverse ? Domain::Coefficient : Domain::Evaluation;
  out.order = inverse ? Order::Natural : Order::BitReversed;
  return out;
}
inline PolynomialLayout pointwise_layout(const PolynomialLayout &a, const PolynomialLayout &b) {
  require_layout(a, b);
  require(a.domain == Domain::Evaluation, "pointwise input must be evaluation format");
  return a;
}

enum class Outcome { Pending, Succeeded, Failed };
struct CompletionRecord {
  Token operation;
  Stream stream;
  Outcome outcome;
};
struct Execution {
  Stream stream;
  uint64_t operation_id;
  std::vector<CompletionRecord> waits;
};
// Every dependency is an earlier, non-failed operation of the same device; a
// pending producer on another stream needs an explicit event wait.
inline void validate_dependency(const CompletionRecord &source, const Execution &consumer) {
  validate(consumer.stream);
  validate(source.stream);
  validate(source.operation);
  require(source.stream.device == consumer.stream.device, "cross-device dependency");
  require(consumer.operation_id > source.operation.id, "dependency must already be submitted");
  require(source.outcome == Outcome::Pending || source.outcome == Outcome::Succeeded ||
              source.outcome == Outcome::Failed,
          "invalid completion outcome");
  require(source.outcome != Outcome::Failed, "failed producer");
  for (const CompletionRecord &w : consumer.waits) {
    validate(w.stream);
    validate(w.operation);
    require(w.stream.device == consumer.stream.device && w.operation.id < consumer.operation_id,
            "invalid dependency session/order");
    require(w.outcome == Outcome::Pending || w.outcome == Outcome::Succeeded, "failed/invalid explicit dependency");
  }
  if (source.outcome == Outcome::Succeeded || source.stream == consumer.stream) return;
  const bool waited = std::any_of(consumer.waits.begin(), consumer.waits.end(), [&](const CompletionRecord &w) {
    return w.operation == source.operation && w.stream == source.stream;
  });
  require(waited, "missing cross-stream event wait");
}
}  // namespace proposal
}  // namespace ntt
