// C bridge over minnow54426/ntt-gpu's own CPU implementation (test
// infrastructure only). oracle/Makefile compiles this file together with the
// reference's src/resident.cpp, in place under the reference tree, into
// oracle/_ref/libntt_ref.so. Nothing of the reference is copied: this file only
// calls its public classes:
//   - ntt::NegacyclicNtt (include/ntt/ntt.hpp:53-158),
//   - ntt::ApproximateBasisPlan (include/ntt/basis_conversion.hpp:32-114),
//   - ntt::resident::Session over the deferred CPU transport
//     resident_test::HostDriver (tests/support/resident_host_driver.hpp:30-195),
//     composed exactly as run_hybrid_core does
//     (include/ntt/openfhe_hybrid_adapter.hpp:163-181).
#include <cstring>
#include <string>
#include <vector>

#include "ntt/barrett.hpp"
#include "ntt/basis_conversion.hpp"
#include "ntt/ntt.hpp"
#include "ntt/param_gen.hpp"
#include "ntt/resident.hpp"
#include "ntt/shoup.hpp"
#include "support/resident_host_driver.hpp"

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

struct Context {
  ParameterHandle parameters;
  size_t level;
};

Context make_context(uint64_t n, const uint64_t *q, const uint64_t *q_psi, size_t m,
                     const uint64_t *p, const uint64_t *p_psi, size_t k, size_t alpha,
                     size_t level) {
  std::vector<Tower> qs, ps;
  for (size_t i = 0; i < m; ++i) qs.push_back({q[i], q_psi[i]});
  for (size_t i = 0; i < k; ++i) ps.push_back({p[i], p_psi[i]});
  return {Parameters::create(n, qs, ps, alpha), level};
}

PolynomialLayout base_layout(const Context &c) {
  return {c.parameters, c.level, qp_basis(*c.parameters, c.level), Domain::Coefficient,
          Order::Natural};
}

PolynomialLayout q_layout(const Context &c, Domain domain) {
  return {c.parameters, c.level, q_prefix(*c.parameters, c.level), domain,
          domain == Domain::Coefficient ? Order::Natural : Order::BitReversed};
}

ntt::resident::Session make_session(const Context &c) {
  const ntt::resident::Limits limits{size_t{1} << 40, size_t{1} << 40, 1u << 20};
  return ntt::resident::Session(std::make_shared<resident_test::HostDriver>(base_layout(c)),
                                limits);
}

void copy_out(std::span<const uint64_t> values, uint64_t *out) {
  std::memcpy(out, values.data(), values.size_bytes());
}
} // namespace

extern "C" {
const char *ref_last_error() { return last_error.c_str(); }

uint64_t ref_add_mod(uint64_t a, uint64_t b, uint64_t q) { return ntt::add_mod(a, b, q); }
uint64_t ref_sub_mod(uint64_t a, uint64_t b, uint64_t q) { return ntt::sub_mod(a, b, q); }
uint64_t ref_mul_mod(uint64_t a, uint64_t b, uint64_t q) { return ntt::mul_mod(a, b, q); }
uint64_t ref_pow_mod(uint64_t a, uint64_t e, uint64_t q) { return ntt::pow_mod(a, e, q); }
int ref_inv_mod(uint64_t x, uint64_t q, uint64_t *out) {
  return guarded([&] { *out = ntt::inv_mod(x, q); });
}
int ref_shoup(uint64_t x, uint64_t w, uint64_t q, uint64_t *out) {
  return guarded([&] { *out = ntt::shoup_multiply(x, w, ntt::shoup_precompute(w, q), q); });
}
int ref_barrett(uint64_t a, uint64_t b, uint64_t q, uint64_t *out) {
  return guarded([&] { *out = ntt::barrett_multiply(a, b, ntt::barrett_precompute(q)); });
}
int ref_find_primes(uint64_t n, uint64_t count, uint64_t bits, uint64_t *out) {
  return guarded([&] {
    const auto primes = ntt::find_primes(n, count, bits);
    std::copy(primes.begin(), primes.end(), out);
  });
}
uint64_t ref_find_psi(uint64_t q, uint64_t n) { return ntt::find_psi(q, n); }

int ref_ntt(uint64_t *values, uint64_t n, uint64_t q, uint64_t psi, int inverse) {
  return guarded([&] {
    const ntt::NegacyclicNtt plan(n, q, psi);
    std::vector<uint64_t> v(values, values + n);
    if (inverse) plan.inverse(v);
    else plan.forward(v);
    std::copy(v.begin(), v.end(), values);
  });
}

int ref_basis_convert(const uint64_t *input, uint64_t n, const uint64_t *source, size_t s,
                      const uint64_t *target, size_t t, uint64_t *out) {
  return guarded([&] {
    const ntt::ApproximateBasisPlan plan(std::vector<uint64_t>(source, source + s),
                                         std::vector<uint64_t>(target, target + t));
    const auto result = plan.convert(n, std::span<const uint64_t>(input, s * n));
    std::copy(result.begin(), result.end(), out);
  });
}

int ref_mod_up(uint64_t n, const uint64_t *q, const uint64_t *q_psi, size_t m, const uint64_t *p,
               const uint64_t *p_psi, size_t k, size_t alpha, size_t level, const uint64_t *input,
               int input_is_eval, uint64_t *out) {
  return guarded([&] {
    const auto c = make_context(n, q, q_psi, m, p, p_psi, k, alpha, level);
    auto session = make_session(c);
    const auto layout = q_layout(c, input_is_eval ? Domain::Evaluation : Domain::Coefficient);
    const auto x = session.upload(layout, std::span<const uint64_t>(input, level * n));
    const auto download = session.download(session.mod_up(x));
    copy_out(download.wait_values(), out);
    session.close();
  });
}

int ref_mod_down(uint64_t n, const uint64_t *q, const uint64_t *q_psi, size_t m, const uint64_t *p,
                 const uint64_t *p_psi, size_t k, size_t alpha, size_t level,
                 const uint64_t *input, uint64_t *out) {
  return guarded([&] {
    const auto c = make_context(n, q, q_psi, m, p, p_psi, k, alpha, level);
    auto session = make_session(c);
    const PolynomialLayout layout{c.parameters, level, qp_basis(*c.parameters, level),
                                  Domain::Evaluation, Order::BitReversed};
    const auto x = session.upload(layout, std::span<const uint64_t>(input, (level + k) * n));
    const auto download = session.download(session.mod_down(x));
    copy_out(download.wait_values(), out);
    session.close();
  });
}

int ref_hybrid_digits(uint64_t n, const uint64_t *q, const uint64_t *q_psi, size_t m,
                      const uint64_t *p, const uint64_t *p_psi, size_t k, size_t alpha,
                      size_t level, const uint64_t *input, uint64_t *digits) {
  return guarded([&] {
    const auto c = make_context(n, q, q_psi, m, p, p_psi, k, alpha, level);
    auto session = make_session(c);
    const auto x = session.upload(q_layout(c, Domain::Evaluation),
                                  std::span<const uint64_t>(input, level * n));
    const auto result = session.hybrid_digits(x);
    const size_t block = (level + k) * n;
    for (size_t d = 0; d < result.size(); ++d)
      copy_out(session.download(result[d]).wait_values(), digits + d * block);
    session.close();
  });
}

// Full-context keys: digits_full x (M+K) towers per channel. c0 may be null.
int ref_keyswitch(uint64_t n, const uint64_t *q, const uint64_t *q_psi, size_t m,
                  const uint64_t *p, const uint64_t *p_psi, size_t k, size_t alpha, size_t level,
                  const uint64_t *input, const uint64_t *key_b, const uint64_t *key_a,
                  const uint64_t *c0, uint32_t automorphism, uint64_t *out_b, uint64_t *out_a) {
  return guarded([&] {
    const auto c = make_context(n, q, q_psi, m, p, p_psi, k, alpha, level);
    const size_t full_digits = 1 + (m - 1) / alpha;
    const size_t full_block = (m + k) * n;
    const PolynomialLayout full_key_layout{c.parameters, m, qp_basis(*c.parameters, m),
                                           Domain::Evaluation, Order::BitReversed};
    std::vector<ntt::resident::HybridKeyDigit> rows;
    for (size_t d = 0; d < full_digits; ++d)
      rows.push_back({std::span<const uint64_t>(key_b + d * full_block, full_block),
                      std::span<const uint64_t>(key_a + d * full_block, full_block)});
    auto session = make_session(c);
    const auto source = q_layout(c, Domain::Evaluation);
    const auto key = session.upload_hybrid_key(full_key_layout, rows);
    const auto digits =
        session.hybrid_digits(session.upload(source, std::span<const uint64_t>(input, level * n)));
    auto extended = session.hybrid_accumulate(digits, key);
    if (c0)
      extended = session.hybrid_rotate_extended(
          extended, session.upload(source, std::span<const uint64_t>(c0, level * n)), automorphism);
    const auto reduced_b = session.mod_down(extended.b);
    const auto reduced_a = session.mod_down(extended.a);
    const auto download_b = session.download(reduced_b);
    const auto download_a = session.download(reduced_a);
    copy_out(download_a.wait_values(), out_a);
    copy_out(download_b.wait_values(), out_b);
    session.close();
  });
}
} // extern "C"
