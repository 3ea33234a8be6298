// C bridge over minnow54426/ntt-gpu's own resident Session (test
// infrastructure). oracle/Makefile (target refb200) compiles this file with
// the reference's UNCHANGED src/resident.cpp, in place under the reference
// tree, and with this repository's Driver binding
// (ntt_gpu_b200/binding/resident_b200.cpp), linked against libntt_b200.so,
// into oracle/_ref/libntt_ref_b200.so. The GPU tests then drive the
// reference's Session - its journal, pins, budgets and composites - over the
// B200 transport exactly as a user of the reference would after the drop-in,
// and compare every output with the oracle.
//
// Only the reference's public API is called (include/ntt/resident.hpp:85-143):
// make_cuda_session, Session::upload / mod_up / mod_down / hybrid_digits /
// upload_hybrid_key / hybrid_accumulate / hybrid_rotate_extended / multiply /
// download / stats / close, composed as run_hybrid_core does
// (include/ntt/openfhe_hybrid_adapter.hpp:163-181).
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
using ntt::resident::Session;
}  // namespace

extern "C" {
// One CKKS context: M Q towers, K P towers, digit width alpha, and the device.
struct refsess_ctx {
  uint64_t n;
  const uint64_t *q, *q_psi;
  size_t m;
  const uint64_t *p, *p_psi;
  size_t k, alpha;
  int device;
};
}

namespace {
struct Env {
  ParameterHandle prm;
  size_t level, n;
  PolynomialLayout base, q_coeff, q_eval, qp_eval, full_key;
};

Env env(const refsess_ctx &c, size_t level) {
  std::vector<Tower> qs, ps;
  for (size_t i = 0; i < c.m; ++i) qs.push_back({c.q[i], c.q_psi[i]});
  for (size_t i = 0; i < c.k; ++i) ps.push_back({c.p[i], c.p_psi[i]});
  ParameterHandle prm = Parameters::create(c.n, qs, ps, c.alpha);
  Env e{prm,
        level,
        c.n,
        {prm, level, qp_basis(*prm, level), Domain::Coefficient, Order::Natural},
        {prm, level, q_prefix(*prm, level), Domain::Coefficient, Order::Natural},
        {prm, level, q_prefix(*prm, level), Domain::Evaluation, Order::BitReversed},
        {prm, level, qp_basis(*prm, level), Domain::Evaluation, Order::BitReversed},
        {prm, c.m, qp_basis(*prm, c.m), Domain::Evaluation, Order::BitReversed}};
  return e;
}

Session open(const Env &e, int device) {
  const ntt::resident::Limits limits{size_t{1} << 40, size_t{1} << 40, 1u << 20};
  return ntt::resident::make_cuda_session(e.base, device, limits);
}

void fetch(Session &s, const ntt::resident::Polynomial &p, uint64_t *out) {
  const auto d = s.download(p);
  const auto v = d.wait_values();
  std::memcpy(out, v.data(), v.size_bytes());
}
}  // namespace

extern "C" {
const char *refsess_last_error() { return last_error.c_str(); }

// ModUp of a Q_level polynomial (coefficient if is_eval == 0, else evaluation)
// into evaluation QP: out is (level + K) x N.
int refsess_mod_up(const refsess_ctx *c, size_t level, const uint64_t *in, int is_eval, uint64_t *out) {
  return guarded([&] {
    const Env e = env(*c, level);
    Session s = open(e, c->device);
    const auto x = s.upload(is_eval ? e.q_eval : e.q_coeff, std::span<const uint64_t>(in, level * e.n));
    fetch(s, s.mod_up(x), out);
    s.close();
  });
}

// ModDown of an evaluation-QP polynomial into evaluation Q_level.
int refsess_mod_down(const refsess_ctx *c, size_t level, const uint64_t *in, uint64_t *out) {
  return guarded([&] {
    const Env e = env(*c, level);
    Session s = open(e, c->device);
    const auto x = s.upload(e.qp_eval, std::span<const uint64_t>(in, (level + c->k) * e.n));
    fetch(s, s.mod_down(x), out);
    s.close();
  });
}

// Hybrid digits of an evaluation-Q_level polynomial: out is beta x (level + K) x N.
int refsess_digits(const refsess_ctx *c, size_t level, const uint64_t *in, uint64_t *out) {
  return guarded([&] {
    const Env e = env(*c, level);
    Session s = open(e, c->device);
    const auto x = s.upload(e.q_eval, std::span<const uint64_t>(in, level * e.n));
    const auto digits = s.hybrid_digits(x);
    const size_t block = (level + c->k) * e.n;
    for (size_t d = 0; d < digits.size(); ++d) fetch(s, digits[d], out + d * block);
    s.close();
  });
}

// Hybrid key switch (and, with c0 set, rotation by `automorphism`) of an
// evaluation-Q_level component with a full-context key (digits x (M+K) x N per
// channel): upload_hybrid_key, hybrid_digits, hybrid_accumulate,
// [hybrid_rotate_extended], mod_down of both channels. *operations receives the
// Session's executed-operation count.
int refsess_keyswitch(const refsess_ctx *c, size_t level, const uint64_t *in, const uint64_t *key_b,
                      const uint64_t *key_a, const uint64_t *c0, uint32_t automorphism, uint64_t *out_b,
                      uint64_t *out_a, uint64_t *operations) {
  return guarded([&] {
    const Env e = env(*c, level);
    Session s = open(e, c->device);
    const size_t full_digits = 1 + (c->m - 1) / c->alpha, block = (c->m + c->k) * e.n;
    std::vector<ntt::resident::HybridKeyDigit> rows;
    for (size_t d = 0; d < full_digits; ++d)
      rows.push_back({std::span<const uint64_t>(key_b + d * block, block),
                      std::span<const uint64_t>(key_a + d * block, block)});
    const auto key = s.upload_hybrid_key(e.full_key, rows);
    const auto x = s.upload(e.q_eval, std::span<const uint64_t>(in, level * e.n));
    auto extended = s.hybrid_accumulate(s.hybrid_digits(x), key);
    if (c0) {
      const auto c0p = s.upload(e.q_eval, std::span<const uint64_t>(c0, level * e.n));
      extended = s.hybrid_rotate_extended(extended, c0p, automorphism);
    }
    fetch(s, s.mod_down(extended.b), out_b);
    fetch(s, s.mod_down(extended.a), out_a);
    if (operations) *operations = s.stats().submitted;
    s.close();
  });
}

// Ring product over the session's coefficient QP_level basis (forward, forward,
// pointwise, inverse): left, right, out are (level + K) x N.
int refsess_multiply(const refsess_ctx *c, size_t level, const uint64_t *left, const uint64_t *right,
                     uint64_t *out) {
  return guarded([&] {
    const Env e = env(*c, level);
    Session s = open(e, c->device);
    const size_t words = (level + c->k) * e.n;
    const auto d = s.multiply(std::span<const uint64_t>(left, words), std::span<const uint64_t>(right, words));
    const auto v = d.wait_values();
    std::memcpy(out, v.data(), v.size_bytes());
    s.close();
  });
}

// Opens a session on `device` and closes it again: an invalid ordinal must
// come back as the transport's error, with nothing enqueued.
int refsess_open(const refsess_ctx *c, size_t level, int device) {
  return guarded([&] {
    const Env e = env(*c, level);
    Session s = open(e, device);
    s.close();
  });
}
}  // extern "C"
