// The resident Session over the B200 driver (make_cuda_session): every
// composite result equals the C oracle bit for bit. Needs a CUDA device.
#include <iostream>

#include "ntt_b200/resident.hpp"

extern "C" {
#include "../../oracle/oracle.h"
}

using namespace ntt::resident;
using namespace ntt::proposal;

namespace {
size_t checks = 0;
void check(bool ok, const char *why) {
  ++checks;
  if (!ok) throw std::runtime_error(why);
}
template <class F> void rejects(F f, const char *why) {
  ++checks;
  try {
    f();
  } catch (const std::invalid_argument &) {
    return;
  }
  throw std::runtime_error(why);
}
void equal(std::span<const uint64_t> a, const std::vector<uint64_t> &b, const char *why) {
  check(a.size() == b.size() && std::equal(a.begin(), a.end(), b.begin()), why);
}

struct Ctx {
  uint64_t n;
  std::vector<uint64_t> q, qpsi, p, ppsi;
  size_t alpha;
  ParameterHandle params;
  orc_context oracle() const { return {n, q.size(), p.size(), alpha, q.data(), qpsi.data(), p.data(), ppsi.data()}; }
};
Ctx make(uint64_t n, size_t m, size_t k, size_t alpha, int qbits, int pbits) {
  Ctx c{n, std::vector<uint64_t>(m), {}, std::vector<uint64_t>(k), {}, alpha, nullptr};
  orc_find_primes(n, m, qbits, c.q.data());
  orc_find_primes(n, k, pbits, c.p.data());
  std::vector<Tower> qt, pt;
  for (uint64_t v : c.q) c.qpsi.push_back(orc_find_psi(v, n)), qt.push_back({v, c.qpsi.back()});
  for (uint64_t v : c.p) c.ppsi.push_back(orc_find_psi(v, n)), pt.push_back({v, c.ppsi.back()});
  c.params = Parameters::create(n, qt, pt, alpha);
  return c;
}
Ctx pinned() {
  Ctx c{65536,
        {1152921504606584833ULL, 1125899902124033ULL, 1125899911168001ULL, 1125899903827969ULL, 1125899908022273ULL},
        {18043022392882ULL, 15995550378ULL, 21670117260ULL, 938640682ULL, 6511788946ULL},
        {1152921504598720513ULL, 1152921504597016577ULL, 1152921504595968001ULL},
        {800790938143ULL, 17749908910371ULL, 11469071954203ULL},
        3,
        nullptr};
  std::vector<Tower> qt, pt;
  for (size_t i = 0; i < 5; ++i) qt.push_back({c.q[i], c.qpsi[i]});
  for (size_t i = 0; i < 3; ++i) pt.push_back({c.p[i], c.ppsi[i]});
  c.params = Parameters::create(65536, qt, pt, 3);
  return c;
}

void hybrid_core(const Ctx &c, size_t level, uint32_t g) {
  const size_t n = c.n, m = c.q.size(), k = c.p.size(), full_digits = 1 + (m - 1) / c.alpha;
  const PolynomialLayout base{c.params, level, qp_basis(*c.params, level), Domain::Coefficient, Order::Natural};
  const PolynomialLayout src{c.params, level, q_prefix(*c.params, level), Domain::Evaluation, Order::BitReversed};
  const PolynomialLayout key_layout{c.params, m, qp_basis(*c.params, m), Domain::Evaluation, Order::BitReversed};
  std::vector<uint64_t> mods(c.q);
  mods.insert(mods.end(), c.p.begin(), c.p.end());
  const size_t block = (m + k) * n;
  std::vector<uint64_t> kb(full_digits * block), ka(full_digits * block), x(level * n), c0(level * n);
  for (size_t d = 0; d < full_digits; ++d) {
    orc_splitmix_fill(kb.data() + d * block, n, m + k, mods.data(), 11 + 1000 * d);
    orc_splitmix_fill(ka.data() + d * block, n, m + k, mods.data(), 12 + 1000 * d);
  }
  orc_lcg_fill(x.data(), n, level, mods.data(), 0x7251d9);
  orc_lcg_fill(c0.data(), n, level, mods.data(), 0x7251da);
  Session s = make_cuda_session(base, 0, {size_t(8) << 30, size_t(8) << 30, 4096});
  std::vector<HybridKeyDigit> rows;
  for (size_t d = 0; d < full_digits; ++d)
    rows.push_back({std::span<const uint64_t>(kb).subspan(d * block, block),
                    std::span<const uint64_t>(ka).subspan(d * block, block)});
  const auto key = s.upload_hybrid_key(key_layout, rows);
  const auto input = s.upload(src, x);
  const auto digits = s.hybrid_digits(input);
  // digits against the oracle
  const auto oc = c.oracle();
  const size_t beta = digits.size(), tq = level + k;
  std::vector<uint64_t> want_digits(beta * tq * n);
  check(orc_hybrid_digits(&oc, level, x.data(), want_digits.data()) == 0, "oracle digits");
  for (size_t d = 0; d < beta; ++d)
    equal(s.download(digits[d]).wait_values(),
          {want_digits.begin() + d * tq * n, want_digits.begin() + (d + 1) * tq * n}, "B200 digits equal the oracle");
  auto ext = s.hybrid_accumulate(digits, key);
  if (g) ext = s.hybrid_rotate_extended(ext, s.upload(src, c0), g);
  const auto rb = s.mod_down(ext.b), ra = s.mod_down(ext.a);
  const auto db = s.download(rb), da = s.download(ra);
  std::vector<uint64_t> wb(level * n), wa(level * n);
  check(orc_keyswitch(&oc, level, x.data(), kb.data(), ka.data(), g ? c0.data() : nullptr, g, wb.data(), wa.data()) == 0,
        "oracle key switch");
  equal(db.wait_values(), wb, "B200 Session key switch b equals the oracle");
  equal(da.wait_values(), wa, "B200 Session key switch a equals the oracle");
  equal(s.download(input).wait_values(), x, "source stays unchanged");
  // ModUp from coefficient and evaluation input
  std::vector<uint64_t> coeff(x);
  check(orc_ntt_towers(coeff.data(), n, level, c.q.data(), c.qpsi.data(), 1) == 0, "oracle inverse");
  std::vector<uint64_t> want_up(tq * n);
  orc_mod_up(&oc, level, x.data(), 1, want_up.data());
  const PolynomialLayout coeff_layout{c.params, level, q_prefix(*c.params, level), Domain::Coefficient,
                                      Order::Natural};
  equal(s.download(s.mod_up(input)).wait_values(), want_up, "ModUp from evaluation");
  equal(s.download(s.mod_up(s.upload(coeff_layout, coeff))).wait_values(), want_up, "ModUp from coefficients");
  const auto stats = s.stats();
  check(!stats.poisoned && stats.uploads >= 3, "session healthy");
  s.close();
}

void transform_chain_and_contract() {
  const Ctx c = make(4096, 3, 0, 1, 50, 60);
  const PolynomialLayout base{c.params, 3, q_prefix(*c.params, 3), Domain::Coefficient, Order::Natural};
  Session s = make_cuda_session(base);
  std::vector<uint64_t> a(3 * 4096), b(3 * 4096);
  orc_lcg_fill(a.data(), 4096, 3, c.q.data(), 1);
  orc_lcg_fill(b.data(), 4096, 3, c.q.data(), 2);
  const auto r = s.multiply(a, b);
  std::vector<uint64_t> fa(a), fb(b);
  orc_ntt_towers(fa.data(), 4096, 3, c.q.data(), c.qpsi.data(), 0);
  orc_ntt_towers(fb.data(), 4096, 3, c.q.data(), c.qpsi.data(), 0);
  for (size_t i = 0; i < fa.size(); ++i) fa[i] = orc_mul_mod(fa[i], fb[i], c.q[i / 4096]);
  orc_ntt_towers(fa.data(), 4096, 3, c.q.data(), c.qpsi.data(), 1);
  equal(r.wait_values(), fa, "B200 ring product equals the oracle");
  auto bad = a;
  bad[5] = c.q[0];
  rejects([&] { s.upload(bad); }, "noncanonical upload rejected before enqueue");
  check(!s.stats().poisoned, "contract errors do not poison");
  s.close();
}
}  // namespace

int main() {
  try {
    transform_chain_and_contract();
    const Ctx small = make(4096, 6, 3, 2, 50, 60);
    for (size_t level : {6, 5, 3, 1}) hybrid_core(small, level, 5);
    hybrid_core(small, 4, 0);
    const Ctx pin = pinned();
    hybrid_core(pin, 5, 5);
    hybrid_core(pin, 4, 0);
    std::cout << checks << " B200 SESSION CHECKS PASSED\n";
  } catch (const std::exception &e) {
    std::cerr << "FAILED: " << e.what() << '\n';
    return 1;
  }
  return 0;
}
