// Resident Session runtime over the deferred CPU transport: the control-plane
// behaviours the reference's tests/resident_tests.cpp:49-417 pins (journal,
// pins and leases, budgets, failure injection, quarantine, abandonment, views,
// conversions, Hybrid digits and keys, closed/moved admission), restated here
// against this library's Session. No GPU.
#include <array>
#include <functional>
#include <iostream>
#include <type_traits>

#include "host_driver.hpp"

using namespace ntt::resident;
using namespace ntt::proposal;
using host_test::HostDriver;

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
  } catch (const std::exception &) {
    return;
  }
  throw std::runtime_error(why);
}

PolynomialLayout layout(size_t q_count = 2, size_t p_count = 0, uint64_t n = 8) {
  std::vector<uint64_t> primes(q_count + p_count);
  if (orc_find_primes(n, primes.size(), 20, primes.data())) throw std::runtime_error("prime search");
  std::vector<Tower> q, p;
  for (size_t i = 0; i < primes.size(); ++i) (i < q_count ? q : p).push_back({primes[i], orc_find_psi(primes[i], n)});
  auto params = Parameters::create(n, q, p, 1);
  return {params, q_count, p_count ? qp_basis(*params, q_count) : q_prefix(*params, q_count), Domain::Coefficient,
          Order::Natural};
}
std::vector<uint64_t> input(const PolynomialLayout &p, size_t seed) {
  std::vector<uint64_t> out(bytes(p) / sizeof(uint64_t));
  const size_t n = p.parameters->n();
  for (size_t t = 0; t < p.towers.size(); ++t)
    for (size_t i = 0; i < n; ++i) out[t * n + i] = (seed + i * 17 + t * 31) % p.parameters->tower(p.towers[t]).q;
  return out;
}
std::vector<uint64_t> naive(const PolynomialLayout &p, std::span<const uint64_t> a, std::span<const uint64_t> b) {
  const size_t n = p.parameters->n();
  std::vector<uint64_t> out(a.size());
  for (size_t t = 0; t < p.towers.size(); ++t) {
    const uint64_t q = p.parameters->tower(p.towers[t]).q;
    for (size_t i = 0; i < n; ++i)
      for (size_t j = 0; j < n; ++j) {
        const uint64_t v = orc_mul_mod(a[t * n + i], b[t * n + j], q);
        uint64_t &dst = out[t * n + (i + j) % n];
        dst = i + j < n ? orc_add_mod(dst, v, q) : orc_sub_mod(dst, v, q);
      }
  }
  return out;
}
void equal(std::span<const uint64_t> actual, const std::vector<uint64_t> &expected, const char *why) {
  check(actual.size() == expected.size() && std::equal(actual.begin(), actual.end(), expected.begin()), why);
}

void chain_and_leases() {
  static_assert(!std::is_aggregate_v<Polynomial> && !std::is_aggregate_v<Completion>);
  auto p = layout();
  auto driver = std::make_shared<HostDriver>(p);
  Session s(driver);
  rejects([&] { Session duplicate(driver); }, "a transport belongs to one session");
  auto a = input(p, 5), b = input(p, 9), original = a;
  auto da = s.upload(a), db = s.upload(b);
  std::fill(a.begin(), a.end(), 0);  // caller memory is no longer borrowed
  check(da.readiness().query().outcome == Outcome::Pending, "deferred upload stays pending");
  check(driver->trace->executed == 0, "submission does not execute the deferred queue");
  auto fa = s.forward(da), fb = s.forward(db);
  auto product = s.pointwise(fa, fb);
  auto coefficient = s.inverse(product);
  auto result = s.download(coefficient);
  check(s.stats().submitted == 7 && s.stats().pending == 7, "operation journal of the chain");
  check(s.stats().uploads == 2 && s.stats().downloads == 1 && s.stats().device_copies == 4, "transfer counts");
  check(da.view().allocation != fa.view().allocation && fa.view().allocation != product.view().allocation,
        "out-of-place outputs");
  equal(result.wait_values(), naive(p, original, b), "chain equals the negacyclic convolution");
  check(s.stats().pending == 0 && s.stats().quiescent, "completion retires prior work");
  equal(s.download(da).wait_values(), original, "inputs are immutable");
  equal(s.download(db).wait_values(), b, "right input immutable");
  auto source_completion = da.readiness();
  auto expected = s.download(fa);
  auto ev = expected.wait_values();  // `expected` keeps the storage alive
  auto with_dependency = s.download(s.forward(da, std::span<const Completion>(&source_completion, 1)));
  equal(with_dependency.wait_values(), {ev.begin(), ev.end()}, "explicit same-stream dependency");
  expected = {};
  with_dependency = {};
  equal(s.multiply(original, b).wait_values(), naive(p, original, b), "convenience chain");
  equal(s.download(s.inverse(s.pointwise(fa, fa))).wait_values(), naive(p, original, original),
        "read-only alias with fresh output");
  auto copied = da.view();
  ++copied.allocation.generation;
  check(da.view().allocation != copied.allocation, "descriptor copies cannot alter the registry");
  da = {}; db = {}; fa = {}; fb = {}; product = {}; coefficient = {}; result = {};
  check(driver->trace->live_buffers == 0 && driver->trace->live_events == 0, "completed pins release resources");
  check(s.stats().device_bytes == 0 && s.stats().host_bytes == 0, "budget leases retire");
}

void rejection_and_views() {
  auto p = layout(3, 2);
  auto driver = std::make_shared<HostDriver>(p);
  Session s(driver);
  auto a = input(p, 3), b = a;
  b[0] = p.parameters->tower(p.towers[0]).q;
  rejects([&] { s.multiply(a, b); }, "bad second input rejects the chain before enqueue");
  check(driver->trace->calls == 0, "invalid inputs submit nothing");
  rejects([&] { s.upload(std::span<const uint64_t>(a).first(1)); }, "short input");
  auto da = s.upload(a);
  const auto calls = driver->trace->calls;
  rejects([&] { s.inverse(da); }, "inverse domain rejection");
  rejects([&] { s.pointwise(da, da); }, "pointwise domain rejection");
  rejects([&] { s.forward(Polynomial{}); }, "empty polynomial");
  auto other_driver = std::make_shared<HostDriver>(p);
  Session other(other_driver);
  rejects([&] { other.forward(da); }, "foreign session");
  auto completion = da.readiness();
  rejects([&] { other.upload(a, std::span<const Completion>(&completion, 1)); }, "foreign dependency");
  rejects([&] { s.subview(da, 0, 4, 2); }, "reduced QP cannot be fabricated");
  rejects([&] { s.subview(da, 4, 2, 3); }, "subview beyond extent");
  check(driver->trace->calls == calls && other_driver->trace->calls == 0, "preflight failures call no transport");
  auto view = s.subview(da, 1, 2, 3);
  auto nested = s.subview(view, 1, 1, 3);
  equal(s.download(s.inverse(s.forward(nested))).wait_values(), {a.begin() + 16, a.begin() + 24},
        "nested views use allocation-relative offsets");
  check(nested.view().first_tower == 2, "nested view offset");
  auto e = s.forward(view), e2 = s.forward(nested);
  rejects([&] { s.pointwise(e, e2); }, "incompatible layouts");
  s.close();
  rejects([&] { s.forward(da); }, "stale handles after close");
  rejects([&] { s.upload(a); }, "closed session refuses admission");
  check(da.readiness().query().outcome == Outcome::Succeeded, "completion metadata survives close");
  rejects([] { Completion{}.wait(); }, "empty completion");
  rejects([] { Download{}.wait_values(); }, "empty download");
}

void budgets() {
  auto p = layout();
  auto a = input(p, 4);
  auto driver = std::make_shared<HostDriver>(p);
  Session s(driver, {bytes(p), bytes(p), 1});
  auto da = s.upload(a);
  const auto calls = driver->trace->calls;
  rejects([&] { s.forward(da); }, "device budget exhausted before admission");
  rejects([&] { s.download(da); }, "host budget exhausted before admission");
  check(driver->trace->calls == calls && !s.stats().poisoned, "budget refusal is preflight");
  da.readiness().wait();
  rejects([&] { s.download(da); }, "operation journal stays bounded");
  check(driver->trace->calls == calls + 1, "operation budget submits nothing");
}

void failure_matrix() {
  auto p = layout();
  auto a = input(p, 1), b = input(p, 2);
  size_t steps;
  {
    auto d = std::make_shared<HostDriver>(p);
    Session s(d);
    auto r = s.multiply(a, b);
    steps = d->trace->calls;
    r.wait_values();
  }
  for (size_t step = 1; step <= steps + 1; ++step) {
    auto d = std::make_shared<HostDriver>(p);
    auto trace = d->trace;
    {
      Session s(d);
      trace->fail_step = step;
      rejects([&] { s.multiply(a, b).wait_values(); }, "injected synchronous failure propagates");
      check(s.stats().poisoned && s.stats().quiescent, "failure drains and poisons");
      check(!s.history().empty() && s.history().back().outcome == Outcome::Failed, "failed record kept");
      rejects([&] { s.upload(a); }, "no resubmission after failure");
      rejects([&] { s.close(); }, "close rethrows the failure");
    }
    check(trace->live_buffers == 0 && trace->live_events == 0, "failure unwinds buffers and events");
  }
  for (size_t sequence : {size_t{1}, size_t{4}, size_t{11}}) {
    auto d = std::make_shared<HostDriver>(p);
    Session s(d);
    d->trace->async_fail_at = sequence;
    auto r = s.multiply(a, b);
    rejects([&] { r.wait_values(); }, "asynchronous failure hides output");
    check(s.stats().poisoned, "asynchronous failure poisons");
    check(r.completion().query().outcome != Outcome::Succeeded, "failed output is not successful");
  }
}

void partial_and_quarantine() {
  auto p = layout();
  auto a = input(p, 1), b = input(p, 2);
  std::vector<size_t> enqueue_calls;
  {
    auto d = std::make_shared<HostDriver>(p);
    Session s(d);
    auto r = s.multiply(a, b);
    enqueue_calls = d->trace->enqueue_calls;
    r.wait_values();
  }
  for (size_t step : enqueue_calls) {
    auto d = std::make_shared<HostDriver>(p);
    Session s(d);
    d->trace->partial_step = step;
    rejects([&] { s.multiply(a, b); }, "failure after partial submission");
    check(d->trace->executed > 0 && d->trace->live_buffers == 0 && d->trace->live_events == 0,
          "partial submission drains before release");
    check(s.history().back().outcome == Outcome::Failed, "partial failure keeps its record");
  }
  auto d = std::make_shared<HostDriver>(p);
  auto trace = d->trace;
  {
    Session s(d);
    auto r = s.multiply(a, b);
    trace->async_fail_at = 3;
    trace->allow_drain = false;
    rejects([&] { r.wait_values(); }, "failed wait with unproven quiescence");
    r = {};
    check(s.stats().poisoned && !s.stats().quiescent && trace->live_buffers == 6,
          "abandoned handles cannot free quarantined buffers");
    check(s.stats().host_bytes == 3 * bytes(p), "quarantine keeps upload and download staging");
    rejects([&] { s.close(); }, "failed close keeps pins");
    check(trace->live_buffers == 6, "unproven drain cannot release");
    trace->allow_drain = true;
    rejects([&] { s.close(); }, "recovered cleanup still reports the original failure");
    check(s.stats().quiescent && trace->live_buffers == 0 && trace->live_events == 0, "proven drain reclaims");
  }
  check(trace->live_buffers == 0 && trace->live_events == 0, "no leaked quarantine");
}

void abandonment_and_bad_output() {
  auto p = layout();
  auto a = input(p, 1), b = input(p, 2);
  auto d = std::make_shared<HostDriver>(p);
  Download output;
  {
    Session s(d);
    output = s.multiply(a, b);
  }
  equal(output.wait_values(), naive(p, a, b), "close with live output drains before destruction");
  output = {};
  check(d->trace->live_buffers == 0 && d->trace->live_events == 0, "abandonment cleanup");
  auto corrupt = std::make_shared<HostDriver>(p);
  Session s(corrupt);
  corrupt->trace->corrupt_download = true;
  auto r = s.multiply(a, b);
  rejects([&] { r.wait_values(); }, "noncanonical driver output stays hidden");
  check(s.stats().poisoned && s.history().back().outcome == Outcome::Failed, "bad output fails its completion");
}

void query_failure_and_evaluation_input() {
  auto p = layout();
  auto a = input(p, 8);
  auto d = std::make_shared<HostDriver>(p);
  Session s(d);
  auto eval = s.upload_evaluation(a);
  check(eval.layout().domain == Domain::Evaluation && eval.layout().order == Order::BitReversed,
        "evaluation upload declares its representation");
  auto expected = a;
  for (size_t t = 0; t < p.towers.size(); ++t) {
    const auto tw = p.parameters->tower(p.towers[t]);
    orc_ntt_inverse(expected.data() + t * 8, 8, tw.q, tw.psi);
  }
  equal(s.download(s.inverse(eval)).wait_values(), expected, "evaluation input inverse");
  auto other = std::make_shared<HostDriver>(p);
  Session failed(other);
  auto value = failed.upload(a);
  other->trace->fail_step = other->trace->calls + 1;
  check(value.readiness().query().outcome == Outcome::Failed, "query reports driver failure");
  rejects([&] { value.readiness().wait(); }, "wait rethrows");
  check(failed.stats().poisoned, "query errors poison admission");
  auto cleanup = std::make_shared<HostDriver>(p);
  Session close_error(cleanup);
  cleanup->trace->cleanup_error = true;
  rejects([&] { close_error.close(); }, "close reports cleanup errors");
  check(close_error.stats().poisoned && close_error.stats().closed, "cleanup error stops admission");
}

orc_context oracle_context(const PolynomialLayout &p, std::vector<uint64_t> &store) {
  const auto &prm = *p.parameters;
  store.clear();
  for (const auto &t : prm.q()) store.push_back(t.q);
  for (const auto &t : prm.q()) store.push_back(t.psi);
  for (const auto &t : prm.p()) store.push_back(t.q);
  for (const auto &t : prm.p()) store.push_back(t.psi);
  const size_t m = prm.q().size(), k = prm.p().size();
  return orc_context{prm.n(), m, k, prm.alpha(), store.data(), store.data() + m, store.data() + 2 * m,
                     store.data() + 2 * m + k};
}

void conversion_chain() {
  auto p = layout(3, 2), q = p;
  q.towers = q_prefix(*p.parameters, 3);
  auto driver = std::make_shared<HostDriver>(p);
  Session s(driver);
  auto values = input(p, 17);
  auto uploaded = s.upload(p, values);
  auto source = s.subview(uploaded, 0, 3, 3);
  auto extended = s.mod_up(source);
  auto reduced = s.mod_down(extended);
  check(s.stats().downloads == 0 && s.stats().uploads == 1 && s.stats().parameter_uploads == 3,
        "ModUp/ModDown stay resident; only parameter tables are uploaded");
  check(driver->trace->executed == 0, "conversion composition does not wait on the host");
  std::vector<uint64_t> store;
  const auto ctx = oracle_context(p, store);
  std::vector<uint64_t> want_up(5 * 8), want_down(3 * 8);
  orc_mod_up(&ctx, 3, values.data(), 0, want_up.data());
  orc_mod_down(&ctx, 3, want_up.data(), want_down.data());
  equal(s.download(extended).wait_values(), want_up, "ModUp equals the oracle");
  equal(s.download(reduced).wait_values(), want_down, "ModDown equals the oracle");
  equal(s.download(uploaded).wait_values(), values, "conversion preserves its input");
  const auto before = driver->trace->calls;
  rejects([&] { s.mod_down(uploaded); }, "ModDown rejects coefficient input");
  rejects([&] { s.mod_up(uploaded); }, "ModUp rejects QP input");
  rejects([&] { s.switch_basis(source, q); }, "overlapping bases rejected");
  rejects([&] { s.switch_basis(extended, q); }, "basis switch rejects evaluation input");
  check(driver->trace->calls == before, "bad conversion metadata submits nothing");
  auto chain = [&](Session &session) {
    auto a = session.upload(q, std::span<const uint64_t>(values).first(24));
    return session.download(session.mod_down(session.mod_up(a)));
  };
  auto baseline = std::make_shared<HostDriver>(p);
  {
    Session base(baseline);
    chain(base).wait_values();
  }
  for (size_t step = 1; step <= baseline->trace->calls; ++step) {
    auto failing = std::make_shared<HostDriver>(p);
    failing->trace->fail_step = step;
    bool failed = false;
    {
      Session t(failing);
      try {
        chain(t).wait_values();
      } catch (...) {
        failed = true;
      }
    }
    check(failed && failing->trace->live_buffers == 0 && failing->trace->live_events == 0,
          "failed conversion releases tables, outputs and events");
  }
  auto limited = std::make_shared<HostDriver>(p);
  Session low(limited, {400, 4096, 100});
  auto source_low = low.upload(q, std::span<const uint64_t>(values).first(24));
  source_low.readiness().wait();
  auto p_target = p;
  p_target.towers.erase(p_target.towers.begin(), p_target.towers.begin() + 3);
  const auto prior = limited->trace->calls;
  rejects([&] { low.switch_basis(source_low, p_target); }, "table bytes count against the device limit");
  check(limited->trace->calls == prior && low.stats().device_bytes == 192 && !low.stats().poisoned,
        "admission failure restores credits without enqueue");
}

void hybrid_digits_and_keyswitch() {
  // A complement larger than 40 towers keeps its order across switch chunks.
  const auto full = layout(3, 40);
  auto active = full;
  active.towers = q_prefix(*full.parameters, full.active_q);
  const auto coefficients = input(active, 9);
  auto driver = std::make_shared<HostDriver>(full);
  Session session(driver);
  const auto source = session.upload(active, coefficients);
  rejects([&] { session.hybrid_digits(source); }, "digits reject coefficient input");
  const auto evaluations = session.forward(source);
  const auto digits = session.hybrid_digits(evaluations);
  check(digits.size() == 3 && session.stats().parameter_uploads == 7, "40+ tower complement split in order");
  std::vector<uint64_t> store;
  const auto ctx = oracle_context(full, store);
  const size_t tq = 43, n = 8;
  std::vector<uint64_t> eval(3 * n), want(3 * tq * n);
  const auto ev_download = session.download(evaluations);  // owns the host values
  const auto ev = ev_download.wait_values();
  std::copy(ev.begin(), ev.end(), eval.begin());
  orc_hybrid_digits(&ctx, 3, eval.data(), want.data());
  for (size_t d = 0; d < 3; ++d)
    equal(session.download(digits[d]).wait_values(), {want.begin() + d * tq * n, want.begin() + (d + 1) * tq * n},
          "digits equal the oracle");
  session.close();

  // Full Hybrid core with rotation against the oracle key switch.
  const auto base = layout(5, 3, 64);
  auto params = Parameters::create(64, base.parameters->q(), base.parameters->p(), 2);
  const PolynomialLayout qp{params, 4, qp_basis(*params, 4), Domain::Coefficient, Order::Natural};
  const PolynomialLayout src_layout{params, 4, q_prefix(*params, 4), Domain::Evaluation, Order::BitReversed};
  const PolynomialLayout key_layout{params, 5, qp_basis(*params, 5), Domain::Evaluation, Order::BitReversed};
  auto d2 = std::make_shared<HostDriver>(qp);
  Session s(d2);
  std::vector<uint64_t> store2;
  const auto c2 = oracle_context(key_layout, store2);
  std::vector<uint64_t> mods(store2.begin(), store2.begin() + 5);
  mods.insert(mods.end(), store2.begin() + 10, store2.begin() + 13);
  const size_t full_digits = 3, block = 8 * 64;
  std::vector<uint64_t> kb(full_digits * block), ka(full_digits * block), x(4 * 64), c0(4 * 64);
  for (size_t dd = 0; dd < full_digits; ++dd) {
    orc_splitmix_fill(kb.data() + dd * block, 64, 8, mods.data(), 100 + dd);
    orc_splitmix_fill(ka.data() + dd * block, 64, 8, mods.data(), 200 + dd);
  }
  orc_lcg_fill(x.data(), 64, 4, mods.data(), 7);
  orc_lcg_fill(c0.data(), 64, 4, mods.data(), 8);
  std::vector<HybridKeyDigit> rows;
  for (size_t dd = 0; dd < full_digits; ++dd)
    rows.push_back({std::span<const uint64_t>(kb).subspan(dd * block, block),
                    std::span<const uint64_t>(ka).subspan(dd * block, block)});
  const auto key = s.upload_hybrid_key(key_layout, rows);
  check(s.stats().uploads == 2 * 2, "only the active key digits are uploaded");
  auto ext = s.hybrid_accumulate(s.hybrid_digits(s.upload(src_layout, x)), key);
  ext = s.hybrid_rotate_extended(ext, s.upload(src_layout, c0), 5);
  auto out_b = s.download(s.mod_down(ext.b)), out_a = s.download(s.mod_down(ext.a));
  std::vector<uint64_t> wb(4 * 64), wa(4 * 64);
  check(orc_keyswitch(&c2, 4, x.data(), kb.data(), ka.data(), c0.data(), 5, wb.data(), wa.data()) == 0,
        "oracle key switch");
  equal(out_b.wait_values(), wb, "Session key switch b equals the oracle");
  equal(out_a.wait_values(), wa, "Session key switch a equals the oracle");
  s.close();
}

void closed_and_moved_admission() {
  const auto base = layout(2, 1);
  const auto values = input(base, 1);
  auto driver = std::make_shared<HostDriver>(base);
  Session moved(driver);
  Session owner(std::move(moved));
  const Polynomial empty;
  const HybridKey key;
  const HybridContributions channels;
  const std::vector<std::function<void(Session &)>> admissions{
      [&](Session &s) { s.upload(values); },
      [&](Session &s) { s.upload(base, values); },
      [&](Session &s) { s.upload_evaluation(values); },
      [&](Session &s) { s.forward(empty); },
      [&](Session &s) { s.inverse(empty); },
      [&](Session &s) { s.pointwise(empty, empty); },
      [&](Session &s) { s.switch_basis(empty, base); },
      [&](Session &s) { s.mod_up(empty); },
      [&](Session &s) { s.mod_down(empty); },
      [&](Session &s) { s.hybrid_digits(empty); },
      [&](Session &s) { s.upload_hybrid_key(base, {}); },
      [&](Session &s) { s.hybrid_accumulate({}, key); },
      [&](Session &s) { s.hybrid_rotate_extended(channels, empty, 1); },
      [&](Session &s) { s.subview(empty, 0, 1, 1); },
      [&](Session &s) { s.download(empty); },
      [&](Session &s) { s.multiply(values, values); },
  };
  owner.close();
  for (Session *s : {&moved, &owner})
    for (const auto &admit : admissions) rejects([&] { admit(*s); }, "closed or moved session rejects work");
  check(driver->trace->calls == 0, "rejected admission never touches the driver");
  check(owner.stats().closed && owner.history().empty(), "closed-session diagnostics stay readable");
}
}  // namespace

int main() {
  try {
    chain_and_leases();
    rejection_and_views();
    budgets();
    failure_matrix();
    partial_and_quarantine();
    abandonment_and_bad_output();
    query_failure_and_evaluation_input();
    conversion_chain();
    hybrid_digits_and_keyswitch();
    closed_and_moved_admission();
    std::cout << checks << " RESIDENT HOST CHECKS PASSED; NO GPU EXECUTION\n";
  } catch (const std::exception &e) {
    std::cerr << "FAILED: " << e.what() << '\n';
    return 1;
  }
  return 0;
}
