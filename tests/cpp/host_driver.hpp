#pragma once
// Deferred CPU transport for the resident Session tests (test infrastructure;
// never GPU execution). Work is queued and executed only on wait/quiesce, like
// the reference's resident_test::HostDriver (tests/support/resident_host_driver.hpp:30-195),
// with the same failure-injection knobs: synchronous failure at a call number,
// failure after an enqueue, asynchronous failure, refused drain, corrupt
// download and cleanup error. Arithmetic comes from the C oracle.
#include <functional>
#include <stdexcept>
#include <vector>

#include "ntt_b200/resident_driver.hpp"

extern "C" {
#include "../../oracle/oracle.h"
}

namespace host_test {
using namespace ntt::resident;
using ntt::proposal::PolynomialLayout;

struct Trace {
  size_t calls = 0, live_buffers = 0, live_events = 0, executed = 0;
  size_t fail_step = 0, partial_step = 0, async_fail_at = 0, drains = 0;
  bool allow_drain = true, corrupt_download = false, cleanup_error = false;
  std::vector<size_t> enqueue_calls;
};

struct HostBuffer final : detail::Buffer {
  std::shared_ptr<Trace> trace;
  std::vector<uint64_t> values;
  HostBuffer(std::shared_ptr<Trace> t, size_t n) : trace(std::move(t)), values(n) { ++trace->live_buffers; }
  ~HostBuffer() override { --trace->live_buffers; }
};
struct HostEvent final : detail::Event {
  std::shared_ptr<Trace> trace;
  size_t fence = 0;
  bool recorded = false;
  explicit HostEvent(std::shared_ptr<Trace> t) : trace(std::move(t)) { ++trace->live_events; }
  ~HostEvent() override { --trace->live_events; }
};

class HostDriver final : public detail::Driver {
  PolynomialLayout layout_;
  std::vector<std::function<void()>> queue_;
  size_t done_ = 0;
  bool failed_ = false;

  void tick() {
    if (++trace->calls == trace->fail_step) throw std::runtime_error("injected transport failure");
  }
  void enqueue(std::function<void()> work) {
    tick();
    queue_.push_back(std::move(work));
    trace->enqueue_calls.push_back(trace->calls);
    if (trace->calls == trace->partial_step) throw std::runtime_error("failure after enqueue");
  }
  void through(size_t fence) {
    if (failed_) throw std::runtime_error("host test queue failed");
    while (done_ < fence) {
      if (done_ + 1 == trace->async_fail_at) {
        failed_ = true;
        throw std::runtime_error("injected asynchronous failure");
      }
      queue_[done_]();
      queue_[done_] = {};
      ++done_;
      ++trace->executed;
    }
  }
  static HostBuffer &buf(detail::Buffer &b) { return dynamic_cast<HostBuffer &>(b); }
  static const HostBuffer &buf(const detail::Buffer &b) { return dynamic_cast<const HostBuffer &>(b); }
  static uint64_t modulus(const PolynomialLayout &p, size_t t) { return p.parameters->tower(p.towers[t]).q; }
  static uint64_t root(const PolynomialLayout &p, size_t t) { return p.parameters->tower(p.towers[t]).psi; }

 public:
  std::shared_ptr<Trace> trace = std::make_shared<Trace>();
  explicit HostDriver(PolynomialLayout p) : layout_(std::move(p)) { ntt::proposal::validate(layout_); }
  int ordinal() const override { return 0; }
  const PolynomialLayout &layout() const override { return layout_; }
  size_t constant_bytes() const override { return 0; }
  std::unique_ptr<detail::Buffer> allocate(size_t n) override {
    tick();
    return std::make_unique<HostBuffer>(trace, n);
  }
  std::unique_ptr<detail::Event> make_event() override {
    tick();
    return std::make_unique<HostEvent>(trace);
  }
  void upload(detail::Buffer &out, std::span<const uint64_t> source) override {
    auto *b = &buf(out);
    enqueue([b, source] { std::copy(source.begin(), source.end(), b->values.begin()); });
  }
  void copy(detail::Buffer &out, const detail::Buffer &in, size_t offset, size_t n) override {
    auto *a = &buf(out);
    auto *b = &buf(in);
    enqueue([a, b, offset, n] { std::copy_n(b->values.begin() + offset, n, a->values.begin()); });
  }
  void copy_range(detail::Buffer &out, size_t dst, const detail::Buffer &in, size_t src, size_t n) override {
    auto *a = &buf(out);
    auto *b = &buf(in);
    ntt::proposal::require(dst <= a->values.size() && n <= a->values.size() - dst && src <= b->values.size() &&
                               n <= b->values.size() - src,
                           "host copy range extent");
    enqueue([a, b, dst, src, n] { std::copy_n(b->values.begin() + src, n, a->values.begin() + dst); });
  }
  void transform(detail::Buffer &out, const PolynomialLayout &p, bool inverse) override {
    auto *b = &buf(out);
    enqueue([b, p, inverse] {
      const size_t n = p.parameters->n();
      for (size_t t = 0; t < p.towers.size(); ++t) {
        const int rc = inverse ? orc_ntt_inverse(b->values.data() + t * n, n, modulus(p, t), root(p, t))
                               : orc_ntt_forward(b->values.data() + t * n, n, modulus(p, t), root(p, t));
        if (rc) throw std::runtime_error("host transform rejected");
      }
    });
  }
  void pointwise(detail::Buffer &out, const detail::Buffer &right, size_t offset, const PolynomialLayout &p) override {
    auto *a = &buf(out);
    auto *b = &buf(right);
    enqueue([a, b, offset, p] {
      const size_t n = p.parameters->n();
      for (size_t t = 0; t < p.towers.size(); ++t)
        for (size_t i = 0; i < n; ++i)
          a->values[t * n + i] = orc_mul_mod(a->values[t * n + i], b->values[offset + t * n + i], modulus(p, t));
    });
  }
  void hybrid_mac(detail::Buffer &rb, detail::Buffer &ra, const detail::Buffer &digit, const detail::Buffer &kb,
                  const detail::Buffer &ka, const PolynomialLayout &layout, bool first) override {
    auto *b = &buf(rb), *a = &buf(ra);
    const auto *d = &buf(digit), *key_b = &buf(kb), *key_a = &buf(ka);
    enqueue([b, a, d, key_b, key_a, layout, first] {
      const size_t n = layout.parameters->n();
      for (size_t i = 0; i < d->values.size(); ++i) {
        const uint64_t q = modulus(layout, i / n);
        const uint64_t pb = orc_mul_mod(d->values[i], key_b->values[i], q);
        const uint64_t pa = orc_mul_mod(d->values[i], key_a->values[i], q);
        b->values[i] = first ? pb : orc_add_mod(b->values[i], pb, q);
        a->values[i] = first ? pa : orc_add_mod(a->values[i], pa, q);
      }
    });
  }
  void hybrid_rotate(detail::Buffer &ob, detail::Buffer &oa, const detail::Buffer &eb, const detail::Buffer &ea,
                     const detail::Buffer &c0, size_t c0_offset, const detail::Buffer &scales,
                     const PolynomialLayout &layout, uint32_t g) override {
    auto *b = &buf(ob), *a = &buf(oa);
    const auto *xb = &buf(eb), *xa = &buf(ea), *first = &buf(c0), *table = &buf(scales);
    enqueue([=] {
      const size_t n = layout.parameters->n();
      const uint64_t log_n = orc_log2(n);
      for (size_t t = 0; t < layout.towers.size(); ++t)
        for (size_t k = 0; k < n; ++k) {
          const size_t src = t * n + orc_automorphism_source_index(k, n, log_n, g);
          uint64_t v = xb->values[src];
          if (t < layout.active_q)
            v = orc_add_mod(v, orc_mul_mod(first->values[c0_offset + src], table->values[t], modulus(layout, t)),
                            modulus(layout, t));
          b->values[t * n + k] = v;
          a->values[t * n + k] = xa->values[src];
        }
    });
  }
  void switch_basis(detail::Buffer &out, const detail::Buffer &in, size_t offset, const detail::Buffer &constants,
                    const PolynomialLayout &source, const PolynomialLayout &target) override {
    auto *a = &buf(out);
    const auto *b = &buf(in), *table = &buf(constants);
    enqueue([a, b, table, offset, source, target] {
      // The packed table starts with the source then the target moduli.
      const size_t s = source.towers.size(), t = target.towers.size(), n = source.parameters->n();
      if (orc_basis_convert(b->values.data() + offset, n, table->values.data(), s, table->values.data() + s, t,
                            a->values.data()))
        throw std::runtime_error("host basis switch rejected");
    });
  }
  void correct(detail::Buffer &out, const detail::Buffer &left, size_t lo, const detail::Buffer &right, size_t ro,
               const detail::Buffer &constants, const PolynomialLayout &layout) override {
    auto *a = &buf(out);
    const auto *l = &buf(left), *r = &buf(right), *table = &buf(constants);
    enqueue([=] {
      const size_t n = layout.parameters->n(), count = layout.towers.size();
      for (size_t i = 0; i < a->values.size(); ++i) {
        const size_t t = i / n;
        const uint64_t q = table->values[t];
        a->values[i] = orc_mul_mod(orc_sub_mod(l->values[lo + i], r->values[ro + i], q), table->values[count + t], q);
      }
    });
  }
  void download(std::span<uint64_t> dst, const detail::Buffer &in, size_t offset) override {
    const auto *b = &buf(in);
    const bool corrupt = trace->corrupt_download;
    enqueue([b, dst, offset, corrupt] {
      std::copy_n(b->values.begin() + offset, dst.size(), dst.begin());
      if (corrupt) dst[0] = UINT64_MAX;
    });
  }
  void record(detail::Event &event) override {
    tick();
    auto &e = dynamic_cast<HostEvent &>(event);
    e.fence = queue_.size();
    e.recorded = true;
  }
  bool ready(detail::Event &event) override {
    tick();
    auto &e = dynamic_cast<HostEvent &>(event);
    if (failed_) throw std::runtime_error("host test queue failed");
    return e.recorded && done_ >= e.fence;
  }
  void wait(detail::Event &event) override {
    tick();
    auto &e = dynamic_cast<HostEvent &>(event);
    if (!e.recorded) throw std::runtime_error("unrecorded host test event");
    through(e.fence);
  }
  bool quiesce() noexcept override {
    ++trace->drains;
    if (!trace->allow_drain) return false;
    try {
      through(queue_.size());
    } catch (...) {
    }
    queue_.clear();  // a synchronous fake can prove cancellation
    done_ = 0;
    return true;
  }
  void check_health() const override {
    if (trace->cleanup_error) throw std::runtime_error("injected cleanup error");
  }
};
}  // namespace host_test
