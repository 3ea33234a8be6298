// The reference's resident Driver over the B200 C ABI (libntt_b200.so).
//
// This is the file a maintainer adds to minnow54426/ntt-gpu in place of its
// CUDA transport (src/cuda/resident_adapter.inc, included by
// src/cuda/ntt_kernels.cu): it implements ntt::resident::detail::Driver
// (include/ntt/resident_driver.hpp:13-57) with one C-ABI call per primitive and
// defines make_cuda_session (include/ntt/resident.hpp:142-143). It compiles
// against the reference's own headers; Session, the OpenFHE Hybrid adapters and
// every caller above the seam stay unchanged. Contract errors come back as
// ContractError, CUDA failures as std::runtime_error with the library's
// "CUDA: ..." message (the reference's conventions, backend_contract.hpp:20-26,
// ntt_kernels.cu:40-46). Per-call constant tables the Session uploads
// (resident.cpp:353-365, 411-424, 588-606) are ignored: the context keeps its
// own tables resident in HBM.
#include <stdexcept>
#include <string>

#include "ntt/resident_driver.hpp"
#include "ntt_b200.h"

namespace ntt::resident {
namespace b200_binding {
using namespace ::ntt::proposal;
namespace transport = ::ntt::resident::detail;

inline void check(int rc) {
  if (rc == NTT_B200_OK) return;
  const std::string msg = ntt_b200_last_error();
  if (rc == NTT_B200_ERR_CONTRACT || rc == NTT_B200_ERR_UNSUPPORTED || rc == NTT_B200_ERR_WORKSPACE)
    throw ContractError(msg);
  throw std::runtime_error(msg);
}

struct Context {
  PolynomialLayout base;
  int device;
  void *stream = nullptr;
  ntt_b200_context ctx = nullptr;
  size_t m = 0;
  Context(PolynomialLayout p, int ordinal) : base(std::move(p)), device(ordinal) {
    const auto &prm = *base.parameters;
    std::vector<uint64_t> q, qp, p_, pp;
    for (const auto &t : prm.q()) q.push_back(t.q), qp.push_back(t.psi);
    for (const auto &t : prm.p()) p_.push_back(t.q), pp.push_back(t.psi);
    m = q.size();
    check(ntt_b200_stream_create(device, &stream));
    check(ntt_b200_context_create(&ctx, device, prm.n(), q.data(), qp.data(), q.size(), p_.data(), pp.data(),
                                  p_.size(), prm.alpha()));
  }
  ~Context() {
    ntt_b200_stream_synchronize(stream);
    ntt_b200_context_destroy(ctx);
    ntt_b200_stream_destroy(stream);
  }
  std::vector<uint32_t> ids(const PolynomialLayout &p) const {
    std::vector<uint32_t> out;
    for (const auto &t : p.towers) out.push_back(uint32_t(t.family == Family::Q ? t.index : m + t.index));
    return out;
  }
};
struct Buffer final : transport::Buffer {
  std::shared_ptr<Context> c;
  uint64_t *data = nullptr;
  size_t elements;
  Buffer(std::shared_ptr<Context> ctx, size_t n) : c(std::move(ctx)), elements(n) {
    check(ntt_b200_alloc(c->device, n * sizeof(uint64_t), c->stream, reinterpret_cast<void **>(&data)));
  }
  ~Buffer() override { ntt_b200_free(data, c->stream); }
};
struct Event final : transport::Event {
  std::shared_ptr<Context> c;
  void *e = nullptr;
  explicit Event(std::shared_ptr<Context> ctx) : c(std::move(ctx)) { check(ntt_b200_event_create(c->device, &e)); }
  ~Event() override { ntt_b200_event_destroy(e); }
};

class Driver final : public transport::Driver {
  std::shared_ptr<Context> c_;
  static const Buffer &b(const transport::Buffer &x) { return dynamic_cast<const Buffer &>(x); }
  static void *s(const Context &c) { return c.stream; }

 public:
  Driver(PolynomialLayout p, int ordinal) : c_(std::make_shared<Context>(std::move(p), ordinal)) {}
  int ordinal() const override { return c_->device; }
  const PolynomialLayout &layout() const override { return c_->base; }
  size_t constant_bytes() const override {
    size_t bytes = 0;
    check(ntt_b200_context_table_bytes(c_->ctx, &bytes));
    return bytes;
  }
  std::unique_ptr<transport::Buffer> allocate(size_t n) override { return std::make_unique<Buffer>(c_, n); }
  std::unique_ptr<transport::Event> make_event() override { return std::make_unique<Event>(c_); }
  void upload(transport::Buffer &o, std::span<const uint64_t> v) override {
    check(ntt_b200_memcpy(b(o).data, v.data(), v.size_bytes(), 1, s(*c_)));
  }
  void copy(transport::Buffer &o, const transport::Buffer &i, size_t off, size_t n) override {
    check(ntt_b200_memcpy(b(o).data, b(i).data + off, n * 8, 3, s(*c_)));
  }
  void copy_range(transport::Buffer &o, size_t d, const transport::Buffer &i, size_t src, size_t n) override {
    check(ntt_b200_memcpy(b(o).data + d, b(i).data + src, n * 8, 3, s(*c_)));
  }
  void transform(transport::Buffer &o, const PolynomialLayout &p, bool inverse) override {
    const auto ids = c_->ids(p);
    check(ntt_b200_ntt(c_->ctx, b(o).data, b(o).data, ids.data(), ids.size(), 1, 0, inverse, s(*c_)));
  }
  void pointwise(transport::Buffer &o, const transport::Buffer &r, size_t off, const PolynomialLayout &p) override {
    const auto ids = c_->ids(p);
    check(ntt_b200_pointwise(c_->ctx, b(o).data, b(o).data, b(r).data + off, ids.data(), ids.size(), 1, 0, s(*c_)));
  }
  void hybrid_mac(transport::Buffer &rb, transport::Buffer &ra, const transport::Buffer &d,
                  const transport::Buffer &kb, const transport::Buffer &ka, const PolynomialLayout &p,
                  bool first) override {
    const uint64_t *dp[1] = {b(d).data}, *kbp[1] = {b(kb).data}, *kap[1] = {b(ka).data};
    check(ntt_b200_hybrid_mac_digits(c_->ctx, p.active_q, b(rb).data, b(ra).data, dp, kbp, kap, 1, 0, !first,
                                     s(*c_)));
  }
  void hybrid_rotate(transport::Buffer &ob, transport::Buffer &oa, const transport::Buffer &eb,
                     const transport::Buffer &ea, const transport::Buffer &c0, size_t c0_off, const transport::Buffer &,
                     const PolynomialLayout &p, uint32_t g) override {
    check(ntt_b200_hybrid_rotate(c_->ctx, p.active_q, b(ob).data, b(oa).data, b(eb).data, b(ea).data,
                                 b(c0).data + c0_off, g, s(*c_)));
  }
  void switch_basis(transport::Buffer &o, const transport::Buffer &i, size_t off, const transport::Buffer &,
                    const PolynomialLayout &src, const PolynomialLayout &tgt) override {
    const auto si = c_->ids(src), ti = c_->ids(tgt);
    check(ntt_b200_switch_basis(c_->ctx, b(o).data, b(i).data + off, si.data(), si.size(), ti.data(), ti.size(),
                                s(*c_)));
  }
  void correct(transport::Buffer &o, const transport::Buffer &l, size_t lo, const transport::Buffer &r, size_t ro,
               const transport::Buffer &, const PolynomialLayout &p) override {
    check(ntt_b200_correct(c_->ctx, p.towers.size(), b(o).data, b(l).data + lo, b(r).data + ro, s(*c_)));
  }
  void download(std::span<uint64_t> t, const transport::Buffer &i, size_t off) override {
    check(ntt_b200_memcpy(t.data(), b(i).data + off, t.size_bytes(), 2, s(*c_)));
  }
  void record(transport::Event &e) override { check(ntt_b200_event_record(dynamic_cast<Event &>(e).e, s(*c_))); }
  bool ready(transport::Event &e) override {
    const int rc = ntt_b200_event_query(dynamic_cast<Event &>(e).e);
    if (rc == NTT_B200_NOT_READY) return false;
    check(rc);
    return true;
  }
  void wait(transport::Event &e) override { check(ntt_b200_event_synchronize(dynamic_cast<Event &>(e).e)); }
  bool quiesce() noexcept override { return ntt_b200_stream_synchronize(c_->stream) == NTT_B200_OK; }
};
}  // namespace b200_binding

Session make_cuda_session(const PolynomialLayout &p, int device, Limits limits) {
  proposal::validate(p);
  proposal::require(p.domain == proposal::Domain::Coefficient && p.order == proposal::Order::Natural &&
                        p.parameters->n() <= 65536 && device >= 0 && limits.operations,
                    "unsupported resident CUDA session");
  return Session(std::make_shared<b200_binding::Driver>(p, device), limits);
}
}  // namespace ntt::resident
