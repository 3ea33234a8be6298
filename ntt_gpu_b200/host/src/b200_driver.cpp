// The B200 transport behind make_cuda_session: implements the resident Driver
// seam (the reference's CUDA Driver, src/cuda/resident_adapter.inc:157-317) over
// the C ABI of include/ntt_b200.h. One non-blocking stream per session; buffers
// from the stream-ordered pool; twiddle, conversion and correction tables built
// once in HBM by the context (the per-call constant uploads of the Session are
// accepted but the kernels read the resident tables). ModUp, ModDown, Hybrid
// digits and the all-digit MAC run as fused device pipelines. Status codes map
// back to the reference's exceptions: contract errors -> ContractError
// (std::invalid_argument), CUDA failures -> std::runtime_error("CUDA: ...").
#include <cstring>
#include <stdexcept>
#include <string>

#include "../../../include/ntt_b200.h"
#include "ntt_b200/resident_driver.hpp"

namespace ntt::resident {
namespace b200_impl {
using namespace proposal;
namespace transport = ntt::resident::detail;

void check(int rc) {
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
  size_t m = 0, k = 0, table_bytes = 0;
  bool cleanup_failed = false;

  Context(PolynomialLayout p, int ordinal) : base(std::move(p)), device(ordinal) {
    const Parameters &params = *base.parameters;
    std::vector<uint64_t> q, qpsi, pp, ppsi;
    for (const Tower &t : params.q()) q.push_back(t.q), qpsi.push_back(t.psi);
    for (const Tower &t : params.p()) pp.push_back(t.q), ppsi.push_back(t.psi);
    m = q.size();
    k = pp.size();
    check(ntt_b200_stream_create(device, &stream));
    try {
      check(ntt_b200_context_create(&ctx, device, params.n(), q.data(), qpsi.data(), m, pp.data(), ppsi.data(), k,
                                    params.alpha()));
      check(ntt_b200_context_table_bytes(ctx, &table_bytes));
      if (k > 0 && base.towers == qp_basis(params, base.active_q)) check(ntt_b200_context_prepare(ctx, base.active_q));
    } catch (...) {
      if (ctx) ntt_b200_context_destroy(ctx);
      ntt_b200_stream_destroy(stream);
      throw;
    }
  }
  // Reachable only after the session proved quiescence (or never enqueued).
  ~Context() noexcept {
    if (ntt_b200_stream_synchronize(stream) != NTT_B200_OK) cleanup_failed = true;
    if (ntt_b200_context_destroy(ctx) != NTT_B200_OK) cleanup_failed = true;
    if (ntt_b200_stream_destroy(stream) != NTT_B200_OK) cleanup_failed = true;
  }
  void healthy() const {
    if (cleanup_failed) throw std::runtime_error("resident CUDA cleanup failed");
  }
  uint32_t id(TowerRef ref) const { return uint32_t(ref.family == Family::Q ? ref.index : m + ref.index); }
  std::vector<uint32_t> ids(const PolynomialLayout &p) const {
    std::vector<uint32_t> out;
    for (const TowerRef &t : p.towers) out.push_back(id(t));
    return out;
  }
};

// One stream-ordered device allocation, shared by every Buffer view into it.
struct Region {
  std::shared_ptr<Context> context;
  void *ptr = nullptr;
  Region(std::shared_ptr<Context> c, size_t bytes) : context(std::move(c)) {
    context->healthy();
    check(ntt_b200_alloc(context->device, bytes, context->stream, &ptr));
  }
  ~Region() noexcept {
    if (ntt_b200_free(ptr, context->stream) != NTT_B200_OK) context->cleanup_failed = true;
  }
};

struct Buffer final : transport::Buffer {
  std::shared_ptr<Region> region;
  uint64_t *data;
  size_t elements;
  Buffer(std::shared_ptr<Region> r, size_t offset, size_t n)
      : region(std::move(r)), data(static_cast<uint64_t *>(region->ptr) + offset), elements(n) {}
};

struct Event final : transport::Event {
  std::shared_ptr<Context> context;
  void *event = nullptr;
  bool recorded = false;
  explicit Event(std::shared_ptr<Context> c) : context(std::move(c)) {
    context->healthy();
    check(ntt_b200_event_create(context->device, &event));
  }
  ~Event() noexcept override {
    if (ntt_b200_event_destroy(event) != NTT_B200_OK) context->cleanup_failed = true;
  }
};

class Driver final : public transport::Driver {
  std::shared_ptr<Context> c_;

  const Buffer &buf(const transport::Buffer &b) const {
    const auto &out = dynamic_cast<const Buffer &>(b);
    require(out.region->context == c_, "foreign CUDA buffer");
    return out;
  }
  Event &ev(transport::Event &e) const {
    auto &out = dynamic_cast<Event &>(e);
    require(out.context == c_, "foreign CUDA event");
    return out;
  }
  // Stream-ordered scratch for one composite call; freed (stream-ordered) on return.
  struct Scratch {
    std::shared_ptr<Region> region;
    size_t bytes;
  };
  Scratch scratch(int op, size_t level) {
    size_t bytes = 0;
    check(ntt_b200_workspace_bytes(c_->ctx, op, level, 1, &bytes));
    return {std::make_shared<Region>(c_, bytes), bytes};
  }

 public:
  Driver(PolynomialLayout p, int ordinal) : c_(std::make_shared<Context>(std::move(p), ordinal)) {}
  int ordinal() const override { return c_->device; }
  const PolynomialLayout &layout() const override { return c_->base; }
  size_t constant_bytes() const override { return c_->table_bytes; }
  void check_health() const override { c_->healthy(); }

  std::unique_ptr<transport::Buffer> allocate(size_t n) override {
    auto region = std::make_shared<Region>(c_, checked_product(n, sizeof(uint64_t)));
    return std::make_unique<Buffer>(std::move(region), 0, n);
  }
  std::vector<std::unique_ptr<transport::Buffer>> allocate_group(size_t count, size_t elements) override {
    auto region = std::make_shared<Region>(c_, checked_product(checked_product(count, elements), sizeof(uint64_t)));
    std::vector<std::unique_ptr<transport::Buffer>> out;
    for (size_t i = 0; i < count; ++i) out.push_back(std::make_unique<Buffer>(region, i * elements, elements));
    return out;
  }
  std::unique_ptr<transport::Event> make_event() override { return std::make_unique<Event>(c_); }

  void upload(transport::Buffer &out, std::span<const uint64_t> source) override {
    const auto &a = buf(out);
    require(a.elements == source.size(), "CUDA upload extent");
    c_->healthy();
    check(ntt_b200_memcpy(a.data, source.data(), source.size_bytes(), 1, c_->stream));
  }
  void copy(transport::Buffer &out, const transport::Buffer &in, size_t offset, size_t n) override {
    const auto &a = buf(out), &b = buf(in);
    require(a.elements == n && offset <= b.elements && n <= b.elements - offset, "CUDA copy extent");
    c_->healthy();
    check(ntt_b200_memcpy(a.data, b.data + offset, n * sizeof(uint64_t), 3, c_->stream));
  }
  void copy_range(transport::Buffer &out, size_t dst, const transport::Buffer &in, size_t src, size_t n) override {
    const auto &a = buf(out), &b = buf(in);
    require(dst <= a.elements && n <= a.elements - dst && src <= b.elements && n <= b.elements - src,
            "CUDA range copy extent");
    c_->healthy();
    check(ntt_b200_memcpy(a.data + dst, b.data + src, n * sizeof(uint64_t), 3, c_->stream));
  }
  void transform(transport::Buffer &out, const PolynomialLayout &p, bool inverse) override {
    const auto &a = buf(out);
    require(a.elements == bytes(p) / sizeof(uint64_t), "CUDA transform extent");
    c_->healthy();
    const auto ids = c_->ids(p);
    check(ntt_b200_ntt(c_->ctx, a.data, a.data, ids.data(), ids.size(), 1, 0, inverse ? 1 : 0, c_->stream));
  }
  void pointwise(transport::Buffer &out, const transport::Buffer &right, size_t offset,
                 const PolynomialLayout &p) override {
    const auto &a = buf(out), &b = buf(right);
    require(a.elements == bytes(p) / sizeof(uint64_t) && offset <= b.elements && a.elements <= b.elements - offset,
            "CUDA pointwise extent");
    c_->healthy();
    const auto ids = c_->ids(p);
    check(ntt_b200_pointwise(c_->ctx, a.data, a.data, b.data + offset, ids.data(), ids.size(), 1, 0, c_->stream));
  }
  void hybrid_mac(transport::Buffer &result_b, transport::Buffer &result_a, const transport::Buffer &digit,
                  const transport::Buffer &key_b, const transport::Buffer &key_a, const PolynomialLayout &layout,
                  bool first_digit) override {
    const auto &b = buf(result_b), &a = buf(result_a), &d = buf(digit), &kb = buf(key_b), &ka = buf(key_a);
    const size_t count = bytes(layout) / sizeof(uint64_t);
    require(b.elements == count && a.elements == count && d.elements == count && kb.elements == count &&
                ka.elements == count,
            "CUDA Hybrid MAC extent");
    c_->healthy();
    const uint64_t *dp[1] = {d.data}, *kbp[1] = {kb.data}, *kap[1] = {ka.data};
    check(ntt_b200_hybrid_mac_digits(c_->ctx, layout.active_q, b.data, a.data, dp, kbp, kap, 1, 0,
                                     first_digit ? 0 : 1, c_->stream));
  }
  void hybrid_rotate(transport::Buffer &out_b, transport::Buffer &out_a, const transport::Buffer &extended_b,
                     const transport::Buffer &extended_a, const transport::Buffer &c0, size_t c0_offset,
                     const transport::Buffer &, const PolynomialLayout &layout, uint32_t automorphism) override {
    const auto &b = buf(out_b), &a = buf(out_a), &eb = buf(extended_b), &ea = buf(extended_a), &first = buf(c0);
    const size_t elements = bytes(layout) / sizeof(uint64_t), n = layout.parameters->n();
    require(b.elements == elements && a.elements == elements && eb.elements == elements && ea.elements == elements &&
                c0_offset <= first.elements && layout.active_q * n <= first.elements - c0_offset,
            "CUDA Hybrid rotation extent");
    c_->healthy();
    check(ntt_b200_hybrid_rotate(c_->ctx, layout.active_q, b.data, a.data, eb.data, ea.data, first.data + c0_offset,
                                 automorphism, c_->stream));
  }
  void switch_basis(transport::Buffer &out, const transport::Buffer &input, size_t offset, const transport::Buffer &,
                    const PolynomialLayout &source, const PolynomialLayout &target) override {
    const auto &a = buf(out), &b = buf(input);
    const size_t n = target.parameters->n(), s = source.towers.size(), t = target.towers.size();
    require(a.elements == n * t && offset <= b.elements && n * s <= b.elements - offset, "CUDA basis extent");
    c_->healthy();
    const auto sid = c_->ids(source), tid = c_->ids(target);
    check(ntt_b200_switch_basis(c_->ctx, a.data, b.data + offset, sid.data(), s, tid.data(), t, c_->stream));
  }
  void correct(transport::Buffer &out, const transport::Buffer &left, size_t left_offset,
               const transport::Buffer &right, size_t right_offset, const transport::Buffer &,
               const PolynomialLayout &p) override {
    const auto &a = buf(out), &b = buf(left), &r = buf(right);
    require(a.elements == p.parameters->n() * p.towers.size() && left_offset <= b.elements &&
                a.elements <= b.elements - left_offset && right_offset <= r.elements &&
                a.elements <= r.elements - right_offset,
            "CUDA correction extent");
    require(p.towers == q_prefix(*p.parameters, p.towers.size()), "correction applies to the active Q prefix");
    c_->healthy();
    check(ntt_b200_correct(c_->ctx, p.towers.size(), a.data, b.data + left_offset, r.data + right_offset,
                           c_->stream));
  }
  void download(std::span<uint64_t> target, const transport::Buffer &input, size_t offset) override {
    const auto &a = buf(input);
    require(offset <= a.elements && target.size() <= a.elements - offset, "CUDA download extent");
    c_->healthy();
    check(ntt_b200_memcpy(target.data(), a.data + offset, target.size_bytes(), 2, c_->stream));
  }
  void record(transport::Event &e) override {
    auto &x = ev(e);
    c_->healthy();
    check(ntt_b200_event_record(x.event, c_->stream));
    x.recorded = true;
  }
  bool ready(transport::Event &e) override {
    auto &x = ev(e);
    require(x.recorded, "unrecorded CUDA event");
    c_->healthy();
    const int rc = ntt_b200_event_query(x.event);
    if (rc == NTT_B200_NOT_READY) return false;
    check(rc);
    return true;
  }
  void wait(transport::Event &e) override {
    auto &x = ev(e);
    require(x.recorded, "unrecorded CUDA event");
    c_->healthy();
    check(ntt_b200_event_synchronize(x.event));
  }
  bool quiesce() noexcept override { return ntt_b200_stream_synchronize(c_->stream) == NTT_B200_OK; }

  // ---- fused pipelines ---------------------------------------------------------------
  bool fused() const override { return true; }
  void fused_mod_up(transport::Buffer &out, const transport::Buffer &in, size_t offset,
                    const PolynomialLayout &in_layout) override {
    const auto &a = buf(out), &b = buf(in);
    c_->healthy();
    auto ws = scratch(NTT_B200_OP_MOD_UP, in_layout.active_q);
    check(ntt_b200_mod_up(c_->ctx, in_layout.active_q, a.data, b.data + offset,
                          in_layout.domain == Domain::Evaluation ? 1 : 0, ws.region->ptr, ws.bytes, c_->stream));
  }
  void fused_mod_down(transport::Buffer &out, const transport::Buffer &in, size_t offset,
                      const PolynomialLayout &in_layout) override {
    const auto &a = buf(out), &b = buf(in);
    c_->healthy();
    auto ws = scratch(NTT_B200_OP_MOD_DOWN, in_layout.active_q);
    check(ntt_b200_mod_down(c_->ctx, in_layout.active_q, a.data, b.data + offset, ws.region->ptr, ws.bytes,
                            c_->stream));
  }
  void fused_hybrid_digits(std::span<transport::Buffer *const> outs, const transport::Buffer &in, size_t offset,
                           const PolynomialLayout &in_layout) override {
    const size_t level = in_layout.active_q, tq = level + c_->k, n = in_layout.parameters->n();
    const auto &first = buf(*outs.front());
    for (size_t d = 0; d < outs.size(); ++d)
      require(buf(*outs[d]).data == first.data + d * tq * n, "Hybrid digits must share one contiguous region");
    c_->healthy();
    auto ws = scratch(NTT_B200_OP_DIGITS, level);
    check(ntt_b200_hybrid_digits(c_->ctx, level, first.data, buf(in).data + offset, ws.region->ptr, ws.bytes,
                                 c_->stream));
  }
  void fused_hybrid_accumulate(transport::Buffer &result_b, transport::Buffer &result_a,
                               std::span<const transport::Buffer *const> digits,
                               std::span<const transport::Buffer *const> key_b,
                               std::span<const transport::Buffer *const> key_a,
                               const PolynomialLayout &layout) override {
    std::vector<const uint64_t *> d, kb, ka;
    for (size_t i = 0; i < digits.size(); ++i) {
      d.push_back(buf(*digits[i]).data);
      kb.push_back(buf(*key_b[i]).data);
      ka.push_back(buf(*key_a[i]).data);
    }
    c_->healthy();
    check(ntt_b200_hybrid_mac_digits(c_->ctx, layout.active_q, buf(result_b).data, buf(result_a).data, d.data(),
                                     kb.data(), ka.data(), d.size(), 0, 0, c_->stream));
  }
};
}  // namespace b200_impl

Session make_cuda_session(const PolynomialLayout &p, int device, Limits limits) {
  proposal::validate(p);
  proposal::require(p.domain == proposal::Domain::Coefficient && p.order == proposal::Order::Natural &&
                        p.parameters->n() <= 65536 && p.towers.size() <= 65535 && device >= 0 && limits.operations,
                    "unsupported resident CUDA session");
  return Session(std::make_shared<b200_impl::Driver>(p, device), limits);
}
}  // namespace ntt::resident
