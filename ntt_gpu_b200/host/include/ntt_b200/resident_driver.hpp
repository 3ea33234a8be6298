#pragma once
// Transport seam between the resident Session and a device (the reference's
// ntt::resident::detail::Driver, include/ntt/resident_driver.hpp:13-57). The
// B200 driver implements it over the C ABI of include/ntt_b200.h; tests inject a
// deferred CPU transport. Raw buffers and events never become public handles.
#include <atomic>
#include <stdexcept>
#include <vector>

#include "ntt_b200/resident.hpp"

namespace ntt::resident::detail {
struct Buffer {
  virtual ~Buffer() = default;
};
struct Event {
  virtual ~Event() = default;
};

class Driver {
  std::atomic<bool> attached_{false};

 public:
  Driver() = default;
  Driver(const Driver &) = delete;
  Driver &operator=(const Driver &) = delete;
  virtual ~Driver() = default;
  void attach_once() { proposal::require(!attached_.exchange(true), "transport already belongs to a session"); }

  virtual int ordinal() const = 0;
  virtual const PolynomialLayout &layout() const = 0;
  virtual size_t constant_bytes() const = 0;
  virtual std::unique_ptr<Buffer> allocate(size_t elements) = 0;
  virtual std::unique_ptr<Event> make_event() = 0;
  virtual void upload(Buffer &, std::span<const uint64_t>) = 0;
  virtual void copy(Buffer &, const Buffer &, size_t offset, size_t elements) = 0;
  virtual void copy_range(Buffer &, size_t destination_offset, const Buffer &, size_t source_offset,
                          size_t elements) = 0;
  virtual void transform(Buffer &, const PolynomialLayout &, bool inverse) = 0;
  virtual void pointwise(Buffer &, const Buffer &, size_t offset, const PolynomialLayout &) = 0;
  virtual void hybrid_mac(Buffer &result_b, Buffer &result_a, const Buffer &digit, const Buffer &key_b,
                          const Buffer &key_a, const PolynomialLayout &, bool first_digit) = 0;
  virtual void hybrid_rotate(Buffer &out_b, Buffer &out_a, const Buffer &extended_b, const Buffer &extended_a,
                             const Buffer &c0, size_t c0_offset, const Buffer &scales, const PolynomialLayout &,
                             uint32_t automorphism) = 0;
  virtual void switch_basis(Buffer &, const Buffer &, size_t source_offset, const Buffer &constants,
                            const PolynomialLayout &source, const PolynomialLayout &target) = 0;
  virtual void correct(Buffer &, const Buffer &, size_t left_offset, const Buffer &, size_t right_offset,
                       const Buffer &constants, const PolynomialLayout &) = 0;
  virtual void download(std::span<uint64_t>, const Buffer &, size_t offset) = 0;
  virtual void record(Event &) = 0;
  virtual bool ready(Event &) = 0;
  virtual void wait(Event &) = 0;
  // True proves that no queued command can still touch a pinned resource.
  virtual bool quiesce() noexcept = 0;
  virtual void check_health() const {}

  // ---- fused composites (B200 extension) -----------------------------------------
  // A driver whose fused() is true runs ModUp, ModDown, Hybrid digits and the
  // all-digit MAC as single device pipelines with its own resident tables; the
  // Session then journals each as one operation. Otherwise the Session composes
  // them from the primitives above exactly as the reference does
  // (src/resident.cpp:431-570).
  virtual bool fused() const { return false; }
  // `count` buffers of `elements` words each; a fused driver returns views of
  // one contiguous region (its single-pass MAC reads all digits with one stride).
  virtual std::vector<std::unique_ptr<Buffer>> allocate_group(size_t count, size_t elements) {
    std::vector<std::unique_ptr<Buffer>> out;
    for (size_t i = 0; i < count; ++i) out.push_back(allocate(elements));
    return out;
  }
  virtual void fused_mod_up(Buffer &, const Buffer &, size_t, const PolynomialLayout &) {
    throw std::logic_error("fused pipelines not offered by this driver");
  }
  virtual void fused_mod_down(Buffer &, const Buffer &, size_t, const PolynomialLayout &) {
    throw std::logic_error("fused pipelines not offered by this driver");
  }
  virtual void fused_hybrid_digits(std::span<Buffer *const>, const Buffer &, size_t, const PolynomialLayout &) {
    throw std::logic_error("fused pipelines not offered by this driver");
  }
  virtual void fused_hybrid_accumulate(Buffer &, Buffer &, std::span<const Buffer *const>,
                                       std::span<const Buffer *const>, std::span<const Buffer *const>,
                                       const PolynomialLayout &) {
    throw std::logic_error("fused pipelines not offered by this driver");
  }
};
}  // namespace ntt::resident::detail
