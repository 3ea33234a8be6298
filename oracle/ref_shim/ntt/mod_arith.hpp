#pragma once
// Stand-in for include/ntt/mod_arith.hpp, which minnow54426/ntt-gpu includes
// everywhere but does not ship. Used ONLY to compile the reference's own CPU
// sources into oracle/_ref (test infrastructure). Restated from the contract in
// docs/modular-arithmetic-contract.md:25-31 (operation table) and :49-70
// (widths): canonical add/sub for q < 2^63, full 128-bit product before the
// remainder, square-and-multiply pow with 1 % q for e = 0, Fermat inverse that
// rejects multiples of q with std::invalid_argument.
#include <cstdint>
#include <stdexcept>

#if !defined(NTT_HD)
#if defined(__CUDACC__)
#define NTT_HD __host__ __device__ inline
#else
#define NTT_HD inline
#endif
#endif

namespace ntt {
NTT_HD uint64_t add_mod(uint64_t a, uint64_t b, uint64_t q) {
  const unsigned __int128 sum = static_cast<unsigned __int128>(a) + b;
  return static_cast<uint64_t>(sum >= q ? sum - q : sum);
}
NTT_HD uint64_t sub_mod(uint64_t a, uint64_t b, uint64_t q) {
  return a >= b ? a - b : a + (q - b);
}
NTT_HD uint64_t mul_mod(uint64_t a, uint64_t b, uint64_t q) {
  return static_cast<uint64_t>((static_cast<unsigned __int128>(a) * b) % q);
}
NTT_HD uint64_t pow_mod(uint64_t a, uint64_t e, uint64_t q) {
  uint64_t result = 1 % q, base = a % q;
  for (; e; e >>= 1) {
    if (e & 1) result = mul_mod(result, base, q);
    base = mul_mod(base, base, q);
  }
  return result;
}
inline uint64_t inv_mod(uint64_t x, uint64_t q) {
  if (q < 2 || x % q == 0) throw std::invalid_argument("inverse of zero modulo q");
  return pow_mod(x, q - 2, q);
}
} // namespace ntt
