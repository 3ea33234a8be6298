/*
 * CPU oracle for the CKKS NTT / ModUp / ModDown / Hybrid key-switch path.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker that the CUDA path is
 * compared against; only tests, the smoke check and the benchmark's CPU
 * baseline may load it. The product never links or calls it.
 *
 * Every function restates the algorithm of minnow54426/ntt-gpu (cited by
 * file:line inside that project) in plain C with 128-bit integers:
 *   - modular arithmetic: docs/modular-arithmetic-contract.md:25-70 (the
 *     header include/ntt/mod_arith.hpp is absent from the reference tree),
 *     include/ntt/shoup.hpp:7-27, include/ntt/barrett.hpp:10-50;
 *   - parameter search: include/ntt/param_gen.hpp:29-95;
 *   - negacyclic NTT: include/ntt/ntt.hpp:57-158;
 *   - approximate CRT basis switch: include/ntt/basis_conversion.hpp:13-114;
 *   - resident helpers: include/ntt/resident_conversion.hpp:8-54;
 *   - ModUp / ModDown / Hybrid digits / MAC / rotation: src/resident.cpp:431-617.
 *
 * Layouts are limb-major: tower t of a polynomial occupies values[t*n .. t*n+n).
 * Functions return 0 on success and -1 when the reference would reject the
 * input (it throws std::invalid_argument there).
 */
#ifndef NTT_ORACLE_H
#define NTT_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- exact modular arithmetic ---------------------------------------- */
uint64_t orc_add_mod(uint64_t a, uint64_t b, uint64_t q);
uint64_t orc_sub_mod(uint64_t a, uint64_t b, uint64_t q);
uint64_t orc_mul_mod(uint64_t a, uint64_t b, uint64_t q);
uint64_t orc_pow_mod(uint64_t a, uint64_t e, uint64_t q);
int orc_inv_mod(uint64_t x, uint64_t q, uint64_t *out);
int orc_shoup_precompute(uint64_t w, uint64_t q, uint64_t *out);
uint64_t orc_shoup_multiply(uint64_t x, uint64_t w, uint64_t wq, uint64_t q);
int orc_barrett_precompute(uint64_t q, uint64_t *lo, uint64_t *hi);
uint64_t orc_barrett_quotient(uint64_t low, uint64_t high, uint64_t q, uint64_t lo, uint64_t hi);
uint64_t orc_barrett_multiply(uint64_t a, uint64_t b, uint64_t q, uint64_t lo, uint64_t hi);
uint64_t orc_bit_reverse(uint64_t x, uint64_t lg);
uint64_t orc_log2(uint64_t n);

/* ---- parameter search ------------------------------------------------- */
int orc_is_prime(uint64_t n);
int orc_find_primes(uint64_t n, uint64_t count, uint64_t bits, uint64_t *out);
uint64_t orc_find_psi(uint64_t q, uint64_t n);

/* ---- negacyclic NTT ---------------------------------------------------- */
int orc_ntt_check(uint64_t n, uint64_t q, uint64_t psi);
int orc_ntt_forward(uint64_t *values, uint64_t n, uint64_t q, uint64_t psi);
int orc_ntt_inverse(uint64_t *values, uint64_t n, uint64_t q, uint64_t psi);
int orc_ntt_towers(uint64_t *values, uint64_t n, size_t towers, const uint64_t *q,
                   const uint64_t *psi, int inverse);

/* ---- approximate CRT basis switch ------------------------------------- */
int orc_basis_convert(const uint64_t *input, uint64_t n, const uint64_t *source,
                      size_t source_count, const uint64_t *target, size_t target_count,
                      uint64_t *out);

/* ---- resident helpers -------------------------------------------------- */
uint64_t orc_automorphism_source_index(uint64_t destination, uint64_t n, uint64_t log_n,
                                       uint32_t automorphism);

/* ---- CKKS Hybrid chain --------------------------------------------------
 * A context is (n, M full Q towers, K P towers, alpha). Active level L is a
 * prefix q[0..L). QP order is active Q then all P. */
typedef struct {
  uint64_t n;
  size_t m, k, alpha;
  const uint64_t *q, *q_psi; /* m entries */
  const uint64_t *p, *p_psi; /* k entries */
} orc_context;

int orc_context_check(const orc_context *ctx, size_t level);
size_t orc_digit_count(const orc_context *ctx, size_t level);
int orc_mod_up(const orc_context *ctx, size_t level, const uint64_t *input, int input_is_eval,
               uint64_t *out);
int orc_mod_down(const orc_context *ctx, size_t level, const uint64_t *input, uint64_t *out);
int orc_hybrid_digits(const orc_context *ctx, size_t level, const uint64_t *input,
                      uint64_t *digits);
int orc_pack_key(const orc_context *ctx, size_t level, const uint64_t *full_channel,
                 uint64_t *out);
int orc_hybrid_accumulate(const orc_context *ctx, size_t level, const uint64_t *digits,
                          const uint64_t *key_b, const uint64_t *key_a, uint64_t *out_b,
                          uint64_t *out_a);
int orc_hybrid_rotate_extended(const orc_context *ctx, size_t level, const uint64_t *ext_b,
                               const uint64_t *ext_a, const uint64_t *c0, uint32_t automorphism,
                               uint64_t *out_b, uint64_t *out_a);
int orc_keyswitch(const orc_context *ctx, size_t level, const uint64_t *input,
                  const uint64_t *key_b, const uint64_t *key_a, const uint64_t *c0,
                  uint32_t automorphism, uint64_t *out_b, uint64_t *out_a);

/* ---- seeded inputs ----------------------------------------------------- */
void orc_lcg_fill(uint64_t *out, uint64_t n, size_t towers, const uint64_t *moduli,
                  uint64_t seed);
uint64_t orc_splitmix(uint64_t x);
void orc_splitmix_fill(uint64_t *out, uint64_t n, size_t towers, const uint64_t *moduli,
                       uint64_t seed);

#ifdef __cplusplus
}
#endif
#endif
