/*
 * CPU oracle (test infrastructure only; see oracle.h). Plain C restatement of
 * minnow54426/ntt-gpu's CPU algorithms, each function citing the reference
 * file:line it follows. Exact 128-bit integer arithmetic throughout.
 */
#include "oracle.h"

#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;

/* ---- exact modular arithmetic -------------------------------------------
 * Contract: docs/modular-arithmetic-contract.md:25-31 (table) and :49-70
 * (why intermediates fit). add/sub take canonical operands with q < 2^63;
 * mul forms the full 128-bit product before the remainder. */
uint64_t orc_add_mod(uint64_t a, uint64_t b, uint64_t q) {
  const u128 sum = (u128)a + b;
  return (uint64_t)(sum >= q ? sum - q : sum);
}

uint64_t orc_sub_mod(uint64_t a, uint64_t b, uint64_t q) {
  return a >= b ? a - b : a + (q - b);
}

uint64_t orc_mul_mod(uint64_t a, uint64_t b, uint64_t q) {
  return (uint64_t)(((u128)a * b) % q);
}

/* Square-and-multiply; reduces the base first and returns 1 % q for e = 0
 * (docs/modular-arithmetic-contract.md:65-67). */
uint64_t orc_pow_mod(uint64_t a, uint64_t e, uint64_t q) {
  uint64_t result = 1 % q, base = a % q;
  while (e) {
    if (e & 1) result = orc_mul_mod(result, base, q);
    base = orc_mul_mod(base, base, q);
    e >>= 1;
  }
  return result;
}

/* Fermat inverse x^(q-2) for prime q; x divisible by q is rejected
 * (docs/modular-arithmetic-contract.md:31; tests/oracle/test_arithmetic.py:76-80). */
int orc_inv_mod(uint64_t x, uint64_t q, uint64_t *out) {
  if (q < 2 || x % q == 0) return -1;
  *out = orc_pow_mod(x, q - 2, q);
  return 0;
}

/* include/ntt/shoup.hpp:7-12: floor(w * 2^64 / q) for canonical w, 1 < q < 2^63. */
int orc_shoup_precompute(uint64_t w, uint64_t q, uint64_t *out) {
  if (q <= 1 || q >= (UINT64_C(1) << 63) || w >= q) return -1;
  *out = (uint64_t)(((u128)w << 64) / q);
  return 0;
}

/* include/ntt/shoup.hpp:14-27: estimate one below at most, one subtraction. */
uint64_t orc_shoup_multiply(uint64_t x, uint64_t w, uint64_t wq, uint64_t q) {
  const uint64_t estimate = (uint64_t)(((u128)x * wq) >> 64);
  const uint64_t residual = x * w - estimate * q;
  return residual >= q ? residual - q : residual;
}

/* include/ntt/barrett.hpp:10-17: mu = floor(2^128 / q) as two words. */
int orc_barrett_precompute(uint64_t q, uint64_t *lo, uint64_t *hi) {
  if (q <= 1 || q >= (UINT64_C(1) << 63)) return -1;
  const u128 maximum = ~(u128)0;
  const u128 reciprocal = maximum / q + (maximum % q == q - 1);
  *lo = (uint64_t)reciprocal;
  *hi = (uint64_t)(reciprocal >> 64);
  return 0;
}

static uint64_t high_product(uint64_t a, uint64_t b) { return (uint64_t)(((u128)a * b) >> 64); }

/* include/ntt/barrett.hpp:23-33: low limb of high128(x * mu). */
uint64_t orc_barrett_quotient(uint64_t low, uint64_t high, uint64_t q, uint64_t lo, uint64_t hi) {
  (void)q;
  const uint64_t first = low * hi;
  const uint64_t second = high * lo;
  const uint64_t sum = first + second;
  const uint64_t middle = sum + high_product(low, lo);
  const uint64_t carry = (uint64_t)(sum < first) + (uint64_t)(middle < sum);
  return high * hi + high_product(low, hi) + high_product(high, lo) + carry;
}

/* include/ntt/barrett.hpp:39-49. */
uint64_t orc_barrett_multiply(uint64_t a, uint64_t b, uint64_t q, uint64_t lo, uint64_t hi) {
  const uint64_t low = a * b;
  const uint64_t estimate = orc_barrett_quotient(low, high_product(a, b), q, lo, hi);
  const uint64_t residual = low - estimate * q;
  return residual >= q ? residual - q : residual;
}

/* include/ntt/bitrev.hpp:22-38. */
uint64_t orc_log2(uint64_t n) {
  uint64_t lg = 0;
  while ((UINT64_C(1) << lg) < n) ++lg;
  return lg;
}

uint64_t orc_bit_reverse(uint64_t x, uint64_t lg) {
  uint64_t r = 0;
  for (uint64_t i = 0; i < lg; ++i) {
    r = (r << 1) | (x & 1);
    x >>= 1;
  }
  return r;
}

/* ---- parameter search: include/ntt/param_gen.hpp:29-95 ------------------ */
static const uint64_t kMillerRabinBases[12] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};

int orc_is_prime(uint64_t n) {
  if (n < 2) return 0;
  for (int i = 0; i < 12; ++i)
    if (n % kMillerRabinBases[i] == 0) return n == kMillerRabinBases[i];
  uint64_t d = n - 1, s = 0;
  while ((d & 1) == 0) {
    d >>= 1;
    ++s;
  }
  for (int i = 0; i < 12; ++i) {
    uint64_t x = orc_pow_mod(kMillerRabinBases[i] % n, d, n);
    if (x == 1 || x == n - 1) continue;
    int witness = 1;
    for (uint64_t r = 0; r + 1 < s; ++r) {
      x = orc_mul_mod(x, x, n);
      if (x == n - 1) {
        witness = 0;
        break;
      }
    }
    if (witness) return 0;
  }
  return 1;
}

/* param_gen.hpp:64-77: ascending walk from the first 2n-multiple + 1 above 2^(bits-1). */
int orc_find_primes(uint64_t n, uint64_t count, uint64_t bits, uint64_t *out) {
  if (bits < 2 || bits > 63 || n == 0) return -1;
  const uint64_t step = 2 * n;
  uint64_t q = ((UINT64_C(1) << (bits - 1)) / step + 1) * step + 1;
  uint64_t found = 0;
  while (found < count) {
    if (q >= (UINT64_C(1) << bits)) return -1;
    if (orc_is_prime(q)) out[found++] = q;
    q += step;
  }
  return 0;
}

/* param_gen.hpp:82-95: xorshift candidate walk, accept zeta^n == q-1. */
uint64_t orc_find_psi(uint64_t q, uint64_t n) {
  uint64_t s = q ^ n;
  if (s == 0) s = 1;
  for (;;) {
    s ^= s << 13;
    s ^= s >> 7;
    s ^= s << 17;
    const uint64_t g = 2 + s % (q - 3);
    const uint64_t zeta = orc_pow_mod(g, (q - 1) / (2 * n), q);
    if (orc_pow_mod(zeta, n, q) == q - 1) return zeta;
  }
}

/* ---- negacyclic NTT: include/ntt/ntt.hpp ---------------------------------- */
/* Constructor checks, ntt.hpp:57-79. */
int orc_ntt_check(uint64_t n, uint64_t q, uint64_t psi) {
  if (n < 2 || (n & (n - 1)) != 0) return -1;
  if (q < 2 || (q - 1) % (2 * n) != 0) return -1;
  if (orc_pow_mod(psi, n, q) != q - 1) return -1;
  if (q <= n) return -1;
  return 0;
}

/* DIF forward, ntt.hpp:96-121: natural coefficients in, bit-reversed
 * evaluations at psi^(2j+1) out. */
int orc_ntt_forward(uint64_t *values, uint64_t n, uint64_t q, uint64_t psi) {
  if (orc_ntt_check(n, q, psi)) return -1;
  for (uint64_t d = n / 2; d >= 1; d >>= 1) {
    const uint64_t ladder = orc_pow_mod(psi, d, q);
    const uint64_t step = orc_pow_mod(psi, n / d, q);
    for (uint64_t start = 0; start < n; start += 2 * d) {
      uint64_t w = 1;
      for (uint64_t j = 0; j < d; ++j) {
        const uint64_t upper = start + j, lower = upper + d;
        const uint64_t u = values[upper];
        const uint64_t v = orc_mul_mod(ladder, values[lower], q);
        values[upper] = orc_add_mod(u, v, q);
        values[lower] = orc_mul_mod(orc_sub_mod(u, v, q), w, q);
        w = orc_mul_mod(w, step, q);
      }
    }
  }
  return 0;
}

/* DIT inverse with the final n^-1 scale, ntt.hpp:130-158. */
int orc_ntt_inverse(uint64_t *values, uint64_t n, uint64_t q, uint64_t psi) {
  if (orc_ntt_check(n, q, psi)) return -1;
  uint64_t n_inv, psi_inv;
  if (orc_inv_mod(n % q, q, &n_inv) || orc_inv_mod(psi, q, &psi_inv)) return -1;
  for (uint64_t d = 1; d <= n / 2; d <<= 1) {
    const uint64_t ladder = orc_pow_mod(psi_inv, d, q);
    const uint64_t step = orc_pow_mod(psi_inv, n / d, q);
    for (uint64_t start = 0; start < n; start += 2 * d) {
      uint64_t w = 1;
      for (uint64_t j = 0; j < d; ++j) {
        const uint64_t upper = start + j, lower = upper + d;
        const uint64_t u = values[upper];
        const uint64_t v = orc_mul_mod(values[lower], w, q);
        values[upper] = orc_add_mod(u, v, q);
        values[lower] = orc_mul_mod(orc_sub_mod(u, v, q), ladder, q);
        w = orc_mul_mod(w, step, q);
      }
    }
  }
  for (uint64_t i = 0; i < n; ++i) values[i] = orc_mul_mod(values[i], n_inv, q);
  return 0;
}

int orc_ntt_towers(uint64_t *values, uint64_t n, size_t towers, const uint64_t *q,
                   const uint64_t *psi, int inverse) {
  for (size_t t = 0; t < towers; ++t) {
    const int rc = inverse ? orc_ntt_inverse(values + t * n, n, q[t], psi[t])
                           : orc_ntt_forward(values + t * n, n, q[t], psi[t]);
    if (rc) return rc;
  }
  return 0;
}

/* ---- approximate CRT: include/ntt/basis_conversion.hpp -------------------- */
static int cmp_u64(const void *a, const void *b) {
  const uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
  return x < y ? -1 : x > y;
}

/* Plan admission, basis_conversion.hpp:39-53. */
static int basis_plan_check(const uint64_t *source, size_t s, const uint64_t *target, size_t t) {
  if (s == 0 || s > 40 || t == 0 || t > 40) return -1;
  uint64_t all[80];
  memcpy(all, source, s * sizeof(uint64_t));
  memcpy(all + s, target, t * sizeof(uint64_t));
  qsort(all, s + t, sizeof(uint64_t), cmp_u64);
  for (size_t i = 1; i < s + t; ++i)
    if (all[i] == all[i - 1]) return -1;
  for (size_t i = 0; i < s + t; ++i)
    if (all[i] < 3 || all[i] >= (UINT64_C(1) << 63) || !orc_is_prime(all[i])) return -1;
  return 0;
}

/* Tables (basis_conversion.hpp:55-73) and the per-coefficient unreduced sum
 * (basis_conversion.hpp:13-30); input validation basis_conversion.hpp:91-100. */
int orc_basis_convert(const uint64_t *input, uint64_t n, const uint64_t *source,
                      size_t source_count, const uint64_t *target, size_t target_count,
                      uint64_t *out) {
  if (basis_plan_check(source, source_count, target, target_count)) return -1;
  if (n < 2 || n > 65536 || (n & (n - 1))) return -1;
  for (size_t s = 0; s < source_count; ++s)
    for (uint64_t i = 0; i < n; ++i)
      if (input[s * n + i] >= source[s]) return -1;

  uint64_t inverses[40], quotients[40], hats[40 * 40];
  for (size_t s = 0; s < source_count; ++s) {
    const uint64_t modulus = source[s];
    uint64_t hat = 1;
    for (size_t o = 0; o < source_count; ++o)
      if (o != s) hat = orc_mul_mod(hat, source[o] % modulus, modulus);
    if (orc_inv_mod(hat, modulus, &inverses[s])) return -1;
    if (orc_shoup_precompute(inverses[s], modulus, &quotients[s])) return -1;
    for (size_t t = 0; t < target_count; ++t) {
      uint64_t reduced = 1;
      for (size_t o = 0; o < source_count; ++o)
        if (o != s) reduced = orc_mul_mod(reduced, source[o] % target[t], target[t]);
      hats[s * target_count + t] = reduced;
    }
  }
  for (size_t t = 0; t < target_count; ++t) {
    const uint64_t m = target[t];
    for (uint64_t i = 0; i < n; ++i) {
      uint64_t sum = 0;
      for (size_t s = 0; s < source_count; ++s) {
        const uint64_t scaled = orc_shoup_multiply(input[s * n + i], inverses[s], quotients[s], source[s]);
        const uint64_t term = orc_mul_mod(scaled % m, hats[s * target_count + t], m);
        sum = orc_add_mod(sum, term, m);
      }
      out[t * n + i] = sum;
    }
  }
  return 0;
}

/* include/ntt/resident_conversion.hpp:15-20. */
uint64_t orc_automorphism_source_index(uint64_t destination, uint64_t n, uint64_t log_n,
                                       uint32_t automorphism) {
  const uint64_t odd = 2 * orc_bit_reverse(destination, log_n) + 1;
  const uint64_t source = (odd * automorphism) & (2 * n - 1);
  return orc_bit_reverse(source / 2, log_n);
}

/* ---- Hybrid chain: src/resident.cpp ---------------------------------------- */
/* Parameters::create (include/ntt/backend_contract.hpp:48-66), the session's
 * N <= 65536 bound (src/resident.cpp:98) and conversion_input's 40-tower
 * limits (src/resident.cpp:113-123). */
int orc_context_check(const orc_context *ctx, size_t level) {
  const uint64_t n = ctx->n;
  if (n < 2 || (n & (n - 1)) || n > 65536) return -1;
  if (ctx->m == 0 || ctx->alpha == 0 || ctx->alpha > ctx->m) return -1;
  if (ctx->k == 0 || ctx->k > 40) return -1;
  if (level == 0 || level > ctx->m || level > 40) return -1;
  const size_t total = ctx->m + ctx->k;
  for (size_t i = 0; i < total; ++i) {
    const uint64_t q = i < ctx->m ? ctx->q[i] : ctx->p[i - ctx->m];
    const uint64_t psi = i < ctx->m ? ctx->q_psi[i] : ctx->p_psi[i - ctx->m];
    if (q <= n || q >= (UINT64_C(1) << 63) || q % (2 * n) != 1) return -1;
    if (!orc_is_prime(q)) return -1;
    if (psi == 0 || psi >= q || orc_pow_mod(psi, n, q) != q - 1) return -1;
    for (size_t j = 0; j < i; ++j) {
      const uint64_t other = j < ctx->m ? ctx->q[j] : ctx->p[j - ctx->m];
      if (other == q) return -1;
    }
  }
  return 0;
}

/* Active digit count 1 + (L-1)/alpha (src/resident.cpp:466-468, 536). */
size_t orc_digit_count(const orc_context *ctx, size_t level) {
  return 1 + (level - 1) / ctx->alpha;
}

static void qp_moduli(const orc_context *ctx, size_t level, uint64_t *mod, uint64_t *psi) {
  for (size_t i = 0; i < level; ++i) {
    mod[i] = ctx->q[i];
    psi[i] = ctx->q_psi[i];
  }
  for (size_t j = 0; j < ctx->k; ++j) {
    mod[level + j] = ctx->p[j];
    psi[level + j] = ctx->p_psi[j];
  }
}

/* resident.cpp:431-447: coefficient or evaluation Q in, evaluation QP out:
 * join(eval Q, forward(switch_basis(coeff Q -> P))). */
int orc_mod_up(const orc_context *ctx, size_t level, const uint64_t *input, int input_is_eval,
               uint64_t *out) {
  if (orc_context_check(ctx, level)) return -1;
  const uint64_t n = ctx->n;
  const size_t qn = level * n;
  uint64_t *coeff = malloc(qn * sizeof(uint64_t));
  if (!coeff) return -1;
  int rc = 0;
  memcpy(coeff, input, qn * sizeof(uint64_t));
  memcpy(out, input, qn * sizeof(uint64_t));
  if (input_is_eval)
    rc = orc_ntt_towers(coeff, n, level, ctx->q, ctx->q_psi, 1);
  else
    rc = orc_ntt_towers(out, n, level, ctx->q, ctx->q_psi, 0);
  if (!rc) rc = orc_basis_convert(coeff, n, ctx->q, level, ctx->p, ctx->k, out + qn);
  if (!rc) rc = orc_ntt_towers(out + qn, n, ctx->k, ctx->p, ctx->p_psi, 0);
  free(coeff);
  return rc;
}

/* resident.cpp:448-457 with Session::correct (resident.cpp:404-430) and
 * resident_correction_value (resident_conversion.hpp:45-49):
 * (Z_q - NTT(switch(INTT(Z_p))))·[P^-1]_q. */
int orc_mod_down(const orc_context *ctx, size_t level, const uint64_t *input, uint64_t *out) {
  if (orc_context_check(ctx, level)) return -1;
  const uint64_t n = ctx->n;
  const size_t qn = level * n, pn = ctx->k * n;
  uint64_t *p_part = malloc(pn * sizeof(uint64_t));
  uint64_t *corr = malloc(qn * sizeof(uint64_t));
  int rc = (!p_part || !corr) ? -1 : 0;
  if (!rc) {
    memcpy(p_part, input + qn, pn * sizeof(uint64_t));
    rc = orc_ntt_towers(p_part, n, ctx->k, ctx->p, ctx->p_psi, 1);
  }
  if (!rc) rc = orc_basis_convert(p_part, n, ctx->p, ctx->k, ctx->q, level, corr);
  if (!rc) rc = orc_ntt_towers(corr, n, level, ctx->q, ctx->q_psi, 0);
  for (size_t t = 0; !rc && t < level; ++t) {
    const uint64_t q = ctx->q[t];
    uint64_t product = 1, p_inv; /* special_prime_product, resident_conversion.hpp:8-13 */
    for (size_t j = 0; j < ctx->k; ++j) product = orc_mul_mod(product, ctx->p[j] % q, q);
    if (orc_inv_mod(product, q, &p_inv)) {
      rc = -1;
      break;
    }
    for (uint64_t i = 0; i < n; ++i)
      out[t * n + i] = orc_mul_mod(orc_sub_mod(input[t * n + i], corr[t * n + i], q), p_inv, q);
  }
  free(p_part);
  free(corr);
  return rc;
}

/* resident.cpp:458-491: for each digit, INTT its <= alpha source towers, lift
 * the coefficients to every complement tower (active Q outside the digit, then
 * P) and forward-transform them; keep the digit's own evaluations in place.
 * The reference splits complements into <= 40-tower chunks (resident.cpp:474-483);
 * each target tower is computed independently, so chunking does not change values. */
int orc_hybrid_digits(const orc_context *ctx, size_t level, const uint64_t *input,
                      uint64_t *digits) {
  if (orc_context_check(ctx, level)) return -1;
  const uint64_t n = ctx->n;
  const size_t total = level + ctx->k;
  uint64_t mod[80], psi[80];
  qp_moduli(ctx, level, mod, psi);
  uint64_t *coeff = malloc(ctx->alpha * n * sizeof(uint64_t));
  uint64_t *converted = malloc(total * n * sizeof(uint64_t));
  if (!coeff || !converted) {
    free(coeff);
    free(converted);
    return -1;
  }
  int rc = 0;
  size_t digit = 0;
  for (size_t first = 0; first < level && !rc; first += ctx->alpha, ++digit) {
    const size_t count = ctx->alpha < level - first ? ctx->alpha : level - first;
    uint64_t *out = digits + digit * total * n;
    memcpy(coeff, input + first * n, count * n * sizeof(uint64_t));
    rc = orc_ntt_towers(coeff, n, count, ctx->q + first, ctx->q_psi + first, 1);
    /* complement moduli in QP order */
    uint64_t tmod[80], tpsi[80];
    size_t targets = 0;
    for (size_t t = 0; t < total; ++t)
      if (t < first || t >= first + count) {
        tmod[targets] = mod[t];
        tpsi[targets] = psi[t];
        ++targets;
      }
    for (size_t chunk = 0; chunk < targets && !rc; chunk += 40) {
      const size_t c = targets - chunk < 40 ? targets - chunk : 40;
      rc = orc_basis_convert(coeff, n, ctx->q + first, count, tmod + chunk, c, converted + chunk * n);
      if (!rc) rc = orc_ntt_towers(converted + chunk * n, n, c, tmod + chunk, tpsi + chunk, 0);
    }
    size_t next = 0;
    for (size_t t = 0; t < total && !rc; ++t) {
      if (t >= first && t < first + count)
        memcpy(out + t * n, input + t * n, n * sizeof(uint64_t));
      else
        memcpy(out + t * n, converted + (next++) * n, n * sizeof(uint64_t));
    }
  }
  free(coeff);
  free(converted);
  return rc;
}

/* key_indices (backend_contract.hpp:112-119) packing of a full-context QP key
 * channel into the active QP layout (resident.cpp:512-519): Q tower i keeps
 * index i; P tower j is row M + j of the full key. */
int orc_pack_key(const orc_context *ctx, size_t level, const uint64_t *full_channel, uint64_t *out) {
  if (orc_context_check(ctx, level)) return -1;
  const uint64_t n = ctx->n;
  for (size_t t = 0; t < level + ctx->k; ++t) {
    const size_t row = t < level ? t : t - level + ctx->m;
    memcpy(out + t * n, full_channel + row * n, n * sizeof(uint64_t));
  }
  return 0;
}

/* resident.cpp:530-570 with hybrid_mac_value (resident_conversion.hpp:50-54):
 * the first digit assigns, later digits add. Keys are packed active QP rows,
 * one (L+K)-tower block per digit. */
int orc_hybrid_accumulate(const orc_context *ctx, size_t level, const uint64_t *digits,
                          const uint64_t *key_b, const uint64_t *key_a, uint64_t *out_b,
                          uint64_t *out_a) {
  if (orc_context_check(ctx, level)) return -1;
  const uint64_t n = ctx->n;
  const size_t total = level + ctx->k, beta = orc_digit_count(ctx, level);
  uint64_t mod[80], psi[80];
  qp_moduli(ctx, level, mod, psi);
  for (size_t d = 0; d < beta; ++d)
    for (size_t t = 0; t < total; ++t)
      for (uint64_t i = 0; i < n; ++i) {
        const size_t index = (d * total + t) * n + i, o = t * n + i;
        const uint64_t q = mod[t];
        const uint64_t pb = orc_mul_mod(digits[index], key_b[index], q);
        const uint64_t pa = orc_mul_mod(digits[index], key_a[index], q);
        out_b[o] = d == 0 ? pb : orc_add_mod(out_b[o], pb, q);
        out_a[o] = d == 0 ? pa : orc_add_mod(out_a[o], pa, q);
      }
  return 0;
}

/* resident.cpp:571-617 with rotated_b_value (resident_conversion.hpp:22-29):
 * out_b[k] = ext_b[src] + [P]_q * c0[src] on Q towers, out_a[k] = ext_a[src],
 * src = automorphism_source_index(k). */
int orc_hybrid_rotate_extended(const orc_context *ctx, size_t level, const uint64_t *ext_b,
                               const uint64_t *ext_a, const uint64_t *c0, uint32_t automorphism,
                               uint64_t *out_b, uint64_t *out_a) {
  if (orc_context_check(ctx, level)) return -1;
  const uint64_t n = ctx->n, log_n = orc_log2(n);
  if (!(automorphism & 1) || automorphism >= 2 * n) return -1;
  const size_t total = level + ctx->k;
  uint64_t mod[80], psi[80];
  qp_moduli(ctx, level, mod, psi);
  for (size_t t = 0; t < total; ++t) {
    const uint64_t q = mod[t];
    uint64_t scale = 1;
    for (size_t j = 0; j < ctx->k; ++j) scale = orc_mul_mod(scale, ctx->p[j] % q, q);
    for (uint64_t k = 0; k < n; ++k) {
      const uint64_t src = t * n + orc_automorphism_source_index(k, n, log_n, automorphism);
      uint64_t b = ext_b[src];
      if (t < level) b = orc_add_mod(b, orc_mul_mod(c0[src], scale, q), q);
      out_b[t * n + k] = b;
      out_a[t * n + k] = ext_a[src];
    }
  }
  return 0;
}

/* The Hybrid core as run_hybrid_core composes it
 * (include/ntt/openfhe_hybrid_adapter.hpp:163-181): upload the active key
 * digits, digits(input), MAC, optional rotation with c0, ModDown of each
 * channel. Full keys hold 1 + (M-1)/alpha digits of (M+K) towers each. */
int orc_keyswitch(const orc_context *ctx, size_t level, const uint64_t *input,
                  const uint64_t *key_b, const uint64_t *key_a, const uint64_t *c0,
                  uint32_t automorphism, uint64_t *out_b, uint64_t *out_a) {
  if (orc_context_check(ctx, level)) return -1;
  if (c0 && (!(automorphism & 1) || automorphism >= 2 * ctx->n)) return -1;
  const uint64_t n = ctx->n;
  const size_t total = level + ctx->k, beta = orc_digit_count(ctx, level);
  const size_t full_total = ctx->m + ctx->k;
  const size_t block = total * n;
  uint64_t *digits = malloc(beta * block * sizeof(uint64_t));
  uint64_t *kb = malloc(beta * block * sizeof(uint64_t));
  uint64_t *ka = malloc(beta * block * sizeof(uint64_t));
  uint64_t *eb = malloc(block * sizeof(uint64_t));
  uint64_t *ea = malloc(block * sizeof(uint64_t));
  uint64_t *rb = c0 ? malloc(block * sizeof(uint64_t)) : NULL;
  uint64_t *ra = c0 ? malloc(block * sizeof(uint64_t)) : NULL;
  int rc = (!digits || !kb || !ka || !eb || !ea || (c0 && (!rb || !ra))) ? -1 : 0;
  for (size_t d = 0; d < beta && !rc; ++d) {
    rc = orc_pack_key(ctx, level, key_b + d * full_total * n, kb + d * block);
    if (!rc) rc = orc_pack_key(ctx, level, key_a + d * full_total * n, ka + d * block);
  }
  if (!rc) rc = orc_hybrid_digits(ctx, level, input, digits);
  if (!rc) rc = orc_hybrid_accumulate(ctx, level, digits, kb, ka, eb, ea);
  if (!rc && c0) {
    rc = orc_hybrid_rotate_extended(ctx, level, eb, ea, c0, automorphism, rb, ra);
    if (!rc) {
      memcpy(eb, rb, block * sizeof(uint64_t));
      memcpy(ea, ra, block * sizeof(uint64_t));
    }
  }
  if (!rc) rc = orc_mod_down(ctx, level, eb, out_b);
  if (!rc) rc = orc_mod_down(ctx, level, ea, out_a);
  free(digits);
  free(kb);
  free(ka);
  free(eb);
  free(ea);
  free(rb);
  free(ra);
  return rc;
}

/* ---- seeded inputs ---------------------------------------------------------
 * LCG of include/ntt/benchmark_inputs.hpp:14-20, one state step per value;
 * SplitMix64 finaliser of tests/openfhe_hybrid_tests.cpp:153-158. */
void orc_lcg_fill(uint64_t *out, uint64_t n, size_t towers, const uint64_t *moduli,
                  uint64_t seed) {
  uint64_t state = seed;
  for (size_t t = 0; t < towers; ++t)
    for (uint64_t i = 0; i < n; ++i) {
      state = state * UINT64_C(6364136223846793005) + UINT64_C(1442695040888963407);
      out[t * n + i] = state % moduli[t];
    }
}

uint64_t orc_splitmix(uint64_t x) {
  x += UINT64_C(0x9e3779b97f4a7c15);
  x = (x ^ (x >> 30)) * UINT64_C(0xbf58476d1ce4e5b9);
  x = (x ^ (x >> 27)) * UINT64_C(0x94d049bb133111eb);
  return x ^ (x >> 31);
}

void orc_splitmix_fill(uint64_t *out, uint64_t n, size_t towers, const uint64_t *moduli,
                       uint64_t seed) {
  for (size_t t = 0; t < towers; ++t)
    for (uint64_t i = 0; i < n; ++i)
      out[t * n + i] = orc_splitmix(seed + t * n + i) % moduli[t];
}
