/* CPU oracle: GF(2^128) and prime-field arithmetic. Test infrastructure only. */
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

/* Set by o_set_clmul_mode(): 0 = per-bit loop (crates/field/src/gf128/portable.rs:11-24,
 * the reference's x86 kernel), 1 = PCLMULQDQ (same products, for the fast baseline). */
static int g_clmul_mode = 0;
void o_set_clmul_mode(int mode) { g_clmul_mode = mode; }

#if defined(__x86_64__)
#include <wmmintrin.h>
__attribute__((target("pclmul,sse2"))) static void clmul64_hw(uint64_t a, uint64_t b,
                                                              uint64_t *lo, uint64_t *hi) {
  __m128i x = _mm_set_epi64x(0, (long long)a), y = _mm_set_epi64x(0, (long long)b);
  __m128i r = _mm_clmulepi64_si128(x, y, 0);
  *lo = (uint64_t)_mm_cvtsi128_si64(r);
  *hi = (uint64_t)_mm_cvtsi128_si64(_mm_unpackhi_epi64(r, r));
}
#endif

/* portable.rs:11-24: schoolbook over the bits of b. */
static void clmul64(uint64_t a, uint64_t b, uint64_t *lo, uint64_t *hi) {
#if defined(__x86_64__)
  if (g_clmul_mode) {
    clmul64_hw(a, b, lo, hi);
    return;
  }
#endif
  uint64_t l = 0, h = 0;
  for (int i = 0; i < 64; i++) {
    if ((b >> i) & 1) {
      l ^= a << i;
      if (i > 0) h ^= a >> (64 - i);
    }
  }
  *lo = l;
  *hi = h;
}

/* portable.rs:28-35 */
o_wide o_gf_mul_wide(o_f128 a, o_f128 b) {
  uint64_t l0, l1, h0, h1, m0, m1, n0, n1;
  clmul64(a.lo, b.lo, &l0, &l1);
  clmul64(a.hi, b.hi, &h0, &h1);
  clmul64(a.lo, b.hi, &m0, &m1);
  clmul64(a.hi, b.lo, &n0, &n1);
  o_wide w = {{l0, l1 ^ m0 ^ n0, h0 ^ m1 ^ n1, h1}};
  return w;
}

/* portable.rs:37-61: fold X^128 = X^7+X^2+X+1 twice. */
static void times_g(uint64_t w, uint64_t *lo, uint64_t *hi) {
  *lo = w ^ (w << 1) ^ (w << 2) ^ (w << 7);
  *hi = (w >> 63) ^ (w >> 62) ^ (w >> 57);
}

o_f128 o_gf_reduce(o_wide r) {
  uint64_t a0, a1, b0, b1;
  times_g(r.w[2], &a0, &a1);
  times_g(r.w[3], &b0, &b1);
  uint64_t w0 = r.w[0] ^ a0;
  uint64_t w1 = r.w[1] ^ a1 ^ b0;
  o_f128 out = {w0 ^ b1 ^ (b1 << 1) ^ (b1 << 2) ^ (b1 << 7), w1};
  return out;
}

o_f128 o_gf_mul(o_f128 a, o_f128 b) { return o_gf_reduce(o_gf_mul_wide(a, b)); }

o_f128 o_gf_square(o_f128 a) { return o_gf_mul(a, a); }

static o_f128 sqn(o_f128 a, int k) {
  for (int i = 0; i < k; i++) a = o_gf_square(a);
  return a;
}

/* pow.rs:87-103: Itoh-Tsujii addition chain. */
o_f128 o_gf_inv(o_f128 a) {
  o_f128 b1 = a;
  o_f128 b2 = o_gf_mul(sqn(b1, 1), b1);
  o_f128 b3 = o_gf_mul(sqn(b2, 1), b1);
  o_f128 b6 = o_gf_mul(sqn(b3, 3), b3);
  o_f128 b12 = o_gf_mul(sqn(b6, 6), b6);
  o_f128 b24 = o_gf_mul(sqn(b12, 12), b12);
  o_f128 b48 = o_gf_mul(sqn(b24, 24), b24);
  o_f128 b96 = o_gf_mul(sqn(b48, 48), b48);
  o_f128 b120 = o_gf_mul(sqn(b96, 24), b24);
  o_f128 b126 = o_gf_mul(sqn(b120, 6), b6);
  o_f128 b127 = o_gf_mul(sqn(b126, 1), b1);
  return o_gf_square(b127);
}

/* pow.rs:40-53: square and multiply, low bit first. */
o_f128 o_gf_pow(o_f128 a, u128 e) {
  o_f128 acc = {1, 0};
  o_f128 base = a;
  while (e) {
    if (e & 1) acc = o_gf_mul(acc, base);
    base = o_gf_square(base);
    e >>= 1;
  }
  return acc;
}

/* pow.rs:27-28,112-117: primitive-element test against the nine prime factors. */
int o_gf_is_generator(o_f128 a) {
  static const uint64_t f[9] = {3, 5, 17, 257, 641, 65537, 274177, 6700417, 67280421310721ull};
  if (a.lo == 0 && a.hi == 0) return 0;
  for (int i = 0; i < 9; i++) {
    u128 order = ~(u128)0;
    o_f128 r = o_gf_pow(a, order / f[i]);
    if (r.lo == 1 && r.hi == 0) return 0;
  }
  return 1;
}

/* pow.rs:122-127 */
o_f128 o_gf_smallest_generator(void) {
  for (uint64_t n = 2;; n++) {
    o_f128 a = {n, 0};
    if (o_gf_is_generator(a)) return a;
  }
}

/* pow.rs:153-199: table[i][d] = base^(d * 2^(win*i)). */
void o_comb_init(o_comb *c, o_f128 base, int win) {
  c->win = win;
  c->windows = (128 + win - 1) / win;
  size_t per = (size_t)1 << win;
  c->table = (o_f128 *)malloc(sizeof(o_f128) * per * c->windows);
  o_f128 b = base;
  for (int i = 0; i < c->windows; i++) {
    o_f128 cur = {1, 0};
    for (size_t d = 0; d < per; d++) {
      c->table[i * per + d] = cur;
      cur = o_gf_mul(cur, b);
    }
    b = sqn(b, win);
  }
}

void o_comb_free(o_comb *c) { free(c->table); }

o_f128 o_comb_pow(const o_comb *c, u128 e) {
  o_f128 acc = {1, 0};
  size_t per = (size_t)1 << c->win;
  u128 mask = per - 1;
  int i = 0;
  while (e) {
    u128 d = e & mask;
    if (d) acc = o_gf_mul(acc, c->table[i * per + (size_t)d]);
    e >>= c->win;
    i++;
  }
  return acc;
}

/* crates/poly/src/eq.rs:63-98: entry j = prod_i (r_i if bit i of j else 1 - r_i). */
void o_gf_eq_table(const o_f128 *r, int n, o_f128 *out) {
  out[0].lo = 1;
  out[0].hi = 0;
  for (int i = 0; i < n; i++) {
    size_t half = (size_t)1 << i;
    for (size_t k = 0; k < half; k++) {
      o_f128 p = out[k];
      o_f128 one = o_gf_mul(p, r[i]);
      out[k].lo = p.lo ^ one.lo;
      out[k].hi = p.hi ^ one.hi;
      out[k + half] = one;
    }
  }
}

/* crates/poly/src/mle.rs:174-200: fold the lowest variable first. */
o_f128 o_gf_mle_eval(const o_f128 *v, const o_f128 *point, int nvars) {
  size_t n = (size_t)1 << nvars;
  o_f128 *t = (o_f128 *)malloc(sizeof(o_f128) * n);
  memcpy(t, v, sizeof(o_f128) * n);
  for (int i = 0; i < nvars; i++) {
    size_t h = n >> (i + 1);
    for (size_t k = 0; k < h; k++) {
      o_f128 a = t[2 * k], b = t[2 * k + 1];
      o_f128 d = {a.lo ^ b.lo, a.hi ^ b.hi};
      o_f128 m = o_gf_mul(point[i], d);
      t[k].lo = a.lo ^ m.lo;
      t[k].hi = a.hi ^ m.hi;
    }
  }
  o_f128 r = t[0];
  free(t);
  return r;
}

/* ------------------------------------------------------------ prime field */

/* crates/field/src/helpers.rs:74-85 */
static void mul_wide(u128 a, u128 b, u128 *lo, u128 *hi) {
  u128 alo = (uint64_t)a, ahi = a >> 64, blo = (uint64_t)b, bhi = b >> 64;
  u128 ll = alo * blo, hh = ahi * bhi;
  u128 m1 = alo * bhi, m2 = ahi * blo;
  u128 mid = m1 + m2;
  u128 mid_carry = mid < m1;
  u128 l = ll + (mid << 64);
  u128 lo_carry = l < ll;
  *lo = l;
  *hi = hh + (mid >> 64) + (mid_carry << 64) + lo_carry;
}

static u128 shr_wide(u128 lo, u128 hi, unsigned n) {
  return n == 0 ? lo : (lo >> n) | (hi << (128 - n));
}

/* helpers.rs:103-120: floor(2^(2k)/q). */
static u128 barrett_mu(u128 q, unsigned k) {
  u128 rem = 0, quo = 0;
  for (int i = 2 * (int)k;; i--) {
    rem = (rem << 1) | (u128)(i == 2 * (int)k);
    int fits = rem >= q;
    if (fits) rem -= q;
    quo = (quo << 1) | (u128)fits;
    if (i == 0) return quo;
  }
}

static unsigned bitlen(u128 q) {
  unsigned b = 0;
  while (q) {
    b++;
    q >>= 1;
  }
  return b;
}

/* helpers.rs:133-146: Barrett reduction, two conditional subtractions.
 * The reciprocal is cached for the last modulus seen. */
u128 o_fp_mul(u128 a, u128 b, u128 q) {
  static __thread u128 cq = 0, cmu = 0;
  static __thread unsigned ck = 0;
  if (cq != q) {
    cq = q;
    ck = bitlen(q);
    cmu = barrett_mu(q, ck);
  }
  u128 lo, hi;
  mul_wide(a, b, &lo, &hi);
  u128 q1 = shr_wide(lo, hi, ck - 1);
  u128 q2lo, q2hi;
  mul_wide(q1, cmu, &q2lo, &q2hi);
  u128 q3 = shr_wide(q2lo, q2hi, ck + 1);
  u128 pl, ph;
  mul_wide(q3, q, &pl, &ph);
  u128 r = lo - pl;
  if (r >= q) r -= q;
  if (r >= q) r -= q;
  return r;
}

u128 o_fp_add(u128 a, u128 b, u128 q) {
  u128 s = a + b;
  return s >= q ? s - q : s;
}

u128 o_fp_sub(u128 a, u128 b, u128 q) { return a >= b ? a - b : a + q - b; }

static u128 fp_pow(u128 base, u128 e, u128 q) {
  u128 r = 1 % q;
  int bit = (int)bitlen(e);
  while (bit > 0) {
    bit--;
    r = o_fp_mul(r, r, q);
    if ((e >> bit) & 1) r = o_fp_mul(r, base, q);
  }
  return r;
}

/* helpers.rs:198-215: one strong probable-prime round per base. */
int o_fp_is_prime_mr(u128 q, const u128 *bases, int nbases) {
  u128 qm1 = q - 1;
  int shift = 0;
  while (((qm1 >> shift) & 1) == 0) shift++;
  u128 odd = qm1 >> shift;
  for (int i = 0; i < nbases; i++) {
    u128 x = fp_pow(bases[i] % q, odd, q);
    if (x == 1 || x == qm1) continue;
    int ok = 0;
    for (int s = 1; s < shift; s++) {
      x = o_fp_mul(x, x, q);
      if (x == qm1) {
        ok = 1;
        break;
      }
    }
    if (!ok) return 0;
  }
  return 1;
}
