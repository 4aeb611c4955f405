// Field arithmetic shared by host and device code.
//
// GF(2^128) = F_2[X]/(X^128 + X^7 + X^2 + X + 1) in the reference's basis
// (crates/field/src/gf128.rs:1-8,52): bit i of lo||hi is the coefficient of
// X^i. B200 has no carryless-multiply instruction, so the 32x32 carryless
// product is formed from four interleaved "multiply with holes" integer
// products (T. Pornin's masked-multiply method, BearSSL ghash_ctmul), lifted
// to 128x128 by two levels of Karatsuba. Reduction is the reference's
// two-fold substitution (crates/field/src/gf128/portable.rs:37-61), which is
// F_2-linear, so sums of products are reduced once.
//
// The prime field is the transcript-drawn modulus q < 2^126
// (crates/field/src/helpers.rs:8). Device tables hold Montgomery residues
// a*2^128 mod q; every value that crosses to the host is converted back to
// the canonical residue, so the transcript sees exactly the reference's bytes.
#pragma once
#include <stdint.h>
#if !defined(__CUDA_ARCH__)
#include <immintrin.h>
#endif

#if defined(__CUDACC__)
#define BZ_HD __host__ __device__ __forceinline__
#else
#define BZ_HD inline
#endif

namespace bz {

struct __align__(16) f128 {
  uint64_t lo, hi;
};

struct wide {
  uint64_t w0, w1, w2, w3;
};

BZ_HD f128 mk(uint64_t lo, uint64_t hi) {
  f128 r;
  r.lo = lo;
  r.hi = hi;
  return r;
}
BZ_HD f128 gadd(f128 a, f128 b) { return mk(a.lo ^ b.lo, a.hi ^ b.hi); }
BZ_HD bool gis_zero(f128 a) { return (a.lo | a.hi) == 0; }
BZ_HD bool geq(f128 a, f128 b) { return a.lo == b.lo && a.hi == b.hi; }
BZ_HD wide wzero() { return wide{0, 0, 0, 0}; }
BZ_HD void wacc(wide &acc, const wide &p) {
  acc.w0 ^= p.w0;
  acc.w1 ^= p.w1;
  acc.w2 ^= p.w2;
  acc.w3 ^= p.w3;
}

// 32x32 -> 64 carryless product. Each operand is split into four bit classes
// (positions = 0,1,2,3 mod 4); an integer product of two classes only has
// terms at one class of positions, at most 8 per position, so the 4-bit gaps
// absorb every carry and the class bits hold exact parities.
BZ_HD uint64_t clmul32(uint32_t x, uint32_t y) {
  const uint32_t m0 = 0x11111111u, m1 = 0x22222222u, m2 = 0x44444444u, m3 = 0x88888888u;
  uint32_t x0 = x & m0, x1 = x & m1, x2 = x & m2, x3 = x & m3;
  uint32_t y0 = y & m0, y1 = y & m1, y2 = y & m2, y3 = y & m3;
  uint64_t z0 = ((uint64_t)x0 * y0) ^ ((uint64_t)x1 * y3) ^ ((uint64_t)x2 * y2) ^ ((uint64_t)x3 * y1);
  uint64_t z1 = ((uint64_t)x0 * y1) ^ ((uint64_t)x1 * y0) ^ ((uint64_t)x2 * y3) ^ ((uint64_t)x3 * y2);
  uint64_t z2 = ((uint64_t)x0 * y2) ^ ((uint64_t)x1 * y1) ^ ((uint64_t)x2 * y0) ^ ((uint64_t)x3 * y3);
  uint64_t z3 = ((uint64_t)x0 * y3) ^ ((uint64_t)x1 * y2) ^ ((uint64_t)x2 * y1) ^ ((uint64_t)x3 * y0);
  return (z0 & 0x1111111111111111ull) | (z1 & 0x2222222222222222ull) |
         (z2 & 0x4444444444444444ull) | (z3 & 0x8888888888888888ull);
}

// 64x64 -> 128 carryless product, one Karatsuba level over clmul32.
BZ_HD void clmul64(uint64_t a, uint64_t b, uint64_t &lo, uint64_t &hi) {
  uint32_t a0 = (uint32_t)a, a1 = (uint32_t)(a >> 32);
  uint32_t b0 = (uint32_t)b, b1 = (uint32_t)(b >> 32);
  uint64_t l = clmul32(a0, b0);
  uint64_t h = clmul32(a1, b1);
  uint64_t m = clmul32(a0 ^ a1, b0 ^ b1) ^ l ^ h;
  lo = l ^ (m << 32);
  hi = h ^ (m >> 32);
}

#if !defined(__CUDA_ARCH__)
// The host's scalar steps use the CPU's carryless multiply (PCLMULQDQ) when
// it has one; the result is the same 256-bit product.
__attribute__((target("pclmul,sse4.1"))) inline wide gmul_wide_pclmul(f128 a, f128 b) {
  const __m128i A = _mm_set_epi64x((long long)a.hi, (long long)a.lo);
  const __m128i B = _mm_set_epi64x((long long)b.hi, (long long)b.lo);
  const __m128i lo = _mm_clmulepi64_si128(A, B, 0x00);
  const __m128i hi = _mm_clmulepi64_si128(A, B, 0x11);
  const __m128i mid = _mm_xor_si128(_mm_clmulepi64_si128(A, B, 0x10),
                                    _mm_clmulepi64_si128(A, B, 0x01));
  wide r;
  r.w0 = (uint64_t)_mm_cvtsi128_si64(lo);
  r.w1 = (uint64_t)_mm_extract_epi64(lo, 1) ^ (uint64_t)_mm_cvtsi128_si64(mid);
  r.w2 = (uint64_t)_mm_cvtsi128_si64(hi) ^ (uint64_t)_mm_extract_epi64(mid, 1);
  r.w3 = (uint64_t)_mm_extract_epi64(hi, 1);
  return r;
}
inline bool host_has_pclmul() {
  static const bool yes = __builtin_cpu_supports("pclmul") && __builtin_cpu_supports("sse4.1");
  return yes;
}
#endif

// 128x128 -> 256 carryless product, second Karatsuba level.
BZ_HD wide gmul_wide_portable(f128 a, f128 b);
BZ_HD wide gmul_wide(f128 a, f128 b) {
#if !defined(__CUDA_ARCH__)
#if defined(__PCLMUL__) && defined(__SSE4_1__)
  return gmul_wide_pclmul(a, b);  // compiled for it: no run-time check, inlined
#else
  if (host_has_pclmul()) return gmul_wide_pclmul(a, b);
#endif
#endif
  return gmul_wide_portable(a, b);
}
BZ_HD wide gmul_wide_portable(f128 a, f128 b) {
  uint64_t l0, l1, h0, h1, m0, m1;
  clmul64(a.lo, b.lo, l0, l1);
  clmul64(a.hi, b.hi, h0, h1);
  clmul64(a.lo ^ a.hi, b.lo ^ b.hi, m0, m1);
  m0 ^= l0 ^ h0;
  m1 ^= l1 ^ h1;
  return wide{l0, l1 ^ m0, h0 ^ m1, h1};
}

// X^128 = X^7 + X^2 + X + 1 folded twice; at most 7 bits spill back.
BZ_HD f128 greduce(const wide &r) {
  uint64_t a0 = r.w2 ^ (r.w2 << 1) ^ (r.w2 << 2) ^ (r.w2 << 7);
  uint64_t a1 = (r.w2 >> 63) ^ (r.w2 >> 62) ^ (r.w2 >> 57);
  uint64_t b0 = r.w3 ^ (r.w3 << 1) ^ (r.w3 << 2) ^ (r.w3 << 7);
  uint64_t b1 = (r.w3 >> 63) ^ (r.w3 >> 62) ^ (r.w3 >> 57);
  uint64_t w0 = r.w0 ^ a0;
  uint64_t w1 = r.w1 ^ a1 ^ b0;
  return mk(w0 ^ b1 ^ (b1 << 1) ^ (b1 << 2) ^ (b1 << 7), w1);
}

BZ_HD f128 gmul(f128 a, f128 b) { return greduce(gmul_wide(a, b)); }

// r * X^k for 0 <= k < 128: the 256-bit shift of r, reduced.
BZ_HD f128 gmul_xk(f128 r, int k) {
  if (k == 0) return r;
  wide w;
  if (k < 64) {
    w = wide{r.lo << k, (r.hi << k) | (r.lo >> (64 - k)), r.hi >> (64 - k), 0};
  } else if (k == 64) {
    w = wide{0, r.lo, r.hi, 0};
  } else {
    const int s = k - 64;
    w = wide{0, r.lo << s, (r.hi << s) | (r.lo >> (64 - s)), r.hi >> (64 - s)};
  }
  return greduce(w);
}

// ------------------------------------------------------------ prime field

struct fp {
  uint64_t lo, hi;
};

// Montgomery context for one modulus q < 2^126 (R = 2^128).
struct FpCtx {
  uint64_t q0, q1;  // q
  uint64_t qinv;    // -q^{-1} mod 2^64
  fp one;           // R mod q
  fp r2;            // R^2 mod q
};

BZ_HD void mul64(uint64_t a, uint64_t b, uint64_t &lo, uint64_t &hi) {
#if defined(__CUDA_ARCH__)
  lo = a * b;
  hi = __umul64hi(a, b);
#else
  unsigned __int128 p = (unsigned __int128)a * b;
  lo = (uint64_t)p;
  hi = (uint64_t)(p >> 64);
#endif
}

// add with carry helpers on 64-bit limbs
BZ_HD uint64_t addc(uint64_t a, uint64_t b, uint64_t &carry) {
  uint64_t s = a + b;
  uint64_t c1 = s < a;
  uint64_t t = s + carry;
  uint64_t c2 = t < s;
  carry = c1 + c2;
  return t;
}

BZ_HD bool fp_ge(fp a, uint64_t q0, uint64_t q1) { return a.hi > q1 || (a.hi == q1 && a.lo >= q0); }

BZ_HD fp fp_sub_raw(fp a, uint64_t q0, uint64_t q1) {
  fp r;
  r.lo = a.lo - q0;
  uint64_t borrow = a.lo < q0;
  r.hi = a.hi - q1 - borrow;
  return r;
}

BZ_HD fp fp_add(fp a, fp b, const FpCtx &c) {
  // a, b < q < 2^126: the sum fits in 127 bits.
  fp r;
  r.lo = a.lo + b.lo;
  r.hi = a.hi + b.hi + (r.lo < a.lo);
  if (fp_ge(r, c.q0, c.q1)) r = fp_sub_raw(r, c.q0, c.q1);
  return r;
}

BZ_HD fp fp_sub(fp a, fp b, const FpCtx &c) {
  fp r;
  r.lo = a.lo - b.lo;
  uint64_t borrow = a.lo < b.lo;
  r.hi = a.hi - b.hi - borrow;
  bool neg = (a.hi < b.hi) || (a.hi == b.hi && a.lo < b.lo);
  if (neg) {
    uint64_t lo = r.lo + c.q0;
    r.hi = r.hi + c.q1 + (lo < r.lo);
    r.lo = lo;
  }
  return r;
}

// Montgomery product a*b*2^-128 mod q: schoolbook 256-bit product, then two
// word-by-word reduction steps. a, b < q < 2^126 keep every partial sum inside
// its 128-bit accumulator and the result below 2q.
BZ_HD fp fp_mul(fp a, fp b, const FpCtx &c) {
  typedef unsigned __int128 u128;
  u128 p00 = (u128)a.lo * b.lo, p01 = (u128)a.lo * b.hi;
  u128 p10 = (u128)a.hi * b.lo, p11 = (u128)a.hi * b.hi;
  u128 mid = (p00 >> 64) + (uint64_t)p01 + (uint64_t)p10;
  uint64_t t0 = (uint64_t)p00;
  uint64_t t1 = (uint64_t)mid;
  u128 hi = (mid >> 64) + (p01 >> 64) + (p10 >> 64) + p11;
  uint64_t t2 = (uint64_t)hi, t3 = (uint64_t)(hi >> 64);
  uint64_t m = t0 * c.qinv;
  u128 s = (u128)m * c.q0 + t0;
  s = (s >> 64) + (u128)m * c.q1 + t1;
  t1 = (uint64_t)s;
  s = (s >> 64) + t2;
  t2 = (uint64_t)s;
  t3 += (uint64_t)(s >> 64);
  m = t1 * c.qinv;
  s = (u128)m * c.q0 + t1;
  s = (s >> 64) + (u128)m * c.q1 + t2;
  t2 = (uint64_t)s;
  t3 += (uint64_t)(s >> 64);
  fp r{t2, t3};
  if (fp_ge(r, c.q0, c.q1)) r = fp_sub_raw(r, c.q0, c.q1);
  return r;
}

BZ_HD fp fp_zero() { return fp{0, 0}; }
BZ_HD bool fp_is_zero(fp a) { return (a.lo | a.hi) == 0; }

}  // namespace bz
