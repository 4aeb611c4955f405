// Keccak-f[1600] (FIPS 202 section 3.3) for the host transcript sponge, each
// round fully unrolled over the 25 lanes held in registers: theta, then rho
// and pi folded into one lane permutation (lane (x, y) moves to
// (y, 2x + 3y) rotated by its rho offset), then chi and iota. Three builds of
// the same round: AVX-512VL (one lane per vector register), BMI1/BMI2 and
// plain x86-64, the first the host supports (BITZ_HOST_SIMD=0 skips AVX-512).
#include "transcript.hpp"

#include <immintrin.h>

namespace bz {

static const uint64_t KRC[24] = {
    0x0000000000000001ull, 0x0000000000008082ull, 0x800000000000808aull, 0x8000000080008000ull,
    0x000000000000808bull, 0x0000000080000001ull, 0x8000000080008081ull, 0x8000000000008009ull,
    0x000000000000008aull, 0x0000000000000088ull, 0x0000000080008009ull, 0x000000008000000aull,
    0x000000008000808bull, 0x800000000000008bull, 0x8000000000008089ull, 0x8000000000008003ull,
    0x8000000000008002ull, 0x8000000000000080ull, 0x000000000000800aull, 0x800000008000000aull,
    0x8000000080008081ull, 0x8000000000008080ull, 0x0000000080000001ull, 0x8000000080008008ull};

#define rol(x, n) (((x) << (n)) | ((x) >> ((64 - (n)) & 63)))

#define KECCAK_ROUND(RC) \
  { \
    uint64_t c0 = a0 ^ a5 ^ a10 ^ a15 ^ a20; \
    uint64_t c1 = a1 ^ a6 ^ a11 ^ a16 ^ a21; \
    uint64_t c2 = a2 ^ a7 ^ a12 ^ a17 ^ a22; \
    uint64_t c3 = a3 ^ a8 ^ a13 ^ a18 ^ a23; \
    uint64_t c4 = a4 ^ a9 ^ a14 ^ a19 ^ a24; \
    uint64_t d0 = c4 ^ rol(c1, 1); \
    uint64_t d1 = c0 ^ rol(c2, 1); \
    uint64_t d2 = c1 ^ rol(c3, 1); \
    uint64_t d3 = c2 ^ rol(c4, 1); \
    uint64_t d4 = c3 ^ rol(c0, 1); \
    uint64_t b0 = (a0 ^ d0); \
    uint64_t b1 = rol((a6 ^ d1), 44); \
    uint64_t b2 = rol((a12 ^ d2), 43); \
    uint64_t b3 = rol((a18 ^ d3), 21); \
    uint64_t b4 = rol((a24 ^ d4), 14); \
    uint64_t b5 = rol((a3 ^ d3), 28); \
    uint64_t b6 = rol((a9 ^ d4), 20); \
    uint64_t b7 = rol((a10 ^ d0), 3); \
    uint64_t b8 = rol((a16 ^ d1), 45); \
    uint64_t b9 = rol((a22 ^ d2), 61); \
    uint64_t b10 = rol((a1 ^ d1), 1); \
    uint64_t b11 = rol((a7 ^ d2), 6); \
    uint64_t b12 = rol((a13 ^ d3), 25); \
    uint64_t b13 = rol((a19 ^ d4), 8); \
    uint64_t b14 = rol((a20 ^ d0), 18); \
    uint64_t b15 = rol((a4 ^ d4), 27); \
    uint64_t b16 = rol((a5 ^ d0), 36); \
    uint64_t b17 = rol((a11 ^ d1), 10); \
    uint64_t b18 = rol((a17 ^ d2), 15); \
    uint64_t b19 = rol((a23 ^ d3), 56); \
    uint64_t b20 = rol((a2 ^ d2), 62); \
    uint64_t b21 = rol((a8 ^ d3), 55); \
    uint64_t b22 = rol((a14 ^ d4), 39); \
    uint64_t b23 = rol((a15 ^ d0), 41); \
    uint64_t b24 = rol((a21 ^ d1), 2); \
    a0 = b0 ^ (~b1 & b2); \
    a1 = b1 ^ (~b2 & b3); \
    a2 = b2 ^ (~b3 & b4); \
    a3 = b3 ^ (~b4 & b0); \
    a4 = b4 ^ (~b0 & b1); \
    a5 = b5 ^ (~b6 & b7); \
    a6 = b6 ^ (~b7 & b8); \
    a7 = b7 ^ (~b8 & b9); \
    a8 = b8 ^ (~b9 & b5); \
    a9 = b9 ^ (~b5 & b6); \
    a10 = b10 ^ (~b11 & b12); \
    a11 = b11 ^ (~b12 & b13); \
    a12 = b12 ^ (~b13 & b14); \
    a13 = b13 ^ (~b14 & b10); \
    a14 = b14 ^ (~b10 & b11); \
    a15 = b15 ^ (~b16 & b17); \
    a16 = b16 ^ (~b17 & b18); \
    a17 = b17 ^ (~b18 & b19); \
    a18 = b18 ^ (~b19 & b15); \
    a19 = b19 ^ (~b15 & b16); \
    a20 = b20 ^ (~b21 & b22); \
    a21 = b21 ^ (~b22 & b23); \
    a22 = b22 ^ (~b23 & b24); \
    a23 = b23 ^ (~b24 & b20); \
    a24 = b24 ^ (~b20 & b21); \
    a0 ^= (RC); \
  }


#define KECCAK_BODY \
  uint64_t a0 = st[0], a1 = st[1], a2 = st[2], a3 = st[3], a4 = st[4], a5 = st[5], a6 = st[6], \
           a7 = st[7], a8 = st[8], a9 = st[9], a10 = st[10], a11 = st[11], a12 = st[12], \
           a13 = st[13], a14 = st[14], a15 = st[15], a16 = st[16], a17 = st[17], a18 = st[18], \
           a19 = st[19], a20 = st[20], a21 = st[21], a22 = st[22], a23 = st[23], a24 = st[24]; \
  for (int round = 0; round < 24; round++) KECCAK_ROUND(KRC[round]); \
  st[0] = a0, st[1] = a1, st[2] = a2, st[3] = a3, st[4] = a4, st[5] = a5, st[6] = a6; \
  st[7] = a7, st[8] = a8, st[9] = a9, st[10] = a10, st[11] = a11, st[12] = a12; \
  st[13] = a13, st[14] = a14, st[15] = a15, st[16] = a16, st[17] = a17, st[18] = a18; \
  st[19] = a19, st[20] = a20, st[21] = a21, st[22] = a22, st[23] = a23, st[24] = a24;

static void keccak_generic(uint64_t st[25]) { KECCAK_BODY }

// The same permutation compiled for BMI1/BMI2 (ANDN for chi, RORX): about a
// third faster where the CPU has them.
__attribute__((target("bmi,bmi2"))) static void keccak_bmi(uint64_t st[25]) { KECCAK_BODY }

// The same round with every lane in its own 128-bit vector register (32 of
// them with AVX-512VL, so the state stays out of memory): three-input XORs
// and chi as one ternary-logic instruction each, rotations by VPROLQ. Lane
// (x, y) ^ D[x] is formed as lane ^ C[x-1] ^ rot(C[x+1], 1) in one step.
#define XOR3(a, b, c) _mm_ternarylogic_epi64(a, b, c, 0x96)
#define CHI(a, b, c) _mm_ternarylogic_epi64(a, b, c, 0xD2) /* a ^ (~b & c) */
#define KECCAK_ROUND_VL(RC) \
  { \
    const __m128i c0 = XOR3(XOR3(a0, a5, a10), a15, a20); \
    const __m128i c1 = XOR3(XOR3(a1, a6, a11), a16, a21); \
    const __m128i c2 = XOR3(XOR3(a2, a7, a12), a17, a22); \
    const __m128i c3 = XOR3(XOR3(a3, a8, a13), a18, a23); \
    const __m128i c4 = XOR3(XOR3(a4, a9, a14), a19, a24); \
    const __m128i r0 = _mm_rol_epi64(c0, 1); \
    const __m128i r1 = _mm_rol_epi64(c1, 1); \
    const __m128i r2 = _mm_rol_epi64(c2, 1); \
    const __m128i r3 = _mm_rol_epi64(c3, 1); \
    const __m128i r4 = _mm_rol_epi64(c4, 1); \
    const __m128i b0 = XOR3(a0, c4, r1); \
    const __m128i b1 = _mm_rol_epi64(XOR3(a6, c0, r2), 44); \
    const __m128i b2 = _mm_rol_epi64(XOR3(a12, c1, r3), 43); \
    const __m128i b3 = _mm_rol_epi64(XOR3(a18, c2, r4), 21); \
    const __m128i b4 = _mm_rol_epi64(XOR3(a24, c3, r0), 14); \
    const __m128i b5 = _mm_rol_epi64(XOR3(a3, c2, r4), 28); \
    const __m128i b6 = _mm_rol_epi64(XOR3(a9, c3, r0), 20); \
    const __m128i b7 = _mm_rol_epi64(XOR3(a10, c4, r1), 3); \
    const __m128i b8 = _mm_rol_epi64(XOR3(a16, c0, r2), 45); \
    const __m128i b9 = _mm_rol_epi64(XOR3(a22, c1, r3), 61); \
    const __m128i b10 = _mm_rol_epi64(XOR3(a1, c0, r2), 1); \
    const __m128i b11 = _mm_rol_epi64(XOR3(a7, c1, r3), 6); \
    const __m128i b12 = _mm_rol_epi64(XOR3(a13, c2, r4), 25); \
    const __m128i b13 = _mm_rol_epi64(XOR3(a19, c3, r0), 8); \
    const __m128i b14 = _mm_rol_epi64(XOR3(a20, c4, r1), 18); \
    const __m128i b15 = _mm_rol_epi64(XOR3(a4, c3, r0), 27); \
    const __m128i b16 = _mm_rol_epi64(XOR3(a5, c4, r1), 36); \
    const __m128i b17 = _mm_rol_epi64(XOR3(a11, c0, r2), 10); \
    const __m128i b18 = _mm_rol_epi64(XOR3(a17, c1, r3), 15); \
    const __m128i b19 = _mm_rol_epi64(XOR3(a23, c2, r4), 56); \
    const __m128i b20 = _mm_rol_epi64(XOR3(a2, c1, r3), 62); \
    const __m128i b21 = _mm_rol_epi64(XOR3(a8, c2, r4), 55); \
    const __m128i b22 = _mm_rol_epi64(XOR3(a14, c3, r0), 39); \
    const __m128i b23 = _mm_rol_epi64(XOR3(a15, c4, r1), 41); \
    const __m128i b24 = _mm_rol_epi64(XOR3(a21, c0, r2), 2); \
    a0 = CHI(b0, b1, b2); \
    a1 = CHI(b1, b2, b3); \
    a2 = CHI(b2, b3, b4); \
    a3 = CHI(b3, b4, b0); \
    a4 = CHI(b4, b0, b1); \
    a5 = CHI(b5, b6, b7); \
    a6 = CHI(b6, b7, b8); \
    a7 = CHI(b7, b8, b9); \
    a8 = CHI(b8, b9, b5); \
    a9 = CHI(b9, b5, b6); \
    a10 = CHI(b10, b11, b12); \
    a11 = CHI(b11, b12, b13); \
    a12 = CHI(b12, b13, b14); \
    a13 = CHI(b13, b14, b10); \
    a14 = CHI(b14, b10, b11); \
    a15 = CHI(b15, b16, b17); \
    a16 = CHI(b16, b17, b18); \
    a17 = CHI(b17, b18, b19); \
    a18 = CHI(b18, b19, b15); \
    a19 = CHI(b19, b15, b16); \
    a20 = CHI(b20, b21, b22); \
    a21 = CHI(b21, b22, b23); \
    a22 = CHI(b22, b23, b24); \
    a23 = CHI(b23, b24, b20); \
    a24 = CHI(b24, b20, b21); \
    a0 = _mm_xor_si128(a0, _mm_cvtsi64_si128((long long)(RC))); \
  }

#define VL_LANES(M)                                                                        \
  M(0) M(1) M(2) M(3) M(4) M(5) M(6) M(7) M(8) M(9) M(10) M(11) M(12) M(13) M(14) M(15) M(16) \
  M(17) M(18) M(19) M(20) M(21) M(22) M(23) M(24)
#define VL_RATE_LANES(M) \
  M(0) M(1) M(2) M(3) M(4) M(5) M(6) M(7) M(8) M(9) M(10) M(11) M(12) M(13) M(14) M(15) M(16)
#define VL_DECL(i) __m128i a##i = _mm_cvtsi64_si128((long long)st[i]);
#define VL_STORE(i) st[i] = (uint64_t)_mm_cvtsi128_si64(a##i);
#define VL_XOR_IN(i) \
  a##i = _mm_xor_si128(a##i, _mm_loadl_epi64(reinterpret_cast<const __m128i *>(in + 8 * (i))));

// nblocks == 0: one permutation. Otherwise, per block of the rate (136 bytes
// of `in`): the permutation, then the block XORed into the rate, the state
// staying in registers from the first block to the last.
__attribute__((target("avx512f,avx512vl"))) static void keccak_vl(uint64_t st[25],
                                                                  const uint8_t *in,
                                                                  size_t nblocks) {
  VL_LANES(VL_DECL)
  size_t b = 0;
  do {
    // the 24 rounds written out: no loop-carried register shuffling between them
    KECCAK_ROUND_VL(KRC[0]) KECCAK_ROUND_VL(KRC[1]) KECCAK_ROUND_VL(KRC[2])
    KECCAK_ROUND_VL(KRC[3]) KECCAK_ROUND_VL(KRC[4]) KECCAK_ROUND_VL(KRC[5])
    KECCAK_ROUND_VL(KRC[6]) KECCAK_ROUND_VL(KRC[7]) KECCAK_ROUND_VL(KRC[8])
    KECCAK_ROUND_VL(KRC[9]) KECCAK_ROUND_VL(KRC[10]) KECCAK_ROUND_VL(KRC[11])
    KECCAK_ROUND_VL(KRC[12]) KECCAK_ROUND_VL(KRC[13]) KECCAK_ROUND_VL(KRC[14])
    KECCAK_ROUND_VL(KRC[15]) KECCAK_ROUND_VL(KRC[16]) KECCAK_ROUND_VL(KRC[17])
    KECCAK_ROUND_VL(KRC[18]) KECCAK_ROUND_VL(KRC[19]) KECCAK_ROUND_VL(KRC[20])
    KECCAK_ROUND_VL(KRC[21]) KECCAK_ROUND_VL(KRC[22]) KECCAK_ROUND_VL(KRC[23])
    if (nblocks) {
      VL_RATE_LANES(VL_XOR_IN)
      in += Transcript::RATE;
    }
  } while (++b < nblocks);
  VL_LANES(VL_STORE)
}
#undef VL_XOR_IN
#undef VL_STORE
#undef VL_DECL
#undef VL_RATE_LANES
#undef VL_LANES
#undef KECCAK_ROUND_VL
#undef CHI
#undef XOR3

void keccak_f1600(uint64_t st[25]) {
  static const int path = [] {
    if (host_simd_enabled() && __builtin_cpu_supports("avx512f") &&
        __builtin_cpu_supports("avx512vl"))
      return 2;
    return __builtin_cpu_supports("bmi") && __builtin_cpu_supports("bmi2") ? 1 : 0;
  }();
  if (path == 2)
    keccak_vl(st, nullptr, 0);
  else if (path == 1)
    keccak_bmi(st);
  else
    keccak_generic(st);
}
void keccak_absorb_blocks(uint64_t st[25], const uint8_t *in, size_t nblocks) {
  static_assert(__BYTE_ORDER__ == __ORDER_LITTLE_ENDIAN__, "lanes read as memory bytes");
  if (nblocks == 0) return;
  static const bool vl = host_simd_enabled() && __builtin_cpu_supports("avx512f") &&
                         __builtin_cpu_supports("avx512vl");
  if (vl) {
    keccak_vl(st, in, nblocks);
    return;
  }
  for (size_t b = 0; b < nblocks; b++, in += Transcript::RATE) {
    keccak_f1600(st);
    for (int i = 0; i < Transcript::RATE / 8; i++) {
      uint64_t v;
      memcpy(&v, in + 8 * i, 8);
      st[i] ^= v;
    }
  }
}
#undef KECCAK_BODY
#undef KECCAK_ROUND
#undef rol

}  // namespace bz
