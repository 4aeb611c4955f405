// Host transcript primitives: Keccak-f[1600], grinding and prime sampling.
#include "transcript.hpp"

namespace bz {

static const uint64_t KRC[24] = {
    0x0000000000000001ull, 0x0000000000008082ull, 0x800000000000808aull, 0x8000000080008000ull,
    0x000000000000808bull, 0x0000000080000001ull, 0x8000000080008081ull, 0x8000000000008009ull,
    0x000000000000008aull, 0x0000000000000088ull, 0x0000000080008009ull, 0x000000008000000aull,
    0x000000008000808bull, 0x800000000000008bull, 0x8000000000008089ull, 0x8000000000008003ull,
    0x8000000000008002ull, 0x8000000000000080ull, 0x000000000000800aull, 0x800000008000000aull,
    0x8000000080008081ull, 0x8000000000008080ull, 0x0000000080000001ull, 0x8000000080008008ull};

static inline uint64_t rol(uint64_t x, int n) { return (x << n) | (x >> ((64 - n) & 63)); }

// FIPS 202 section 3.3 with the rho/pi lane walk unrolled.
void keccak_f1600(uint64_t a[25]) {
  static const int PI[24] = {10, 7, 11, 17, 18, 3, 5, 16, 8, 21, 24, 4,
                             15, 23, 19, 13, 12, 2, 20, 14, 22, 9, 6, 1};
  static const int RHO[24] = {1, 3, 6, 10, 15, 21, 28, 36, 45, 55, 2, 14,
                              27, 41, 56, 8, 25, 43, 62, 18, 39, 61, 20, 44};
  for (int round = 0; round < 24; round++) {
    uint64_t c[5];
    for (int x = 0; x < 5; x++) c[x] = a[x] ^ a[x + 5] ^ a[x + 10] ^ a[x + 15] ^ a[x + 20];
    for (int x = 0; x < 5; x++) {
      uint64_t d = c[(x + 4) % 5] ^ rol(c[(x + 1) % 5], 1);
      for (int y = 0; y < 25; y += 5) a[y + x] ^= d;
    }
    uint64_t t = a[1];
    for (int i = 0; i < 24; i++) {
      int j = PI[i];
      uint64_t tmp = a[j];
      a[j] = rol(t, RHO[i]);
      t = tmp;
    }
    for (int y = 0; y < 25; y += 5) {
      uint64_t b0 = a[y], b1 = a[y + 1], b2 = a[y + 2], b3 = a[y + 3], b4 = a[y + 4];
      a[y] = b0 ^ (~b1 & b2);
      a[y + 1] = b1 ^ (~b2 & b3);
      a[y + 2] = b2 ^ (~b3 & b4);
      a[y + 3] = b3 ^ (~b4 & b0);
      a[y + 4] = b4 ^ (~b0 & b1);
    }
    a[0] ^= KRC[round];
  }
}

bool pow_valid(const uint8_t seed[16], uint64_t nonce, uint32_t bits) {
  if (bits > 32) return false;
  if (bits == 0) return nonce == 0;
  // The message is 15 + 16 + 8 = 39 bytes: one BLAKE3 block of one chunk.
  uint8_t blk[64];
  memset(blk, 0, sizeof blk);
  memcpy(blk, "bitz-pcs-pow-v1", 15);
  memcpy(blk + 15, seed, 16);
  for (int i = 0; i < 8; i++) blk[31 + i] = (uint8_t)(nonce >> (8 * i));
  static const uint32_t IV[8] = {0x6A09E667, 0xBB67AE85, 0x3C6EF372, 0xA54FF53A,
                                 0x510E527F, 0x9B05688C, 0x1F83D9AB, 0x5BE0CD19};
  uint32_t m[16], o[8];
  b3_load_le(blk, m, 16);
  b3_compress(IV, m, 0, 39, B3_CHUNK_START | B3_CHUNK_END | B3_ROOT, o);
  uint32_t v = __builtin_bswap32(o[0]);
  uint32_t lz = v == 0 ? 32 : (uint32_t)__builtin_clz(v);
  return lz >= bits;
}

void Transcript::grind(const char *label, uint32_t bits) {
  if (bits == 0) return;
  size_t ll = strlen(label);
  public_message("bitz-transcript-pow-v1", 22);
  public_u64((uint64_t)ll);
  public_message(label, ll);
  uint8_t b4[4];
  for (int i = 0; i < 4; i++) b4[i] = (uint8_t)(bits >> (8 * i));
  public_message(b4, 4);
  uint8_t seed[16];
  squeeze(seed, 16);
  uint64_t nonce = 0;
  while (!pow_valid(seed, nonce, bits)) nonce++;
  uint8_t n8[8];
  for (int i = 0; i < 8; i++) n8[i] = (uint8_t)(nonce >> (8 * i));
  prover_message(n8, 8);
}

// --------------------------------------------------------- prime sampling

static void mulw(u128 a, u128 b, u128 &lo, u128 &hi) {
  u128 al = (uint64_t)a, ah = a >> 64, bl = (uint64_t)b, bh = b >> 64;
  u128 ll = al * bl, hh = ah * bh, m1 = al * bh, m2 = ah * bl;
  u128 mid = m1 + m2;
  u128 mc = mid < m1;
  u128 l = ll + (mid << 64);
  lo = l;
  hi = hh + (mid >> 64) + (mc << 64) + (l < ll);
}

// (a*b) mod q by binary long division of the 256-bit product (q < 2^126).
static u128 mulmod(u128 a, u128 b, u128 q) {
  u128 lo, hi;
  mulw(a, b, lo, hi);
  u128 r = 0;
  for (int i = 255; i >= 0; i--) {
    u128 bit = i >= 128 ? (hi >> (i - 128)) & 1 : (lo >> i) & 1;
    r = (r << 1) | bit;  // r < 2q < 2^127: no overflow
    if (r >= q) r -= q;
  }
  return r;
}

static u128 powmod(u128 b, u128 e, u128 q) {
  u128 r = 1 % q;
  b %= q;
  while (e) {
    if (e & 1) r = mulmod(r, b, q);
    b = mulmod(b, b, q);
    e >>= 1;
  }
  return r;
}

// crates/field/src/helpers.rs:198-215
static bool strong_round(u128 q, u128 base) {
  u128 qm1 = q - 1;
  int shift = 0;
  while (((qm1 >> shift) & 1) == 0) shift++;
  u128 w = powmod(base, qm1 >> shift, q);
  if (w == 1 || w == qm1) return true;
  for (int r = 1; r < shift; r++) {
    w = mulmod(w, w, q);
    if (w == qm1) return true;
  }
  return false;
}

u128 Transcript::prime(uint32_t bits) {
  static const int P[13] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41};
  u128 bottom = (u128)1 << (bits - 1);
  for (;;) {
    u128 cand = bottom | (challenge_u128() & (bottom - 1)) | 1;
    int decided = 0;
    bool prime = false;
    for (int i = 0; i < 13; i++) {
      if (cand == (u128)P[i]) {
        decided = 1;
        prime = true;
        break;
      }
      if (cand % P[i] == 0) {
        decided = 1;
        prime = false;
        break;
      }
    }
    if (!decided) {
      prime = true;
      u128 bound = cand - 3;
      u128 b = bound - 1;
      int lz = 0;
      while (lz < 128 && !((b >> (127 - lz)) & 1)) lz++;
      u128 mask = lz >= 128 ? 0 : (~(u128)0) >> lz;
      for (int r = 0; r < 80 && prime; r++) {
        u128 c;
        do {
          c = challenge_u128() & mask;
        } while (c >= bound);
        if (!strong_round(cand, 2 + c)) prime = false;
      }
    }
    if (prime) return cand;
  }
}

}  // namespace bz
