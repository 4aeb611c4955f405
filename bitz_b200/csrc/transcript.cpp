// Host transcript primitives: Keccak-f[1600], grinding and prime sampling.
#include "transcript.hpp"

#include <immintrin.h>

#include <stdlib.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <deque>
#include <functional>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <thread>
#include <vector>

namespace bz {

static const uint32_t kB3IV[8] = {0x6A09E667, 0xBB67AE85, 0x3C6EF372, 0xA54FF53A,
                                  0x510E527F, 0x9B05688C, 0x1F83D9AB, 0x5BE0CD19};
constexpr uint32_t kPowLen = 39;  // 15 + 16 + 8 bytes: one block of one chunk
constexpr uint32_t kPowFlags = B3_CHUNK_START | B3_CHUNK_END | B3_ROOT;

// The grinding message "bitz-pcs-pow-v1" || seed || nonce (little-endian) as
// the block's sixteen words (crates/transcript/src/pow.rs:38-50).
static void pow_words(const uint8_t seed[16], uint64_t nonce, uint32_t m[16]) {
  uint8_t blk[64];
  memset(blk, 0, sizeof blk);
  memcpy(blk, "bitz-pcs-pow-v1", 15);
  memcpy(blk + 15, seed, 16);
  for (int i = 0; i < 8; i++) blk[31 + i] = (uint8_t)(nonce >> (8 * i));
  b3_load_le(blk, m, 16);
}

// A hash passes when its first `bits` bits, read big-endian from byte 0, are
// zero: the output's word 0 has no bit in common with this mask.
static uint32_t pow_mask(uint32_t bits) { return __builtin_bswap32(~0u << (32 - bits)); }

bool pow_valid(const uint8_t seed[16], uint64_t nonce, uint32_t bits) {
  if (bits > 32) return false;
  if (bits == 0) return nonce == 0;
  uint32_t m[16], o[8];
  pow_words(seed, nonce, m);
  b3_compress(kB3IV, m, 0, kPowLen, kPowFlags, o);
  return (o[0] & pow_mask(bits)) == 0;
}

// Sixteen nonces base .. base + 15 per step, one per 32-bit lane. With base a
// multiple of 16 the nonces differ only in their byte 0, the top byte of
// message word 7; words 8 and 9 (nonce bytes 1-7) are the same in every lane.
// Returns the smallest passing nonce, the one the one-at-a-time loop finds.
#define BZ_B3_G16(a, b, c, d, x, y)                                 \
  do {                                                              \
    s[a] = _mm512_add_epi32(_mm512_add_epi32(s[a], s[b]), x);       \
    s[d] = _mm512_ror_epi32(_mm512_xor_si512(s[d], s[a]), 16);      \
    s[c] = _mm512_add_epi32(s[c], s[d]);                            \
    s[b] = _mm512_ror_epi32(_mm512_xor_si512(s[b], s[c]), 12);      \
    s[a] = _mm512_add_epi32(_mm512_add_epi32(s[a], s[b]), y);       \
    s[d] = _mm512_ror_epi32(_mm512_xor_si512(s[d], s[a]), 8);       \
    s[c] = _mm512_add_epi32(s[c], s[d]);                            \
    s[b] = _mm512_ror_epi32(_mm512_xor_si512(s[b], s[c]), 7);       \
  } while (0)

__attribute__((target("avx512f"))) static uint64_t pow_search16(const uint32_t w[16],
                                                                 uint32_t mask) {
  const __m512i lane = _mm512_setr_epi32(0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15);
  const __m512i vmask = _mm512_set1_epi32((int)mask);
  for (uint64_t base = 0;; base += 16) {
    __m512i m[16];
    for (int i = 0; i < 16; i++) m[i] = _mm512_set1_epi32((int)w[i]);
    m[7] = _mm512_or_si512(
        m[7], _mm512_slli_epi32(_mm512_add_epi32(_mm512_set1_epi32((int)(base & 0xff)), lane), 24));
    m[8] = _mm512_set1_epi32((int)(uint32_t)(base >> 8));
    m[9] = _mm512_set1_epi32((int)(uint32_t)(base >> 40));
    __m512i s[16];
    for (int i = 0; i < 8; i++) s[i] = _mm512_set1_epi32((int)kB3IV[i]);
    for (int i = 0; i < 4; i++) s[8 + i] = _mm512_set1_epi32((int)kB3IV[i]);
    s[12] = _mm512_setzero_si512();
    s[13] = _mm512_setzero_si512();
    s[14] = _mm512_set1_epi32((int)kPowLen);
    s[15] = _mm512_set1_epi32((int)kPowFlags);
    for (int r = 0; r < 7; r++) {
      BZ_B3_G16(0, 4, 8, 12, m[0], m[1]);
      BZ_B3_G16(1, 5, 9, 13, m[2], m[3]);
      BZ_B3_G16(2, 6, 10, 14, m[4], m[5]);
      BZ_B3_G16(3, 7, 11, 15, m[6], m[7]);
      BZ_B3_G16(0, 5, 10, 15, m[8], m[9]);
      BZ_B3_G16(1, 6, 11, 12, m[10], m[11]);
      BZ_B3_G16(2, 7, 8, 13, m[12], m[13]);
      BZ_B3_G16(3, 4, 9, 14, m[14], m[15]);
      // the message schedule permutation of b3_compress
      const __m512i t[16] = {m[2], m[6], m[3],  m[10], m[7],  m[0],  m[4],  m[13],
                             m[1], m[11], m[12], m[5], m[9], m[14], m[15], m[8]};
      for (int i = 0; i < 16; i++) m[i] = t[i];
    }
    const __mmask16 fail = _mm512_test_epi32_mask(_mm512_xor_si512(s[0], s[8]), vmask);
    if (fail != 0xffff) return base + (uint64_t)__builtin_ctz(~(unsigned)fail & 0xffffu);
  }
}
#undef BZ_B3_G16

// The AVX-512 paths (grinding, the prime's strong rounds, the Keccak
// permutation) run where the host has the instructions, unless
// BITZ_HOST_SIMD=0 selects the scalar ones.
bool host_simd_enabled() {
  static const bool on = [] {
    const char *v = getenv("BITZ_HOST_SIMD");
    return !(v && v[0] == '0');
  }();
  return on;
}
static bool host_simd() { return host_simd_enabled(); }

uint64_t pow_search(const uint8_t seed[16], uint32_t bits) {
  if (bits == 0) return 0;
  if (bits > 32) throw std::invalid_argument("grinding difficulty exceeds 32 bits");
  static const bool simd = host_simd() && __builtin_cpu_supports("avx512f");
  if (simd) {
    uint32_t w[16];
    pow_words(seed, 0, w);
    return pow_search16(w, pow_mask(bits));
  }
  uint64_t nonce = 0;
  while (!pow_valid(seed, nonce, bits)) nonce++;
  return nonce;
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
  const uint64_t nonce = pow_search(seed, bits);
  uint8_t n8[8];
  for (int i = 0; i < 8; i++) n8[i] = (uint8_t)(nonce >> (8 * i));
  prover_message(n8, 8);
}

// --------------------------------------------------------- prime sampling


// Montgomery context of an odd candidate q < 2^126 (R = 2^128).
static FpCtx candidate_ctx(u128 q) {
  FpCtx c;
  c.q0 = (uint64_t)q;
  c.q1 = (uint64_t)(q >> 64);
  uint64_t inv = 1;
  for (int i = 0; i < 7; i++) inv *= 2 - c.q0 * inv;  // Newton: q0 * inv = 1 mod 2^64
  c.qinv = (uint64_t)0 - inv;
  u128 one = ((~(u128)0) % q + 1) % q;
  c.one = fp{(uint64_t)one, (uint64_t)(one >> 64)};
  u128 x = one;
  for (int i = 0; i < 128; i++) {
    x <<= 1;
    if (x >= q) x -= q;
  }
  c.r2 = fp{(uint64_t)x, (uint64_t)(x >> 64)};
  return c;
}

static inline u128 to_u128(fp v) { return (u128)v.lo | ((u128)v.hi << 64); }

// crates/field/src/helpers.rs:198-215: base^odd is 1 or -1, or one of its
// next shift - 1 squares is -1. Arithmetic in Montgomery form; the results
// compare against R and -R.
static bool strong_round(const FpCtx &c, u128 q, u128 base) {
  u128 qm1 = q - 1;
  int shift = 0;
  while (((qm1 >> shift) & 1) == 0) shift++;
  u128 e = qm1 >> shift;
  fp b = fp_mul(fp{(uint64_t)(base % q), (uint64_t)((base % q) >> 64)}, c.r2, c);
  fp w = c.one;
  for (int i = 127; i >= 0; i--) {
    w = fp_mul(w, w, c);
    if ((e >> i) & 1) w = fp_mul(w, b, c);
  }
  u128 one = to_u128(c.one), minus_one = q - one;
  if (to_u128(w) == one || to_u128(w) == minus_one) return true;
  for (int r = 1; r < shift; r++) {
    w = fp_mul(w, w, c);
    if (to_u128(w) == minus_one) return true;
  }
  return false;
}

// The same rounds for many bases of one modulus on AVX-512 IFMA (52-bit
// multiply-add): Montgomery arithmetic in radix 2^52 with three limbs and
// R = 2^156, after the IFMA multiplication of Gueron and Krasnov
// ("Accelerating big integer arithmetic using Intel IFMA extensions", 2016).
// As 4q < R, products of values below 2q stay below 2q without a final
// subtraction, so a value is 1 (or -1) exactly when it equals one of that
// residue's two forms below 2q. Every base follows the same square-and-
// multiply schedule (the exponent is the modulus's), eight per vector.
namespace {
struct MrSimd {
  uint64_t q[3], qinv;        // modulus limbs; -q^-1 mod 2^52
  uint64_t one[3], one_q[3];  // R mod q, and that plus q
  uint64_t neg[3], neg_q[3];  // q - (R mod q), and that plus q
  uint64_t r2[3];             // R^2 mod q
  u128 e;                     // (q - 1) >> shift
  int shift, top;             // top: the highest set bit of e
};

struct V3 {
  __m512i l[3];
};
}  // namespace

static void limbs52(u128 v, uint64_t o[3]) {
  const uint64_t m = (1ull << 52) - 1;
  o[0] = (uint64_t)v & m;
  o[1] = (uint64_t)(v >> 52) & m;
  o[2] = (uint64_t)(v >> 104);
}

static MrSimd mr_simd_setup(u128 q) {
  MrSimd s;
  limbs52(q, s.q);
  uint64_t inv = 1;
  for (int i = 0; i < 7; i++) inv *= 2 - (uint64_t)q * inv;  // Newton: q * inv = 1 mod 2^64
  s.qinv = (0 - inv) & ((1ull << 52) - 1);
  u128 x = 1 % q;
  for (int i = 0; i < 156; i++) {
    x <<= 1;
    if (x >= q) x -= q;
  }
  const u128 rm = x;
  for (int i = 0; i < 156; i++) {
    x <<= 1;
    if (x >= q) x -= q;
  }
  limbs52(x, s.r2);
  limbs52(rm, s.one);
  limbs52(rm + q, s.one_q);
  limbs52(q - rm, s.neg);
  limbs52(q - rm + q, s.neg_q);
  const u128 qm1 = q - 1;
  s.shift = 0;
  while (((qm1 >> s.shift) & 1) == 0) s.shift++;
  s.e = qm1 >> s.shift;
  s.top = 127;
  while (s.top > 0 && !((s.e >> s.top) & 1)) s.top--;
  return s;
}

#define BZ_IFMA __attribute__((target("avx512f,avx512ifma")))

// a b R^-1 mod q, below 2q for a, b below 2q; limbs below 2^52 in and out.
BZ_IFMA static inline V3 mont52(const V3 &a, const V3 &b, const __m512i q[3], __m512i qinv) {
  const __m512i z = _mm512_setzero_si512(), m52 = _mm512_set1_epi64((1ll << 52) - 1);
  __m512i t0 = z, t1 = z, t2 = z, t3 = z;
  for (int i = 0; i < 3; i++) {
    const __m512i bi = b.l[i];
    t0 = _mm512_madd52lo_epu64(t0, a.l[0], bi);
    t1 = _mm512_madd52hi_epu64(t1, a.l[0], bi);
    t1 = _mm512_madd52lo_epu64(t1, a.l[1], bi);
    t2 = _mm512_madd52hi_epu64(t2, a.l[1], bi);
    t2 = _mm512_madd52lo_epu64(t2, a.l[2], bi);
    t3 = _mm512_madd52hi_epu64(t3, a.l[2], bi);
    // m = t0 (-q^-1) mod 2^52 makes t0 + m q0 a multiple of 2^52
    const __m512i m = _mm512_madd52lo_epu64(z, t0, qinv);
    t0 = _mm512_madd52lo_epu64(t0, q[0], m);
    t1 = _mm512_madd52hi_epu64(t1, q[0], m);
    t1 = _mm512_madd52lo_epu64(t1, q[1], m);
    t2 = _mm512_madd52hi_epu64(t2, q[1], m);
    t2 = _mm512_madd52lo_epu64(t2, q[2], m);
    t3 = _mm512_madd52hi_epu64(t3, q[2], m);
    t0 = _mm512_add_epi64(t1, _mm512_srli_epi64(t0, 52));
    t1 = t2;
    t2 = t3;
    t3 = z;
  }
  V3 r;
  r.l[0] = _mm512_and_si512(t0, m52);
  t1 = _mm512_add_epi64(t1, _mm512_srli_epi64(t0, 52));
  r.l[1] = _mm512_and_si512(t1, m52);
  r.l[2] = _mm512_add_epi64(t2, _mm512_srli_epi64(t1, 52));
  return r;
}

BZ_IFMA static inline __mmask8 eq52(const V3 &a, const uint64_t c[3]) {
  return _mm512_cmpeq_epi64_mask(a.l[0], _mm512_set1_epi64((long long)c[0])) &
         _mm512_cmpeq_epi64_mask(a.l[1], _mm512_set1_epi64((long long)c[1])) &
         _mm512_cmpeq_epi64_mask(a.l[2], _mm512_set1_epi64((long long)c[2]));
}

// pass[i] = strong_round(q, bases[i]) for i < n, bases below q. Two vectors
// of eight bases go through the schedule side by side, so each product's
// dependent chain overlaps the other's.
BZ_IFMA static void strong_rounds_ifma(u128 qv, const u128 *bases, int n, char *pass) {
  const MrSimd s = mr_simd_setup(qv);
  __m512i q[3];
  for (int i = 0; i < 3; i++) q[i] = _mm512_set1_epi64((long long)s.q[i]);
  const __m512i qinv = _mm512_set1_epi64((long long)s.qinv);
  V3 r2;
  for (int i = 0; i < 3; i++) r2.l[i] = _mm512_set1_epi64((long long)s.r2[i]);
  for (int at = 0; at < n; at += 16) {
    alignas(64) uint64_t bl[2][3][8];
    for (int k = 0; k < 16; k++) {
      uint64_t t[3];
      limbs52(at + k < n ? bases[at + k] : 2, t);
      for (int i = 0; i < 3; i++) bl[k >> 3][i][k & 7] = t[i];
    }
    V3 b0, b1;
    for (int i = 0; i < 3; i++) {
      b0.l[i] = _mm512_load_si512(bl[0][i]);
      b1.l[i] = _mm512_load_si512(bl[1][i]);
    }
    b0 = mont52(b0, r2, q, qinv);  // to Montgomery form
    b1 = mont52(b1, r2, q, qinv);
    V3 w0 = b0, w1 = b1;  // the top bit of e is set
    for (int i = s.top - 1; i >= 0; i--) {
      w0 = mont52(w0, w0, q, qinv);
      w1 = mont52(w1, w1, q, qinv);
      if ((s.e >> i) & 1) {
        w0 = mont52(w0, b0, q, qinv);
        w1 = mont52(w1, b1, q, qinv);
      }
    }
    __mmask8 ok0 = eq52(w0, s.one) | eq52(w0, s.one_q) | eq52(w0, s.neg) | eq52(w0, s.neg_q);
    __mmask8 ok1 = eq52(w1, s.one) | eq52(w1, s.one_q) | eq52(w1, s.neg) | eq52(w1, s.neg_q);
    for (int r = 1; r < s.shift; r++) {
      w0 = mont52(w0, w0, q, qinv);
      w1 = mont52(w1, w1, q, qinv);
      ok0 |= eq52(w0, s.neg) | eq52(w0, s.neg_q);
      ok1 |= eq52(w1, s.neg) | eq52(w1, s.neg_q);
    }
    const unsigned ok = (unsigned)ok0 | ((unsigned)ok1 << 8);
    for (int k = 0; k < 16 && at + k < n; k++) pass[at + k] = (char)((ok >> k) & 1);
  }
}
#undef BZ_IFMA

// A few host threads for independent work items of one call (the
// Miller-Rabin rounds of a candidate). The calling thread works on its own
// job too, so a call finishes even when every pool thread is busy with
// another lane's job; idle pool threads sleep on a condition variable.
namespace {
struct PoolJob {
  const std::function<void(int)> *fn;
  int n;
  std::atomic<int> next{0}, done{0};
};

class HostPool {
 public:
  static HostPool &get() {
    static HostPool *p = new HostPool();
    return *p;
  }
  void run(int n, const std::function<void(int)> &fn) {
    auto job = std::make_shared<PoolJob>();
    job->fn = &fn;
    job->n = n;
    {
      std::lock_guard<std::mutex> lk(mu_);
      jobs_.push_back(job);
    }
    cv_.notify_all();
    work(*job);
    while (job->done.load(std::memory_order_acquire) < n) _mm_pause();
  }

 private:
  HostPool() {
    const unsigned hw = std::max(2u, std::thread::hardware_concurrency());
    const unsigned nt = std::min(8u, hw - 1);
    for (unsigned i = 0; i < nt; i++) std::thread([this] { loop(); }).detach();
  }
  static void work(PoolJob &j) {
    for (;;) {
      const int i = j.next.fetch_add(1);
      if (i >= j.n) return;
      (*j.fn)(i);
      j.done.fetch_add(1, std::memory_order_release);
    }
  }
  void loop() {
    for (;;) {
      std::shared_ptr<PoolJob> j;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return !jobs_.empty(); });
        j = jobs_.front();
        if (j->next.load() >= j->n) {  // handed out: drop it
          jobs_.pop_front();
          continue;
        }
      }
      work(*j);
    }
  }
  std::mutex mu_;
  std::condition_variable cv_;
  std::deque<std::shared_ptr<PoolJob>> jobs_;
};
}  // namespace

// crates/transcript/src/challenge/prime.rs:33-61 with the strong test of
// crates/field/src/helpers.rs:198-215: a candidate is the top bit, transcript
// bits and the low bit; trial division by the primes to 41, then 80 rounds,
// each on a base drawn from the transcript (rejection-sampled below q - 3)
// and stopping at the first failure. The draws depend on the outcomes, so
// they follow the reference exactly: once a candidate passes its first round
// (almost surely a prime), the sponge state is saved, the other 79 bases are
// drawn in order and their rounds run together (sixteen bases at a time on
// AVX-512 IFMA, else spread over the host pool); if some round j failed,
// the state goes back and exactly the bases up to j are drawn again, as the
// sequential loop would have.
u128 Transcript::prime(uint32_t bits) {
  static const int P[13] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41};
  constexpr int kRounds = 80;
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
      FpCtx ctx = candidate_ctx(cand);
      u128 bound = cand - 3;
      u128 b = bound - 1;
      int lz = 0;
      while (lz < 128 && !((b >> (127 - lz)) & 1)) lz++;
      u128 mask = lz >= 128 ? 0 : (~(u128)0) >> lz;
      auto draw = [&] {
        u128 c;
        do {
          c = challenge_u128() & mask;
        } while (c >= bound);
        return c;
      };
      prime = strong_round(ctx, cand, 2 + draw());
      if (prime) {
        uint64_t st_saved[25];
        memcpy(st_saved, st_, sizeof st_);
        const int absorb_saved = absorb_pos_, squeeze_saved = squeeze_pos_;
        std::vector<u128> base(kRounds);
        for (int r = 1; r < kRounds; r++) base[r] = 2 + draw();
        std::vector<char> pass(kRounds, 1);
        static const bool ifma = host_simd() && __builtin_cpu_supports("avx512f") &&
                                 __builtin_cpu_supports("avx512ifma");
        if (ifma)
          strong_rounds_ifma(cand, base.data() + 1, kRounds - 1, pass.data() + 1);
        else
          HostPool::get().run(kRounds - 1, [&](int i) {
            pass[i + 1] = strong_round(ctx, cand, base[i + 1]) ? 1 : 0;
          });
        int fail = 0;
        for (int r = 1; r < kRounds && !fail; r++)
          if (!pass[r]) fail = r;
        if (fail) {
          prime = false;
          memcpy(st_, st_saved, sizeof st_);
          absorb_pos_ = absorb_saved;
          squeeze_pos_ = squeeze_saved;
          for (int r = 1; r <= fail; r++) draw();
        }
      }
    }
    if (prime) return cand;
  }
}

}  // namespace bz
