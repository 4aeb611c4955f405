// Host transcript primitives: Keccak-f[1600], grinding and prime sampling.
#include "transcript.hpp"

#include <immintrin.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <deque>
#include <functional>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

namespace bz {




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
// drawn in order and their rounds run in parallel; if some round j failed,
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
        for (int r = 1; r < kRounds; r++) base[r] = draw();
        std::vector<char> pass(kRounds, 1);
        HostPool::get().run(kRounds - 1, [&](int i) {
          pass[i + 1] = strong_round(ctx, cand, 2 + base[i + 1]) ? 1 : 0;
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
