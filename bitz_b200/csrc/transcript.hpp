// Host Fiat-Shamir transcript: the prover side of crates/transcript.
//
// Framing follows crates/transcript/src/lib.rs:7-27 (rules F1-F6): the
// protocol id "bitz/v1", the session and the instance are absorbed as domain
// tags at construction (domain.rs:13-26); prover messages are absorbed and
// appended to the narg string; public messages are absorbed only; hints ride
// in a second byte string the sponge never sees. The sponge is a
// Keccak-f[1600] duplex with a 136-byte rate, standing in for spongefish
// 0.7.4's std sponge (not vendored in the reference), so the byte-level sponge
// framing is this library's own.
#pragma once
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "field.cuh"
#include "hash.cuh"

namespace bz {

typedef unsigned __int128 u128;

void keccak_f1600(uint64_t st[25]);
// For each 136-byte block of `in`: the permutation, then the block XORed into
// the rate (the sponge's absorb of whole blocks once its rate is full).
void keccak_absorb_blocks(uint64_t st[25], const uint8_t *in, size_t nblocks);
// False when BITZ_HOST_SIMD=0: the host paths then avoid AVX-512 (grinding,
// the prime's strong rounds, the Keccak permutation).
bool host_simd_enabled();

class Transcript {
 public:
  static constexpr int RATE = 136;

  Transcript(const uint8_t *session, size_t slen, const uint8_t *instance, size_t ilen) {
    memset(st_, 0, sizeof st_);
    uint8_t pid[64];
    memset(pid, 0, sizeof pid);
    memcpy(pid, "bitz/v1", 7);
    absorb(pid, 64);
    absorb_len_prefixed(session, slen);
    absorb_len_prefixed(instance, ilen);
  }

  void public_message(const void *msg, size_t len) { absorb((const uint8_t *)msg, len); }
  void public_u64(uint64_t v) {
    uint8_t b[8];
    for (int i = 0; i < 8; i++) b[i] = (uint8_t)(v >> (8 * i));
    absorb(b, 8);
  }
  void public_f128(f128 v) { public_message(&v, 16); }

  void prover_message(const void *msg, size_t len) {
    absorb((const uint8_t *)msg, len);
    const uint8_t *p = (const uint8_t *)msg;
    narg_.insert(narg_.end(), p, p + len);
  }
  void prover_f128(f128 v) { prover_message(&v, 16); }

  void hint(const void *msg, size_t len) {
    const uint8_t *p = (const uint8_t *)msg;
    hints_.insert(hints_.end(), p, p + len);
  }

  // Byte i of the rate is byte i % 8 (little-endian) of lane i / 8, which on
  // a little-endian host is where it lies in memory: spans are copied whole.
  void squeeze(uint8_t *out, size_t n) {
    static_assert(__BYTE_ORDER__ == __ORDER_LITTLE_ENDIAN__, "lanes read as memory bytes");
    while (n > 0) {
      if (squeeze_pos_ == RATE) {
        keccak_f1600(st_);
        squeeze_pos_ = 0;
        absorb_pos_ = 0;
      }
      const size_t take = std::min(n, (size_t)(RATE - squeeze_pos_));
      memcpy(out, reinterpret_cast<const uint8_t *>(st_) + squeeze_pos_, take);
      squeeze_pos_ += (int)take;
      out += take;
      n -= take;
    }
  }

  // crates/field/src/codec.rs:24-35: 16 bytes little endian, lo then hi.
  f128 challenge_f128() {
    uint8_t b[16];
    squeeze(b, 16);
    f128 r;
    memcpy(&r.lo, b, 8);
    memcpy(&r.hi, b + 8, 8);
    return r;
  }
  u128 challenge_u128() {
    f128 f = challenge_f128();
    return (u128)f.lo | ((u128)f.hi << 64);
  }
  // crates/transcript/src/challenge.rs:59-86: uniform residue by rejection.
  u128 challenge_fp(u128 q) {
    u128 maxv = ~(u128)0;
    u128 rej = (maxv % q + 1) % q;
    u128 max_accepted = maxv - rej;
    for (;;) {
      u128 c = challenge_u128();
      if (c <= max_accepted) return c % q;
    }
  }

  // crates/transcript/src/prover.rs:29-41, pow.rs:11-36.
  void grind(const char *label, uint32_t bits);
  // crates/transcript/src/challenge/prime.rs:33-61.
  u128 prime(uint32_t bits);

  const std::vector<uint8_t> &narg() const { return narg_; }
  const std::vector<uint8_t> &hints() const { return hints_; }

 private:
  // Duplex absorb: XOR into the rate, permuting when it fills. Whole
  // little-endian lanes go in eight bytes at a time once aligned.
  void absorb(const uint8_t *in, size_t n) {
    while (n) {
      if (absorb_pos_ == RATE && n >= RATE) {  // whole blocks, the state kept in registers
        const size_t blocks = n / RATE;
        keccak_absorb_blocks(st_, in, blocks);
        in += blocks * RATE;
        n -= blocks * RATE;
        continue;
      }
      if (absorb_pos_ == RATE) {
        keccak_f1600(st_);
        absorb_pos_ = 0;
      }
      if ((absorb_pos_ & 7) == 0 && n >= 8) {
        size_t lanes = (size_t)(RATE - absorb_pos_) / 8;
        if (lanes > n / 8) lanes = n / 8;
        for (size_t i = 0; i < lanes; i++) {
          uint64_t v;
          memcpy(&v, in, 8);
          st_[absorb_pos_ / 8] ^= v;
          absorb_pos_ += 8;
          in += 8;
        }
        n -= lanes * 8;
        continue;
      }
      st_[absorb_pos_ / 8] ^= (uint64_t)*in << (8 * (absorb_pos_ % 8));
      absorb_pos_++;
      in++;
      n--;
    }
    squeeze_pos_ = RATE;
  }
  void absorb_len_prefixed(const uint8_t *msg, size_t len) {
    public_u64((uint64_t)len);
    absorb(msg, len);
  }

  uint64_t st_[25];
  int absorb_pos_ = 0;
  int squeeze_pos_ = RATE;
  std::vector<uint8_t> narg_;
  std::vector<uint8_t> hints_;
};

// crates/transcript/src/pow.rs:38-50
bool pow_valid(const uint8_t seed[16], uint64_t nonce, uint32_t bits);
// The smallest nonce that passes (0 for no grinding); at most 32 bits.
uint64_t pow_search(const uint8_t seed[16], uint32_t bits);

// crates/common/src/security.rs:25-31
inline uint32_t grinding_bits(uint32_t security_bits, uint64_t coefficient) {
  if (coefficient == 0) return 0;
  uint32_t log_c = 0;
  uint64_t c = coefficient - 1;
  while (c) {
    log_c++;
    c >>= 1;
  }
  uint32_t need = security_bits + log_c;
  return need > 128 ? need - 128 : 0;
}

}  // namespace bz
