/* CPU oracle: the Fiat-Shamir transcript. Test infrastructure only.
 *
 * Framing follows crates/transcript/src/lib.rs:7-27 (F1-F6): domain tags at
 * construction, prover messages absorbed and written to the narg string,
 * public messages absorbed only, hints written beside the sponge. The sponge
 * is a Keccak-f[1600] duplex with a 136-byte rate standing in for spongefish
 * 0.7.4's std sponge, whose source is not in the reference tree: its exact
 * byte framing is parity unpinned. The narg and hint bytes of the reference's
 * golden transcript (crates/transcript/tests/golden.rs:14-15) are reproduced;
 * its two challenges (:16-17) are not. */
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

#define RATE 136

static void put(uint8_t **buf, size_t *len, size_t *cap, const void *src, size_t n) {
  if (*len + n > *cap) {
    size_t c = *cap ? *cap : 256;
    while (c < *len + n) c *= 2;
    *buf = (uint8_t *)realloc(*buf, c);
    *cap = c;
  }
  memcpy(*buf + *len, src, n);
  *len += n;
}

static void absorb(o_transcript *t, const uint8_t *in, size_t n) {
  for (size_t i = 0; i < n; i++) {
    if (t->absorb_pos == RATE) {
      o_keccak_f1600(t->st);
      t->absorb_pos = 0;
    }
    t->st[t->absorb_pos / 8] ^= (uint64_t)in[i] << (8 * (t->absorb_pos % 8));
    t->absorb_pos++;
  }
  t->squeeze_pos = RATE;
}

void o_ts_squeeze(o_transcript *t, uint8_t *out, size_t n) {
  for (size_t i = 0; i < n; i++) {
    if (t->squeeze_pos == RATE) {
      o_keccak_f1600(t->st);
      t->squeeze_pos = 0;
      t->absorb_pos = 0;
    }
    out[i] = (uint8_t)(t->st[t->squeeze_pos / 8] >> (8 * (t->squeeze_pos % 8)));
    t->squeeze_pos++;
  }
}

static void absorb_tagged(o_transcript *t, const uint8_t *msg, size_t len) {
  uint8_t l[8];
  for (int i = 0; i < 8; i++) l[i] = (uint8_t)((uint64_t)len >> (8 * i));
  absorb(t, l, 8);
  absorb(t, msg, len);
}

/* crates/transcript/src/domain.rs:13-26: protocol id "bitz/v1", then the
 * session and the instance as domain tags, none of them in the narg string. */
void o_ts_init(o_transcript *t, const uint8_t *session, size_t slen, const uint8_t *instance,
               size_t ilen) {
  memset(t, 0, sizeof *t);
  t->squeeze_pos = RATE;
  uint8_t pid[64];
  memset(pid, 0, sizeof pid);
  memcpy(pid, "bitz/v1", 7);
  absorb(t, pid, 64);
  absorb_tagged(t, session, slen);
  absorb_tagged(t, instance, ilen);
}

void o_ts_free(o_transcript *t) {
  free(t->narg);
  free(t->hints);
  t->narg = t->hints = NULL;
}

void o_ts_public(o_transcript *t, const void *msg, size_t len) { absorb(t, (const uint8_t *)msg, len); }

void o_ts_prover(o_transcript *t, const void *msg, size_t len) {
  absorb(t, (const uint8_t *)msg, len);
  put(&t->narg, &t->narg_len, &t->narg_cap, msg, len);
}

void o_ts_hint(o_transcript *t, const void *msg, size_t len) { put(&t->hints, &t->hints_len, &t->hints_cap, msg, len); }

/* crates/field/src/codec.rs:24-35: 16 bytes little endian, lo then hi. */
o_f128 o_ts_f128(o_transcript *t) {
  uint8_t b[16];
  o_ts_squeeze(t, b, 16);
  o_f128 r = {0, 0};
  for (int i = 0; i < 8; i++) {
    r.lo |= (uint64_t)b[i] << (8 * i);
    r.hi |= (uint64_t)b[8 + i] << (8 * i);
  }
  return r;
}

u128 o_ts_u128(o_transcript *t) {
  o_f128 f = o_ts_f128(t);
  return (u128)f.lo | ((u128)f.hi << 64);
}

/* crates/transcript/src/challenge.rs:59-86: reject the incomplete top interval,
 * then reduce. */
u128 o_ts_fp(o_transcript *t, u128 q) {
  u128 maxv = ~(u128)0;
  u128 rej = (maxv % q + 1) % q;
  u128 max_accepted = maxv - rej;
  for (;;) {
    u128 c = o_ts_u128(t);
    if (c <= max_accepted) return c % q;
  }
}

/* crates/transcript/src/pow.rs:38-50 */
int o_pow_valid(const uint8_t seed[16], uint64_t nonce, uint32_t bits) {
  if (bits > 32) return 0;
  if (bits == 0) return nonce == 0;
  o_blake3_state h;
  o_blake3_init(&h);
  o_blake3_update(&h, (const uint8_t *)"bitz-pcs-pow-v1", 15);
  o_blake3_update(&h, seed, 16);
  uint8_t n[8];
  for (int i = 0; i < 8; i++) n[i] = (uint8_t)(nonce >> (8 * i));
  o_blake3_update(&h, n, 8);
  uint8_t d[32];
  o_blake3_final(&h, d);
  uint32_t v = (uint32_t)d[0] << 24 | (uint32_t)d[1] << 16 | (uint32_t)d[2] << 8 | d[3];
  uint32_t lz = v == 0 ? 32 : (uint32_t)__builtin_clz(v);
  return lz >= bits;
}

/* crates/transcript/src/prover.rs:29-41 and pow.rs:11-36 */
void o_ts_grind(o_transcript *t, const char *label, uint32_t bits) {
  if (bits == 0) return;
  size_t ll = strlen(label);
  o_ts_public(t, "bitz-transcript-pow-v1", 22);
  uint8_t l8[8];
  for (int i = 0; i < 8; i++) l8[i] = (uint8_t)((uint64_t)ll >> (8 * i));
  o_ts_public(t, l8, 8);
  o_ts_public(t, label, ll);
  uint8_t b4[4];
  for (int i = 0; i < 4; i++) b4[i] = (uint8_t)(bits >> (8 * i));
  o_ts_public(t, b4, 4);
  uint8_t seed[16];
  o_ts_squeeze(t, seed, 16);
  uint64_t nonce = 0;
  while (!o_pow_valid(seed, nonce, bits)) nonce++;
  uint8_t n8[8];
  for (int i = 0; i < 8; i++) n8[i] = (uint8_t)(nonce >> (8 * i));
  o_ts_prover(t, n8, 8);
}

/* crates/field/src/helpers.rs:5,14-31 */
static int sieve(u128 c, int *decided) {
  static const int P[13] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41};
  *decided = 1;
  if (c < 2) return 0;
  for (int i = 0; i < 13; i++) {
    if (c == (u128)P[i]) return 1;
    if (c % P[i] == 0) return 0;
  }
  *decided = 0;
  return 0;
}

/* crates/transcript/src/challenge/prime.rs:52-61 */
static u128 sample_below(o_transcript *t, u128 bound) {
  u128 b = bound - 1;
  int lz = 0;
  while (lz < 128 && !((b >> (127 - lz)) & 1)) lz++;
  u128 mask = lz >= 128 ? 0 : (~(u128)0) >> lz;
  for (;;) {
    u128 c = o_ts_u128(t) & mask;
    if (c < bound) return c;
  }
}

/* crates/transcript/src/challenge/prime.rs:33-47: 80 Miller-Rabin rounds whose
 * bases come from the stream, drawn one at a time until one fails. */
u128 o_ts_prime(o_transcript *t, uint32_t bits) {
  u128 bottom = (u128)1 << (bits - 1);
  for (;;) {
    u128 cand = bottom | (o_ts_u128(t) & (bottom - 1)) | 1;
    int decided;
    int prime = sieve(cand, &decided);
    if (!decided) {
      prime = 1;
      for (int r = 0; r < 80; r++) {
        u128 base = 2 + sample_below(t, cand - 3);
        if (!o_fp_is_prime_mr(cand, &base, 1)) {
          prime = 0;
          break;
        }
      }
    }
    if (prime) return cand;
  }
}

/* Heap-allocated transcripts for callers that cannot size the struct. */
o_transcript *o_ts_new(const uint8_t *session, size_t slen, const uint8_t *instance, size_t ilen) {
  o_transcript *t = (o_transcript *)malloc(sizeof(o_transcript));
  o_ts_init(t, session, slen, instance, ilen);
  return t;
}

void o_ts_delete(o_transcript *t) {
  o_ts_free(t);
  free(t);
}

size_t o_ts_narg(const o_transcript *t, uint8_t *out, size_t cap) {
  if (out && cap >= t->narg_len) memcpy(out, t->narg, t->narg_len);
  return t->narg_len;
}

void o_ts_prime_le(o_transcript *t, uint32_t bits, uint8_t out[16]) {
  u128 p = o_ts_prime(t, bits);
  for (int i = 0; i < 16; i++) out[i] = (uint8_t)(p >> (8 * i));
}
