/* CPU oracle: Keccak-f[1600] (FIPS 202), SHA-256 (FIPS 180-4) and BLAKE3
 * (BLAKE3 specification, O'Connor et al. 2020), restated from the published
 * standards. Test infrastructure only. */
#include <string.h>

#include "oracle.h"

/* ------------------------------------------------------------ Keccak-f1600 */
static const uint64_t KRC[24] = {
    0x0000000000000001ull, 0x0000000000008082ull, 0x800000000000808aull, 0x8000000080008000ull,
    0x000000000000808bull, 0x0000000080000001ull, 0x8000000080008081ull, 0x8000000000008009ull,
    0x000000000000008aull, 0x0000000000000088ull, 0x0000000080008009ull, 0x000000008000000aull,
    0x000000008000808bull, 0x800000000000008bull, 0x8000000000008089ull, 0x8000000000008003ull,
    0x8000000000008002ull, 0x8000000000000080ull, 0x000000000000800aull, 0x800000008000000aull,
    0x8000000080008081ull, 0x8000000000008080ull, 0x0000000080000001ull, 0x8000000080008008ull};
static const int KROT[25] = {0,  1,  62, 28, 27, 36, 44, 6,  55, 20, 3,  10, 43,
                             25, 39, 41, 45, 15, 21, 8,  18, 2,  61, 56, 14};

static uint64_t rotl(uint64_t x, int n) { return n == 0 ? x : (x << n) | (x >> (64 - n)); }

/* FIPS 202 section 3.3: theta, rho, pi, chi, iota; lane (x, y) at index x + 5y. */
void o_keccak_f1600(uint64_t a[25]) {
  for (int round = 0; round < 24; round++) {
    uint64_t c[5], d[5], b[25];
    for (int x = 0; x < 5; x++) c[x] = a[x] ^ a[x + 5] ^ a[x + 10] ^ a[x + 15] ^ a[x + 20];
    for (int x = 0; x < 5; x++) d[x] = c[(x + 4) % 5] ^ rotl(c[(x + 1) % 5], 1);
    for (int i = 0; i < 25; i++) a[i] ^= d[i % 5];
    for (int x = 0; x < 5; x++)
      for (int y = 0; y < 5; y++) b[y + 5 * ((2 * x + 3 * y) % 5)] = rotl(a[x + 5 * y], KROT[x + 5 * y]);
    for (int x = 0; x < 5; x++)
      for (int y = 0; y < 5; y++)
        a[x + 5 * y] = b[x + 5 * y] ^ (~b[(x + 1) % 5 + 5 * y] & b[(x + 2) % 5 + 5 * y]);
    a[0] ^= KRC[round];
  }
}

static void st_xor_byte(uint64_t st[25], int pos, uint8_t v) {
  st[pos / 8] ^= (uint64_t)v << (8 * (pos % 8));
}

static uint8_t st_byte(const uint64_t st[25], int pos) { return (uint8_t)(st[pos / 8] >> (8 * (pos % 8))); }

void o_sha3_256(const uint8_t *in, size_t len, uint8_t out[32]) {
  uint64_t st[25];
  memset(st, 0, sizeof st);
  const int rate = 136;
  size_t off = 0;
  while (len - off >= (size_t)rate) {
    for (int i = 0; i < rate; i++) st_xor_byte(st, i, in[off + i]);
    o_keccak_f1600(st);
    off += rate;
  }
  int rem = (int)(len - off);
  for (int i = 0; i < rem; i++) st_xor_byte(st, i, in[off + i]);
  st_xor_byte(st, rem, 0x06);
  st_xor_byte(st, rate - 1, 0x80);
  o_keccak_f1600(st);
  for (int i = 0; i < 32; i++) out[i] = st_byte(st, i);
}

/* ----------------------------------------------------------------- SHA-256 */
static const uint32_t SK[64] = {
    0x428a2f98, 0x71374491, 0xb5c0fbcf, 0xe9b5dba5, 0x3956c25b, 0x59f111f1, 0x923f82a4, 0xab1c5ed5,
    0xd807aa98, 0x12835b01, 0x243185be, 0x550c7dc3, 0x72be5d74, 0x80deb1fe, 0x9bdc06a7, 0xc19bf174,
    0xe49b69c1, 0xefbe4786, 0x0fc19dc6, 0x240ca1cc, 0x2de92c6f, 0x4a7484aa, 0x5cb0a9dc, 0x76f988da,
    0x983e5152, 0xa831c66d, 0xb00327c8, 0xbf597fc7, 0xc6e00bf3, 0xd5a79147, 0x06ca6351, 0x14292967,
    0x27b70a85, 0x2e1b2138, 0x4d2c6dfc, 0x53380d13, 0x650a7354, 0x766a0abb, 0x81c2c92e, 0x92722c85,
    0xa2bfe8a1, 0xa81a664b, 0xc24b8b70, 0xc76c51a3, 0xd192e819, 0xd6990624, 0xf40e3585, 0x106aa070,
    0x19a4c116, 0x1e376c08, 0x2748774c, 0x34b0bcb5, 0x391c0cb3, 0x4ed8aa4a, 0x5b9cca4f, 0x682e6ff3,
    0x748f82ee, 0x78a5636f, 0x84c87814, 0x8cc70208, 0x90befffa, 0xa4506ceb, 0xbef9a3f7, 0xc67178f2};

static uint32_t ror(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }

void o_sha256_compress(uint32_t s[8], const uint32_t m[16]) {
  uint32_t w[64];
  for (int i = 0; i < 16; i++) w[i] = m[i];
  for (int i = 16; i < 64; i++) {
    uint32_t s0 = ror(w[i - 15], 7) ^ ror(w[i - 15], 18) ^ (w[i - 15] >> 3);
    uint32_t s1 = ror(w[i - 2], 17) ^ ror(w[i - 2], 19) ^ (w[i - 2] >> 10);
    w[i] = w[i - 16] + s0 + w[i - 7] + s1;
  }
  uint32_t a = s[0], b = s[1], c = s[2], d = s[3], e = s[4], f = s[5], g = s[6], h = s[7];
  for (int i = 0; i < 64; i++) {
    uint32_t t1 = h + (ror(e, 6) ^ ror(e, 11) ^ ror(e, 25)) + ((e & f) ^ (~e & g)) + SK[i] + w[i];
    uint32_t t2 = (ror(a, 2) ^ ror(a, 13) ^ ror(a, 22)) + ((a & b) ^ (a & c) ^ (b & c));
    h = g;
    g = f;
    f = e;
    e = d + t1;
    d = c;
    c = b;
    b = a;
    a = t1 + t2;
  }
  s[0] += a;
  s[1] += b;
  s[2] += c;
  s[3] += d;
  s[4] += e;
  s[5] += f;
  s[6] += g;
  s[7] += h;
}

static void be_words(const uint8_t *b, uint32_t m[16]) {
  for (int i = 0; i < 16; i++)
    m[i] = (uint32_t)b[4 * i] << 24 | (uint32_t)b[4 * i + 1] << 16 | (uint32_t)b[4 * i + 2] << 8 | b[4 * i + 3];
}

void o_sha256(const uint8_t *in, size_t len, uint8_t out[32]) {
  uint32_t s[8] = {0x6a09e667, 0xbb67ae85, 0x3c6ef372, 0xa54ff53a,
                   0x510e527f, 0x9b05688c, 0x1f83d9ab, 0x5be0cd19};
  uint32_t m[16];
  size_t full = len / 64;
  for (size_t b = 0; b < full; b++) {
    be_words(in + 64 * b, m);
    o_sha256_compress(s, m);
  }
  uint8_t tail[128];
  memset(tail, 0, sizeof tail);
  size_t rem = len - 64 * full;
  memcpy(tail, in + 64 * full, rem);
  tail[rem] = 0x80;
  size_t tlen = rem < 56 ? 64 : 128;
  uint64_t bits = (uint64_t)len * 8;
  for (int i = 0; i < 8; i++) tail[tlen - 1 - i] = (uint8_t)(bits >> (8 * i));
  for (size_t off = 0; off < tlen; off += 64) {
    be_words(tail + off, m);
    o_sha256_compress(s, m);
  }
  for (int i = 0; i < 8; i++) {
    out[4 * i] = (uint8_t)(s[i] >> 24);
    out[4 * i + 1] = (uint8_t)(s[i] >> 16);
    out[4 * i + 2] = (uint8_t)(s[i] >> 8);
    out[4 * i + 3] = (uint8_t)s[i];
  }
}

/* ------------------------------------------------------------------ BLAKE3 */
static const uint32_t B3IV[8] = {0x6A09E667, 0xBB67AE85, 0x3C6EF372, 0xA54FF53A,
                                 0x510E527F, 0x9B05688C, 0x1F83D9AB, 0x5BE0CD19};
static const int B3PERM[16] = {2, 6, 3, 10, 7, 0, 4, 13, 1, 11, 12, 5, 9, 14, 15, 8};
enum { CHUNK_START = 1, CHUNK_END = 2, PARENT = 4, ROOT = 8, KEYED_HASH = 16,
       DERIVE_KEY_CONTEXT = 32, DERIVE_KEY_MATERIAL = 64 };

static void b3g(uint32_t *s, int a, int b, int c, int d, uint32_t x, uint32_t y) {
  s[a] = s[a] + s[b] + x;
  s[d] = ror(s[d] ^ s[a], 16);
  s[c] = s[c] + s[d];
  s[b] = ror(s[b] ^ s[c], 12);
  s[a] = s[a] + s[b] + y;
  s[d] = ror(s[d] ^ s[a], 8);
  s[c] = s[c] + s[d];
  s[b] = ror(s[b] ^ s[c], 7);
}

static void b3_compress(const uint32_t cv[8], const uint32_t m_in[16], uint64_t counter,
                        uint32_t len, uint32_t flags, uint32_t out[16]) {
  uint32_t s[16] = {cv[0], cv[1], cv[2], cv[3], cv[4], cv[5], cv[6], cv[7],
                    B3IV[0], B3IV[1], B3IV[2], B3IV[3], (uint32_t)counter,
                    (uint32_t)(counter >> 32), len, flags};
  uint32_t m[16];
  memcpy(m, m_in, sizeof m);
  for (int r = 0; r < 7; r++) {
    b3g(s, 0, 4, 8, 12, m[0], m[1]);
    b3g(s, 1, 5, 9, 13, m[2], m[3]);
    b3g(s, 2, 6, 10, 14, m[4], m[5]);
    b3g(s, 3, 7, 11, 15, m[6], m[7]);
    b3g(s, 0, 5, 10, 15, m[8], m[9]);
    b3g(s, 1, 6, 11, 12, m[10], m[11]);
    b3g(s, 2, 7, 8, 13, m[12], m[13]);
    b3g(s, 3, 4, 9, 14, m[14], m[15]);
    if (r < 6) {
      uint32_t t[16];
      for (int i = 0; i < 16; i++) t[i] = m[B3PERM[i]];
      memcpy(m, t, sizeof m);
    }
  }
  for (int i = 0; i < 8; i++) {
    out[i] = s[i] ^ s[i + 8];
    out[i + 8] = s[i + 8] ^ cv[i];
  }
}

static void words_le(const uint8_t *b, uint32_t *w, int n) {
  for (int i = 0; i < n; i++)
    w[i] = (uint32_t)b[4 * i] | (uint32_t)b[4 * i + 1] << 8 | (uint32_t)b[4 * i + 2] << 16 | (uint32_t)b[4 * i + 3] << 24;
}

static void b3_init_key(o_blake3_state *h, const uint32_t key[8], uint32_t flags) {
  memset(h, 0, sizeof *h);
  memcpy(h->key, key, 32);
  memcpy(h->cv, key, 32);
  h->flags = flags;
}

void o_blake3_init(o_blake3_state *h) { b3_init_key(h, B3IV, 0); }

void o_blake3_init_derive_key(o_blake3_state *h, const char *context) {
  o_blake3_state c;
  b3_init_key(&c, B3IV, DERIVE_KEY_CONTEXT);
  o_blake3_update(&c, (const uint8_t *)context, strlen(context));
  uint8_t k[32];
  o_blake3_final(&c, k);
  uint32_t kw[8];
  words_le(k, kw, 8);
  b3_init_key(h, kw, DERIVE_KEY_MATERIAL);
}

static void b3_push_cv(o_blake3_state *h, uint32_t cv[8], uint64_t total_chunks) {
  /* merge while the number of completed chunks has trailing zero bits */
  while ((total_chunks & 1) == 0) {
    uint32_t m[16], out[16];
    memcpy(m, h->stack[--h->stack_len], 32);
    memcpy(m + 8, cv, 32);
    b3_compress(h->key, m, 0, 64, h->flags | PARENT, out);
    memcpy(cv, out, 32);
    total_chunks >>= 1;
  }
  memcpy(h->stack[h->stack_len++], cv, 32);
}

void o_blake3_update(o_blake3_state *h, const uint8_t *in, size_t len) {
  while (len > 0) {
    if (h->chunk_len == 1024) {
      /* finish the chunk: its last block is already buffered */
      uint32_t m[16], out[16];
      words_le(h->buf, m, 16);
      uint32_t fl = h->flags | CHUNK_END | (h->blocks_compressed == 0 ? CHUNK_START : 0);
      b3_compress(h->cv, m, h->chunk_counter, (uint32_t)h->buf_len, fl, out);
      uint32_t cv[8];
      memcpy(cv, out, 32);
      h->chunk_counter++;
      b3_push_cv(h, cv, h->chunk_counter);
      memcpy(h->cv, h->key, 32);
      h->chunk_len = 0;
      h->buf_len = 0;
      h->blocks_compressed = 0;
    }
    if (h->buf_len == 64) {
      uint32_t m[16], out[16];
      words_le(h->buf, m, 16);
      uint32_t fl = h->flags | (h->blocks_compressed == 0 ? CHUNK_START : 0);
      b3_compress(h->cv, m, h->chunk_counter, 64, fl, out);
      memcpy(h->cv, out, 32);
      h->blocks_compressed++;
      h->buf_len = 0;
    }
    size_t want = 64 - h->buf_len;
    size_t room = 1024 - h->chunk_len;
    if (want > room) want = room;
    if (want > len) want = len;
    memcpy(h->buf + h->buf_len, in, want);
    h->buf_len += want;
    h->chunk_len += want;
    in += want;
    len -= want;
  }
}

void o_blake3_final(const o_blake3_state *h, uint8_t out[32]) {
  uint32_t m[16], o[16];
  uint8_t blk[64];
  memset(blk, 0, 64);
  memcpy(blk, h->buf, h->buf_len);
  words_le(blk, m, 16);
  uint32_t fl = h->flags | CHUNK_END | (h->blocks_compressed == 0 ? CHUNK_START : 0);
  if (h->stack_len == 0) {
    b3_compress(h->cv, m, h->chunk_counter, (uint32_t)h->buf_len, fl | ROOT, o);
  } else {
    b3_compress(h->cv, m, h->chunk_counter, (uint32_t)h->buf_len, fl, o);
    uint32_t cv[8];
    memcpy(cv, o, 32);
    for (int i = h->stack_len - 1; i >= 0; i--) {
      uint32_t pm[16];
      memcpy(pm, h->stack[i], 32);
      memcpy(pm + 8, cv, 32);
      uint32_t pf = h->flags | PARENT | (i == 0 ? ROOT : 0);
      b3_compress(h->key, pm, 0, 64, pf, o);
      memcpy(cv, o, 32);
    }
  }
  for (int i = 0; i < 8; i++) {
    out[4 * i] = (uint8_t)o[i];
    out[4 * i + 1] = (uint8_t)(o[i] >> 8);
    out[4 * i + 2] = (uint8_t)(o[i] >> 16);
    out[4 * i + 3] = (uint8_t)(o[i] >> 24);
  }
}

void o_blake3(const uint8_t *in, size_t len, uint8_t out[32]) {
  o_blake3_state h;
  o_blake3_init(&h);
  o_blake3_update(&h, in, len);
  o_blake3_final(&h, out);
}

/* Derive-key mode over `in`, fed in pieces of `piece` bytes (0: in one
 * update), so the streaming state is exercised at every split. */
void o_blake3_derive_key(const char *context, const uint8_t *in, size_t len, size_t piece,
                         uint8_t out[32]) {
  o_blake3_state h;
  o_blake3_init_derive_key(&h, context);
  if (!piece) piece = len ? len : 1;
  for (size_t i = 0; i < len; i += piece) o_blake3_update(&h, in + i, len - i < piece ? len - i : piece);
  o_blake3_final(&h, out);
}
