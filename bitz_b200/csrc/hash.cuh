// Keccak-f[1600] (FIPS 202) for the host transcript sponge, and the BLAKE3
// compression function (BLAKE3 specification, O'Connor et al. 2020) shared by
// host and device code. BLAKE3 hashes the grinding nonces
// (crates/transcript/src/pow.rs:38-50), the inner-product weight digest
// (crates/pcs/src/opening.rs:337-368), the virtual-map digest
// (crates/circuit/src/matrix_transpose.rs:424-441) and the Merkle trees.
#pragma once
#include <stdint.h>
#include <string.h>

#include "field.cuh"

namespace bz {

// ------------------------------------------------------------------ BLAKE3
enum : uint32_t {
  B3_CHUNK_START = 1,
  B3_CHUNK_END = 2,
  B3_PARENT = 4,
  B3_ROOT = 8,
  B3_DERIVE_KEY_CONTEXT = 32,
  B3_DERIVE_KEY_MATERIAL = 64
};

BZ_HD uint32_t rotr32(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }

BZ_HD void b3_g(uint32_t *s, int a, int b, int c, int d, uint32_t x, uint32_t y) {
  s[a] = s[a] + s[b] + x;
  s[d] = rotr32(s[d] ^ s[a], 16);
  s[c] = s[c] + s[d];
  s[b] = rotr32(s[b] ^ s[c], 12);
  s[a] = s[a] + s[b] + y;
  s[d] = rotr32(s[d] ^ s[a], 8);
  s[c] = s[c] + s[d];
  s[b] = rotr32(s[b] ^ s[c], 7);
}

// One compression; writes the 8-word chaining value (the first half of the
// 16-word output, which is all this protocol ever reads).
BZ_HD void b3_compress(const uint32_t cv[8], const uint32_t m_in[16], uint64_t counter,
                       uint32_t len, uint32_t flags, uint32_t out[8]) {
  const uint32_t IV[8] = {0x6A09E667, 0xBB67AE85, 0x3C6EF372, 0xA54FF53A,
                          0x510E527F, 0x9B05688C, 0x1F83D9AB, 0x5BE0CD19};
  uint32_t s[16] = {cv[0], cv[1], cv[2], cv[3], cv[4], cv[5], cv[6], cv[7],
                    IV[0], IV[1], IV[2], IV[3], (uint32_t)counter, (uint32_t)(counter >> 32),
                    len, flags};
  uint32_t m[16];
  for (int i = 0; i < 16; i++) m[i] = m_in[i];
#pragma unroll
  for (int r = 0; r < 7; r++) {
    b3_g(s, 0, 4, 8, 12, m[0], m[1]);
    b3_g(s, 1, 5, 9, 13, m[2], m[3]);
    b3_g(s, 2, 6, 10, 14, m[4], m[5]);
    b3_g(s, 3, 7, 11, 15, m[6], m[7]);
    b3_g(s, 0, 5, 10, 15, m[8], m[9]);
    b3_g(s, 1, 6, 11, 12, m[10], m[11]);
    b3_g(s, 2, 7, 8, 13, m[12], m[13]);
    b3_g(s, 3, 4, 9, 14, m[14], m[15]);
    if (r < 6) {
      // message schedule permutation 2,6,3,10,7,0,4,13,1,11,12,5,9,14,15,8
      uint32_t t[16] = {m[2], m[6], m[3], m[10], m[7], m[0], m[4], m[13],
                        m[1], m[11], m[12], m[5], m[9], m[14], m[15], m[8]};
      for (int i = 0; i < 16; i++) m[i] = t[i];
    }
  }
  for (int i = 0; i < 8; i++) out[i] = s[i] ^ s[i + 8];
}

BZ_HD void b3_load_le(const uint8_t *b, uint32_t *w, int n) {
  for (int i = 0; i < n; i++)
    w[i] = (uint32_t)b[4 * i] | (uint32_t)b[4 * i + 1] << 8 | (uint32_t)b[4 * i + 2] << 16 |
           (uint32_t)b[4 * i + 3] << 24;
}

BZ_HD void b3_store_le(const uint32_t *w, uint8_t *b, int n) {
  for (int i = 0; i < n; i++) {
    b[4 * i] = (uint8_t)w[i];
    b[4 * i + 1] = (uint8_t)(w[i] >> 8);
    b[4 * i + 2] = (uint8_t)(w[i] >> 16);
    b[4 * i + 3] = (uint8_t)(w[i] >> 24);
  }
}

// Incremental host hasher (default and derive-key modes).
struct Blake3 {
  uint32_t key[8];
  uint32_t cv[8];
  uint8_t buf[64];
  uint32_t buf_len = 0;
  uint64_t chunk_counter = 0;
  uint32_t chunk_len = 0;
  uint32_t blocks = 0;
  uint32_t flags = 0;
  uint32_t stack[64][8];
  int stack_len = 0;

  Blake3() {
    static const uint32_t IV[8] = {0x6A09E667, 0xBB67AE85, 0x3C6EF372, 0xA54FF53A,
                                   0x510E527F, 0x9B05688C, 0x1F83D9AB, 0x5BE0CD19};
    init(IV, 0);
  }
  void init(const uint32_t k[8], uint32_t f) {
    memcpy(key, k, 32);
    memcpy(cv, k, 32);
    buf_len = 0;
    chunk_counter = 0;
    chunk_len = 0;
    blocks = 0;
    flags = f;
    stack_len = 0;
  }
  static Blake3 derive_key(const char *context) {
    Blake3 c;
    c.flags = B3_DERIVE_KEY_CONTEXT;
    c.update((const uint8_t *)context, strlen(context));
    uint8_t k[32];
    c.finalize(k);
    uint32_t kw[8];
    b3_load_le(k, kw, 8);
    Blake3 h;
    h.init(kw, B3_DERIVE_KEY_MATERIAL);
    return h;
  }
  void push_cv(uint32_t ncv[8], uint64_t total) {
    while ((total & 1) == 0) {
      uint32_t m[16];
      memcpy(m, stack[--stack_len], 32);
      memcpy(m + 8, ncv, 32);
      b3_compress(key, m, 0, 64, flags | B3_PARENT, ncv);
      total >>= 1;
    }
    memcpy(stack[stack_len++], ncv, 32);
  }
  void update(const uint8_t *in, size_t len) {
    while (len > 0) {
      if (chunk_len == 1024) {
        uint32_t m[16], out[8];
        b3_load_le(buf, m, 16);
        uint32_t fl = flags | B3_CHUNK_END | (blocks == 0 ? B3_CHUNK_START : 0);
        b3_compress(cv, m, chunk_counter, buf_len, fl, out);
        chunk_counter++;
        push_cv(out, chunk_counter);
        memcpy(cv, key, 32);
        chunk_len = 0;
        buf_len = 0;
        blocks = 0;
      }
      if (buf_len == 64) {
        uint32_t m[16];
        b3_load_le(buf, m, 16);
        uint32_t fl = flags | (blocks == 0 ? B3_CHUNK_START : 0);
        b3_compress(cv, m, chunk_counter, 64, fl, cv);
        blocks++;
        buf_len = 0;
      }
      size_t want = 64 - buf_len;
      size_t room = 1024 - chunk_len;
      if (want > room) want = room;
      if (want > len) want = len;
      memcpy(buf + buf_len, in, want);
      buf_len += (uint32_t)want;
      chunk_len += (uint32_t)want;
      in += want;
      len -= want;
    }
  }
  void finalize(uint8_t out[32]) const {
    uint32_t m[16], o[8];
    uint8_t blk[64];
    memset(blk, 0, 64);
    memcpy(blk, buf, buf_len);
    b3_load_le(blk, m, 16);
    uint32_t fl = flags | B3_CHUNK_END | (blocks == 0 ? B3_CHUNK_START : 0);
    if (stack_len == 0) {
      b3_compress(cv, m, chunk_counter, buf_len, fl | B3_ROOT, o);
    } else {
      b3_compress(cv, m, chunk_counter, buf_len, fl, o);
      for (int i = stack_len - 1; i >= 0; i--) {
        uint32_t pm[16];
        memcpy(pm, stack[i], 32);
        memcpy(pm + 8, o, 32);
        b3_compress(key, pm, 0, 64, flags | B3_PARENT | (i == 0 ? B3_ROOT : 0), o);
      }
    }
    b3_store_le(o, out, 8);
  }
};

}  // namespace bz
