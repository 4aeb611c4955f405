// Symbolic replay of the SHA-256 circuits (setup only: no witness values).
#include "circuit.hpp"

#include <immintrin.h>
#include <string.h>

#include <algorithm>
#include <stdexcept>

#include "hash.cuh"

namespace bz {

const char *circuit_name(int kind) {
  static const char *n[4] = {"sha256-compression", "sha256-chain", "sha256-block-aligned",
                             "sha256-2kb"};
  return (kind >= 0 && kind < 4) ? n[kind] : "unknown";
}

namespace {

// An F2 linear combination over (1 || f): sorted positions, 0 is the constant.
// SHA-256 never XORs more than three single bits and a constant.
struct Lc {
  uint8_t n = 0;
  uint32_t p[4];
};

Lc lc_const(bool b) {
  Lc r;
  if (b) r.p[r.n++] = 0;
  return r;
}

Lc lc_bit(uint32_t f_index) {
  Lc r;
  r.p[r.n++] = f_index + 1;
  return r;
}

Lc lc_xor(const Lc &a, const Lc &b) {
  Lc r;
  int i = 0, j = 0;
  while (i < a.n || j < b.n) {
    if (j == b.n || (i < a.n && a.p[i] < b.p[j])) {
      r.p[r.n++] = a.p[i++];
    } else if (i == a.n || b.p[j] < a.p[i]) {
      r.p[r.n++] = b.p[j++];
    } else {
      i++, j++;
    }
    if (r.n > 4) throw std::runtime_error("bool combination wider than 4");
  }
  return r;
}

struct Word {
  Lc b[35];
};

// z-side value of a word: sum_i 2^i h[col + i] for i < width, or a constant.
struct Span {
  uint32_t col = 0;
  int width = 0;
  int64_t konst = 0;
};

struct Term {
  Span s;
  int64_t scale;
};

struct UInt {
  Word w;
  Span z;  // the low 32 bits
};

struct Builder {
  CircuitSetup &S;
  uint32_t next_f;
  explicit Builder(CircuitSetup &s, size_t n_inputs) : S(s), next_f((uint32_t)n_inputs) {
    S.m_off.assign(1, 0);
    push_row(lc_const(true));  // row 0: the constant one
    for (auto &m : S.abc) m.off.assign(1, 0);
  }

  uint32_t h_count() const { return (uint32_t)S.m_off.size() - 1; }

  void push_row(const Lc &l) {
    for (int i = 0; i < l.n; i++) S.m_pos.push_back(l.p[i]);
    S.m_off.push_back((uint32_t)S.m_pos.size());
  }

  // Circuit::bitz_unsigned (constraints.rs:842-866): one lift per bit.
  Span lift(const Word &w, int width) {
    Span s;
    s.col = h_count();
    s.width = width;
    for (int i = 0; i < width; i++) push_row(w.b[i]);
    return s;
  }

  Word hint(int width) {
    Word w;
    for (int i = 0; i < width; i++) w.b[i] = lc_bit(next_f++);
    return w;
  }

  // One R1CS row: A = B = 0 (assert_zero, sha256.rs:218-223), C = sum of terms.
  void assert_zero(const std::vector<Term> &terms) {
    std::vector<std::pair<uint32_t, int64_t>> e;
    int64_t c0 = 0;
    for (auto &t : terms) {
      if (t.s.width == 0) {
        c0 += t.s.konst * t.scale;
        continue;
      }
      for (int i = 0; i < t.s.width; i++) e.push_back({t.s.col + i, t.scale * ((int64_t)1 << i)});
    }
    if (c0) e.push_back({0, c0});
    std::sort(e.begin(), e.end());
    Matrix &C = S.abc[2];
    size_t start = C.col.size();
    for (size_t i = 0; i < e.size();) {
      size_t j = i;
      int64_t sum = 0;
      while (j < e.size() && e[j].first == e[i].first) sum += e[j++].second;
      if (sum) {
        C.col.push_back(e[i].first);
        C.coef.push_back(sum);
      }
      i = j;
    }
    (void)start;
    C.off.push_back((uint32_t)C.col.size());
    for (int k = 0; k < 2; k++) S.abc[k].off.push_back((uint32_t)S.abc[k].col.size());
  }

  UInt uint_of(const Word &w) {
    UInt u;
    u.w = w;
    u.z = lift(w, 32);
    return u;
  }

  UInt uint_const(uint32_t v) {
    UInt u;
    for (int i = 0; i < 32; i++) u.w.b[i] = lc_const((v >> i) & 1);
    u.z.konst = v;
    return u;
  }

  // sum_32 (sha256.rs:228-262)
  UInt sum32(int width, std::initializer_list<const UInt *> terms) {
    Word bits = hint(width);
    Span full = lift(bits, width);
    std::vector<Term> t;
    for (auto *u : terms) t.push_back({u->z, 1});
    t.push_back({full, -1});
    assert_zero(t);
    UInt r;
    r.w = bits;
    r.z = full;
    r.z.width = 32;
    return r;
  }

  // sum_doubled_32 (sha256.rs:268-316): 2 * ordinary + doubled = 2 * half
  UInt sum_doubled(std::initializer_list<const UInt *> ordinary, const std::vector<Term> &doubled) {
    Word bits = hint(35);
    Span half = lift(bits, 35);
    std::vector<Term> t;
    for (auto *u : ordinary) t.push_back({u->z, 2});
    for (auto &d : doubled) t.push_back(d);
    t.push_back({half, -2});
    assert_zero(t);
    UInt r;
    r.w = bits;
    r.z = half;
    r.z.width = 32;
    return r;
  }

  static Word wxor(const Word &x, const Word &y) {
    Word r;
    for (int i = 0; i < 32; i++) r.b[i] = lc_xor(x.b[i], y.b[i]);
    return r;
  }
  static Word rotr(const Word &x, int k) {
    Word r;
    for (int i = 0; i < 32; i++) r.b[i] = x.b[(i + k) & 31];
    return r;
  }
  static Word shr(const Word &x, int k) {
    Word r;
    for (int i = 0; i < 32; i++) r.b[i] = i + k < 32 ? x.b[i + k] : lc_const(false);
    return r;
  }

  // compress (sha256.rs:344-456)
  void compress(const Word block[16], const Word state_in[8], Word out[8]) {
    S.block_f_offset.push_back(next_f);
    UInt st[8];
    for (int i = 0; i < 8; i++) st[i] = uint_of(state_in[i]);
    std::vector<UInt> w;
    w.reserve(64);
    for (int i = 0; i < 16; i++) w.push_back(uint_of(block[i]));
    for (int i = 16; i < 64; i++) {
      const Word &a = w[i - 15].w;
      UInt s0 = uint_of(wxor(wxor(rotr(a, 7), rotr(a, 18)), shr(a, 3)));
      const Word &b = w[i - 2].w;
      UInt s1 = uint_of(wxor(wxor(rotr(b, 17), rotr(b, 19)), shr(b, 10)));
      w.push_back(sum32(34, {&w[i - 16], &s0, &w[i - 7], &s1}));
    }
    static const uint32_t K[64] = {
        0x428a2f98, 0x71374491, 0xb5c0fbcf, 0xe9b5dba5, 0x3956c25b, 0x59f111f1, 0x923f82a4,
        0xab1c5ed5, 0xd807aa98, 0x12835b01, 0x243185be, 0x550c7dc3, 0x72be5d74, 0x80deb1fe,
        0x9bdc06a7, 0xc19bf174, 0xe49b69c1, 0xefbe4786, 0x0fc19dc6, 0x240ca1cc, 0x2de92c6f,
        0x4a7484aa, 0x5cb0a9dc, 0x76f988da, 0x983e5152, 0xa831c66d, 0xb00327c8, 0xbf597fc7,
        0xc6e00bf3, 0xd5a79147, 0x06ca6351, 0x14292967, 0x27b70a85, 0x2e1b2138, 0x4d2c6dfc,
        0x53380d13, 0x650a7354, 0x766a0abb, 0x81c2c92e, 0x92722c85, 0xa2bfe8a1, 0xa81a664b,
        0xc24b8b70, 0xc76c51a3, 0xd192e819, 0xd6990624, 0xf40e3585, 0x106aa070, 0x19a4c116,
        0x1e376c08, 0x2748774c, 0x34b0bcb5, 0x391c0cb3, 0x4ed8aa4a, 0x5b9cca4f, 0x682e6ff3,
        0x748f82ee, 0x78a5636f, 0x84c87814, 0x8cc70208, 0x90befffa, 0xa4506ceb, 0xbef9a3f7,
        0xc67178f2};
    UInt a = st[0], b = st[1], c = st[2], d = st[3], e = st[4], f = st[5], g = st[6], h = st[7];
    for (int i = 0; i < 64; i++) {
      UInt S1 = uint_of(wxor(wxor(rotr(e.w, 6), rotr(e.w, 11)), rotr(e.w, 25)));
      // choice_twice: y + z - (x ^ y) + (x ^ z)
      UInt xy = uint_of(wxor(e.w, f.w));
      UInt xz = uint_of(wxor(e.w, g.w));
      std::vector<Term> ch = {{f.z, 1}, {g.z, 1}, {xy.z, -1}, {xz.z, 1}};
      UInt S0 = uint_of(wxor(wxor(rotr(a.w, 2), rotr(a.w, 13)), rotr(a.w, 22)));
      // majority_twice: x + y + z - (x ^ y ^ z)
      UInt xyz = uint_of(wxor(wxor(a.w, b.w), c.w));
      std::vector<Term> mj = {{a.z, 1}, {b.z, 1}, {c.z, 1}, {xyz.z, -1}};
      UInt kc = uint_const(K[i]);
      UInt ne = sum_doubled({&d, &h, &S1, &kc, &w[i]}, ch);
      std::vector<Term> both = ch;
      both.insert(both.end(), mj.begin(), mj.end());
      UInt na = sum_doubled({&h, &S1, &kc, &w[i], &S0}, both);
      h = g;
      g = f;
      f = e;
      e = ne;
      d = c;
      c = b;
      b = a;
      a = na;
    }
    const UInt *work[8] = {&a, &b, &c, &d, &e, &f, &g, &h};
    for (int i = 0; i < 8; i++) out[i] = sum32(33, {&st[i], work[i]}).w;
  }

  // tooling/cli/src/circuits.rs:204-209: (1) * (bit) = (expected)
  void constrain_bit(const Lc &bit) {
    Word w;
    w.b[0] = bit;
    Span s = lift(w, 1);
    Matrix &A = S.abc[0], &B = S.abc[1], &C = S.abc[2];
    A.col.push_back(0);
    A.coef.push_back(1);
    A.off.push_back((uint32_t)A.col.size());
    B.col.push_back(s.col);
    B.coef.push_back(1);
    B.off.push_back((uint32_t)B.col.size());
    // C = the expected constant: filled in per statement (column 0, 0 or 1),
    // recorded here as column 0 with coefficient 1 and dropped when 0.
    C.off.push_back((uint32_t)C.col.size());
  }
};

const uint32_t IV[8] = {0x6a09e667, 0xbb67ae85, 0x3c6ef372, 0xa54ff53a,
                        0x510e527f, 0x9b05688c, 0x1f83d9ab, 0x5be0cd19};

Word const_word(uint32_t v) {
  Word w;
  for (int i = 0; i < 32; i++) w.b[i] = lc_const((v >> i) & 1);
  return w;
}

int ceil_log2(size_t n) {
  int l = 0;
  while (((size_t)1 << l) < n) l++;
  return l;
}

void put_u64(std::vector<uint8_t> &b, uint64_t v) {
  for (int i = 0; i < 8; i++) b.push_back((uint8_t)(v >> (8 * i)));
}

}  // namespace

void build_circuit_setup(int kind, size_t n_inputs, CircuitSetup &S) {
  S = CircuitSetup();
  S.kind = kind;
  S.n_inputs = n_inputs;
  Builder B(S, n_inputs);
  std::vector<Lc> in(n_inputs);
  for (size_t i = 0; i < n_inputs; i++) in[i] = lc_bit((uint32_t)i);
  for (size_t i = 0; i < n_inputs; i++) B.constrain_bit(in[i]);
  Word state[8];
  Lc out[256];
  if (kind == kCompression || kind == kChain) {
    size_t nblocks = kind == kCompression ? 1 : n_inputs / 512;
    for (int i = 0; i < 8; i++)
      for (int j = 0; j < 32; j++)
        state[i].b[j] = kind == kCompression ? in[512 + 32 * i + j] : lc_const((IV[i] >> j) & 1);
    for (size_t blk = 0; blk < nblocks; blk++) {
      Word block[16], next[8];
      for (int w = 0; w < 16; w++)
        for (int j = 0; j < 32; j++) block[w].b[j] = in[blk * 512 + 32 * w + j];
      B.compress(block, state, next);
      for (int i = 0; i < 8; i++) state[i] = next[i];
    }
    for (int i = 0; i < 256; i++) out[i] = state[i / 32].b[i % 32];
  } else {
    for (int i = 0; i < 8; i++) state[i] = const_word(IV[i]);
    for (size_t blk = 0; blk < n_inputs / 512; blk++) {
      Word block[16], next[8];
      for (int w = 0; w < 16; w++)
        for (int j = 0; j < 32; j++) block[w].b[j] = in[blk * 512 + 32 * w + (31 - j)];
      B.compress(block, state, next);
      for (int i = 0; i < 8; i++) state[i] = next[i];
    }
    uint64_t len = n_inputs;
    uint32_t pad[16] = {0x80000000u, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0,
                        (uint32_t)(len >> 32), (uint32_t)len};
    Word block[16], next[8];
    for (int w = 0; w < 16; w++) block[w] = const_word(pad[w]);
    B.compress(block, state, next);
    for (int i = 0; i < 256; i++) out[i] = next[i / 32].b[31 - (i % 32)];
  }
  for (int i = 0; i < 256; i++) B.constrain_bit(out[i]);
  S.n_blocks = S.block_f_offset.size();
  S.f_bits = B.next_f;
  S.h_len = B.h_count();
  S.rows = S.abc[2].off.size() - 1;
  int mh = ceil_log2(S.h_len), mf = ceil_log2(S.f_bits);
  S.claim_log_cols = (mh < 20 ? 20 : mh) - 7;
  S.committed_m = mf < 20 ? 20 : mf;

  // M^T as CSC, rows ascending inside each column (matrix_transpose.rs:523-560)
  size_t ncols = S.f_bits + 1;
  S.csc_off.assign(ncols + 1, 0);
  for (uint32_t p : S.m_pos) S.csc_off[p + 1]++;
  for (size_t c = 0; c < ncols; c++) S.csc_off[c + 1] += S.csc_off[c];
  S.csc_row.resize(S.m_pos.size());
  {
    std::vector<uint32_t> cur(S.csc_off.begin(), S.csc_off.end() - 1);
    for (size_t r = 0; r < S.h_len; r++)
      for (uint32_t e = S.m_off[r]; e < S.m_off[r + 1]; e++)
        S.csc_row[cur[S.m_pos[e]]++] = (uint32_t)r;
  }
  // csc_digest (matrix_transpose.rs:424-441)
  {
    Blake3 h;
    const char *dom = "bitz/virtual-map/csc/v1";
    h.update((const uint8_t *)dom, strlen(dom));
    std::vector<uint8_t> b;
    put_u64(b, S.h_len);
    put_u64(b, ncols);
    put_u64(b, S.csc_row.size());
    h.update(b.data(), b.size());
    h.update((const uint8_t *)S.csc_off.data(), S.csc_off.size() * 4);
    h.update((const uint8_t *)S.csc_row.data(), S.csc_row.size() * 4);
    h.finalize(S.map_digest);
  }
}

// integer_matrix_digest (crates/spartan/src/matrix.rs:562-661): SHA-256 over
// the positions of M, then A, B, C row by row with canonical coefficient
// words. The C rows of the bit constraints carry the statement's expected
// outputs, so the digest is finished per statement.
void matrix_digest(const CircuitSetup &S, const std::vector<int64_t> &c_bits_expected,
                   uint8_t out[32]);

// ---------------------------------------------------------------- SHA-256

static const uint32_t SHA_K[64] = {
    0x428a2f98, 0x71374491, 0xb5c0fbcf, 0xe9b5dba5, 0x3956c25b, 0x59f111f1, 0x923f82a4, 0xab1c5ed5,
    0xd807aa98, 0x12835b01, 0x243185be, 0x550c7dc3, 0x72be5d74, 0x80deb1fe, 0x9bdc06a7, 0xc19bf174,
    0xe49b69c1, 0xefbe4786, 0x0fc19dc6, 0x240ca1cc, 0x2de92c6f, 0x4a7484aa, 0x5cb0a9dc, 0x76f988da,
    0x983e5152, 0xa831c66d, 0xb00327c8, 0xbf597fc7, 0xc6e00bf3, 0xd5a79147, 0x06ca6351, 0x14292967,
    0x27b70a85, 0x2e1b2138, 0x4d2c6dfc, 0x53380d13, 0x650a7354, 0x766a0abb, 0x81c2c92e, 0x92722c85,
    0xa2bfe8a1, 0xa81a664b, 0xc24b8b70, 0xc76c51a3, 0xd192e819, 0xd6990624, 0xf40e3585, 0x106aa070,
    0x19a4c116, 0x1e376c08, 0x2748774c, 0x34b0bcb5, 0x391c0cb3, 0x4ed8aa4a, 0x5b9cca4f, 0x682e6ff3,
    0x748f82ee, 0x78a5636f, 0x84c87814, 0x8cc70208, 0x90befffa, 0xa4506ceb, 0xbef9a3f7, 0xc67178f2};

static inline uint32_t rr(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }

void sha256_compress_host(uint32_t s[8], const uint32_t m[16]) {
  uint32_t w[64];
  for (int i = 0; i < 16; i++) w[i] = m[i];
  for (int i = 16; i < 64; i++)
    w[i] = w[i - 16] + (rr(w[i - 15], 7) ^ rr(w[i - 15], 18) ^ (w[i - 15] >> 3)) + w[i - 7] +
           (rr(w[i - 2], 17) ^ rr(w[i - 2], 19) ^ (w[i - 2] >> 10));
  uint32_t a = s[0], b = s[1], c = s[2], d = s[3], e = s[4], f = s[5], g = s[6], h = s[7];
  for (int i = 0; i < 64; i++) {
    uint32_t t1 = h + (rr(e, 6) ^ rr(e, 11) ^ rr(e, 25)) + ((e & f) ^ (~e & g)) + SHA_K[i] + w[i];
    uint32_t t2 = (rr(a, 2) ^ rr(a, 13) ^ rr(a, 22)) + ((a & b) ^ (a & c) ^ (b & c));
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

void sha256_host(const uint8_t *in, size_t len, uint8_t out[32]) {
  uint32_t s[8] = {0x6a09e667, 0xbb67ae85, 0x3c6ef372, 0xa54ff53a,
                   0x510e527f, 0x9b05688c, 0x1f83d9ab, 0x5be0cd19};
  auto be = [](const uint8_t *p, uint32_t *m) {
    for (int i = 0; i < 16; i++)
      m[i] = (uint32_t)p[4 * i] << 24 | (uint32_t)p[4 * i + 1] << 16 | (uint32_t)p[4 * i + 2] << 8 |
             p[4 * i + 3];
  };
  uint32_t m[16];
  size_t full = len / 64;
  for (size_t b = 0; b < full; b++) {
    be(in + 64 * b, m);
    sha256_compress_host(s, m);
  }
  uint8_t tail[128] = {0};
  size_t rem = len - 64 * full;
  memcpy(tail, in + 64 * full, rem);
  tail[rem] = 0x80;
  size_t tlen = rem < 56 ? 64 : 128;
  uint64_t bits = (uint64_t)len * 8;
  for (int i = 0; i < 8; i++) tail[tlen - 1 - i] = (uint8_t)(bits >> (8 * i));
  for (size_t o = 0; o < tlen; o += 64) {
    be(tail + o, m);
    sha256_compress_host(s, m);
  }
  for (int i = 0; i < 8; i++) {
    out[4 * i] = (uint8_t)(s[i] >> 24);
    out[4 * i + 1] = (uint8_t)(s[i] >> 16);
    out[4 * i + 2] = (uint8_t)(s[i] >> 8);
    out[4 * i + 3] = (uint8_t)s[i];
  }
}

// SHA-256 over many blocks: the SHA extensions where the CPU has them (the
// published SHA-NI round and message-schedule instruction sequence), else the
// portable compression. The dispatch checks the extension against the
// portable code on one block before trusting it.
__attribute__((target("sha,sse4.1"))) static void sha256_blocks_ni(uint32_t st[8],
                                                                   const uint8_t *p,
                                                                   size_t nblocks) {
  const __m128i bswap = _mm_set_epi64x(0x0c0d0e0f08090a0bULL, 0x0405060700010203ULL);
  __m128i tmp = _mm_loadu_si128((const __m128i *)&st[0]);  // D C B A
  __m128i s1 = _mm_loadu_si128((const __m128i *)&st[4]);   // H G F E
  tmp = _mm_shuffle_epi32(tmp, 0xB1);                       // C D A B
  s1 = _mm_shuffle_epi32(s1, 0x1B);                         // E F G H
  __m128i s0 = _mm_alignr_epi8(tmp, s1, 8);                 // A B E F
  s1 = _mm_blend_epi16(s1, tmp, 0xF0);                      // C D G H
  for (; nblocks; nblocks--, p += 64) {
    const __m128i abef = s0, cdgh = s1;
    __m128i w[4];
    for (int g = 0; g < 16; g++) {
      __m128i wg;
      if (g < 4) {
        wg = _mm_shuffle_epi8(_mm_loadu_si128((const __m128i *)(p + 16 * g)), bswap);
      } else {
        // W[4g..4g+3] from the four previous groups
        __m128i a = w[g & 3], b = w[(g + 1) & 3], c = w[(g + 2) & 3], d = w[(g + 3) & 3];
        wg = _mm_sha256msg2_epu32(
            _mm_add_epi32(_mm_sha256msg1_epu32(a, b), _mm_alignr_epi8(d, c, 4)), d);
      }
      w[g & 3] = wg;
      __m128i msg = _mm_add_epi32(wg, _mm_loadu_si128((const __m128i *)&SHA_K[4 * g]));
      s1 = _mm_sha256rnds2_epu32(s1, s0, msg);
      s0 = _mm_sha256rnds2_epu32(s0, s1, _mm_shuffle_epi32(msg, 0x0E));
    }
    s0 = _mm_add_epi32(s0, abef);
    s1 = _mm_add_epi32(s1, cdgh);
  }
  tmp = _mm_shuffle_epi32(s0, 0x1B);   // F E B A
  s1 = _mm_shuffle_epi32(s1, 0xB1);    // D C H G
  s0 = _mm_blend_epi16(tmp, s1, 0xF0); // D C B A
  s1 = _mm_alignr_epi8(s1, tmp, 8);    // H G F E
  _mm_storeu_si128((__m128i *)&st[0], s0);
  _mm_storeu_si128((__m128i *)&st[4], s1);
}

static void sha256_blocks_portable(uint32_t s[8], const uint8_t *p, size_t nblocks) {
  uint32_t m[16];
  for (; nblocks; nblocks--, p += 64) {
    for (int i = 0; i < 16; i++)
      m[i] = (uint32_t)p[4 * i] << 24 | (uint32_t)p[4 * i + 1] << 16 | (uint32_t)p[4 * i + 2] << 8 |
             p[4 * i + 3];
    sha256_compress_host(s, m);
  }
}

static bool sha_ni_usable() {
  if (!__builtin_cpu_supports("sha") || !__builtin_cpu_supports("sse4.1")) return false;
  uint8_t blk[128];
  for (int i = 0; i < 128; i++) blk[i] = (uint8_t)(i * 37 + 11);
  uint32_t a[8] = {0x6a09e667, 0xbb67ae85, 0x3c6ef372, 0xa54ff53a,
                   0x510e527f, 0x9b05688c, 0x1f83d9ab, 0x5be0cd19};
  uint32_t b[8];
  memcpy(b, a, sizeof a);
  sha256_blocks_ni(a, blk, 2);
  sha256_blocks_portable(b, blk, 2);
  return memcmp(a, b, sizeof a) == 0;
}

static void sha256_blocks(uint32_t s[8], const uint8_t *p, size_t nblocks) {
  static const bool ni = sha_ni_usable();
  if (ni)
    sha256_blocks_ni(s, p, nblocks);
  else
    sha256_blocks_portable(s, p, nblocks);
}

// SHA-256 over a byte stream fed in pieces (the digest input is large).
struct Sha256Stream {
  uint32_t s[8] = {0x6a09e667, 0xbb67ae85, 0x3c6ef372, 0xa54ff53a,
                   0x510e527f, 0x9b05688c, 0x1f83d9ab, 0x5be0cd19};
  uint8_t buf[64];
  size_t n = 0;
  uint64_t total = 0;
  void update(const uint8_t *p, size_t len) {
    total += len;
    if (n) {
      size_t take = 64 - n < len ? 64 - n : len;
      memcpy(buf + n, p, take);
      n += take;
      p += take;
      len -= take;
      if (n < 64) return;
      sha256_blocks(s, buf, 1);
      n = 0;
    }
    size_t full = len / 64;
    if (full) sha256_blocks(s, p, full);
    p += 64 * full;
    len -= 64 * full;
    memcpy(buf, p, len);
    n = len;
  }
  void u64(uint64_t v) {
    uint8_t b[8];
    for (int i = 0; i < 8; i++) b[i] = (uint8_t)(v >> (8 * i));
    update(b, 8);
  }
  void finish(uint8_t out[32]) {
    uint64_t bits = total * 8;
    uint8_t pad[72] = {0x80};
    size_t padlen = n < 56 ? 56 - n : 120 - n;
    uint8_t l[8];
    for (int i = 0; i < 8; i++) l[i] = (uint8_t)(bits >> (56 - 8 * i));
    update(pad, padlen);
    update(l, 8);
    for (int i = 0; i < 8; i++) {
      out[4 * i] = (uint8_t)(s[i] >> 24);
      out[4 * i + 1] = (uint8_t)(s[i] >> 16);
      out[4 * i + 2] = (uint8_t)(s[i] >> 8);
      out[4 * i + 3] = (uint8_t)s[i];
    }
  }
};

// Little-endian u64 words gathered into 16 KB before they reach the hash.
struct WordSink {
  Sha256Stream &h;
  uint8_t buf[16384];
  size_t n = 0;
  explicit WordSink(Sha256Stream &hh) : h(hh) {}
  ~WordSink() { flush(); }
  void flush() {
    if (n) h.update(buf, n);
    n = 0;
  }
  void bytes(const void *p, size_t len) {
    flush();
    h.update((const uint8_t *)p, len);
  }
  void u64(uint64_t v) {
    if (n + 8 > sizeof buf) flush();
    for (int i = 0; i < 8; i++) buf[n + i] = (uint8_t)(v >> (8 * i));
    n += 8;
  }
};

// The statement-independent prefix of the integer-matrix digest (the domain,
// M, A and B): hashed once per circuit shape, resumed per statement.
static void digest_prefix(const CircuitSetup &S, Sha256Stream &h) {
  WordSink w(h);
  const char *dom = "bitz/spartan/integer-constraint-matrices/v1";
  w.bytes(dom, strlen(dom));
  w.bytes("M", 1);
  w.u64(S.h_len);
  w.u64(S.f_bits + 1);
  for (size_t r = 0; r < S.h_len; r++) {
    w.u64(S.m_off[r + 1] - S.m_off[r]);
    for (uint32_t e = S.m_off[r]; e < S.m_off[r + 1]; e++) w.u64(S.m_pos[e]);
  }
  const char lab[2] = {'A', 'B'};
  for (int k = 0; k < 2; k++) {
    w.bytes(&lab[k], 1);
    w.u64(S.rows);
    w.u64(S.h_len);
    const Matrix &M = S.abc[k];
    for (size_t r = 0; r < S.rows; r++) {
      w.u64(M.off[r + 1] - M.off[r]);
      for (uint32_t e = M.off[r]; e < M.off[r + 1]; e++) {
        w.u64(M.col[e]);
        w.u64(1);  // a nonzero i64 coefficient is one canonical word
        w.u64((uint64_t)M.coef[e]);
      }
    }
  }
}

void matrix_digest(const CircuitSetup &S, const std::vector<int64_t> &expected_c,
                   uint8_t out[32]) {
  // Only C holds statement-dependent entries (the bit constraints' expected
  // values); the hash state after the domain, M, A and B is cached per shape.
  static_assert(sizeof(Sha256Stream) <= sizeof(S.digest_prefix_state), "prefix slot too small");
  std::call_once(*S.digest_prefix_once, [&] {
    Sha256Stream h;
    digest_prefix(S, h);
    memcpy(S.digest_prefix_state, &h, sizeof h);
  });
  Sha256Stream h;
  memcpy(&h, S.digest_prefix_state, sizeof h);
  {
    WordSink w(h);
    size_t n_bits = S.n_inputs;  // bit-constraint rows: inputs first, outputs last
    w.bytes("C", 1);
    w.u64(S.rows);
    w.u64(S.h_len);
    const Matrix &M = S.abc[2];
    for (size_t r = 0; r < S.rows; r++) {
      bool bitrow = r < n_bits || r >= S.rows - 256;
      if (bitrow) {
        size_t bi = r < n_bits ? r : n_bits + (r - (S.rows - 256));
        int64_t v = expected_c[bi];
        w.u64(v ? 1 : 0);
        if (v) {
          w.u64(0);
          w.u64(1);
          w.u64((uint64_t)v);
        }
        continue;
      }
      w.u64(M.off[r + 1] - M.off[r]);
      for (uint32_t e = M.off[r]; e < M.off[r + 1]; e++) {
        w.u64(M.col[e]);
        w.u64(1);
        w.u64((uint64_t)M.coef[e]);
      }
    }
  }
  h.finish(out);
}

}  // namespace bz
