// CPU oracle: the SHA-256 circuits replayed once with values and symbols side
// by side. Test infrastructure only.
//
// One pass produces what the reference obtains from three replays of the same
// circuit description: ProductWitgen's witness f, h = M (1 || f) and exact
// products (crates/circuit/src/witgen.rs:560-676), ConstraintGenerator's
// matrices M, A, B, C (crates/circuit/src/constraints.rs:678-880) and
// MTransposeGenerator's CSC of M (crates/circuit/src/matrix_transpose.rs:475-560).
// Gadgets follow crates/circuit/src/sha256.rs:187-504 and the statement
// adapters tooling/cli/src/circuits.rs:149-210.
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <vector>

#include "oracle.h"

namespace {

// An F2 linear combination over (1 || f): sorted positions, 0 = the constant.
// SHA-256's Boolean words never XOR more than three single bits and a
// constant, so four inline positions suffice (checked).
struct Bit {
  bool v = false;
  uint8_t n = 0;
  uint32_t pos[4] = {0, 0, 0, 0};
};

Bit constant_bit(bool b) {
  Bit r;
  r.v = b;
  if (b) r.pos[r.n++] = 0;
  return r;
}

Bit bxor(const Bit &a, const Bit &b) {
  Bit r;
  r.v = a.v ^ b.v;
  int i = 0, j = 0;
  while (i < a.n || j < b.n) {
    uint32_t x;
    if (j >= b.n || (i < a.n && a.pos[i] < b.pos[j])) {
      x = a.pos[i++];
    } else if (i >= a.n || b.pos[j] < a.pos[i]) {
      x = b.pos[j++];
    } else {
      i++;
      j++;
      continue;
    }
    if (r.n == 4) abort();
    r.pos[r.n++] = x;
  }
  return r;
}

// An integer linear combination over z = (1, h_1, ...): column 0 = constant.
struct Lin {
  int64_t v = 0;  // value under the witness
  std::map<uint32_t, __int128> t;
};

Lin lconst(int64_t c) {
  Lin r;
  r.v = c;
  if (c) r.t[0] = c;
  return r;
}

void ladd(Lin &a, const Lin &b, int64_t scale = 1) {
  a.v += b.v * scale;
  for (auto &kv : b.t) {
    __int128 c = a.t[kv.first] + kv.second * scale;
    if (c == 0)
      a.t.erase(kv.first);
    else
      a.t[kv.first] = c;
  }
}

struct Word {
  Bit b[35];
  int n = 32;
};

struct UInt {
  Word w;      // the Boolean word (32 bits)
  Lin full;    // z value of the word (low 32 bits for sums)
};

struct Row {
  std::vector<std::pair<uint32_t, int64_t>> e;
};

struct Builder {
  std::vector<uint8_t> f;              // witness bits (inputs, then hints)
  std::vector<uint8_t> h;              // integer witness: h[0] = 1, then each lift
  std::vector<std::vector<uint32_t>> m;  // M rows over (1 || f)
  std::vector<Row> a, b, c;
  std::vector<int64_t> av, bv, cv;

  Builder() {
    h.push_back(1);
    m.push_back({0});
  }

  Bit input(size_t i) {
    Bit r;
    r.v = f[i];
    r.pos[r.n++] = (uint32_t)i + 1;
    return r;
  }

  // Circuit::hint (witgen.rs:605-614, constraints.rs:818-835): N fresh f bits.
  Word hint(uint64_t value, int n) {
    Word w;
    w.n = n;
    for (int i = 0; i < n; i++) {
      uint32_t idx = (uint32_t)f.size();
      f.push_back((value >> i) & 1);
      w.b[i].v = (value >> i) & 1;
      w.b[i].n = 1;
      w.b[i].pos[0] = idx + 1;
    }
    return w;
  }

  // Circuit::bitz: one h entry per lift, M row = the bit's support.
  Lin bitz(const Bit &bit) {
    uint32_t col = (uint32_t)h.size();
    h.push_back(bit.v);
    m.push_back(std::vector<uint32_t>(bit.pos, bit.pos + bit.n));
    Lin r;
    r.v = bit.v;
    r.t[col] = 1;
    return r;
  }

  static Row to_row(const Lin &l) {
    Row r;
    for (auto &kv : l.t) r.e.push_back({kv.first, (int64_t)kv.second});
    return r;
  }

  void assert_r1c(const Lin &x, const Lin &y, const Lin &z) {
    a.push_back(to_row(x));
    b.push_back(to_row(y));
    c.push_back(to_row(z));
    av.push_back(x.v);
    bv.push_back(y.v);
    cv.push_back(z.v);
  }

  // sha256.rs:165-176 (uint_from_word via bitz_unsigned, lib.rs:506-527)
  UInt uint_from_word(const Word &w, Lin *full_out = nullptr) {
    UInt u;
    u.w = w;
    Lin full, low;
    for (int i = 0; i < w.n; i++) {
      Lin l = bitz(w.b[i]);
      ladd(full, l, (int64_t)1 << i);
      if (i < 32) ladd(low, l, (int64_t)1 << i);
    }
    u.full = low;
    if (full_out) *full_out = full;
    u.w.n = 32;
    return u;
  }

  UInt uint_constant(uint32_t value) {
    UInt u;
    for (int i = 0; i < 32; i++) u.w.b[i] = constant_bit((value >> i) & 1);
    u.full = lconst(value);
    return u;
  }

  static uint64_t wval(const Word &w) {
    uint64_t v = 0;
    for (int i = 0; i < 32; i++) v |= (uint64_t)w.b[i].v << i;
    return v;
  }

  // sha256.rs:228-262
  UInt sum_32(int width, const std::vector<UInt> &terms) {
    uint64_t s = 0;
    for (auto &t : terms) s += wval(t.w);
    Word bits = hint(s, width);
    Lin wide_full;
    UInt wide = uint_from_word(bits, &wide_full);
    Lin input_sum;
    for (auto &t : terms) ladd(input_sum, t.full);
    Lin diff = input_sum;
    ladd(diff, wide_full, -1);
    assert_r1c(Lin(), Lin(), diff);
    return wide;  // word = low 32 bits, z = low_32
  }

  // sha256.rs:268-316
  UInt sum_doubled_32(const std::vector<UInt> &ord, const std::vector<Lin> &dbl,
                      const std::vector<uint64_t> &dbl_values) {
    uint64_t s = 0;
    for (auto &t : ord) s += wval(t.w);
    for (auto v : dbl_values) s += v;
    Word bits = hint(s, 35);
    Lin half_full;
    UInt half = uint_from_word(bits, &half_full);
    Lin total;
    for (auto &t : ord) ladd(total, t.full, 2);
    for (auto &d : dbl) ladd(total, d);
    ladd(total, half_full, -2);
    assert_r1c(Lin(), Lin(), total);
    return half;
  }

  Word wxor(const Word &x, const Word &y) {
    Word r;
    for (int i = 0; i < 32; i++) r.b[i] = bxor(x.b[i], y.b[i]);
    return r;
  }
  static Word rotr(const Word &x, int k) {
    Word r;
    for (int i = 0; i < 32; i++) r.b[i] = x.b[(i + k) % 32];
    return r;
  }
  static Word shr(const Word &x, int k) {
    Word r;
    for (int i = 0; i < 32; i++) r.b[i] = i + k < 32 ? x.b[i + k] : constant_bit(false);
    return r;
  }

  // sha256.rs:320-341
  Lin choice_twice(const UInt &x, const UInt &y, const UInt &z) {
    UInt xy = uint_from_word(wxor(x.w, y.w));
    UInt xz = uint_from_word(wxor(x.w, z.w));
    Lin r = y.full;
    ladd(r, z.full);
    ladd(r, xy.full, -1);
    ladd(r, xz.full);
    return r;
  }
  Lin majority_twice(const UInt &x, const UInt &y, const UInt &z) {
    UInt xyz = uint_from_word(wxor(wxor(x.w, y.w), z.w));
    Lin r = x.full;
    ladd(r, y.full);
    ladd(r, z.full);
    ladd(r, xyz.full, -1);
    return r;
  }

  // sha256.rs:344-456
  void compress(const Word block[16], const Word state_in[8], Word out[8]) {
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
    UInt state[8];
    for (int i = 0; i < 8; i++) state[i] = uint_from_word(state_in[i]);
    std::vector<UInt> w;
    for (int i = 0; i < 16; i++) w.push_back(uint_from_word(block[i]));
    for (int i = 16; i < 64; i++) {
      const Word &w15 = w[i - 15].w;
      UInt s0 = uint_from_word(wxor(wxor(rotr(w15, 7), rotr(w15, 18)), shr(w15, 3)));
      const Word &w2 = w[i - 2].w;
      UInt s1 = uint_from_word(wxor(wxor(rotr(w2, 17), rotr(w2, 19)), shr(w2, 10)));
      w.push_back(sum_32(34, {w[i - 16], s0, w[i - 7], s1}));
    }
    UInt a = state[0], b = state[1], c = state[2], d = state[3];
    UInt e = state[4], f_ = state[5], g = state[6], hh = state[7];
    for (int i = 0; i < 64; i++) {
      UInt S1 = uint_from_word(wxor(wxor(rotr(e.w, 6), rotr(e.w, 11)), rotr(e.w, 25)));
      Lin ch = choice_twice(e, f_, g);
      UInt S0 = uint_from_word(wxor(wxor(rotr(a.w, 2), rotr(a.w, 13)), rotr(a.w, 22)));
      Lin mj = majority_twice(a, b, c);
      uint64_t ev = wval(e.w), fv = wval(f_.w), gv = wval(g.w);
      uint64_t av_ = wval(a.w), bv_ = wval(b.w), cv_ = wval(c.w);
      uint64_t chv = ((ev & fv) ^ (~ev & gv)) & 0xffffffffu;
      uint64_t mjv = (av_ & bv_) ^ (av_ & cv_) ^ (bv_ & cv_);
      UInt kc = uint_constant(K[i]);
      UInt old_a = a, old_b = b, old_c = c, old_d = d, old_e = e, old_f = f_, old_g = g,
           old_h = hh;
      hh = old_g;
      g = old_f;
      f_ = old_e;
      e = sum_doubled_32({old_d, old_h, S1, kc, w[i]}, {ch}, {chv});
      d = old_c;
      c = old_b;
      b = old_a;
      a = sum_doubled_32({old_h, S1, kc, w[i], S0}, {ch, mj}, {chv, mjv});
    }
    UInt working[8] = {a, b, c, d, e, f_, g, hh};
    for (int i = 0; i < 8; i++) out[i] = sum_32(33, {state[i], working[i]}).w;
  }

  // tooling/cli/src/circuits.rs:204-209
  void constrain_bit(const Bit &bit, bool expected) {
    Lin v = bitz(bit);
    assert_r1c(lconst(1), v, lconst(expected ? 1 : 0));
  }
};

const uint32_t IV[8] = {0x6a09e667, 0xbb67ae85, 0x3c6ef372, 0xa54ff53a,
                        0x510e527f, 0x9b05688c, 0x1f83d9ab, 0x5be0cd19};

Word const_word(uint32_t v) {
  Word w;
  for (int i = 0; i < 32; i++) w.b[i] = constant_bit((v >> i) & 1);
  return w;
}

}  // namespace

struct o_circuit {
  Builder b;
  std::vector<uint8_t> outputs;  // the circuit's computed output bits
};

extern "C" {

/* kind: 0 sha256-compression, 1 sha256-chain, 2 sha256-block-aligned, 3 sha256-2kb.
 * inputs/outputs: one byte (0/1) per bit in the statement's ordering
 * (tooling/cli/src/circuits.rs:67-139). */
o_circuit *o_circuit_build(int kind, const uint8_t *inputs, size_t n_inputs,
                           const uint8_t *expected) {
  o_circuit *c = new o_circuit();
  Builder &b = c->b;
  b.f.assign(inputs, inputs + n_inputs);
  std::vector<Bit> in(n_inputs);
  for (size_t i = 0; i < n_inputs; i++) in[i] = b.input(i);
  for (size_t i = 0; i < n_inputs; i++) b.constrain_bit(in[i], inputs[i]);
  std::vector<Bit> out(256);
  if (kind == 0 || kind == 1) {
    Word state[8];
    size_t nblocks = kind == 0 ? 1 : n_inputs / 512;
    for (int i = 0; i < 8; i++) {
      if (kind == 0) {
        for (int j = 0; j < 32; j++) state[i].b[j] = in[512 + i * 32 + j];
      } else {
        state[i] = const_word(IV[i]);
      }
    }
    for (size_t blk = 0; blk < nblocks; blk++) {
      Word block[16];
      for (int w = 0; w < 16; w++)
        for (int j = 0; j < 32; j++) block[w].b[j] = in[blk * 512 + w * 32 + j];
      Word next[8];
      b.compress(block, state, next);
      for (int i = 0; i < 8; i++) state[i] = next[i];
    }
    for (int i = 0; i < 256; i++) out[i] = state[i / 32].b[i % 32];
  } else {
    /* sha256.rs:482-504 */
    size_t mbits = n_inputs;
    Word state[8];
    for (int i = 0; i < 8; i++) state[i] = const_word(IV[i]);
    for (size_t blk = 0; blk < mbits / 512; blk++) {
      Word block[16];
      for (int w = 0; w < 16; w++)
        for (int j = 0; j < 32; j++) block[w].b[j] = in[blk * 512 + w * 32 + (31 - j)];
      Word next[8];
      b.compress(block, state, next);
      for (int i = 0; i < 8; i++) state[i] = next[i];
    }
    uint64_t len = mbits;
    uint32_t pad[16] = {0x80000000u, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0,
                        (uint32_t)(len >> 32), (uint32_t)len};
    Word block[16];
    for (int w = 0; w < 16; w++) block[w] = const_word(pad[w]);
    Word next[8];
    b.compress(block, state, next);
    for (int i = 0; i < 256; i++) out[i] = next[i / 32].b[31 - (i % 32)];
  }
  c->outputs.resize(256);
  for (int i = 0; i < 256; i++) {
    c->outputs[i] = out[i].v;
    b.constrain_bit(out[i], expected[i]);
  }
  return c;
}

void o_circuit_free(o_circuit *c) { delete c; }

/* sizes: [0] f bits, [1] h entries (constant included), [2] R1CS rows,
 * [3] M nonzeros, [4] A, [5] B, [6] C nonzeros */
void o_circuit_sizes(const o_circuit *c, uint64_t out[7]) {
  const Builder &b = c->b;
  out[0] = b.f.size();
  out[1] = b.h.size();
  out[2] = b.c.size();
  uint64_t nm = 0;
  for (auto &r : b.m) nm += r.size();
  out[3] = nm;
  uint64_t na = 0, nb = 0, nc = 0;
  for (auto &r : b.a) na += r.e.size();
  for (auto &r : b.b) nb += r.e.size();
  for (auto &r : b.c) nc += r.e.size();
  out[4] = na;
  out[5] = nb;
  out[6] = nc;
}

void o_circuit_outputs(const o_circuit *c, uint8_t *out) { memcpy(out, c->outputs.data(), 256); }

/* f and h as one byte per bit. */
void o_circuit_f(const o_circuit *c, uint8_t *out) { memcpy(out, c->b.f.data(), c->b.f.size()); }
void o_circuit_h(const o_circuit *c, uint8_t *out) { memcpy(out, c->b.h.data(), c->b.h.size()); }

/* exact products per row: a, b, c (each rows entries). */
void o_circuit_products(const o_circuit *c, int64_t *a, int64_t *b, int64_t *cc) {
  memcpy(a, c->b.av.data(), c->b.av.size() * 8);
  memcpy(b, c->b.bv.data(), c->b.bv.size() * 8);
  memcpy(cc, c->b.cv.data(), c->b.cv.size() * 8);
}

/* M rows in CSR over (1 || f): offsets (h+1), positions (nnz). */
void o_circuit_m(const o_circuit *c, uint32_t *off, uint32_t *pos) {
  uint32_t k = 0;
  off[0] = 0;
  for (size_t r = 0; r < c->b.m.size(); r++) {
    for (uint32_t p : c->b.m[r]) pos[k++] = p;
    off[r + 1] = k;
  }
}

/* which: 0 = A, 1 = B, 2 = C. CSR with offsets (rows+1), columns, coefficients. */
void o_circuit_matrix(const o_circuit *c, int which, uint32_t *off, uint32_t *cols,
                      int64_t *coef) {
  const std::vector<Row> &m = which == 0 ? c->b.a : which == 1 ? c->b.b : c->b.c;
  uint32_t k = 0;
  off[0] = 0;
  for (size_t r = 0; r < m.size(); r++) {
    for (auto &e : m[r].e) {
      cols[k] = e.first;
      coef[k] = e.second;
      k++;
    }
    off[r + 1] = k;
  }
}

}  // extern "C"
