// CPU oracle: the end-to-end BitZ SHA-256 prover and verifier.
// Test infrastructure only; also the timed CPU baseline.
//
// Follows tooling/cli/src/end_to_end.rs:161-456 (setup, witness, commit,
// prove), crates/prover/src/{prove,fold,reduce}.rs (BitZ virtual opening),
// crates/common/src/virtual_map.rs:174-223 (transpose_query),
// crates/pcs/src/{commitment,opening,ood,mle}.rs (binding, ring switch) and
// the Ligerito restatement in pcs.c. Proof bytes are
// root || Spartan section || bitzPCS wire container (host/src/wire_proof.rs).
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <chrono>
#include <string>
#include <vector>

#include "oracle.h"
#include "pcs.h"

extern "C" {
struct o_circuit;
o_circuit *o_circuit_build(int kind, const uint8_t *inputs, size_t n_inputs, const uint8_t *expected);
void o_circuit_free(o_circuit *c);
void o_circuit_sizes(const o_circuit *c, uint64_t out[7]);
void o_circuit_f(const o_circuit *c, uint8_t *out);
void o_circuit_h(const o_circuit *c, uint8_t *out);
void o_circuit_products(const o_circuit *c, int64_t *a, int64_t *b, int64_t *cc);
void o_circuit_m(const o_circuit *c, uint32_t *off, uint32_t *pos);
void o_circuit_matrix(const o_circuit *c, int which, uint32_t *off, uint32_t *cols, int64_t *coef);
void o_circuit_outputs(const o_circuit *c, uint8_t *out);
int o_spartan_prove(u128 q, size_t rows, size_t cols, const uint32_t *const off[3],
                    const uint32_t *const col_idx[3], const int64_t *const coef[3],
                    const int64_t *const prod[3], const uint8_t *h, const uint8_t digest[32],
                    o_transcript *t, u128 *outer_polys, u128 abc_claims[3], u128 *inner_polys,
                    u128 *rx, u128 *ry, u128 *d_at_ry, u128 *final_claim);
void o_fp_eq_table(const u128 *r, int n, u128 q, u128 *out);
o_f128 o_weighted_sum(const o_f128 *rows, int log_rows, const o_f128 *cols, int log_cols,
                      const o_f128 *packed);
}

namespace {

typedef o_f128 F;
const F ZERO = {0, 0};
const F ONE = {1, 0};
inline F add(F a, F b) { return F{a.lo ^ b.lo, a.hi ^ b.hi}; }
inline F mul(F a, F b) { return o_gf_mul(a, b); }
inline bool eqf(F a, F b) { return a.lo == b.lo && a.hi == b.hi; }
inline int bitof(F e, int v) { return v < 64 ? (int)((e.lo >> v) & 1) : (int)((e.hi >> (v - 64)) & 1); }

const char *NAMES[4] = {"sha256-compression", "sha256-chain", "sha256-block-aligned", "sha256-2kb"};

void u64le(std::vector<uint8_t> &v, uint64_t x) {
  for (int i = 0; i < 8; i++) v.push_back((uint8_t)(x >> (8 * i)));
}
void u128le(uint8_t *b, u128 x) {
  for (int i = 0; i < 16; i++) b[i] = (uint8_t)(x >> (8 * i));
}
void pub_u64(o_transcript *t, uint64_t x) {
  uint8_t b[8];
  for (int i = 0; i < 8; i++) b[i] = (uint8_t)(x >> (8 * i));
  o_ts_public(t, b, 8);
}
void pub_str(o_transcript *t, const char *s) { o_ts_public(t, s, strlen(s)); }
void pub_f(o_transcript *t, F v) { o_ts_public(t, &v, 16); }
void prov_f(o_transcript *t, F v) { o_ts_prover(t, &v, 16); }

int ceil_log2(size_t n) {
  int l = 0;
  while (((size_t)1 << l) < n) l++;
  return l;
}

// crates/common/src/security.rs:25-31
uint32_t grinding_bits(int sec, uint64_t c) {
  if (c == 0) return 0;
  uint32_t lc = 0;
  uint64_t x = c - 1;
  while (x) {
    lc++;
    x >>= 1;
  }
  uint32_t need = (uint32_t)sec + lc;
  return need > 128 ? need - 128 : 0;
}

std::vector<F> eq_table(const F *r, int n) {
  std::vector<F> t((size_t)1 << n);
  o_gf_eq_table(r, n, t.data());
  return t;
}

// ------------------------------------------------------------- the setup
struct Setup {
  int kind, security;
  o_circuit *circ = nullptr;
  uint64_t sizes[7];
  size_t f_bits, h_len, rows;
  int claim_log_cols, committed_m, prime_bits;
  std::vector<uint32_t> m_off, m_pos;  // M rows over (1 || f)
  std::vector<uint32_t> csc_off, csc_row;  // M^T (CSC of M)
  std::vector<uint32_t> off[3], col[3];
  std::vector<int64_t> coef[3];
  uint8_t map_digest[32], matrix_digest[32];
  o_pcs_config_t pcs;
  std::vector<uint8_t> public_bytes;
  F generator;
};

void pcs_encoding(const Setup &s, std::vector<uint8_t> &out) {
  // crates/pcs/src/commitment.rs:214-221
  const char *v = "bitz/pcs/security/v1";
  out.insert(out.end(), v, v + strlen(v));
  u64le(out, (uint64_t)1 << s.committed_m);
  uint32_t b = (uint32_t)s.security;
  for (int i = 0; i < 4; i++) out.push_back((uint8_t)(b >> (8 * i)));
}

void build_setup(Setup &s, int kind, const uint8_t *inputs, size_t n_inputs, const uint8_t *expected,
                 int security) {
  s.kind = kind;
  s.security = security;
  s.circ = o_circuit_build(kind, inputs, n_inputs, expected);
  o_circuit_sizes(s.circ, s.sizes);
  s.f_bits = s.sizes[0];
  s.h_len = s.sizes[1];
  s.rows = s.sizes[2];
  // end_to_end.rs:489-497 (shape_for): pad to a power of two, at least 2^20, 7 row bits
  int mh = ceil_log2(s.h_len);
  if (mh < 20) mh = 20;
  s.claim_log_cols = mh - 7;
  int mf = ceil_log2(s.f_bits);
  if (mf < 20) mf = 20;
  s.committed_m = mf;
  s.prime_bits = 121;  // params.rs:52 for 7 row bits: ilog2((2^128 - 2) / 128 + 1)
  s.m_off.resize(s.h_len + 1);
  s.m_pos.resize(s.sizes[3]);
  o_circuit_m(s.circ, s.m_off.data(), s.m_pos.data());
  for (int k = 0; k < 3; k++) {
    s.off[k].resize(s.rows + 1);
    s.col[k].resize(s.sizes[4 + k] + 1);
    s.coef[k].resize(s.sizes[4 + k] + 1);
    o_circuit_matrix(s.circ, k, s.off[k].data(), s.col[k].data(), s.coef[k].data());
  }
  // matrix_transpose.rs:523-560: CSC of M, rows ascending within a column
  size_t ncols = s.f_bits + 1;
  s.csc_off.assign(ncols + 1, 0);
  for (uint32_t p : s.m_pos) s.csc_off[p + 1]++;
  for (size_t c = 0; c < ncols; c++) s.csc_off[c + 1] += s.csc_off[c];
  s.csc_row.resize(s.m_pos.size());
  std::vector<uint32_t> cur(s.csc_off.begin(), s.csc_off.end() - 1);
  for (size_t r = 0; r < s.h_len; r++)
    for (uint32_t e = s.m_off[r]; e < s.m_off[r + 1]; e++) s.csc_row[cur[s.m_pos[e]]++] = (uint32_t)r;
  // csc_digest (matrix_transpose.rs:424-441)
  {
    o_blake3_state h;
    o_blake3_init(&h);
    const char *dom = "bitz/virtual-map/csc/v1";
    o_blake3_update(&h, (const uint8_t *)dom, strlen(dom));
    std::vector<uint8_t> b;
    u64le(b, s.h_len);
    u64le(b, ncols);
    u64le(b, s.csc_row.size());
    o_blake3_update(&h, b.data(), b.size());
    o_blake3_update(&h, (const uint8_t *)s.csc_off.data(), s.csc_off.size() * 4);
    o_blake3_update(&h, (const uint8_t *)s.csc_row.data(), s.csc_row.size() * 4);
    o_blake3_final(&h, s.map_digest);
  }
  // integer_matrix_digest (crates/spartan/src/matrix.rs:562-661), SHA-256
  {
    std::vector<uint8_t> b;
    const char *dom = "bitz/spartan/integer-constraint-matrices/v1";
    b.insert(b.end(), dom, dom + strlen(dom));
    b.push_back('M');
    u64le(b, s.h_len);
    u64le(b, ncols);
    for (size_t r = 0; r < s.h_len; r++) {
      u64le(b, s.m_off[r + 1] - s.m_off[r]);
      for (uint32_t e = s.m_off[r]; e < s.m_off[r + 1]; e++) u64le(b, s.m_pos[e]);
    }
    const char lab[3] = {'A', 'B', 'C'};
    for (int k = 0; k < 3; k++) {
      b.push_back((uint8_t)lab[k]);
      u64le(b, s.rows);
      u64le(b, s.h_len);
      for (size_t r = 0; r < s.rows; r++) {
        u64le(b, s.off[k][r + 1] - s.off[k][r]);
        for (uint32_t e = s.off[k][r]; e < s.off[k][r + 1]; e++) {
          u64le(b, s.col[k][e]);
          int64_t v = s.coef[k][e];
          if (v == 0) {
            u64le(b, 0);
          } else {
            u64le(b, 1);
            u64le(b, (uint64_t)v);
          }
        }
      }
    }
    o_sha256(b.data(), b.size(), s.matrix_digest);
  }
  o_pcs_config(s.committed_m, security, &s.pcs);
  s.generator = o_gf_smallest_generator();
  // circuits.rs:149-160: u64 input count, then one byte per input and output bit
  u64le(s.public_bytes, n_inputs);
  s.public_bytes.insert(s.public_bytes.end(), inputs, inputs + n_inputs);
  s.public_bytes.insert(s.public_bytes.end(), expected, expected + 256);
}

// ------------------------------------------------------------- PCS parts
struct Level {
  int log_n, k, rate;
  std::vector<F> codeword;       // rows x 2^k
  std::vector<uint8_t> nodes;    // Merkle nodes, 32 bytes each, root at 1
  size_t rows;
};

void commit_level(Level &L, const std::vector<F> &vec, int log_n, int k, int rate) {
  L.log_n = log_n;
  L.k = k;
  L.rate = rate;
  L.rows = (size_t)1 << (log_n - k + rate);
  L.codeword.assign(L.rows << k, ZERO);
  o_pcs_encode(vec.data(), log_n, k, rate, L.codeword.data());
  L.nodes.assign(64 * L.rows, 0);
  o_merkle_build(L.codeword.data(), L.rows, 1 << k, L.nodes.data());
}

F mle_eval(const std::vector<F> &v, const F *pt, int n) { return o_gf_mle_eval(v.data(), pt, n); }

// The sumcheck glue: the queried symbols are linear in the folded vector.
// X_j(x_q) = prod_{t in j} Wh_t(x_q), a tensor over (1, Wh_t(x_q)).
void add_query_basis(std::vector<F> &basis, int l, uint64_t idx, F scale) {
  F x = {idx, 0};
  std::vector<F> w(l);
  for (int t = 0; t < l; t++) w[t] = o_wh(t, x);
  std::vector<F> tab((size_t)1 << l);
  tab[0] = scale;
  for (int t = 0; t < l; t++) {
    size_t h = (size_t)1 << t;
    for (size_t j = 0; j < h; j++) tab[h + j] = mul(tab[j], w[t]);
  }
  for (size_t j = 0; j < tab.size(); j++) basis[j] = add(basis[j], tab[j]);
}

struct Challenger {
  o_transcript *t;
  const o_pcs_config_t *cfg;
  std::vector<std::pair<uint32_t, uint32_t>> sched;
  size_t at = 0;
  explicit Challenger(o_transcript *tt, const o_pcs_config_t *c) : t(tt), cfg(c) {
    // ligerito.rs:47-63: per level, k fold grinds then one query grind
    for (int i = 0; i < c->nlevels; i++) {
      const o_pcs_level_t &L = c->levels[i];
      for (int r = 0; r < L.k; r++) {
        uint32_t native = (uint32_t)(L.fold_grinding - r);
        uint32_t eff = c->security_bits == 128 ? (uint32_t)L.fold_grinding : native;
        sched.push_back({native, eff});
      }
      sched.push_back({(uint32_t)L.grinding, (uint32_t)L.grinding});
    }
  }
  // challenger.rs:142-175
  F sample() { return o_ts_f128(t); }
  std::vector<F> sample_vec(size_t n) {
    pub_str(t, "pcs/flock/sample-vector/v1");
    pub_u64(t, n);
    std::vector<F> v(n);
    for (auto &x : v) x = sample();
    return v;
  }
  void observe(F v) { prov_f(t, v); }
  void observe_slice(const std::vector<F> &v) {
    uint32_t n = (uint32_t)v.size();
    o_ts_prover(t, &n, 4);
    for (auto &x : v) observe(x);
  }
  void observe_bytes(const uint8_t *b, size_t n) {
    uint32_t l = (uint32_t)n;
    std::vector<uint8_t> m(4 + n);
    memcpy(m.data(), &l, 4);
    memcpy(m.data() + 4, b, n);
    o_ts_prover(t, m.data(), m.size());
  }
  void grind(uint32_t native) {
    uint32_t bits = sched[at].second;
    (void)native;
    at++;
    pub_str(t, "pcs/flock/pow/v1");
    uint8_t b4[4];
    for (int i = 0; i < 4; i++) b4[i] = (uint8_t)(bits >> (8 * i));
    o_ts_public(t, b4, 4);
    uint8_t seed[16];
    o_ts_squeeze(t, seed, 16);
    uint64_t nonce = 0;
    while (!o_pow_valid(seed, nonce, bits)) nonce++;
    o_ts_prover(t, &nonce, 8);
  }
};

F advance(F claim, F a0, F a2, F r) { return add(a0, mul(r, add(add(claim, a2), mul(r, a2)))); }

void fold(std::vector<F> &t, F r) {
  size_t n = t.size() / 2;
  for (size_t k = 0; k < n; k++) t[k] = add(t[2 * k], mul(r, add(t[2 * k], t[2 * k + 1])));
  t.resize(n);
}

// The Ligerito opening (restatement, see pcs.c): returns the hint bytes.
std::vector<uint8_t> ligerito_prove(o_transcript *t, const o_pcs_config_t &cfg, std::vector<F> f,
                                    std::vector<F> basis, F target, Level &level0) {
  Challenger ch(t, &cfg);
  pub_str(t, "flock-ligerito-basis-v0");
  pub_f(t, target);
  F claim = target;
  std::vector<uint8_t> proof;
  Level cur = level0;
  for (int i = 0; i < cfg.nlevels; i++) {
    const o_pcs_level_t &L = cfg.levels[i];
    std::vector<F> rs;
    for (int r = 0; r < L.k; r++) {
      // the quadratic round of <basis, f> over the lowest variable
      o_wide s0 = {{0, 0, 0, 0}}, s2 = {{0, 0, 0, 0}};
      for (size_t j = 0; j < f.size() / 2; j++) {
        o_wide p0 = o_gf_mul_wide(basis[2 * j], f[2 * j]);
        o_wide p2 = o_gf_mul_wide(add(basis[2 * j], basis[2 * j + 1]), add(f[2 * j], f[2 * j + 1]));
        for (int w = 0; w < 4; w++) {
          s0.w[w] ^= p0.w[w];
          s2.w[w] ^= p2.w[w];
        }
      }
      F a0 = o_gf_reduce(s0), a2 = o_gf_reduce(s2);
      ch.observe(a0);
      ch.observe(a2);
      ch.grind((uint32_t)(L.fold_grinding - r));
      F c = ch.sample();
      rs.push_back(c);
      claim = advance(claim, a0, a2, c);
      fold(basis, c);
      fold(f, c);
    }
    int l = L.log_msg_cols;  // f now has 2^l entries
    Level next;
    bool last = i + 1 == cfg.nlevels;
    if (!last) {
      const o_pcs_level_t &N = cfg.levels[i + 1];
      commit_level(next, f, l, N.k, N.log_inv_rate);
      ch.observe_bytes(next.nodes.data() + 32, 32);
      if (N.ood_samples) {
        std::vector<F> pt = ch.sample_vec((size_t)l);
        F v = mle_eval(f, pt.data(), l);
        ch.observe(v);
        F mu = ch.sample();
        std::vector<F> e = eq_table(pt.data(), l);
        for (size_t j = 0; j < basis.size(); j++) basis[j] = add(basis[j], mul(mu, e[j]));
        claim = add(claim, mul(mu, v));
      }
    } else {
      ch.observe_slice(f);
    }
    // queries into this level's codeword
    ch.grind((uint32_t)L.grinding);
    std::vector<F> qs = ch.sample_vec((size_t)L.queries);
    int width = 1 << cur.k;
    int depth = ceil_log2(cur.rows);
    u64le(proof, (uint64_t)L.queries);
    std::vector<F> eqr = eq_table(rs.data(), L.k);
    std::vector<F> vals(L.queries);
    std::vector<uint64_t> idx(L.queries);
    for (int q = 0; q < L.queries; q++) {
      idx[q] = qs[q].lo & (cur.rows - 1);
      const F *row = cur.codeword.data() + idx[q] * width;
      proof.insert(proof.end(), (const uint8_t *)row, (const uint8_t *)(row + width));
      size_t node = cur.rows + idx[q];
      for (int d = 0; d < depth; d++) {
        const uint8_t *sib = cur.nodes.data() + 32 * (node ^ 1);
        proof.insert(proof.end(), sib, sib + 32);
        node >>= 1;
      }
      F v = ZERO;
      for (int c = 0; c < width; c++) v = add(v, mul(row[c], eqr[c]));
      vals[q] = v;
    }
    int av = ceil_log2((size_t)L.queries);
    std::vector<F> alpha = ch.sample_vec((size_t)av);
    F mu = ch.sample();
    std::vector<F> beta = eq_table(alpha.data(), av);
    for (int q = 0; q < L.queries; q++) {
      F s = mul(mu, beta[q]);
      add_query_basis(basis, l, idx[q], s);
      claim = add(claim, mul(s, vals[q]));
    }
    if (!last) cur = std::move(next);
  }
  // the final vector meets its basis
  F chk = ZERO;
  for (size_t j = 0; j < f.size(); j++) chk = add(chk, mul(basis[j], f[j]));
  if (!eqf(chk, claim)) proof.clear();
  return proof;
}


// ------------------------------------------------------------- verifier
//
// CircuitProofSystem::verify (tooling/cli/src/end_to_end.rs:339-377) over the
// proof bytes: the Spartan checks (crates/spartan/src/piop.rs verify side),
// the BitZ fold checks and GKR replay (crates/verifier/src/{fold,reduce}.rs,
// crates/gkr/src/lib.rs:717-772), the transposed query
// (virtual_map.rs:174-223), the inner-product sumcheck
// (crates/post_gkr/src/sumcheck.rs:112-200), the ring switch and OOD batching
// (crates/pcs/src/{opening,mle,ood}.rs) and the Ligerito restatement above,
// replayed message by message. It reads prover messages from the narg string
// and absorbs them exactly as the prover did, so every challenge is the
// prover's; every check failure returns its own code.

struct Reader {
  o_transcript t;
  const uint8_t *narg = nullptr, *hints = nullptr;
  size_t narg_len = 0, pos = 0, hints_len = 0, hpos = 0;
  bool short_read = false;
  // a prover message of n bytes
  void take(void *out, size_t n) {
    if (pos + n > narg_len) {
      short_read = true;
      memset(out, 0, n);
      pos = narg_len;
      return;
    }
    memcpy(out, narg + pos, n);
    pos += n;
    o_ts_prover(&t, out, n);
  }
  F f() {
    F v;
    take(&v, 16);
    return v;
  }
  // hint bytes (not absorbed)
  const uint8_t *hint(size_t n) {
    if (hpos + n > hints_len) {
      short_read = true;
      return nullptr;
    }
    const uint8_t *p = hints + hpos;
    hpos += n;
    return p;
  }
  // transcript grind (crates/transcript/src/pow.rs:21-50) on the verifier side
  bool grind(const char *label, uint32_t bits) {
    if (bits == 0) return true;
    size_t ll = strlen(label);
    o_ts_public(&t, "bitz-transcript-pow-v1", 22);
    pub_u64(&t, (uint64_t)ll);
    o_ts_public(&t, label, ll);
    uint8_t b4[4];
    for (int i = 0; i < 4; i++) b4[i] = (uint8_t)(bits >> (8 * i));
    o_ts_public(&t, b4, 4);
    uint8_t seed[16];
    o_ts_squeeze(&t, seed, 16);
    uint8_t n8[8];
    take(n8, 8);
    uint64_t nonce = 0;
    for (int i = 0; i < 8; i++) nonce |= (uint64_t)n8[i] << (8 * i);
    return !short_read && o_pow_valid(seed, nonce, bits);
  }
};

u128 get_u128(const uint8_t *b) {
  u128 v = 0;
  for (int i = 15; i >= 0; i--) v = (v << 8) | b[i];
  return v;
}

// sum-check round over the prime field: p(0) + p(1) must equal the claim;
// the coefficients are absorbed as one public message (sumcheck.rs:771-811)
bool fp_round(o_transcript *t, u128 q, const uint8_t *coefs, int ncoef, u128 *claim, u128 *r_out) {
  u128 c[4], at_one = 0;
  for (int i = 0; i < ncoef; i++) {
    c[i] = get_u128(coefs + 16 * i);
    if (c[i] >= q) return false;
    at_one = o_fp_add(at_one, c[i], q);
  }
  if (o_fp_add(c[0], at_one, q) != *claim) return false;
  o_ts_public(t, coefs, 16 * (size_t)ncoef);
  u128 r = o_ts_fp(t, q);
  u128 v = 0;
  for (int i = ncoef - 1; i >= 0; i--) v = o_fp_add(o_fp_mul(v, r, q), c[i], q);
  *claim = v;
  *r_out = r;
  return true;
}

u128 fp_eq_at(const u128 *a, const u128 *b, int n, u128 q) {
  // prod_i (a_i b_i + (1 - a_i)(1 - b_i))
  u128 e = 1;
  for (int i = 0; i < n; i++) {
    u128 ab = o_fp_mul(a[i], b[i], q);
    u128 na = o_fp_sub(1, a[i], q), nb = o_fp_sub(1, b[i], q);
    e = o_fp_mul(e, o_fp_add(ab, o_fp_mul(na, nb, q), q), q);
  }
  return e;
}

int verify_proof(int kind, const uint8_t *inputs, size_t n_inputs, const uint8_t *expected,
                 int security, const uint8_t *proof, size_t proof_len) {
  Setup s;
  build_setup(s, kind, inputs, n_inputs, expected, security);
  struct Free {
    Setup &s;
    ~Free() {
      if (s.circ) o_circuit_free(s.circ);
    }
  } free_circuit{s};
  const int nr = ceil_log2(s.rows ? s.rows : 1), nc = ceil_log2(s.h_len);
  // ---- proof bytes: root || Spartan section || bitzPCS container
  size_t spartan_len = 16 * (4 * (size_t)nr + 3 + 3 * (size_t)nc);
  size_t head = 32 + spartan_len;
  if (proof_len < head + 32) return 101;
  const uint8_t *root = proof;
  const uint8_t *outer = proof + 32, *abc = outer + 64 * nr, *inner = abc + 48;
  const uint8_t *box = proof + head;
  const uint8_t magic[16] = {'b', 'i', 't', 'z', 'P', 'C', 'S', 0, 1, 0, 32, 0, 0, 0, 0, 0};
  if (memcmp(box, magic, 16) != 0) return 102;
  uint64_t narg_len = 0, hints_len = 0;
  for (int i = 7; i >= 0; i--) narg_len = (narg_len << 8) | box[16 + i];
  for (int i = 7; i >= 0; i--) hints_len = (hints_len << 8) | box[24 + i];
  if (head + 32 + narg_len + hints_len != proof_len) return 103;
  Reader rd;
  rd.narg = box + 32;
  rd.narg_len = narg_len;
  rd.hints = rd.narg + narg_len;
  rd.hints_len = hints_len;
  o_transcript *t = &rd.t;
  const char *dom = NAMES[kind];
  o_ts_init(t, (const uint8_t *)"bitz/circuit-e2e/v2", 19, (const uint8_t *)dom, strlen(dom));
  struct FreeTs {
    o_transcript *t;
    ~FreeTs() { o_ts_free(t); }
  } free_ts{t};
  const int log_n = s.committed_m - 7;
  std::vector<uint8_t> pcs_enc;
  pcs_encoding(s, pcs_enc);
  // ---- receive_commitment (commitment.rs:153-190, ood.rs:56-75)
  pub_str(t, "bitz/pcs/commit/v1");
  o_ts_public(t, root, 32);
  o_ts_public(t, pcs_enc.data(), pcs_enc.size());
  std::vector<F> ood_pt;
  F ood_val = ZERO;
  if (security == 100) {
    pub_str(t, "bitz/pcs/ood/v1");
    for (int i = 0; i < log_n; i++) ood_pt.push_back(o_ts_f128(t));
    ood_val = rd.f();
  }
  // ---- bind and the prime (end_to_end.rs:401-455)
  pub_u64(t, s.public_bytes.size());
  o_ts_public(t, s.public_bytes.data(), s.public_bytes.size());
  o_ts_public(t, root, 32);
  pub_u64(t, 7);
  pub_u64(t, (uint64_t)s.claim_log_cols);
  pub_f(t, s.generator);
  o_ts_public(t, pcs_enc.data(), pcs_enc.size());
  o_ts_public(t, s.map_digest, 32);
  o_ts_public(t, s.matrix_digest, 32);
  pub_str(t, "bitz/circuit-opening-path/v1");
  uint8_t path = 1;
  o_ts_public(t, &path, 1);
  u128 q = o_ts_prime(t, (uint32_t)s.prime_bits);
  std::vector<uint8_t> params;
  u64le(params, 7);
  u64le(params, (uint64_t)s.claim_log_cols);
  uint8_t qb[16];
  u128le(qb, q);
  params.insert(params.end(), qb, qb + 16);
  params.insert(params.end(), (uint8_t *)&s.generator, (uint8_t *)&s.generator + 16);
  o_ts_public(t, params.data(), params.size());
  // ---- Spartan (piop.rs:67-113): outer cubic rounds, then the inner quadratic
  o_ts_public(t, s.matrix_digest, 32);
  std::vector<u128> tau(nr), rx(nr), ry(nc);
  for (int i = 0; i < nr; i++) tau[i] = o_ts_fp(t, q);
  u128 claim = 0;
  for (int i = 0; i < nr; i++)
    if (!fp_round(t, q, outer + 64 * i, 4, &claim, &rx[i])) return 201;
  u128 az = get_u128(abc), bz = get_u128(abc + 16), cz = get_u128(abc + 32);
  if (az >= q || bz >= q || cz >= q) return 202;
  if (claim != o_fp_mul(fp_eq_at(tau.data(), rx.data(), nr, q),
                        o_fp_sub(o_fp_mul(az, bz, q), cz, q), q))
    return 203;
  o_ts_public(t, abc, 48);
  u128 rho = o_ts_fp(t, q), rho2 = o_fp_mul(rho, rho, q);
  claim = o_fp_add(o_fp_add(az, o_fp_mul(rho, bz, q), q), o_fp_mul(rho2, cz, q), q);
  for (int i = 0; i < nc; i++)
    if (!fp_round(t, q, inner + 48 * i, 3, &claim, &ry[i])) return 204;
  const u128 fin = claim;
  // D(r_y) = sum_{i,j} eq(r_x, i) eq(r_y, j) (A + rho B + rho^2 C)[i, j]
  u128 d_ry = 0;
  {
    std::vector<u128> ex((size_t)1 << nr), ey((size_t)1 << nc);
    o_fp_eq_table(rx.data(), nr, q, ex.data());
    o_fp_eq_table(ry.data(), nc, q, ey.data());
    const u128 scales[3] = {1, rho, rho2};
    for (int k = 0; k < 3; k++)
      for (size_t i = 0; i < s.rows; i++) {
        u128 acc = 0;
        for (uint32_t e = s.off[k][i]; e < s.off[k][i + 1]; e++) {
          int64_t v = s.coef[k][e];
          u128 cv = v >= 0 ? (u128)v % q : (q - (u128)(-(v + 1) + 1) % q) % q;
          acc = o_fp_add(acc, o_fp_mul(cv, ey[s.col[k][e]], q), q);
        }
        d_ry = o_fp_add(d_ry, o_fp_mul(o_fp_mul(ex[i], scales[k], q), acc, q), q);
      }
  }
  // ---- the opening claim (end_to_end.rs:509-528)
  const int sc = s.claim_log_cols, mh = 7 + sc;
  const size_t ncol = (size_t)1 << sc;
  std::vector<u128> pt(mh, 0);
  for (int i = 0; i < nc; i++) pt[i] = ry[i];
  std::vector<u128> rows_w(128), cols_w(ncol);
  o_fp_eq_table(pt.data(), 7, q, rows_w.data());
  for (auto &w : rows_w) w = o_fp_mul(w, d_ry, q);
  o_fp_eq_table(pt.data() + 7, sc, q, cols_w.data());
  pub_str(t, "bitz/virtual-statement/v1");
  o_ts_public(t, root, 32);
  {
    std::vector<uint8_t> vp = params;
    u64le(vp, 7);
    u64le(vp, (uint64_t)(s.committed_m - 7));
    o_ts_public(t, vp.data(), vp.size());
  }
  o_ts_public(t, s.map_digest, 32);
  {
    std::vector<uint8_t> ce;
    u64le(ce, 128);
    uint8_t b[16];
    for (auto w : rows_w) {
      u128le(b, w);
      ce.insert(ce.end(), b, b + 16);
    }
    u64le(ce, ncol);
    for (auto w : cols_w) {
      u128le(b, w);
      ce.insert(ce.end(), b, b + 16);
    }
    u128le(b, fin);
    ce.insert(ce.end(), b, b + 16);
    o_ts_public(t, ce.data(), ce.size());
  }
  o_ts_public(t, pcs_enc.data(), pcs_enc.size());
  // ---- receive_fold (crates/verifier/src/fold.rs:42-77)
  std::vector<u128> folds(ncol);
  {
    const u128 bound = (u128)128 * (q - 1);
    u128 acc = 0;
    for (size_t j = 0; j < ncol; j++) {
      uint8_t b[16];
      rd.take(b, 16);
      folds[j] = get_u128(b);
      if (folds[j] > bound) return 301;
      acc = o_fp_add(acc, o_fp_mul(cols_w[j], folds[j] % q, q), q);
    }
    if (rd.short_read) return 302;
    if (acc != fin) return 303;
  }
  o_comb comb;
  o_comb_init(&comb, s.generator, 8);
  std::vector<F> col_images(ncol), row_images(128);
  for (size_t j = 0; j < ncol; j++) col_images[j] = o_comb_pow(&comb, folds[j]);
  for (int b = 0; b < 128; b++) row_images[b] = o_comb_pow(&comb, rows_w[b]);
  o_comb_free(&comb);
  if (!rd.grind("bitz/columns/v1", grinding_bits(security, (uint64_t)sc))) return 304;
  std::vector<F> point(sc);
  for (auto &z : point) z = o_ts_f128(t);
  // ---- gpgkr_verify (crates/gkr/src/lib.rs:717-772) from e0 = MLE(images)(zeta)
  F gclaim = mle_eval(col_images, point.data(), sc);
  for (int layer = 0; layer < 7; layer++) {
    const int n = (int)point.size();
    std::vector<F> next(n + 1);
    F eq_bound = ONE;
    for (int i = n - 1; i >= 0; i--) {
      F z = point[i];
      F sum_b = rd.f(), sum_inf = rd.f();
      F sum0, sum1;
      if (eqf(z, ZERO)) {
        sum0 = gclaim;
        sum1 = sum_b;
      } else {
        sum0 = sum_b;
        sum1 = mul(add(gclaim, mul(add(ONE, z), sum_b)), o_gf_inv(z));
      }
      if (!rd.grind("gkr/cubic/v1", grinding_bits(security, 3))) return 401;
      F r = o_ts_f128(t);
      next[i] = r;
      F eq_r = add(add(ONE, r), z);
      gclaim = mul(eq_r, add(sum0, mul(r, add(add(sum1, sum0), mul(add(r, ONE), sum_inf)))));
      eq_bound = mul(eq_bound, eq_r);
    }
    F left = rd.f(), right = rd.f();
    if (rd.short_read) return 402;
    if (!eqf(mul(mul(eq_bound, left), right), gclaim)) return 403;
    F tt = o_ts_f128(t);
    next[n] = tt;
    gclaim = add(left, mul(tt, add(right, left)));
    point = next;
  }
  // ---- gkr_reduce's claim (crates/verifier/src/reduce.rs:27-54) and the
  // transposed query (virtual_map.rs:174-223)
  F ip_target = add(gclaim, ONE);
  std::vector<F> eqb = eq_table(point.data() + sc, 7), u2 = eq_table(point.data(), sc);
  std::vector<F> u1(128);
  for (int b = 0; b < 128; b++) u1[b] = mul(add(row_images[b], ONE), eqb[b]);
  size_t fcols = s.f_bits + 1;
  std::vector<F> wt(fcols);
  o_mt_transpose(s.csc_off.data(), s.csc_row.data(), fcols, u1.data(), 7, u2.data(), wt.data());
  F target2 = add(ip_target, wt[0]);
  size_t nbits = (size_t)1 << s.committed_m;
  std::vector<F> weights(nbits, ZERO);
  for (size_t c = 1; c < fcols; c++) weights[c - 1] = wt[c];
  // ---- verify_lin, InnerProduct (opening.rs:162-245)
  pub_str(t, "bitz/pcs/bit-inner-product/v3");
  o_ts_public(t, root, 32);
  o_ts_public(t, pcs_enc.data(), pcs_enc.size());
  pub_u64(t, nbits);
  pub_u64(t, 1);
  {
    o_blake3_state h;
    o_blake3_init_derive_key(&h, "bitz/pcs/bit-inner-product-weights/v1");
    o_blake3_update(&h, (const uint8_t *)weights.data(), nbits * 16);
    o_blake3_update(&h, (const uint8_t *)&ONE, 16);
    uint8_t dg[32];
    o_blake3_final(&h, dg);
    o_ts_public(t, dg, 32);
  }
  pub_f(t, target2);
  pub_str(t, "bitz/pcs/inner-product-sumcheck/v2");
  // post_gkr::verify (post_gkr/src/lib.rs:150-164, sumcheck.rs:112-200)
  const int m = s.committed_m;
  std::vector<F> rho_pt(m);
  F pclaim = target2;
  for (int k = 0; k < m; k++) {
    F a0 = rd.f(), a2 = rd.f();
    if (!rd.grind("bitz/pcs/sumcheck/v1", grinding_bits(security, 2))) return 501;
    F r = o_ts_f128(t);
    rho_pt[k] = r;
    pclaim = advance(pclaim, a0, a2, r);
  }
  F v = rd.f();
  if (rd.short_read) return 502;
  if (!eqf(mul(mle_eval(weights, rho_pt.data(), m), v), pclaim)) return 503;
  // ---- the MLE opening with binding, ring switch (opening.rs:119-135,
  // mle.rs:63-123) and OOD batching (ood.rs:77-95)
  pub_str(t, "bitz/pcs/mle-opening/v1");
  o_ts_public(t, root, 32);
  o_ts_public(t, pcs_enc.data(), pcs_enc.size());
  pub_u64(t, (uint64_t)m);
  for (auto &c : rho_pt) pub_f(t, c);
  pub_f(t, v);
  pub_str(t, "bitz/pcs/mle-claims/v1");
  std::vector<F> claims(128);
  for (auto &c : claims) c = rd.f();
  {
    std::vector<F> pre = eq_table(rho_pt.data(), 7);
    F chk = ZERO;
    for (int b = 0; b < 128; b++) chk = add(chk, mul(pre[b], claims[b]));
    if (!eqf(chk, v)) return 601;
  }
  if (!rd.grind("bitz/pcs/ring/v1", grinding_bits(security, 7 + (security == 100 ? 1 : 0))))
    return 602;
  pub_str(t, "bitz/pcs/ring-switch-challenges/v1");
  std::vector<F> bpt(7);
  for (auto &c : bpt) c = o_ts_f128(t);
  std::vector<F> bw = eq_table(bpt.data(), 7);
  F ptarget = ZERO;
  for (int u = 0; u < 128; u++) {
    F tu = ZERO;
    for (int vv = 0; vv < 128; vv++)
      if (bitof(claims[vv], u)) (vv < 64 ? tu.lo : tu.hi) |= 1ull << (vv % 64);
    ptarget = add(ptarget, mul(tu, bw[u]));
  }
  const size_t packed_f = (size_t)1 << log_n;
  std::vector<F> suffix = eq_table(rho_pt.data() + 7, log_n);
  std::vector<F> basis(packed_f, ZERO);
  for (size_t y = 0; y < packed_f; y++) {
    F acc = ZERO;
    for (int u = 0; u < 128; u++)
      if (bitof(suffix[y], u)) acc = add(acc, bw[u]);
    basis[y] = acc;
  }
  if (security == 100) {
    pub_str(t, "bitz/pcs/ood-batching/v1");
    F coef = o_ts_f128(t);
    std::vector<F> e = eq_table(ood_pt.data(), log_n);
    for (size_t y = 0; y < packed_f; y++) basis[y] = add(basis[y], mul(coef, e[y]));
    ptarget = add(ptarget, mul(coef, ood_val));
  }
  // ---- the Ligerito opening (the restatement in ligerito_prove)
  const uint8_t *lhead = rd.hint(4);
  if (!lhead) return 701;
  uint32_t llen = (uint32_t)lhead[0] | ((uint32_t)lhead[1] << 8) | ((uint32_t)lhead[2] << 16) |
                  ((uint32_t)lhead[3] << 24);
  if ((size_t)llen != hints_len - 4) return 702;
  const o_pcs_config_t &cfg = s.pcs;
  std::vector<std::pair<uint32_t, uint32_t>> sched;
  for (int i = 0; i < cfg.nlevels; i++) {
    const o_pcs_level_t &L = cfg.levels[i];
    for (int r = 0; r < L.k; r++)
      sched.push_back({0u, security == 128 ? (uint32_t)L.fold_grinding
                                            : (uint32_t)(L.fold_grinding - r)});
    sched.push_back({0u, (uint32_t)L.grinding});
  }
  size_t at = 0;
  auto lig_grind = [&](void) -> bool {
    uint32_t bits = sched[at++].second;
    pub_str(t, "pcs/flock/pow/v1");
    uint8_t b4[4];
    for (int i = 0; i < 4; i++) b4[i] = (uint8_t)(bits >> (8 * i));
    o_ts_public(t, b4, 4);
    uint8_t seed[16];
    o_ts_squeeze(t, seed, 16);
    uint8_t n8[8];
    rd.take(n8, 8);
    uint64_t nonce = 0;
    for (int i = 0; i < 8; i++) nonce |= (uint64_t)n8[i] << (8 * i);
    return !rd.short_read && o_pow_valid(seed, nonce, bits);
  };
  auto sample_vec = [&](size_t n) {
    pub_str(t, "pcs/flock/sample-vector/v1");
    pub_u64(t, n);
    std::vector<F> out(n);
    for (auto &x : out) x = o_ts_f128(t);
    return out;
  };
  pub_str(t, "flock-ligerito-basis-v0");
  pub_f(t, ptarget);
  F lclaim = ptarget;
  uint8_t cur_root[32];
  memcpy(cur_root, root, 32);
  int cur_k = cfg.levels[0].k, cur_rate = cfg.levels[0].log_inv_rate, cur_log_n = log_n;
  std::vector<F> f_final;
  for (int i = 0; i < cfg.nlevels; i++) {
    const o_pcs_level_t &L = cfg.levels[i];
    std::vector<F> rs;
    for (int r = 0; r < L.k; r++) {
      F a0 = rd.f(), a2 = rd.f();
      if (!lig_grind()) return 703;
      F c = o_ts_f128(t);
      rs.push_back(c);
      lclaim = advance(lclaim, a0, a2, c);
      fold(basis, c);
    }
    const int l = L.log_msg_cols;
    const bool last = i + 1 == cfg.nlevels;
    uint8_t next_root[32] = {0};
    if (!last) {
      const o_pcs_level_t &N = cfg.levels[i + 1];
      uint8_t rb[36];
      rd.take(rb, 36);
      if (rd.short_read || rb[0] != 32 || rb[1] || rb[2] || rb[3]) return 704;
      memcpy(next_root, rb + 4, 32);
      if (N.ood_samples) {
        std::vector<F> opt = sample_vec((size_t)l);
        F ov = rd.f();
        F mu = o_ts_f128(t);
        std::vector<F> e = eq_table(opt.data(), l);
        for (size_t j = 0; j < basis.size(); j++) basis[j] = add(basis[j], mul(mu, e[j]));
        lclaim = add(lclaim, mul(mu, ov));
      }
    } else {
      uint8_t nb[4];
      rd.take(nb, 4);
      uint32_t fl = (uint32_t)nb[0] | ((uint32_t)nb[1] << 8) | ((uint32_t)nb[2] << 16) |
                    ((uint32_t)nb[3] << 24);
      if (rd.short_read || fl != (1u << l)) return 705;
      f_final.resize(fl);
      for (auto &x : f_final) x = rd.f();
    }
    if (!lig_grind()) return 706;
    std::vector<F> qs = sample_vec((size_t)L.queries);
    const size_t rows = (size_t)1 << (cur_log_n - cur_k + cur_rate);
    const int width = 1 << cur_k, depth = ceil_log2(rows);
    const uint8_t *qh = rd.hint(8);
    if (!qh) return 707;
    uint64_t nq = 0;
    for (int b = 7; b >= 0; b--) nq = (nq << 8) | qh[b];
    if (nq != (uint64_t)L.queries) return 708;
    std::vector<F> eqr = eq_table(rs.data(), L.k);
    std::vector<F> vals(L.queries);
    std::vector<uint64_t> idx(L.queries);
    for (int qi = 0; qi < L.queries; qi++) {
      idx[qi] = qs[qi].lo & (rows - 1);
      const uint8_t *row = rd.hint((size_t)width * 16);
      if (!row) return 709;
      uint8_t node[32];
      o_blake3(row, (size_t)width * 16, node);
      size_t at_node = rows + idx[qi];
      for (int d = 0; d < depth; d++) {
        const uint8_t *sib = rd.hint(32);
        if (!sib) return 710;
        uint8_t pair[64];
        if (at_node & 1) {
          memcpy(pair, sib, 32);
          memcpy(pair + 32, node, 32);
        } else {
          memcpy(pair, node, 32);
          memcpy(pair + 32, sib, 32);
        }
        o_blake3(pair, 64, node);
        at_node >>= 1;
      }
      if (memcmp(node, cur_root, 32) != 0) return 711;
      F val = ZERO;
      for (int c = 0; c < width; c++) {
        F e;
        memcpy(&e, row + 16 * c, 16);
        val = add(val, mul(e, eqr[c]));
      }
      vals[qi] = val;
    }
    const int av = ceil_log2((size_t)L.queries);
    std::vector<F> alpha = sample_vec((size_t)av);
    F mu = o_ts_f128(t);
    std::vector<F> beta = eq_table(alpha.data(), av);
    for (int qi = 0; qi < L.queries; qi++) {
      F sc2 = mul(mu, beta[qi]);
      add_query_basis(basis, l, idx[qi], sc2);
      lclaim = add(lclaim, mul(sc2, vals[qi]));
    }
    if (!last) {
      memcpy(cur_root, next_root, 32);
      cur_log_n = l;
      cur_k = cfg.levels[i + 1].k;
      cur_rate = cfg.levels[i + 1].log_inv_rate;
    }
  }
  if (rd.short_read) return 712;
  F chk = ZERO;
  for (size_t j = 0; j < f_final.size(); j++) chk = add(chk, mul(basis[j], f_final[j]));
  if (!eqf(chk, lclaim)) return 713;
  // both streams spent (verify.rs:69-71)
  if (rd.pos != rd.narg_len || rd.hpos != rd.hints_len) return 801;
  return 0;
}

}  // namespace

struct o_prover {
  Setup s;
  std::vector<uint8_t> proof;
  double t_witness = 0, t_commit = 0, t_prove = 0;
};

extern "C" {

/* Runs setup, witness, commit and prove for one statement. Returns 0 and the
 * proof bytes through o_prover_proof(); the stage timings go to
 * o_prover_times(). */
o_prover *o_prover_run(int kind, const uint8_t *inputs, size_t n_inputs, const uint8_t *expected,
                       int security, int *status) {
  using clk = std::chrono::steady_clock;
  o_prover *P = new o_prover();
  Setup &s = P->s;
  auto t0 = clk::now();
  build_setup(s, kind, inputs, n_inputs, expected, security);
  // witness (end_to_end.rs:215-243): the replay above holds it; check it
  std::vector<uint8_t> fb(s.f_bits), hb(s.h_len);
  o_circuit_f(s.circ, fb.data());
  o_circuit_h(s.circ, hb.data());
  std::vector<int64_t> pa(s.rows), pb(s.rows), pc(s.rows);
  o_circuit_products(s.circ, pa.data(), pb.data(), pc.data());
  for (size_t r = 0; r < s.rows; r++)
    if ((__int128)pa[r] * pb[r] != pc[r]) {
      *status = 3;
      return P;
    }
  size_t packed_f = (size_t)1 << (s.committed_m - 7);
  size_t packed_h = (size_t)1 << s.claim_log_cols;
  std::vector<F> fpk(packed_f, ZERO), hpk(packed_h, ZERO);
  for (size_t i = 0; i < s.f_bits; i++)
    if (fb[i]) (i % 128 < 64 ? fpk[i / 128].lo : fpk[i / 128].hi) |= 1ull << (i % 64);
  for (size_t i = 0; i < s.h_len; i++)
    if (hb[i]) (i % 128 < 64 ? hpk[i / 128].lo : hpk[i / 128].hi) |= 1ull << (i % 64);
  auto t1 = clk::now();

  // ------------------------------------------------------------- commit
  o_transcript t;
  const char *dom = NAMES[kind];
  o_ts_init(&t, (const uint8_t *)"bitz/circuit-e2e/v2", 19, (const uint8_t *)dom, strlen(dom));
  Level level0;
  int log_n = s.committed_m - 7;
  commit_level(level0, fpk, log_n, s.pcs.levels[0].k, s.pcs.levels[0].log_inv_rate);
  uint8_t root[32];
  memcpy(root, level0.nodes.data() + 32, 32);
  std::vector<uint8_t> pcs_enc;
  pcs_encoding(s, pcs_enc);
  pub_str(&t, "bitz/pcs/commit/v1");
  o_ts_public(&t, root, 32);
  o_ts_public(&t, pcs_enc.data(), pcs_enc.size());
  std::vector<F> ood_pt;
  F ood_val = ZERO;
  if (security == 100) {
    pub_str(&t, "bitz/pcs/ood/v1");
    for (int i = 0; i < log_n; i++) ood_pt.push_back(o_ts_f128(&t));
    ood_val = mle_eval(fpk, ood_pt.data(), log_n);
    prov_f(&t, ood_val);
  }
  auto t2 = clk::now();

  // -------------------------------------------------------------- prove
  // bind (end_to_end.rs:442-455)
  pub_u64(&t, s.public_bytes.size());
  o_ts_public(&t, s.public_bytes.data(), s.public_bytes.size());
  o_ts_public(&t, root, 32);
  pub_u64(&t, 7);
  pub_u64(&t, (uint64_t)s.claim_log_cols);
  pub_f(&t, s.generator);
  o_ts_public(&t, pcs_enc.data(), pcs_enc.size());
  o_ts_public(&t, s.map_digest, 32);
  o_ts_public(&t, s.matrix_digest, 32);
  pub_str(&t, "bitz/circuit-opening-path/v1");
  uint8_t path = 1;
  o_ts_public(&t, &path, 1);
  // sample_and_install_prime, project_contraints (end_to_end.rs:401-435)
  u128 q = o_ts_prime(&t, (uint32_t)s.prime_bits);
  std::vector<uint8_t> params;
  u64le(params, 7);
  u64le(params, (uint64_t)s.claim_log_cols);
  uint8_t qb[16];
  u128le(qb, q);
  params.insert(params.end(), qb, qb + 16);
  params.insert(params.end(), (uint8_t *)&s.generator, (uint8_t *)&s.generator + 16);
  o_ts_public(&t, params.data(), params.size());
  // Spartan
  int nr = ceil_log2(s.rows ? s.rows : 1), nc = ceil_log2(s.h_len);
  std::vector<u128> outer(4 * (nr + 1)), inner(3 * (nc + 1)), rx(nr + 1), ry(nc + 1);
  u128 abc[3], d_ry, fin;
  const uint32_t *offs[3] = {s.off[0].data(), s.off[1].data(), s.off[2].data()};
  const uint32_t *cols[3] = {s.col[0].data(), s.col[1].data(), s.col[2].data()};
  const int64_t *coefs[3] = {s.coef[0].data(), s.coef[1].data(), s.coef[2].data()};
  const int64_t *prods[3] = {pa.data(), pb.data(), pc.data()};
  int rc = o_spartan_prove(q, s.rows, s.h_len, offs, cols, coefs, prods, hb.data(), s.matrix_digest,
                           &t, outer.data(), abc, inner.data(), rx.data(), ry.data(), &d_ry, &fin);
  if (rc) {
    *status = rc;
    return P;
  }
  // opening_claim (end_to_end.rs:509-528): rows scaled by D(r_y), point padded with zeros
  int mh = 7 + s.claim_log_cols;
  std::vector<u128> pt(mh, 0);
  for (int i = 0; i < nc; i++) pt[i] = ry[i];
  std::vector<u128> rows_w(128), cols_w((size_t)1 << s.claim_log_cols);
  o_fp_eq_table(pt.data(), 7, q, rows_w.data());
  for (auto &w : rows_w) w = o_fp_mul(w, d_ry, q);
  o_fp_eq_table(pt.data() + 7, s.claim_log_cols, q, cols_w.data());
  // BitZ prove_virtual (crates/prover/src/prove.rs:96-152)
  pub_str(&t, "bitz/virtual-statement/v1");
  o_ts_public(&t, root, 32);
  {
    // VirtualParams (params.rs:225-231): the claim parameters, then the
    // committed shape shape_for(f) = (7, m_f - 7)
    std::vector<uint8_t> vp = params;
    u64le(vp, 7);
    u64le(vp, (uint64_t)(s.committed_m - 7));
    o_ts_public(&t, vp.data(), vp.size());
  }
  o_ts_public(&t, s.map_digest, 32);
  {
    std::vector<uint8_t> ce;
    u64le(ce, 128);
    for (auto w : rows_w) {
      uint8_t b[16];
      u128le(b, w);
      ce.insert(ce.end(), b, b + 16);
    }
    u64le(ce, cols_w.size());
    for (auto w : cols_w) {
      uint8_t b[16];
      u128le(b, w);
      ce.insert(ce.end(), b, b + 16);
    }
    uint8_t b[16];
    u128le(b, fin);
    ce.insert(ce.end(), b, b + 16);
    o_ts_public(&t, ce.data(), ce.size());
  }
  o_ts_public(&t, pcs_enc.data(), pcs_enc.size());
  // send_fold (crates/prover/src/fold.rs:38-75)
  int sc = s.claim_log_cols;
  size_t ncol = (size_t)1 << sc;
  std::vector<u128> folds(ncol);
  o_fold_columns(hpk.data(), sc, rows_w.data(), folds.data());
  for (auto fd : folds) {
    uint8_t b[16];
    u128le(b, fd);
    o_ts_prover(&t, b, 16);
  }
  o_comb comb;
  o_comb_init(&comb, s.generator, 8);
  std::vector<F> row_images(128);
  for (int b = 0; b < 128; b++) row_images[b] = o_comb_pow(&comb, rows_w[b]);
  o_comb_free(&comb);
  o_ts_grind(&t, "bitz/columns/v1", grinding_bits(security, (uint64_t)sc));
  std::vector<F> zeta(sc);
  for (auto &z : zeta) z = o_ts_f128(&t);
  // gkr_reduce (crates/prover/src/reduce.rs:17-47)
  std::vector<F> gpt(sc + 7);
  F gclaim = o_gkr_prove(row_images.data(), hpk.data(), sc, zeta.data(), grinding_bits(security, 3),
                         &t, gpt.data());
  F ip_target = add(gclaim, ONE);
  std::vector<F> eqb = eq_table(gpt.data() + sc, 7), u2 = eq_table(gpt.data(), sc);
  std::vector<F> u1(128);
  for (int b = 0; b < 128; b++) u1[b] = mul(add(row_images[b], ONE), eqb[b]);
  // transpose_query (virtual_map.rs:174-223)
  size_t fcols = s.f_bits + 1;
  std::vector<F> wt(fcols);
  o_mt_transpose(s.csc_off.data(), s.csc_row.data(), fcols, u1.data(), 7, u2.data(), wt.data());
  F target2 = add(ip_target, wt[0]);
  size_t nbits = (size_t)1 << s.committed_m;
  std::vector<F> weights(nbits, ZERO);
  for (size_t c = 1; c < fcols; c++) weights[c - 1] = wt[c];
  // Pcs::prove_lin, InnerProduct (opening.rs:136-160, 337-368)
  pub_str(&t, "bitz/pcs/bit-inner-product/v3");
  o_ts_public(&t, root, 32);
  o_ts_public(&t, pcs_enc.data(), pcs_enc.size());
  pub_u64(&t, nbits);
  pub_u64(&t, 1);
  {
    o_blake3_state h;
    o_blake3_init_derive_key(&h, "bitz/pcs/bit-inner-product-weights/v1");
    o_blake3_update(&h, (const uint8_t *)weights.data(), nbits * 16);
    o_blake3_update(&h, (const uint8_t *)&ONE, 16);
    uint8_t dg[32];
    o_blake3_final(&h, dg);
    o_ts_public(&t, dg, 32);
  }
  pub_f(&t, target2);
  pub_str(&t, "bitz/pcs/inner-product-sumcheck/v2");
  std::vector<F> rho(s.committed_m);
  F v;
  F onecol[1] = {ONE};
  rc = o_post_gkr_prove(weights.data(), s.committed_m, onecol, 0, target2, fpk.data(),
                        grinding_bits(security, 2), &t, rho.data(), &v);
  if (rc) {
    *status = 10 + rc;
    return P;
  }
  // prove(Mle) with binding (opening.rs:119-135, 323-335)
  pub_str(&t, "bitz/pcs/mle-opening/v1");
  o_ts_public(&t, root, 32);
  o_ts_public(&t, pcs_enc.data(), pcs_enc.size());
  pub_u64(&t, (uint64_t)s.committed_m);
  for (auto &c : rho) pub_f(&t, c);
  pub_f(&t, v);
  // ring switch (mle.rs:63-123): s_v = sum_y eq(r_hi, y) bit_v(f[y])
  std::vector<F> suffix = eq_table(rho.data() + 7, log_n);
  std::vector<F> claims(128, ZERO);
  for (size_t y = 0; y < packed_f; y++)
    for (int b = 0; b < 128; b++)
      if (bitof(fpk[y], b)) claims[b] = add(claims[b], suffix[y]);
  {
    std::vector<F> pre = eq_table(rho.data(), 7);
    F chk = ZERO;
    for (int b = 0; b < 128; b++) chk = add(chk, mul(pre[b], claims[b]));
    if (!eqf(chk, v)) {
      *status = 20;
      return P;
    }
  }
  pub_str(&t, "bitz/pcs/mle-claims/v1");
  o_ts_prover(&t, claims.data(), 128 * 16);
  o_ts_grind(&t, "bitz/pcs/ring/v1", grinding_bits(security, 7 + (security == 100 ? 1 : 0)));
  pub_str(&t, "bitz/pcs/ring-switch-challenges/v1");
  std::vector<F> bpt(7);
  for (auto &c : bpt) c = o_ts_f128(&t);
  std::vector<F> bw = eq_table(bpt.data(), 7);
  // transposed claims: out[u].bit(v) = claims[v].bit(u) (transpose.rs:14)
  F ptarget = ZERO;
  for (int u = 0; u < 128; u++) {
    F tu = ZERO;
    for (int vv = 0; vv < 128; vv++)
      if (bitof(claims[vv], u)) (vv < 64 ? tu.lo : tu.hi) |= 1ull << (vv % 64);
    ptarget = add(ptarget, mul(tu, bw[u]));
  }
  std::vector<F> basis(packed_f, ZERO);
  for (size_t y = 0; y < packed_f; y++) {
    F acc = ZERO;
    for (int u = 0; u < 128; u++)
      if (bitof(suffix[y], u)) acc = add(acc, bw[u]);
    basis[y] = acc;
  }
  if (security == 100) {
    pub_str(&t, "bitz/pcs/ood-batching/v1");
    F coef = o_ts_f128(&t);
    std::vector<F> e = eq_table(ood_pt.data(), log_n);
    for (size_t y = 0; y < packed_f; y++) basis[y] = add(basis[y], mul(coef, e[y]));
    ptarget = add(ptarget, mul(coef, ood_val));
  }
  std::vector<uint8_t> lproof = ligerito_prove(&t, s.pcs, fpk, basis, ptarget, level0);
  if (lproof.empty()) {
    *status = 21;
    return P;
  }
  uint32_t ll = (uint32_t)lproof.size();
  o_ts_hint(&t, &ll, 4);
  o_ts_hint(&t, lproof.data(), lproof.size());
  auto t3 = clk::now();
  // proof bytes: root || Spartan section || wire container
  std::vector<uint8_t> &pr = P->proof;
  pr.insert(pr.end(), root, root + 32);
  for (int i = 0; i < 4 * nr; i++) {
    uint8_t b[16];
    u128le(b, outer[i]);
    pr.insert(pr.end(), b, b + 16);
  }
  for (int k = 0; k < 3; k++) {
    uint8_t b[16];
    u128le(b, abc[k]);
    pr.insert(pr.end(), b, b + 16);
  }
  for (int i = 0; i < 3 * nc; i++) {
    uint8_t b[16];
    u128le(b, inner[i]);
    pr.insert(pr.end(), b, b + 16);
  }
  const uint8_t magic[8] = {'b', 'i', 't', 'z', 'P', 'C', 'S', 0};
  pr.insert(pr.end(), magic, magic + 8);
  pr.push_back(1);
  pr.push_back(0);
  pr.push_back(32);
  pr.push_back(0);
  for (int i = 0; i < 4; i++) pr.push_back(0);
  u64le(pr, t.narg_len);
  u64le(pr, t.hints_len);
  pr.insert(pr.end(), t.narg, t.narg + t.narg_len);
  pr.insert(pr.end(), t.hints, t.hints + t.hints_len);
  o_ts_free(&t);
  P->t_witness = std::chrono::duration<double>(t1 - t0).count();
  P->t_commit = std::chrono::duration<double>(t2 - t1).count();
  P->t_prove = std::chrono::duration<double>(t3 - t2).count();
  *status = 0;
  return P;
}

size_t o_prover_proof(const o_prover *P, uint8_t *out, size_t cap) {
  if (out && cap >= P->proof.size()) memcpy(out, P->proof.data(), P->proof.size());
  return P->proof.size();
}

void o_prover_times(const o_prover *P, double out[3]) {
  out[0] = P->t_witness;
  out[1] = P->t_commit;
  out[2] = P->t_prove;
}

void o_prover_free(o_prover *P) {
  if (P->s.circ) o_circuit_free(P->s.circ);
  delete P;
}

/* The PCS profile encoding for a committed size of 2^m bits
 * (crates/pcs/src/commitment.rs:214-221). Returns its length. */
size_t o_pcs_encoding(int m, int security, uint8_t *out, size_t cap) {
  Setup s;
  s.committed_m = m;
  s.security = security;
  std::vector<uint8_t> enc;
  pcs_encoding(s, enc);
  if (out && cap >= enc.size()) memcpy(out, enc.data(), enc.size());
  return enc.size();
}

/* CircuitProofSystem::verify (end_to_end.rs:339-377) on proof bytes: 0 when
 * accepted, else the code of the first failed check. */
int o_verify(int kind, const uint8_t *inputs, size_t n_inputs, const uint8_t *expected,
             int security, const uint8_t *proof, size_t proof_len) {
  return verify_proof(kind, inputs, n_inputs, expected, security, proof, proof_len);
}

/* The statement's integer-matrix digest (crates/spartan/src/matrix.rs:562-661). */
void o_matrix_digest(int kind, const uint8_t *inputs, size_t n_inputs, const uint8_t *expected,
                     uint8_t out[32]) {
  Setup s;
  build_setup(s, kind, inputs, n_inputs, expected, 100);
  memcpy(out, s.matrix_digest, 32);
  o_circuit_free(s.circ);
}

}  // extern "C"
