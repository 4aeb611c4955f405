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

}  // extern "C"
