/* CPU oracle: the binary PCS. Test infrastructure only.
 *
 * The reference delegates this layer to flock-core (git rev 8790722, not in
 * the reference tree), so only its interface, parameters and transcript hooks
 * are pinned: crates/pcs/src/{commitment,profiles,ligerito,challenger,ood,
 * mle,transpose}.rs. The algorithms below are this project's restatement of
 * the published constructions they name (parity unpinned):
 *
 * - Parameter ladder: crates/pcs/src/profiles.rs:26-126, with the query and
 *   grinding counts re-derived from the closed forms that profiles.rs:188-327
 *   tests against (pinned for m = 20 and m = 22).
 * - Reed-Solomon: interleaved columns (log_batch_size = initial k), each
 *   column read as coefficients in the Lin-Chung-Han novel polynomial basis
 *   and evaluated on the subspace spanned by X^0..X^(d-1) with the additive
 *   FFT (Lin, Chung, Han, FOCS 2014).
 * - Merkle: BLAKE3 of each codeword row (2^k elements, 16 bytes each, LE), and
 *   BLAKE3 of the 64-byte concatenation for every parent.
 * - Ring switch: crates/pcs/src/mle.rs:63-123 and transpose.rs:14-48.
 * - Ligerito (Novakovic and Angeris, 2025): per level, k sumcheck folds of the
 *   low variables, the folded vector committed at the next rate, queried rows
 *   glued into the next level's sumcheck by a batched linear claim.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"
#include "pcs.h"

/* ------------------------------------------------------------ the ladder */

static double ilog2c(double x) { return ceil(log2(x)); }

/* profiles.rs:26-59: levels fold INITIAL_K = 4, then RECURSIVE_K = 3 at most,
 * until FINAL_LOG_N = 5 variables remain; level i has log_inv_rate = i + 1. */
int o_pcs_config(int m, int security_bits, o_pcs_config_t *cfg) {
  if (m < 20 || m > 35) return 1;
  memset(cfg, 0, sizeof *cfg);
  cfg->m = m;
  cfg->security_bits = security_bits;
  int log_n = m - 7;
  cfg->log_n = log_n;
  int remaining = log_n;
  while (remaining > 5) {
    int folds = cfg->nlevels == 0 ? 4 : (3 < remaining - 5 ? 3 : remaining - 5);
    remaining -= folds;
    o_pcs_level_t *L = &cfg->levels[cfg->nlevels];
    L->k = folds;
    L->log_inv_rate = cfg->nlevels + 1;
    L->log_msg_cols = remaining;
    cfg->nlevels++;
  }
  cfg->final_log_n = remaining;
  for (int i = 0; i < cfg->nlevels; i++) {
    o_pcs_level_t *L = &cfg->levels[i];
    double n = ldexp(1.0, L->log_msg_cols + L->log_inv_rate);
    double rho = ldexp(1.0, -L->log_inv_rate);
    if (security_bits == 128) {
      /* unique decoding: profiles.rs:188-227 */
      double delta = 1.0 - rho;
      double gamma = delta / 2.0 - 3.0 / (delta * n);
      int g = 0;
      for (;; g++) {
        double beta = (i > 0 && g == 0) ? 1.0 : 0.0;
        if ((gamma * n + 3.0 + beta) * ldexp(1.0, -128 - g) <= ldexp(1.0, -128)) break;
      }
      L->fold_grinding = g;
      int q = 1;
      while (pow(1.0 - gamma, q) > ldexp(1.0, -128)) q++;
      L->queries = q;
      L->grinding = 4;
      L->ood_samples = 0;
    } else {
      /* Johnson regime, eta = 0.02: profiles.rs:244-327 */
      double eta = 0.02, srho = sqrt(rho);
      double list = 1.0 / (2.0 * eta * srho);
      double gamma = 1.0 - srho - eta;
      double half = fmax(ceil(srho / (2.0 * eta)), 3.0) + 0.5;
      double base = (2.0 * pow(half, 5) + 3.0 * half * gamma * rho) / (3.0 * pow(rho, 1.5)) * n +
                    half / srho;
      int k = L->k, g = 0;
      for (;; g++) {
        int fits = 1;
        for (int round = 0; round < k; round++) {
          double row_union = ldexp(1.0, k - 1 - round);
          int eff = g - round > 0 ? g - round : 0;
          double beta = (i > 0 && round == 0 && eff == 0) ? 1.0 : 0.0;
          if (base * row_union + (2.0 + beta) * list > ldexp(1.0, 28 + eff)) fits = 0;
        }
        if (fits) break;
      }
      L->fold_grinding = g;
      double next_list = 1.0;
      if (i + 1 < cfg->nlevels) {
        double nrho = ldexp(1.0, -(i + 2));
        next_list = 1.0 / (2.0 * eta * sqrt(nrho));
      }
      int q = 1;
      for (;; q++) {
        int np2 = 1;
        while (np2 < q) np2 <<= 1;
        int alpha = 0;
        while ((1 << alpha) < np2) alpha++;
        double err = pow(srho + eta, q) + (double)(alpha + 1) * next_list * ldexp(1.0, -128);
        if (err <= ldexp(1.0, -100)) break;
      }
      L->queries = q;
      L->grinding = 0;
      L->ood_samples = i > 0 ? 1 : 0;
    }
  }
  (void)ilog2c;
  return 0;
}

/* ---------------------------------------------------- additive FFT basis */

static o_f128 gadd(o_f128 a, o_f128 b) {
  o_f128 r = {a.lo ^ b.lo, a.hi ^ b.hi};
  return r;
}
static o_f128 elem(uint64_t idx) {
  o_f128 r = {idx, 0};
  return r;
}

/* W_0(x) = x, W_{t+1}(x) = W_t(x) (W_t(x) + W_t(v_t)), v_t = X^t: the
 * subspace polynomials of span(v_0..v_{t-1}), evaluated by carrying W_s(x)
 * and W_s(v_j) for every j up the recursion; Wh_t = W_t / W_t(v_t). */
static void subspace_eval(int t, o_f128 x, o_f128 *wx_out) {
  /* maintain W_s(x) and W_s(v_j) for j >= s */
  o_f128 wx = x;
  o_f128 wv[64];
  for (int j = 0; j < 64; j++) wv[j] = elem(1ull << j);
  for (int s = 0; s < t; s++) {
    o_f128 c = wv[s]; /* W_s(v_s) */
    wx = o_gf_mul(wx, gadd(wx, c));
    for (int j = s + 1; j < 64; j++) wv[j] = o_gf_mul(wv[j], gadd(wv[j], c));
  }
  *wx_out = wx;
}

/* Normalised subspace polynomial Wh_t(x). */
o_f128 o_wh(int t, o_f128 x) {
  o_f128 wx, wvt;
  subspace_eval(t, x, &wx);
  subspace_eval(t, elem(1ull << t), &wvt);
  return o_gf_mul(wx, o_gf_inv(wvt));
}

/* Table wh[t][s] = Wh_t(v_s) for t < s < d: every twiddle is a sum of these. */
static void twiddle_basis(int d, o_f128 *tab /* d*d */) {
  for (int t = 0; t < d; t++)
    for (int s = 0; s < d; s++) tab[t * d + s] = s > t ? o_wh(t, elem(1ull << s)) : elem(s == t);
}

/* Reed-Solomon encode one column: coefficients c[0..2^l) in the novel basis,
 * evaluations at x_q = F128(q) for q < 2^d (d = l + rate), strided access. */
void o_rs_encode_column(const o_f128 *msg, size_t stride_in, int l, int d, o_f128 *out,
                        size_t stride_out) {
  size_t N = (size_t)1 << d, M = (size_t)1 << l;
  o_f128 *a = (o_f128 *)calloc(N, sizeof(o_f128));
  /* levels t >= l only copy (the upper coefficients are zero) */
  for (size_t q = 0; q < N; q++) a[q] = msg[(q % M) * stride_in];
  o_f128 *tab = (o_f128 *)malloc(sizeof(o_f128) * d * d);
  twiddle_basis(d, tab);
  for (int t = l - 1; t >= 0; t--) {
    size_t half = (size_t)1 << t;
    for (size_t base = 0; base < N; base += 2 * half) {
      o_f128 lam = {0, 0};
      for (int s = t + 1; s < d; s++)
        if ((base >> s) & 1) lam = gadd(lam, tab[t * d + s]);
      for (size_t j = 0; j < half; j++) {
        o_f128 u = a[base + j], w = a[base + half + j];
        o_f128 u2 = gadd(u, o_gf_mul(lam, w));
        a[base + j] = u2;
        a[base + half + j] = gadd(u2, w);
      }
    }
  }
  for (size_t q = 0; q < N; q++) out[q * stride_out] = a[q];
  free(a);
  free(tab);
}

/* X_j(x) = prod over set bits t of j of Wh_t(x), evaluated naively. */
o_f128 o_novel_eval(const o_f128 *c, int l, o_f128 x) {
  o_f128 wh[64];
  for (int t = 0; t < l; t++) wh[t] = o_wh(t, x);
  o_f128 acc = {0, 0};
  for (size_t j = 0; j < ((size_t)1 << l); j++) {
    o_f128 b = {1, 0};
    for (int t = 0; t < l; t++)
      if ((j >> t) & 1) b = o_gf_mul(b, wh[t]);
    acc = gadd(acc, o_gf_mul(c[j], b));
  }
  return acc;
}

/* ---------------------------------------------------------------- Merkle */

static void hash_row(const o_f128 *row, int n, uint8_t out[32]) {
  o_blake3((const uint8_t *)row, (size_t)n * 16, out);
}

/* Builds a tree over `rows` leaves of `width` elements: nodes[1] is the root,
 * leaves at nodes[rows .. 2 rows). */
void o_merkle_build(const o_f128 *codeword, size_t rows, int width, uint8_t *nodes) {
  for (size_t i = 0; i < rows; i++) hash_row(codeword + i * width, width, nodes + 32 * (rows + i));
  for (size_t i = rows - 1; i >= 1; i--) o_blake3(nodes + 32 * (2 * i), 64, nodes + 32 * i);
}

/* ---------------------------------------------------------------- commit */

/* Interleaved encoding of level 0: the packed witness as 2^(log_n - k) rows by
 * 2^k columns (the low k variables index the column), every column encoded
 * at rate 2^-log_inv_rate; codeword row q holds the q-th symbol of every
 * column. */
void o_pcs_encode(const o_f128 *vec, int log_n, int k, int log_inv_rate, o_f128 *codeword) {
  int l = log_n - k, d = l + log_inv_rate;
  size_t cols = (size_t)1 << k;
  for (size_t c = 0; c < cols; c++) o_rs_encode_column(vec + c, cols, l, d, codeword + c, cols);
}
