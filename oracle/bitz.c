/* CPU oracle: BitZ reduction stages over GF(2^128). Test infrastructure only.
 *
 * Each stage is written in its plainest dense form. Round messages are exact
 * field values, so a dense table gives the same bytes as the reference's
 * lookup-table and bucket shortcuts (crates/gkr/src/lib.rs:265-604). */
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

static o_f128 add(o_f128 a, o_f128 b) {
  o_f128 r = {a.lo ^ b.lo, a.hi ^ b.hi};
  return r;
}
static const o_f128 ONE = {1, 0};
static const o_f128 ZERO = {0, 0};
static int is_zero(o_f128 a) { return a.lo == 0 && a.hi == 0; }
static int eq128(o_f128 a, o_f128 b) { return a.lo == b.lo && a.hi == b.hi; }
static int bit_of(o_f128 e, int v) { return v < 64 ? (int)((e.lo >> v) & 1) : (int)((e.hi >> (v - 64)) & 1); }

static void msg2(o_transcript *t, o_f128 a, o_f128 b) {
  uint8_t m[32];
  memcpy(m, &a.lo, 8);
  memcpy(m + 8, &a.hi, 8);
  memcpy(m + 16, &b.lo, 8);
  memcpy(m + 24, &b.hi, 8);
  o_ts_prover(t, m, 32);
}

static void msg1(o_transcript *t, o_f128 a) {
  uint8_t m[16];
  memcpy(m, &a.lo, 8);
  memcpy(m + 8, &a.hi, 8);
  o_ts_prover(t, m, 16);
}

/* crates/post_gkr/src/lib.rs:320-323: h' = p(rho), a1 = h + a2. */
static o_f128 advance(o_f128 claim, o_f128 a0, o_f128 a2, o_f128 r) {
  o_f128 inner = add(add(claim, a2), o_gf_mul(r, a2));
  return add(a0, o_gf_mul(r, inner));
}

/* crates/post_gkr/src/sumcheck.rs:198-205: entry = t0 + r (t0 + t1). */
static void fold_table(o_f128 *t, size_t n, o_f128 r) {
  for (size_t k = 0; k < n / 2; k++) t[k] = add(t[2 * k], o_gf_mul(r, add(t[2 * k], t[2 * k + 1])));
}

/* crates/post_gkr/src/lib.rs:121-148 (prove_factors), :189-239 (weighted_sum,
 * first_message, fold), :265-283 (bind_first), sumcheck.rs:98-215. */
int o_post_gkr_prove(const o_f128 *rows, int log_rows, const o_f128 *cols, int log_cols,
                     o_f128 target, const o_f128 *packed, uint32_t grind_bits, o_transcript *t,
                     o_f128 *point_out, o_f128 *value_out) {
  size_t per_col = (size_t)1 << (log_rows - 7);
  size_t ncols = (size_t)1 << log_cols;
  size_t npacked = per_col * ncols;
  /* weighted_sum: the claim must hold */
  o_f128 ws = ZERO;
  for (size_t e = 0; e < npacked; e++) {
    const o_f128 *rw = rows + ((e % per_col) << 7);
    o_f128 s = ZERO;
    for (int v = 0; v < 128; v++)
      if (bit_of(packed[e], v)) s = add(s, rw[v]);
    ws = add(ws, o_gf_mul(cols[e / per_col], s));
  }
  if (!eq128(ws, target)) return 2; /* ClaimDoesNotHold */
  /* first_message: a0 over even set bits, a2 over pairs whose bits differ */
  o_f128 a0 = ZERO, a2 = ZERO;
  for (size_t e = 0; e < npacked; e++) {
    const o_f128 *rw = rows + ((e % per_col) << 7);
    o_f128 s0 = ZERO, s2 = ZERO;
    for (int v = 0; v < 128; v += 2) {
      int b0 = bit_of(packed[e], v), b1 = bit_of(packed[e], v + 1);
      if (b0) s0 = add(s0, rw[v]);
      if (b0 != b1) s2 = add(s2, add(rw[v], rw[v + 1]));
    }
    o_f128 c = cols[e / per_col];
    a0 = add(a0, o_gf_mul(c, s0));
    a2 = add(a2, o_gf_mul(c, s2));
  }
  msg2(t, a0, a2);
  o_ts_grind(t, "bitz/pcs/sumcheck/v1", grind_bits);
  o_f128 r = o_ts_f128(t);
  o_f128 claim = advance(target, a0, a2, r);
  point_out[0] = r;
  /* fold the weights: folded rows tensored with columns */
  size_t nrows = (size_t)1 << log_rows;
  size_t n = (nrows / 2) * ncols;
  o_f128 *rowsf = (o_f128 *)malloc(sizeof(o_f128) * nrows);
  memcpy(rowsf, rows, sizeof(o_f128) * nrows);
  fold_table(rowsf, nrows, r);
  o_f128 *w = (o_f128 *)malloc(sizeof(o_f128) * n);
  o_f128 *v = (o_f128 *)malloc(sizeof(o_f128) * n);
  for (size_t c = 0; c < ncols; c++)
    for (size_t k = 0; k < nrows / 2; k++) w[c * (nrows / 2) + k] = o_gf_mul(cols[c], rowsf[k]);
  /* bind_first: pairs of bits map to 0, 1+r, r, 1 */
  o_f128 vals[4] = {ZERO, add(r, ONE), r, ONE};
  for (size_t e = 0; e < npacked; e++)
    for (int p = 0; p < 64; p++) {
      int two = bit_of(packed[e], 2 * p) | (bit_of(packed[e], 2 * p + 1) << 1);
      v[e * 64 + p] = vals[two];
    }
  free(rowsf);
  int rounds = 0;
  while (((size_t)1 << rounds) < n) rounds++;
  for (int k = 0; k < rounds; k++) {
    size_t len = n >> k;
    o_wide s0 = {{0, 0, 0, 0}}, s2 = {{0, 0, 0, 0}};
    for (size_t i = 0; i < len / 2; i++) {
      o_wide p0 = o_gf_mul_wide(w[2 * i], v[2 * i]);
      o_wide p2 = o_gf_mul_wide(add(w[2 * i], w[2 * i + 1]), add(v[2 * i], v[2 * i + 1]));
      for (int j = 0; j < 4; j++) {
        s0.w[j] ^= p0.w[j];
        s2.w[j] ^= p2.w[j];
      }
    }
    o_f128 m0 = o_gf_reduce(s0), m2 = o_gf_reduce(s2);
    msg2(t, m0, m2);
    o_ts_grind(t, "bitz/pcs/sumcheck/v1", grind_bits);
    o_f128 rr = o_ts_f128(t);
    claim = advance(claim, m0, m2, rr);
    point_out[1 + k] = rr;
    fold_table(w, len, rr);
    fold_table(v, len, rr);
  }
  *value_out = v[0];
  msg1(t, v[0]);
  int ok = eq128(o_gf_mul(w[0], v[0]), claim);
  free(w);
  free(v);
  return ok ? 0 : 3;
}

/* ------------------------------------------------------------------- GKR */

/* crates/gkr/src/reduce.rs:1-5 and lib.rs:265-283: leaf (b << s) | c is the row
 * image b where bit (c, b) is set, one elsewhere. */
static o_f128 *gkr_leaves(const o_f128 *img, const o_f128 *cols, int s) {
  size_t nc = (size_t)1 << s;
  o_f128 *l = (o_f128 *)malloc(sizeof(o_f128) * 128 * nc);
  for (size_t b = 0; b < 128; b++)
    for (size_t c = 0; c < nc; c++) l[(b << s) | c] = bit_of(cols[c], (int)b) ? img[b] : ONE;
  return l;
}

/* crates/gkr/src/lib.rs:874-897: node k multiplies nodes k and k + half. */
static o_f128 *gkr_parent(const o_f128 *child, size_t len) {
  o_f128 *p = (o_f128 *)malloc(sizeof(o_f128) * (len / 2));
  for (size_t k = 0; k < len / 2; k++) p[k] = o_gf_mul(child[k], child[k + len / 2]);
  return p;
}

void o_gkr_outputs(const o_f128 *row_images, const o_f128 *columns, int log_cols, o_f128 *out) {
  o_f128 *layer = gkr_leaves(row_images, columns, log_cols);
  size_t len = (size_t)128 << log_cols;
  for (int j = 0; j < 7; j++) {
    o_f128 *p = gkr_parent(layer, len);
    free(layer);
    layer = p;
    len /= 2;
  }
  memcpy(out, layer, sizeof(o_f128) * len);
  free(layer);
}

/* crates/gkr/src/lib.rs:88-157 (prove_layer, prove_rounds), 164-240
 * (round_sums, bind), 617-633 (sends_one, eq_factor). Returns the claim on the
 * children and writes n + 1 coordinates. */
static o_f128 gkr_prove_layer(o_transcript *t, const o_f128 *point, int n, o_f128 *children,
                              uint32_t grind_bits, o_f128 *next_point) {
  size_t half = (size_t)1 << n;
  o_f128 *left = children, *right = children + half;
  o_f128 *eq = (o_f128 *)malloc(sizeof(o_f128) * (half > 1 ? half / 2 : 1));
  o_f128 eq_bound = ONE;
  for (int i = n - 1; i >= 0; i--) {
    o_f128 z = point[i];
    size_t h = (size_t)1 << i;
    o_gf_eq_table(point, i, eq);
    int at_one = is_zero(z);
    o_wide sb = {{0, 0, 0, 0}}, si = {{0, 0, 0, 0}};
    for (size_t x = 0; x < h; x++) {
      o_f128 l0 = left[x], l1 = left[h + x], r0 = right[x], r1 = right[h + x];
      o_f128 lb = at_one ? l1 : l0, rb = at_one ? r1 : r0;
      o_wide pb = o_gf_mul_wide(o_gf_mul(eq[x], lb), rb);
      o_wide pi = o_gf_mul_wide(o_gf_mul(eq[x], add(l1, l0)), add(r1, r0));
      for (int j = 0; j < 4; j++) {
        sb.w[j] ^= pb.w[j];
        si.w[j] ^= pi.w[j];
      }
    }
    msg2(t, o_gf_mul(eq_bound, o_gf_reduce(sb)), o_gf_mul(eq_bound, o_gf_reduce(si)));
    o_ts_grind(t, "gkr/cubic/v1", grind_bits);
    o_f128 r = o_ts_f128(t);
    for (size_t x = 0; x < h; x++) {
      left[x] = add(left[x], o_gf_mul(r, add(left[h + x], left[x])));
      right[x] = add(right[x], o_gf_mul(r, add(right[h + x], right[x])));
    }
    next_point[i] = r;
    eq_bound = o_gf_mul(eq_bound, add(add(ONE, r), z));
  }
  free(eq);
  o_f128 lr = left[0], rr = right[0];
  msg2(t, lr, rr);
  o_f128 tt = o_ts_f128(t);
  next_point[n] = tt;
  return add(lr, o_gf_mul(tt, add(rr, lr)));
}

/* crates/gkr/src/lib.rs:24-81: the seven layer sumchecks from the output down. */
o_f128 o_gkr_prove(const o_f128 *row_images, const o_f128 *columns, int log_cols,
                   const o_f128 *zeta, uint32_t grind_bits, o_transcript *t, o_f128 *point_out) {
  o_f128 *layers[8];
  size_t len = (size_t)128 << log_cols;
  layers[0] = gkr_leaves(row_images, columns, log_cols);
  for (int j = 0; j < 7; j++) {
    layers[j + 1] = gkr_parent(layers[j], len);
    len /= 2;
  }
  int n = log_cols;
  o_f128 *point = (o_f128 *)malloc(sizeof(o_f128) * (n + 8));
  o_f128 *next = (o_f128 *)malloc(sizeof(o_f128) * (n + 8));
  memcpy(point, zeta, sizeof(o_f128) * n);
  o_f128 claim = ZERO;
  for (int j = 6; j >= 0; j--) {
    claim = gkr_prove_layer(t, point, n, layers[j], grind_bits, next);
    n++;
    memcpy(point, next, sizeof(o_f128) * n);
  }
  memcpy(point_out, point, sizeof(o_f128) * n);
  for (int j = 0; j < 8; j++) free(layers[j]);
  free(point);
  free(next);
  return claim;
}

/* ------------------------------------------------------------------ fold */

/* crates/common/src/fold.rs:29-63: eta_c = sum of row exponents at set bits. */
void o_fold_columns(const o_f128 *columns, int log_cols, const u128 *exponents, u128 *folds) {
  size_t nc = (size_t)1 << log_cols;
  for (size_t c = 0; c < nc; c++) {
    u128 s = 0;
    for (int b = 0; b < 128; b++)
      if (bit_of(columns[c], b)) s += exponents[b];
    folds[c] = s;
  }
}

/* ------------------------------------------------------------------- M^T */

/* crates/circuit/src/matrix_transpose.rs:377-416: per column of M, the sum over
 * its nonzero rows of row_w[row & mask] * col_w[row >> log_rows]. */
void o_mt_transpose(const uint32_t *col_off, const uint32_t *row_idx, size_t ncols,
                    const o_f128 *row_w, int log_rows, const o_f128 *col_w, o_f128 *out) {
  uint32_t mask = (1u << log_rows) - 1;
  for (size_t c = 0; c < ncols; c++) {
    o_wide s = {{0, 0, 0, 0}};
    for (uint32_t k = col_off[c]; k < col_off[c + 1]; k++) {
      uint32_t r = row_idx[k];
      o_wide p = o_gf_mul_wide(row_w[r & mask], col_w[r >> log_rows]);
      for (int j = 0; j < 4; j++) s.w[j] ^= p.w[j];
    }
    out[c] = o_gf_reduce(s);
  }
}

/* crates/post_gkr/src/lib.rs:189-209 (weighted_sum): <rows (x) cols, f>. */
o_f128 o_weighted_sum(const o_f128 *rows, int log_rows, const o_f128 *cols, int log_cols,
                      const o_f128 *packed) {
  size_t per_col = (size_t)1 << (log_rows - 7);
  size_t npacked = per_col << log_cols;
  o_f128 ws = ZERO;
  for (size_t e = 0; e < npacked; e++) {
    const o_f128 *rw = rows + ((e % per_col) << 7);
    o_f128 s = ZERO;
    for (int v = 0; v < 128; v++)
      if (bit_of(packed[e], v)) s = add(s, rw[v]);
    ws = add(ws, o_gf_mul(cols[e / per_col], s));
  }
  return ws;
}
