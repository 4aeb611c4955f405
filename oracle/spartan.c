/* CPU oracle: Spartan's outer and inner sumchecks over the transcript-drawn
 * prime, and the matrix bind between them. Test infrastructure only.
 *
 * crates/spartan/src/piop.rs:67-113 (composition), sumcheck.rs:252-384 (outer),
 * sumcheck.rs:442-553 (inner), sumcheck.rs:724-802 (cubic_contribution,
 * reconstruct_round_coefficients, evaluate_polynomial), matrix.rs:429-467
 * (bind_and_batch), matrix.rs:336-419 (build_product_mles,
 * build_assignment_mle). Every value is a canonical residue below q. */
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

static void put_fp(uint8_t *b, u128 v) {
  for (int i = 0; i < 16; i++) b[i] = (uint8_t)(v >> (8 * i));
}

/* crates/spartan/src/sumcheck.rs:771-811: write [c0, c1, ...] with c1 recovered
 * from the running claim, absorb, squeeze, move the claim to p(r). */
static u128 round_and_challenge(o_transcript *t, u128 q, u128 *claim, const u128 *without_linear,
                                int ncoef, u128 *coefs_out) {
  u128 c[4];
  c[0] = without_linear[0];
  c[1] = 0;
  for (int i = 2; i < ncoef; i++) c[i] = without_linear[i - 1];
  u128 at_one = 0;
  for (int i = 0; i < ncoef; i++) at_one = o_fp_add(at_one, c[i], q);
  c[1] = o_fp_sub(o_fp_sub(*claim, c[0], q), at_one, q);
  uint8_t msg[64];
  for (int i = 0; i < ncoef; i++) put_fp(msg + 16 * i, c[i]);
  o_ts_public(t, msg, 16 * (size_t)ncoef);
  u128 r = o_ts_fp(t, q);
  u128 v = 0;
  for (int i = ncoef - 1; i >= 0; i--) v = o_fp_add(o_fp_mul(v, r, q), c[i], q);
  *claim = v;
  for (int i = 0; i < ncoef; i++) coefs_out[i] = c[i];
  return r;
}

static void fold(u128 *t, size_t n, u128 r, u128 q) {
  for (size_t k = 0; k < n / 2; k++)
    t[k] = o_fp_add(t[2 * k], o_fp_mul(r, o_fp_sub(t[2 * k + 1], t[2 * k], q), q), q);
}

static u128 reduce_i64(int64_t v, u128 q) {
  if (v >= 0) return (u128)v % q;
  u128 m = (u128)(-(v + 1)) + 1;
  m %= q;
  return m ? q - m : 0;
}

/* eq over the prime field, little-endian variables (crates/poly/src/eq.rs:63). */
void o_fp_eq_table(const u128 *r, int n, u128 q, u128 *out) {
  out[0] = 1;
  for (int i = 0; i < n; i++) {
    size_t half = (size_t)1 << i;
    for (size_t k = 0; k < half; k++) {
      u128 p = out[k];
      u128 one = o_fp_mul(p, r[i], q);
      out[k] = o_fp_sub(p, one, q);
      out[k + half] = one;
    }
  }
}

/* The whole Spartan PIOP. Inputs: the modulus, the R1CS in CSR with integer
 * coefficients (rows x cols logical sizes), the exact products and the 0/1
 * assignment h (one byte per entry). Outputs: the outer round polynomials
 * (4 per round), the three MLE claims, the inner round polynomials (3 per
 * round), r_x, r_y, D(r_y) and the final claim. */
int o_spartan_prove(u128 q, size_t rows, size_t cols, const uint32_t *const off[3],
                    const uint32_t *const col_idx[3], const int64_t *const coef[3],
                    const int64_t *const prod[3], const uint8_t *h, const uint8_t digest[32],
                    o_transcript *t, u128 *outer_polys, u128 abc_claims[3], u128 *inner_polys,
                    u128 *rx, u128 *ry, u128 *d_at_ry, u128 *final_claim) {
  int nr = 0, nc = 0;
  while (((size_t)1 << nr) < (rows ? rows : 1)) nr++;
  while (((size_t)1 << nc) < (cols ? cols : 1)) nc++;
  size_t R = (size_t)1 << nr, C = (size_t)1 << nc;
  o_ts_public(t, digest, 32);
  u128 *tau = (u128 *)malloc(sizeof(u128) * (nr ? nr : 1));
  for (int i = 0; i < nr; i++) tau[i] = o_ts_fp(t, q);
  u128 *E = (u128 *)malloc(sizeof(u128) * R);
  u128 *T[3];
  o_fp_eq_table(tau, nr, q, E);
  for (int k = 0; k < 3; k++) {
    T[k] = (u128 *)calloc(R, sizeof(u128));
    for (size_t i = 0; i < rows; i++) T[k][i] = reduce_i64(prod[k][i], q);
  }
  /* outer sumcheck: claim 0 = sum_x eq(tau, x) (A(x) B(x) - C(x)) */
  u128 claim = 0;
  for (int round = 0; round < nr; round++) {
    size_t len = R >> round;
    u128 acc[3] = {0, 0, 0};
    for (size_t k = 0; k < len / 2; k++) {
      u128 e0 = E[2 * k], e1 = E[2 * k + 1];
      u128 a0 = T[0][2 * k], a1 = T[0][2 * k + 1];
      u128 b0 = T[1][2 * k], b1 = T[1][2 * k + 1];
      u128 c0 = T[2][2 * k], c1 = T[2][2 * k + 1];
      u128 ed = o_fp_sub(e1, e0, q), ad = o_fp_sub(a1, a0, q), bd = o_fp_sub(b1, b0, q),
           cd = o_fp_sub(c1, c0, q);
      u128 r0 = o_fp_sub(o_fp_mul(a0, b0, q), c0, q);
      u128 rl = o_fp_sub(o_fp_add(o_fp_mul(a0, bd, q), o_fp_mul(ad, b0, q), q), cd, q);
      u128 rq = o_fp_mul(ad, bd, q);
      acc[0] = o_fp_add(acc[0], o_fp_mul(e0, r0, q), q);
      acc[1] = o_fp_add(acc[1], o_fp_add(o_fp_mul(e0, rq, q), o_fp_mul(ed, rl, q), q), q);
      acc[2] = o_fp_add(acc[2], o_fp_mul(ed, rq, q), q);
    }
    u128 r = round_and_challenge(t, q, &claim, acc, 4, outer_polys + 4 * round);
    rx[round] = r;
    fold(E, len, r, q);
    for (int k = 0; k < 3; k++) fold(T[k], len, r, q);
  }
  for (int k = 0; k < 3; k++) abc_claims[k] = T[k][0];
  uint8_t msg[48];
  for (int k = 0; k < 3; k++) put_fp(msg + 16 * k, abc_claims[k]);
  o_ts_public(t, msg, 48);
  u128 rho = o_ts_fp(t, q);
  u128 rho2 = o_fp_mul(rho, rho, q);
  u128 scales[3] = {1, rho, rho2};
  u128 inner_claim = o_fp_add(o_fp_add(abc_claims[0], o_fp_mul(rho, abc_claims[1], q), q),
                              o_fp_mul(rho2, abc_claims[2], q), q);
  /* bind_and_batch: D(j) = sum_i eq(r_x, i) (A + rho B + rho^2 C)[i, j] */
  o_fp_eq_table(rx, nr, q, E);
  u128 *D = (u128 *)calloc(C, sizeof(u128));
  for (int k = 0; k < 3; k++)
    for (size_t i = 0; i < rows; i++) {
      u128 w = o_fp_mul(E[i], scales[k], q);
      for (uint32_t e = off[k][i]; e < off[k][i + 1]; e++)
        D[col_idx[k][e]] = o_fp_add(D[col_idx[k][e]], o_fp_mul(w, reduce_i64(coef[k][e], q), q), q);
    }
  u128 *W = (u128 *)calloc(C, sizeof(u128));
  for (size_t j = 0; j < cols; j++) W[j] = h[j] ? 1 : 0;
  claim = inner_claim;
  for (int round = 0; round < nc; round++) {
    size_t len = C >> round;
    u128 acc[2] = {0, 0};
    for (size_t k = 0; k < len / 2; k++) {
      u128 d0 = D[2 * k], d1 = D[2 * k + 1], w0 = W[2 * k], w1 = W[2 * k + 1];
      acc[0] = o_fp_add(acc[0], o_fp_mul(d0, w0, q), q);
      acc[1] = o_fp_add(acc[1], o_fp_mul(o_fp_sub(d1, d0, q), o_fp_sub(w1, w0, q), q), q);
    }
    u128 r = round_and_challenge(t, q, &claim, acc, 3, inner_polys + 3 * round);
    ry[round] = r;
    fold(D, len, r, q);
    fold(W, len, r, q);
  }
  *d_at_ry = D[0];
  *final_claim = claim;
  int ok = o_fp_mul(D[0], W[0], q) == claim;
  free(tau);
  free(E);
  for (int k = 0; k < 3; k++) free(T[k]);
  free(D);
  free(W);
  return ok ? 0 : 6;
}
