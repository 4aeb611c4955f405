/*
 * CPU oracle for the BitZ SHA-256 proving path.
 *
 * TEST INFRASTRUCTURE ONLY. This library is a plain, scalar C restatement of
 * the reference prover's algorithms. It is the checker the CUDA path is
 * compared against in tests/, in __graft_entry__.smoke() and as the timed CPU
 * baseline in bench.py. Nothing in the product (bitz_b200/, include/) links,
 * loads or calls it.
 *
 * Every function cites the reference file:line it restates (paths are within
 * the worldfnd/BitZ workspace).
 *
 * Parity status: GF(2^128) is pinned by the NIST GCM vectors shipped with the
 * reference (crates/field/tests/vectors), SHA-256 by FIPS 180-4, Keccak-f by
 * FIPS 202 (checked against Python hashlib). The spongefish sponge framing,
 * BLAKE3 outputs and the flock-core PCS are not present in the reference tree:
 * those parts are "parity unpinned" (own restatement, self-consistent only).
 */
#ifndef BITZ_ORACLE_H
#define BITZ_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef unsigned __int128 u128;

/* ---------------------------------------------------------------- GF(2^128)
 * crates/field/src/gf128.rs:1-8: F_2[X]/(X^128+X^7+X^2+X+1), bit i of lo||hi is
 * the X^i coefficient. */
typedef struct {
  uint64_t lo, hi;
} o_f128;

typedef struct {
  uint64_t w[4];
} o_wide;

o_f128 o_gf_mul(o_f128 a, o_f128 b);
o_wide o_gf_mul_wide(o_f128 a, o_f128 b);
o_f128 o_gf_reduce(o_wide w);
o_f128 o_gf_square(o_f128 a);
o_f128 o_gf_inv(o_f128 a);
o_f128 o_gf_pow(o_f128 a, u128 e);
int o_gf_is_generator(o_f128 a);
o_f128 o_gf_smallest_generator(void);
o_f128 o_gf_mle_eval(const o_f128 *v, const o_f128 *point, int nvars);
void o_gf_eq_table(const o_f128 *r, int n, o_f128 *out);

/* Comb for fixed-base exponentiation, crates/field/src/gf128/pow.rs:137-199. */
typedef struct {
  int win, windows;
  o_f128 *table; /* windows * 2^win */
} o_comb;
void o_comb_init(o_comb *c, o_f128 base, int win);
void o_comb_free(o_comb *c);
o_f128 o_comb_pow(const o_comb *c, u128 e);

/* ------------------------------------------------------------- prime field
 * crates/field/src/helpers.rs: moduli below 2^126, canonical residues. */
u128 o_fp_mul(u128 a, u128 b, u128 q);
u128 o_fp_add(u128 a, u128 b, u128 q);
u128 o_fp_sub(u128 a, u128 b, u128 q);
int o_fp_is_prime_mr(u128 q, const u128 *bases, int nbases);

/* ------------------------------------------------------------------ hashes */
void o_keccak_f1600(uint64_t st[25]);
void o_sha3_256(const uint8_t *in, size_t len, uint8_t out[32]);
void o_sha256(const uint8_t *in, size_t len, uint8_t out[32]);
void o_sha256_compress(uint32_t state[8], const uint32_t block[16]);

typedef struct {
  uint32_t cv[8];
  uint32_t key[8];
  uint8_t buf[64];
  size_t buf_len;
  uint64_t chunk_counter;
  size_t chunk_len; /* bytes absorbed into the current chunk */
  int blocks_compressed;
  uint32_t flags;
  uint32_t stack[64][8];
  int stack_len;
} o_blake3_state;
void o_blake3_init(o_blake3_state *h);
void o_blake3_init_derive_key(o_blake3_state *h, const char *context);
void o_blake3_update(o_blake3_state *h, const uint8_t *in, size_t len);
void o_blake3_final(const o_blake3_state *h, uint8_t out[32]);
void o_blake3(const uint8_t *in, size_t len, uint8_t out[32]);
void o_blake3_derive_key(const char *context, const uint8_t *in, size_t len, size_t piece,
                         uint8_t out[32]);

/* -------------------------------------------------------------- transcript
 * crates/transcript/src/{domain,prover,pow,challenge}.rs over a Keccak duplex
 * sponge (spongefish 0.7.4 stand-in, parity unpinned). */
typedef struct {
  uint64_t st[25];
  int absorb_pos;
  int squeeze_pos;
  uint8_t *narg;
  size_t narg_len, narg_cap;
  uint8_t *hints;
  size_t hints_len, hints_cap;
} o_transcript;

void o_ts_init(o_transcript *t, const uint8_t *session, size_t slen,
               const uint8_t *instance, size_t ilen);
void o_ts_free(o_transcript *t);
void o_ts_public(o_transcript *t, const void *msg, size_t len);
void o_ts_prover(o_transcript *t, const void *msg, size_t len);
void o_ts_hint(o_transcript *t, const void *msg, size_t len);
void o_ts_squeeze(o_transcript *t, uint8_t *out, size_t len);
o_f128 o_ts_f128(o_transcript *t);
u128 o_ts_u128(o_transcript *t);
u128 o_ts_fp(o_transcript *t, u128 q);
void o_ts_grind(o_transcript *t, const char *label, uint32_t bits);
u128 o_ts_prime(o_transcript *t, uint32_t bits);
int o_pow_valid(const uint8_t seed[16], uint64_t nonce, uint32_t bits);

/* ---------------------------------------------------------- post-GKR (a15)
 * crates/post_gkr/src/lib.rs:121-148 and sumcheck.rs:98-215.
 * rows: 2^t weights, cols: 2^s weights, packed: 2^(t+s-7) elements.
 * point_out: t+s coordinates, returns the closing evaluation v. */
int o_post_gkr_prove(const o_f128 *rows, int log_rows, const o_f128 *cols,
                     int log_cols, o_f128 target, const o_f128 *packed,
                     uint32_t grind_bits, o_transcript *t, o_f128 *point_out,
                     o_f128 *value_out);

/* ------------------------------------------------------------- GKR (a11-12)
 * crates/gkr/src/lib.rs:24-81,785-897. The table holds 2^s columns of 128
 * bits (one F128 per column), row_images has 128 entries. Writes the leaves'
 * point (7+s coordinates) and returns the claim on the leaves. */
o_f128 o_gkr_prove(const o_f128 *row_images, const o_f128 *columns, int log_cols,
                   const o_f128 *zeta, uint32_t grind_bits, o_transcript *t,
                   o_f128 *point_out);
void o_gkr_outputs(const o_f128 *row_images, const o_f128 *columns, int log_cols,
                   o_f128 *out);

/* -------------------------------------------------------------- fold (a10)
 * crates/common/src/fold.rs:29-104, crates/prover/src/fold.rs:38-75. */
void o_fold_columns(const o_f128 *columns, int log_cols, const u128 *exponents,
                    u128 *folds);

/* ------------------------------------------------------------- M^T (a13)
 * crates/circuit/src/matrix_transpose.rs:377-416. */
void o_mt_transpose(const uint32_t *col_off, const uint32_t *row_idx,
                    size_t ncols, const o_f128 *row_w, int log_rows,
                    const o_f128 *col_w, o_f128 *out);

#ifdef __cplusplus
}
#endif
#endif
