/*
 * bitz_b200 — C ABI of the B200 BitZ SHA-256 prover.
 *
 * Every entry point returns an int status (BZ_OK = 0, codes in
 * bitz_b200/csrc/status.hpp, mirroring the reference's error enums) and never
 * lets an exception cross the boundary; bitz_last_error() returns a
 * thread-local message for the last failure. Field elements are passed as
 * pairs of uint64_t (lo, hi) in the reference's GF(2^128) basis
 * (crates/field/src/gf128.rs:1-8); prime-field values as 16-byte little-endian
 * canonical residues (crates/field/src/codec.rs:69-73).
 *
 * Pointers named `*_dev` are device pointers on the current CUDA device;
 * every other pointer is host memory owned by the caller.
 */
#ifndef BITZ_B200_H
#define BITZ_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ errors */
const char *bitz_last_error(void);
int bitz_device_count(void);

/* -------------------------------------------------------------- transcript
 * The prover half of the Fiat-Shamir transcript.
 * Replaces: transcript::build_prover (crates/transcript/src/domain.rs:13-26),
 * ProverState::{public_message, prover_message, verifier_message, hint, grind,
 * finish} (crates/transcript/src/prover.rs:15-84). */
typedef struct bitz_transcript bitz_transcript;
bitz_transcript *bitz_transcript_new(const uint8_t *session, size_t session_len,
                                     const uint8_t *instance, size_t instance_len);
void bitz_transcript_free(bitz_transcript *t);
int bitz_transcript_public(bitz_transcript *t, const void *msg, size_t len);
int bitz_transcript_prover(bitz_transcript *t, const void *msg, size_t len);
int bitz_transcript_hint(bitz_transcript *t, const void *msg, size_t len);
int bitz_transcript_challenge_f128(bitz_transcript *t, uint64_t out[2]);
int bitz_transcript_grind(bitz_transcript *t, const char *label, uint32_t bits);
/* crates/transcript/src/challenge/prime.rs:33 (squeeze_prime) */
int bitz_transcript_prime(bitz_transcript *t, uint32_t bits, uint8_t out_le[16]);
/* Copies the narg string / hints into out (if cap allows) and returns their
 * length. crates/transcript/src/prover.rs:78 (finish). */
size_t bitz_transcript_narg(const bitz_transcript *t, uint8_t *out, size_t cap);
size_t bitz_transcript_hints(const bitz_transcript *t, uint8_t *out, size_t cap);

/* ------------------------------------------------------- post-GKR sumcheck
 * Replaces post_gkr::prove (crates/post_gkr/src/lib.rs:85-100) on the claim
 * <rows (x) cols, f> = target: 2^log_rows row weights (log_rows >= 7),
 * 2^log_cols column weights, 2^(log_rows+log_cols-7) packed words of f.
 * Writes log_rows+log_cols challenges to point_out and the closing evaluation
 * to value_out. security_bits is 100 or 128 (grinding per
 * crates/common/src/security.rs:25). Returns BZ_ERR_CLAIM if the claim does
 * not hold (ProveError::ClaimDoesNotHold). */
int bitz_post_gkr_prove(const uint64_t *rows, int log_rows, const uint64_t *cols, int log_cols,
                        const uint64_t target[2], const uint64_t *packed,
                        uint32_t security_bits, bitz_transcript *t, uint64_t *point_out,
                        uint64_t value_out[2]);
int bitz_post_gkr_prove_dev(const uint64_t *rows_dev, int log_rows, const uint64_t *cols_dev,
                            int log_cols, const uint64_t target[2], const uint64_t *packed_dev,
                            uint32_t security_bits, bitz_transcript *t, uint64_t *point_out,
                            uint64_t value_out[2]);

/* ------------------------------------------------------- grand-product GKR
 * Replaces gkr::grand_product + gkr::gpgkr_prove (crates/gkr/src/lib.rs:785,24)
 * for a table of 2^log_cols columns of 128 bits (one packed word per column)
 * and its 128 row images, from the output point zeta (log_cols coordinates).
 * Writes 7+log_cols coordinates to point_out and the leaves' claim. */
int bitz_gkr_prove(const uint64_t *row_images, const uint64_t *columns, int log_cols,
                   const uint64_t *zeta, uint32_t security_bits, bitz_transcript *t,
                   uint64_t *point_out, uint64_t claim_out[2]);
int bitz_gkr_prove_dev(const uint64_t *row_images_dev, const uint64_t *columns_dev,
                       int log_cols, const uint64_t *zeta, uint32_t security_bits,
                       bitz_transcript *t, uint64_t *point_out, uint64_t claim_out[2]);
/* gkr::grand_product's output layer only (crates/gkr/src/lib.rs:785-803). */
int bitz_gkr_outputs(const uint64_t *row_images, const uint64_t *columns, int log_cols,
                     uint64_t *out);

#ifdef __cplusplus
}
#endif
#endif
