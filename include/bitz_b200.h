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
/* Selects the device this library's calls use (one process per GPU); call it
 * before the first other call. No reference counterpart: the reference is
 * CPU-only. */
int bitz_set_device(int device);

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

/* The post-GKR sumcheck as bitz_post_gkr_prove_dev, allocating nothing.
 * No counterpart in the reference. For callers that cannot allocate device
 * memory: processes whose device memory belongs to another allocator or to a
 * fixed budget set aside at start-up, and embedders that forbid allocation on
 * the request path. Inputs are device pointers, outputs host pointers;
 * stream may be NULL (the default stream). Its scratch is a fixed array in
 * the library's device memory (32 MiB on every GPU that loads the library,
 * held until the process exits), so log_rows + log_cols must be at most 20:
 * larger claims return BZ_ERR_SCRATCH. Every call shares that array: calls
 * that overlap on the GPU race, so serialise them. Each round copies its
 * message to the host and synchronises the stream (the host transcript draws
 * the next challenge), so the call cannot run while a stream is being
 * captured. The first call on a device (and the first after the device's
 * context was reset) looks up the array's address. */
int bitz_post_gkr_prove_noalloc(const uint64_t *rows_dev, int log_rows, const uint64_t *cols_dev,
                                int log_cols, const uint64_t target[2], const uint64_t *packed_dev,
                                uint32_t security_bits, bitz_transcript *t, void *stream,
                                uint64_t *point_out, uint64_t value_out[2]);

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

/* ----------------------------------------------------- end-to-end prover
 * A prepared statement of one of the four SHA-256 circuits.
 * Replaces CircuitProofSystem::new(statement, SecurityLevel)
 * (tooling/cli/src/end_to_end.rs:161-197) with the statement of
 * tooling/cli/src/circuits.rs:58-210: circuit_kind 0 sha256-compression
 * (768 input bits), 1 sha256-chain (512 n), 2 sha256-block-aligned (512 k),
 * 3 sha256-2kb (16384); input_bits and the 256 output_bits one byte (0/1)
 * per bit in the statement's order. security_bits is the PCS profile (100 or
 * 128). The circuit's structure is built once per (kind, size) and cached. */
typedef struct bitz_system bitz_system;
int bitz_system_new(int circuit_kind, const uint8_t *input_bits, size_t n_inputs,
                    const uint8_t *output_bits, uint32_t security_bits, bitz_system **out);
void bitz_system_free(bitz_system *sys);
/* CircuitProofSystem::stats (end_to_end.rs:199-212): [0] constraints, [1]
 * assignment entries, [2] committed bits, [3] padded committed bits, [4]
 * prime bits, [5] PCS security, [6] claim column bits s, [7] compressions. */
int bitz_system_stats(const bitz_system *sys, uint64_t out[8]);
/* witness + commit + prove (end_to_end.rs:215-336; the stages
 * benchmark::run times, tooling/cli/src/benchmark.rs:28-79). Returns the
 * proof bytes root || Spartan section || bitzPCS wire container
 * (crates/host/src/wire_proof.rs:88-104) in a buffer freed with bitz_free,
 * and the times in milliseconds: witness, commit, prove (host clock) and the
 * CUDA-event span of the whole proof on the prover's stream.
 * BZ_ERR_UNSATISFIED when the statement is false (Error::Unsatisfied).
 * The statement is copied from host memory on every call. */
int bitz_system_prove(bitz_system *sys, uint8_t **proof, size_t *proof_len, double times_ms[4]);
/* As bitz_system_prove; with restage = 0 the statement staged on the device
 * when the system was created is reused instead of copied again. */
int bitz_system_prove_ex(bitz_system *sys, int restage, uint8_t **proof, size_t *proof_len,
                         double times_ms[4]);
void bitz_free(void *p);

/* The same proof as three calls, as the reference's API has it:
 * CircuitProofSystem::witness (end_to_end.rs:215-243), commit (:248-255) and
 * prove, which consumes both (:260-336). The witness and its commitment stay
 * in device memory between the calls, on a prover lane held from bitz_witness
 * until bitz_prove (the process's default lane when free, else a pooled one).
 * A system holds at most one staged proof at a time (BZ_ERR_ARGUMENT
 * otherwise), and bitz_system_prove on it waits for none: it refuses while
 * one is staged. Handles must be used on the thread's current device and
 * freed (or consumed) before their system. */
typedef struct bitz_witness_handle bitz_witness_handle;
typedef struct bitz_committed_witness bitz_committed_witness;
/* input_bits: the witness inputs, one byte (0/1) per bit, as many as the
 * statement's ("wrong witness input length" otherwise, Error::Input);
 * BZ_ERR_UNSATISFIED when they do not satisfy the statement. */
int bitz_witness(bitz_system *sys, const uint8_t *input_bits, size_t n_inputs,
                 bitz_witness_handle **out);
int bitz_commit(bitz_system *sys, const bitz_witness_handle *wit, bitz_committed_witness **out);
/* Consumes wit and com on every return. The proof bytes are those of
 * bitz_system_prove for the same statement, freed with bitz_free. */
int bitz_prove(bitz_system *sys, bitz_witness_handle *wit, bitz_committed_witness *com,
               uint8_t **proof, size_t *proof_len);
/* CircuitProofSystem::verify (end_to_end.rs:339-377) on proof bytes as
 * bitz_system_prove returns them, replayed by this library's own verifier
 * (the bulk steps on the device). BZ_OK: accepted. BZ_ERR_MALFORMED: the
 * bytes do not parse (the wire container's errors,
 * crates/host/src/wire_proof.rs:40-60, named in bitz_last_error).
 * BZ_ERR_VERIFY: a check failed (named in bitz_last_error). Hostile bytes
 * never crash it. */
int bitz_verify(bitz_system *sys, const uint8_t *proof, size_t proof_len);
/* WireProof::from_bytes (crates/host/src/wire_proof.rs:109-140): strict
 * decoding of a bitzPCS container (header, then exactly the declared narg and
 * hint bytes). out: narg offset, narg length, hint offset, hint length.
 * Needs no GPU. */
int bitz_wire_decode(const uint8_t *bytes, size_t len, uint64_t out[4]);
/* Diagnostic (the reference hashes with the blake3 crate, Cargo.lock:239):
 * this library's host BLAKE3, the one its transcript grinding, Merkle checks
 * and weight digest use; derive-key mode when derive_key_context is non-null
 * (crates/pcs/src/opening.rs:354-365), else hash mode. Needs no GPU. */
int bitz_blake3(const char *derive_key_context, const uint8_t *in, size_t len, uint8_t out[32]);
/* Drop a staged proof without proving; freeing either handle ends it. */
void bitz_witness_free(bitz_witness_handle *wit);
void bitz_committed_witness_free(bitz_committed_witness *com);
/* Diagnostic (no reference counterpart): kernel launches issued by this
 * library since the process started. */
unsigned long long bitz_launch_count(void);
/* Diagnostic (no reference counterpart): 1 when kernels that wait for the
 * host thread (resident and queued sumcheck rounds) are in use, 0 when every
 * round is its own launch. BITZ_RESIDENT_ROUNDS=0/1 forces the mode; unset,
 * it is off when a CUDA injection tool announces itself
 * (CUDA_INJECTION64_PATH) or when the first prover lane found that the host
 * cannot reach a running kernel (a kernel profiler holds the host at every
 * launch). Proof bytes are the same in both modes. Needs no GPU (before the
 * first lane exists it reports the environment's answer). */
int bitz_resident_rounds(void);
/* Diagnostic (no reference counterpart): on the default lane since the
 * process started, out[0] the nanoseconds the host spent waiting for round
 * results (device work and the PCIe round trip) and out[1] the number of
 * such waits. The rest of a proof's host time is the host's own transcript
 * work. */
int bitz_round_wait_stats(unsigned long long out[2]);
/* Diagnostic (no reference counterpart): the process's device gate since it
 * started. A lane whose kernels may wait for its host thread holds the gate
 * as a resident stretch; a device or pinned allocation (a lane's scratch
 * growing, a new circuit shape) waits until no stretch is held and holds new
 * ones back meanwhile. out[0] allocation stretches, out[1] nanoseconds they
 * waited, out[2] resident stretches, out[3] nanoseconds they waited. */
int bitz_gate_stats(unsigned long long out[4]);
/* Diagnostic (no reference counterpart): the last proof's packed witness f,
 * packed h = M (1 || f) and the exact products (A h, B h, C h per row). */
int bitz_system_witness(bitz_system *sys, uint32_t *f_words, size_t f_cap, uint32_t *h_words,
                        size_t h_cap, int64_t *products, size_t prod_cap);

/* Diagnostic (no reference counterpart): the structural setup of a circuit
 * size, as ConstraintGenerator and MTransposeGenerator build it
 * (crates/circuit/src/constraints.rs:678-880,
 * crates/circuit/src/matrix_transpose.rs:475-560). sizes: [0] f bits, [1] h
 * entries, [2] rows, [3] M nonzeros, [4] C nonzeros without the statement's
 * bit constants, [5] compressions, [6] claim column bits, [7] committed m.
 * The array outputs are filled when non-null. Needs no GPU. */
int bitz_circuit_layout(int circuit_kind, size_t n_inputs, uint64_t sizes[8],
                        uint8_t map_digest[32], uint32_t *m_off, uint32_t *m_pos,
                        uint32_t *c_off, uint32_t *c_col, int64_t *c_coef);
/* Diagnostic (no reference counterpart): the statement's integer-matrix
 * digest (crates/spartan/src/matrix.rs:562-661, SHA-256 over M, A, B and C
 * with the bit constraints' expected values) as CircuitProofSystem::new
 * absorbs it. Needs no GPU. */
int bitz_statement_digest(int circuit_kind, const uint8_t *input_bits, size_t n_inputs,
                          const uint8_t *output_bits, uint8_t digest[32]);

/* ------------------------------------------------------ batch and serving
 * No reference counterpart: the reference proves one statement per call
 * (CircuitProofSystem::prove, end_to_end.rs:260-336, on a Rayon pool the
 * caller installs, cmd/circuit_e2e.rs:50-56). These run many independent
 * proofs at once on prover lanes: a lane is one CUDA stream, one host
 * thread and its own round mailbox and scratch, so the rounds of different
 * proofs overlap on the device while each proof's Fiat-Shamir transcript
 * advances on its own thread. Every proof's bytes are the same as the
 * single-proof call's for the same statement. */

/* Proves systems[0..n) on `lanes` lanes (1..64), driven by one host thread
 * per lane up to the host's hardware threads (BITZ_LANE_THREADS sets the
 * cap); past it, lanes share threads as cooperative fibers that switch
 * wherever a lane waits for the device. proofs[i] (freed with
 * bitz_free) and proof_lens[i] receive each proof; latency_ms[i] (may be
 * NULL) that proof's own duration, from its start on a lane to its bytes. The
 * lanes take the statements largest first (a lane's scratch then grows at
 * most once per call); results come back in the callers' order. Returns
 * the first failure's status after every proof has finished; failed entries
 * get a NULL proof. The systems must be distinct. */
int bitz_batch_prove(bitz_system *const *systems, size_t n, int lanes, uint8_t **proofs,
                     size_t *proof_lens, double *latency_ms);

/* A prove server: `lanes` lanes take requests from a FIFO queue as they
 * free up (continuous batching). A request is admitted when a lane is free
 * and its padded-witness device footprint fits in hbm_budget_bytes beside
 * the requests in flight (one request is always admitted when none is in
 * flight). Host threads beside the lanes (half the host's hardware threads,
 * at least two) prepare each request's statement (CircuitProofSystem::new:
 * the cached circuit shape and the statement's matrix digest) in submission
 * order; the lanes prove prepared requests, oldest first. */
typedef struct bitz_server bitz_server;
int bitz_server_start(int lanes, uint64_t hbm_budget_bytes, uint32_t security_bits,
                      bitz_server **out);
/* Queues one statement (arguments as bitz_system_new); returns a ticket. */
int bitz_server_submit(bitz_server *srv, int circuit_kind, const uint8_t *input_bits,
                       size_t n_inputs, const uint8_t *output_bits, uint64_t *ticket);
/* Waits up to wait_ms for the ticket's proof. BZ_OK: proof (freed with
 * bitz_free), its length and the submit-to-proof latency are returned and the
 * ticket is retired. BZ_PENDING: not finished yet. Any other status: that
 * request failed (the ticket is retired). */
int bitz_server_poll(bitz_server *srv, uint64_t ticket, int wait_ms, uint8_t **proof,
                     size_t *proof_len, double *latency_ms);
/* Counters: [0] submitted, [1] finished, [2] in flight, [3] queued,
 * [4] bytes admitted in flight, [5] peak requests in flight. */
int bitz_server_stats(bitz_server *srv, uint64_t out[6]);
/* Finishes the requests already admitted, drops the queued ones, joins the
 * lanes and frees the server. */
int bitz_server_stop(bitz_server *srv);

/* --------------------------------------------------------- measurement aids
 * No reference counterpart. */
/* Times every launch of the probed kernels with CUDA events on their stream
 * and counts each launch's algorithmic work. spec: NULL or "" turns the
 * probe off, "*" probes every instrumented launch site, else a comma-separated
 * list of kernel names; enabling resets the totals. While the probe is on,
 * every sumcheck round is its own launch (as under a kernel profiler).
 * Instrumented: gkr_top_sums, gkr_round, gkr_bind_sums, pg_round,
 * k_outer_round, k_inner_round, k_fp_finalize. */
int bitz_probe_kernel(const char *spec);
/* One kernel's totals since the probe was enabled: out[0] milliseconds,
 * out[1] algorithmic bytes, and its GF(2^128) products: out[2] reduced
 * general products, out[3] unreduced (wide) general products, out[4] products
 * by the round's challenge through its window table (none are counted for the
 * prime-field kernels); *launches the launch count. */
int bitz_probe_read(const char *kernel, double out[5], unsigned long long *launches);
/* The probed kernels that launched, comma-separated, into out (truncated to
 * cap - 1 characters); returns the full length. */
size_t bitz_probe_kernels(char *out, size_t cap);
/* Self-test of the fibers that let one host thread drive several prover
 * lanes (no GPU): `threads` threads each run `fibers` fibers that yield
 * `yields` times, throw and catch on their own stacks and keep their own
 * gate counters. BZ_OK when every check holds; *checksum identifies the
 * interleaving (the same for the same arguments). */
int bitz_diag_fibers(int threads, int fibers, int yields, unsigned long long *checksum);
/* Overwrites a 256 MiB device buffer and waits, evicting the L2 cache. */
int bitz_l2_flush(void);
/* Mean microseconds per host<->device round on the default lane: mode 0
 * launches one kernel per round that posts to the mailbox; mode 1 runs one
 * resident kernel that waits (bounded) for each host word and posts it back. */
int bitz_diag_round_trip(int mode, int rounds, double *us_per_round);
/* The GPU's GF(2^128) product throughput (products per second over every SM,
 * four independent chains per thread): kind 0 reduced general products, 1
 * unreduced ones, 2 products by one factor through its window table in
 * shared memory. The ceiling that the integer-bound kernels are held to. */
int bitz_diag_gf_peak(int kind, double *products_per_s);

#ifdef __cplusplus
}
#endif
#endif
