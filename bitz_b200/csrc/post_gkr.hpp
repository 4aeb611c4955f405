// Host interface of the post-GKR sumcheck kernels.
#pragma once
#include <cuda_runtime.h>

#include <string>

#include "device.cuh"
#include "status.hpp"
#include "transcript.hpp"

namespace bz {

struct PostGkrArgs {
  const f128 *rows;  // device, 2^log_rows weights
  int log_rows;      // t >= 7
  const f128 *cols;  // device, 2^log_cols weights
  int log_cols;      // s
  const f128 *packed;  // device, 2^(t+s-7) committed words
  f128 target;
  uint32_t grind_bits;
};

// Device scratch, reusable across proofs: four tables of `capacity` entries,
// a round-accumulator array and a pinned host staging buffer.
struct PostGkrScratch {
  size_t capacity = 0;
  f128 *w0 = nullptr, *v0 = nullptr, *w1 = nullptr, *v1 = nullptr;
  unsigned long long *acc = nullptr;  // 8 words per round, 64 rounds
  uint64_t *host = nullptr;           // pinned, 8 words
  f128 claim_seen{0, 0};              // the weighted sum found when a claim fails
  RoundChannel *channel = nullptr;    // mailbox for round results; null: copy + sync
  RoundCtl *ctl = nullptr;            // round controls for queued rounds; null: none
  // blocks of the cooperative kernel that runs the rounds above the tail
  // resident (128 for a lane proving alone, fewer for a pooled lane); 0: queued
  // launches
  int mid_blocks = 0;
};

// Folds k = km .. t0-1 of a quadratic sumcheck over <W, V> (n_in entries
// each) in one resident cooperative launch of nb blocks: fold
// k takes its challenge from downbox publication d0 + k (relayed through
// ctl[k], which must start zeroed), XORs the next message into
// acc + 8 (k + acc_off) and posts it as publication p0 + k + 1 (the last fold
// only with emit_last); the folded tables end in (w_out, v_out).
// pg_mid_start gives the first fold it can take (t0 when none).
// nb is the grid (0: none fits).
int pg_mid_start(size_t n1, int t0, int nb);
// All `rounds` folds of n-entry tables fit launch_pg_mid with nb blocks (the
// last without a message).
bool pg_mid_fits_folds(size_t n, int rounds, int nb);
void launch_pg_mid(const f128 *w_in, const f128 *v_in, size_t n_in, int km, int t0,
                   int emit_last, int acc_off, f128 *w_out, f128 *v_out, unsigned long long *acc,
                   RoundChannel *ch, unsigned long long p0, unsigned long long d0, RoundCtl *ctl,
                   int nb, cudaStream_t s);
// The grid of a lane's resident post-GKR and Ligerito folds
// (PostGkrScratch::mid_blocks): 128 for a lane proving alone; for a pooled
// lane none, or 32 with BITZ_POOL_MID=1 (as for the GKR middle rounds).
int pg_mid_blocks(bool alone);

// The quadratic sumcheck round of <W, V> (shared with the Ligerito folds):
// quad_sums accumulates (a0, a2) over the pairs as they are; quad_fold folds
// both tables at r and, with emit, accumulates the next round's sums.
void quad_sums(const f128 *w, const f128 *v, size_t n, unsigned long long *acc, Publish pub,
               cudaStream_t s);
void quad_fold(const f128 *w, const f128 *v, f128 r, f128 *w2, f128 *v2, size_t n, int emit,
               unsigned long long *acc, Publish pub, cudaStream_t s);

// Runs the whole reduction: writes t+s challenges to point_out and the
// closing evaluation to value_out, appending every message to `ts`.
int post_gkr_prove(const PostGkrArgs &a, Transcript &ts, PostGkrScratch &sc, cudaStream_t s,
                   f128 *point_out, f128 *value_out);

// The same reduction on fixed file-scope device scratch: allocates nothing.
// Claims up to 2^20 bits; see post_gkr_noalloc.cu for the sharing rules.
int post_gkr_prove_noalloc(const PostGkrArgs &a, Transcript &ts, cudaStream_t s, f128 *point_out,
                           f128 *value_out, std::string &err);

}  // namespace bz
