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
  bool resident_middle = false;       // rounds above the tail in one resident kernel
};

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
