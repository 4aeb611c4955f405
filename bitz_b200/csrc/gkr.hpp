// Host interface of the grand-product GKR kernels.
#pragma once
#include <cuda_runtime.h>

#include "device.cuh"
#include "status.hpp"
#include "transcript.hpp"

namespace bz {

struct GkrScratch {
  size_t capacity = 0;         // leaves the layer tables can hold: 2^(7+s)
  f128 *layer[8] = {nullptr};  // layer j holds 2^(7+s-j) nodes; layer 7 is the output
  f128 *eq = nullptr;          // 2^(6+s-1) entries
  f128 *eq_scratch = nullptr;
  f128 *pair = nullptr;               // 2 entries
  unsigned long long *acc = nullptr;  // 4 words per round
  RoundCtl *ctl = nullptr;            // one per round of a layer
  uint64_t *host = nullptr;           // pinned, 4 words
  RoundChannel *channel = nullptr;    // mailbox for round results; null: copy + sync
  // Columns at or beyond live_cols hold no set bit (the padding of h), so
  // every node of theirs is one in every layer; the kernels skip their
  // products and add their known contribution. 0: every column is live.
  size_t live_cols = 0;
  // Blocks of the cooperative kernel that runs the middle rounds of each
  // layer, resident across them (128 for a lane proving alone, fewer for a
  // pooled lane that shares the GPU); 0: one queued launch per round.
  int mid_blocks = 0;
};

// The grid of a lane's resident middle rounds (GkrScratch::mid_blocks).
int gkr_mid_blocks(bool alone);

// Builds every layer from the packed columns (2^s F128, bit b of column c is
// row b) and the 128 row images. Layer 7 holds the column products.
void gkr_build(const f128 *cols, int s, const f128 *images, GkrScratch &sc, cudaStream_t st);

// The seven layer sumchecks from the output point zeta (s coordinates) to the
// leaves: writes 7 + s coordinates and returns the claim on the leaves. The
// layer tables are consumed (bound in place).
f128 gkr_prove(int s, const f128 *zeta, uint32_t grind_bits, Transcript &ts, GkrScratch &sc,
               cudaStream_t st, f128 *point_out);

}  // namespace bz
