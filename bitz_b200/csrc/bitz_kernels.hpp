// Host interface of the BitZ opening and PCS kernels.
#pragma once
#include <cuda_runtime.h>

#include "device.cuh"
#include "transcript.hpp"

namespace bz {

constexpr int kMaxRsDim = 40;  // largest additive-FFT dimension (row bits of a codeword)

void fold_columns(const f128 *cols, size_t ncols, const u128 *exps, u128 *folds, cudaStream_t s);
void comb_pow(const f128 *table, const u128 *exps, int n, f128 *out, cudaStream_t s);
// weights[c - 1] = sum over the rows r of column c of u1[r & 127] u2[r >> 7]
// (rows below 2^(7 + log_u2)); column 0 into w0. With `dense` (2^(7 + log_u2)
// entries of scratch) the row table is formed once and the columns gather it.
void mt_transpose(const uint32_t *off, const uint32_t *row, size_t ncols, const f128 *u1,
                  const f128 *u2, f128 *weights, size_t padded, f128 *w0, cudaStream_t s,
                  f128 *dense, int log_u2);
// The non-root chaining value of nchunks (a power of two) whole 1 KiB chunks,
// and the 16 bytes at `extra` (device, may be null) into extra_out. ch: the
// lane's channel (null: a copy and a stream synchronisation).
void blake3_tree_cv(const uint8_t *data, size_t nchunks, const uint32_t key[8], uint32_t flags,
                    uint32_t *scratch, uint32_t cv_out[8], cudaStream_t s, RoundChannel *ch,
                    const f128 *extra, f128 *extra_out);
void ring_claims(const f128 *f, const f128 *suffix, size_t n, unsigned long long *claims,
                 cudaStream_t s);
void packed_basis(const f128 *suffix, size_t n, const f128 *bw, const f128 *eq_ood, f128 coef,
                  f128 *basis, cudaStream_t s);
// y += a * x
void axpy(f128 *y, f128 a, const f128 *x, size_t n, cudaStream_t s);
void dot(const f128 *a, const f128 *b, size_t n, unsigned long long *acc, Publish pub,
         cudaStream_t s);
// Interleaved Reed-Solomon encode of msg (2^log_n entries, 2^k columns) at
// rate 2^-rate into cw, staged through shared memory by TMA copies; err (a
// word the host reads; null: no report) is set when a copy did not land
// within its time limit.
void rs_encode(const f128 *msg, int log_n, int k, int rate, const f128 *wh, f128 *cw,
               unsigned int *err, cudaStream_t s);
void merkle_build(const f128 *cw, size_t rows, int k, uint32_t *nodes, cudaStream_t s);
// A small tree (at most kMerkleBlockMaxRows rows) in one launch that posts
// the root (node 1, 32 bytes) as four mailbox words of publication pub; false
// (nothing launched) when the tree is larger or there is no mailbox.
constexpr size_t kMerkleBlockMaxRows = 4096;
bool merkle_build_posted(const f128 *cw, size_t rows, int k, uint32_t *nodes, Publish pub,
                         cudaStream_t s);
// basis += sum_q scale[q] * tensor(Wh_t(x_q), t < l), x_q = idx[q]; wh is the
// kMaxRsDim x kMaxRsDim subspace table (Wh_t(X^s) at t * kMaxRsDim + s).
void query_basis(const uint64_t *idx, const f128 *wh, const f128 *scale, int nq, int l,
                 f128 *basis, cudaStream_t s);
// Per query (idx[q] < rows): the codeword row and its Merkle siblings, packed
// as width + 2 * depth 16-byte units.
void gather_openings(const f128 *cw, const uint32_t *nodes, size_t rows, int width, int depth,
                     const uint64_t *idx, int nq, f128 *out, cudaStream_t s);

// Host helpers (GF(2^128) on the CPU for the few scalar steps).
f128 gf_inv_host(f128 a);
// wh[t * kMaxRsDim + s] = Wh_t(X^s): the normalised subspace polynomial of
// span(X^0..X^(t-1)) at X^s, for t, s < d.
void subspace_table(int d, f128 *wh);
// The comb table of `base` with 8-bit windows: 16 x 256 entries.
void comb_table(f128 base, f128 *out);
f128 smallest_generator_host();
void eq_table_host(const f128 *r, int n, f128 *out);

}  // namespace bz
