// The BitZ virtual opening's device stages and the PCS kernels.
//
// - Column fold (crates/common/src/fold.rs:29-63) and the comb exponentiation
//   of the row images (fold.rs:72-104, crates/field/src/gf128/pow.rs:137-199).
// - M^T gather (crates/circuit/src/matrix_transpose.rs:377-416).
// - BLAKE3 derive-key digest of the inner-product weights
//   (crates/pcs/src/opening.rs:337-368) as a chunk-parallel tree.
// - Ring switch (crates/pcs/src/mle.rs:63-123), OOD evaluation and basis
//   (crates/pcs/src/ood.rs:44-95).
// - Interleaved Reed-Solomon encoding by the additive FFT, BLAKE3 Merkle tree
//   and the Ligerito query glue (the PCS restatement; flock-core is not in
//   the reference tree).
#include "bitz_kernels.hpp"
#include "device.cuh"
#include "hash.cuh"
#include "context.hpp"
#include "tma.cuh"

#include <cudaTypedefs.h>

#include <algorithm>

namespace bz {

// --------------------------------------------------------------- the fold

__global__ void k_fold_columns(const f128 *__restrict__ cols, size_t ncols,
                               const u128 *__restrict__ exps, u128 *__restrict__ folds) {
  __shared__ u128 e[128];
  for (int i = threadIdx.x; i < 128; i += blockDim.x) e[i] = exps[i];
  __syncthreads();
  for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < ncols;
       c += (size_t)gridDim.x * blockDim.x) {
    f128 w = ld(cols + c);
    u128 s = 0;
    uint64_t lo = w.lo, hi = w.hi;
    while (lo) {
      s += e[__ffsll((long long)lo) - 1];
      lo &= lo - 1;
    }
    while (hi) {
      s += e[64 + __ffsll((long long)hi) - 1];
      hi &= hi - 1;
    }
    folds[c] = s;
  }
}

// comb.pow(e): one multiply per non-zero 8-bit window (pow.rs:177-199)
__global__ void k_comb_pow(const f128 *__restrict__ table, const u128 *__restrict__ exps, int n,
                           f128 *__restrict__ out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  u128 e = exps[i];
  f128 acc = mk(1, 0);
  for (int w = 0; w < 16 && e; w++, e >>= 8) {
    int d = (int)(e & 0xff);
    if (d) acc = gmul(acc, ld(table + w * 256 + d));
  }
  st(out + i, acc);
}

void fold_columns(const f128 *cols, size_t ncols, const u128 *exps, u128 *folds, cudaStream_t s) {
  k_fold_columns<<<grid_for(ncols), kThreads, 0, s>>>(cols, ncols, exps, folds);
  BZ_LAUNCH_CHECK();
}

void comb_pow(const f128 *table, const u128 *exps, int n, f128 *out, cudaStream_t s) {
  k_comb_pow<<<(n + 127) / 128, 128, 0, s>>>(table, exps, n, out);
  BZ_LAUNCH_CHECK();
}

// -------------------------------------------------------------------- M^T

// w[c] = sum over the rows of column c of u1[row & 127] * u2[row >> 7]; one
// reduction per column. Column 0 (the constant) goes to w0, the others to
// weights[c - 1]; weights beyond the last column are zero.
__global__ void k_mt_transpose(const uint32_t *__restrict__ off, const uint32_t *__restrict__ row,
                               size_t ncols, const f128 *__restrict__ u1,
                               const f128 *__restrict__ u2, f128 *__restrict__ weights,
                               size_t padded, f128 *w0) {
  __shared__ f128 su1[128];
  for (int i = threadIdx.x; i < 128; i += blockDim.x) su1[i] = u1[i];
  __syncthreads();
  for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c <= padded;
       c += (size_t)gridDim.x * blockDim.x) {
    if (c == 0) continue;  // the constant column: k_mt_col0
    f128 v = mk(0, 0);
    if (c < ncols) {
      wide acc = wzero();
      for (uint32_t e = off[c]; e < off[c + 1]; e++) {
        uint32_t r = row[e];
        wacc(acc, gmul_wide(su1[r & 127], ld(u2 + (r >> 7))));
      }
      v = greduce(acc);
    }
    st(weights + (c - 1), v);
  }
}

// The constant column holds one entry per lift with a constant term (hundreds
// where the others hold under ten), so one block shares it out.
__global__ void k_mt_col0(const uint32_t *__restrict__ off, const uint32_t *__restrict__ row,
                          const f128 *__restrict__ u1, const f128 *__restrict__ u2, f128 *w0) {
  wide acc = wzero();
  for (uint32_t e = off[0] + threadIdx.x; e < off[1]; e += blockDim.x) {
    uint32_t r = row[e];
    wacc(acc, gmul_wide(ld(u1 + (r & 127)), ld(u2 + (r >> 7))));
  }
  f128 v = greduce(acc);
  uint64_t w[2] = {v.lo, v.hi};
  block_xor_reduce<2>(w);
  if (threadIdx.x == 0) st(w0, mk(w[0], w[1]));
}

// The dense eq table of the rows, dense[lo << log_u2 | hi] = u1[lo] * u2[hi]
// (row r = hi * 128 + lo): block (lo, part) takes a slice of hi through
// u1[lo]'s window table, writing along hi.
constexpr int kMtParts = 2;
__global__ void k_mt_dense(const f128 *__restrict__ u1, const f128 *__restrict__ u2, int log_u2,
                           f128 *__restrict__ dense) {
  __shared__ MulTable T;
  const int lo = blockIdx.x / kMtParts, part = blockIdx.x % kMtParts;
  mul_table_build(T, ld(u1 + lo));
  const size_t per = ((size_t)1 << log_u2) / kMtParts;
  f128 *out = dense + ((size_t)lo << log_u2);
  for (size_t hi = part * per + threadIdx.x; hi < (part + 1) * per; hi += blockDim.x)
    st(out + hi, mul_table(T, ld(u2 + hi)));
}

// k_mt_transpose over the dense table: each column XORs its rows' entries.
__global__ void k_mt_gather(const uint32_t *__restrict__ off, const uint32_t *__restrict__ row,
                            size_t ncols, const f128 *__restrict__ dense, int log_u2,
                            f128 *__restrict__ weights, size_t padded) {
  for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c <= padded;
       c += (size_t)gridDim.x * blockDim.x) {
    if (c == 0) continue;  // the constant column: k_mt_col0
    f128 v = mk(0, 0);
    if (c < ncols)
      for (uint32_t e = off[c]; e < off[c + 1]; e++) {
        const uint32_t r = row[e];
        v = gadd(v, ld(dense + (((size_t)(r & 127) << log_u2) | (r >> 7))));
      }
    st(weights + (c - 1), v);
  }
}

void mt_transpose(const uint32_t *off, const uint32_t *row, size_t ncols, const f128 *u1,
                  const f128 *u2, f128 *weights, size_t padded, f128 *w0, cudaStream_t s,
                  f128 *dense, int log_u2) {
  if (dense && log_u2 >= 8) {
    k_mt_dense<<<128 * kMtParts, kThreads, 0, s>>>(u1, u2, log_u2, dense);
    BZ_LAUNCH_CHECK();
    k_mt_gather<<<grid_for(padded + 1), kThreads, 0, s>>>(off, row, ncols, dense, log_u2, weights,
                                                          padded);
    BZ_LAUNCH_CHECK();
  } else {
    k_mt_transpose<<<grid_for(padded + 1), kThreads, 0, s>>>(off, row, ncols, u1, u2, weights,
                                                             padded, w0);
    BZ_LAUNCH_CHECK();
  }
  k_mt_col0<<<1, kThreads, 0, s>>>(off, row, u1, u2, w0);
  BZ_LAUNCH_CHECK();
}

// ------------------------------------------------------------ BLAKE3 tree

struct Key8 {
  uint32_t k[8];
};

// Chaining value of every full 1 KiB chunk of `data` (16 blocks each).
__global__ void k_b3_chunks(const uint8_t *__restrict__ data, size_t nchunks, Key8 key,
                            uint32_t flags, uint32_t *__restrict__ cvs) {
  for (size_t ch = blockIdx.x * (size_t)blockDim.x + threadIdx.x; ch < nchunks;
       ch += (size_t)gridDim.x * blockDim.x) {
    uint32_t cv[8];
    for (int i = 0; i < 8; i++) cv[i] = key.k[i];
    const uint32_t *p = reinterpret_cast<const uint32_t *>(data + ch * 1024);
    for (int b = 0; b < 16; b++) {
      uint32_t m[16];
      for (int i = 0; i < 16; i++) m[i] = p[16 * b + i];
      uint32_t fl = flags | (b == 0 ? B3_CHUNK_START : 0) | (b == 15 ? B3_CHUNK_END : 0);
      b3_compress(cv, m, ch, 64, fl, cv);
    }
    for (int i = 0; i < 8; i++) cvs[8 * ch + i] = cv[i];
  }
}

__global__ void k_b3_parents(const uint32_t *__restrict__ in, size_t nout, Key8 key,
                             uint32_t flags, uint32_t *__restrict__ out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nout;
       i += (size_t)gridDim.x * blockDim.x) {
    uint32_t m[16], cv[8];
    for (int j = 0; j < 16; j++) m[j] = in[16 * i + j];
    b3_compress(key.k, m, 0, 64, flags | B3_PARENT, cv);
    for (int j = 0; j < 8; j++) out[8 * i + j] = cv[j];
  }
}

// The last parent levels of a tree in one block: n chaining values (a power
// of two, at most kB3BlockMax) reduced to one in shared memory, posted as
// mailbox words 0-3, with the 16 bytes at `extra` (when given) as words 4-5.
constexpr int kB3BlockThreads = 512;
constexpr size_t kB3BlockMax = 1024;  // 2 x kB3BlockThreads: one compression per thread per level
__global__ void __launch_bounds__(kB3BlockThreads) k_b3_top(const uint32_t *__restrict__ in,
                                                            size_t n, Key8 key, uint32_t flags,
                                                            const f128 *extra, Publish pub) {
  __shared__ uint32_t cv[kB3BlockMax * 8];
  for (size_t i = threadIdx.x; i < 8 * n; i += blockDim.x) cv[i] = in[i];
  __syncthreads();
  for (size_t m = n / 2; m >= 1; m /= 2) {
    uint32_t out[8];
    const bool mine = threadIdx.x < m;
    if (mine) {
      uint32_t msg[16];
      for (int j = 0; j < 16; j++) msg[j] = cv[16 * threadIdx.x + j];
      b3_compress(key.k, msg, 0, 64, flags | B3_PARENT, out);
    }
    __syncthreads();  // every read of this level before any write
    if (mine)
      for (int j = 0; j < 8; j++) cv[8 * threadIdx.x + j] = out[j];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    for (int w = 0; w < 4; w++)
      mailbox_post(pub.mailbox, pub.seq, w,
                   (unsigned long long)cv[2 * w] | ((unsigned long long)cv[2 * w + 1] << 32));
    if (extra) {
      const f128 e = ld(extra);
      mailbox_post(pub.mailbox, pub.seq, 4, e.lo);
      mailbox_post(pub.mailbox, pub.seq, 5, e.hi);
    }
  }
}

// The non-root chaining value of a power-of-two number of whole chunks. With
// a channel, the last levels run in one block that posts the value (and the
// 16 bytes at `extra`, returned in extra_out) through the lane's mailbox
// instead of a copy and a stream synchronisation.
void blake3_tree_cv(const uint8_t *data, size_t nchunks, const uint32_t key[8], uint32_t flags,
                    uint32_t *scratch, uint32_t cv_out[8], cudaStream_t s, RoundChannel *ch,
                    const f128 *extra, f128 *extra_out) {
  Key8 k;
  for (int i = 0; i < 8; i++) k.k[i] = key[i];
  uint32_t *a = scratch, *b = scratch + 8 * nchunks;
  k_b3_chunks<<<grid_for(nchunks), kThreads, 0, s>>>(data, nchunks, k, flags, a);
  BZ_LAUNCH_CHECK();
  size_t n = nchunks;
  while (n > 1 && (!ch || n > kB3BlockMax)) {
    k_b3_parents<<<grid_for(n / 2), kThreads, 0, s>>>(a, n / 2, k, flags, b);
    BZ_LAUNCH_CHECK();
    std::swap(a, b);
    n /= 2;
  }
  if (ch) {
    k_b3_top<<<1, kB3BlockThreads, 0, s>>>(a, n, k, flags, extra, ch->arm());
    BZ_LAUNCH_CHECK();
    uint64_t w[6];
    ch->wait(s, w, extra ? 6 : 4);
    memcpy(cv_out, w, 32);
    if (extra) *extra_out = mk(w[4], w[5]);
    return;
  }
  BZ_CUDA(cudaMemcpyAsync(cv_out, a, 32, cudaMemcpyDeviceToHost, s));
  if (extra) BZ_CUDA(cudaMemcpyAsync(extra_out, extra, 16, cudaMemcpyDeviceToHost, s));
  BZ_CUDA(stream_wait(s));
}

// ----------------------------------------------------------- ring switch

// claims[v] = sum over y with bit v of f[y] set of suffix[y]; block b covers
// 64 consecutive y, thread v one bit position.
__global__ void k_ring_claims(const f128 *__restrict__ f, const f128 *__restrict__ suffix,
                              size_t n, unsigned long long *claims) {
  int v = threadIdx.x;
  uint64_t lo = 0, hi = 0;
  for (size_t y0 = blockIdx.x * (size_t)64; y0 < n; y0 += (size_t)gridDim.x * 64) {
    size_t y1 = y0 + 64 < n ? y0 + 64 : n;
    for (size_t y = y0; y < y1; y++) {
      f128 w = ld(f + y);
      if (bit128(w, v)) {
        f128 e = ld(suffix + y);
        lo ^= e.lo;
        hi ^= e.hi;
      }
    }
  }
  if (lo) atomicXor(claims + 2 * v, (unsigned long long)lo);
  if (hi) atomicXor(claims + 2 * v + 1, (unsigned long long)hi);
}

// B(y) = sum over u with bit u of suffix[y] set of bw[u] (the packed basis of
// the batched ring-switch claim), plus coef * eq_ood[y] when eq_ood is given.
__global__ void k_packed_basis(const f128 *__restrict__ suffix, size_t n,
                               const f128 *__restrict__ bw, const f128 *__restrict__ eq_ood,
                               f128 coef, f128 *__restrict__ basis) {
  __shared__ f128 w[128];
  for (int i = threadIdx.x; i < 128; i += blockDim.x) w[i] = bw[i];
  __syncthreads();
  for (size_t y = blockIdx.x * (size_t)blockDim.x + threadIdx.x; y < n;
       y += (size_t)gridDim.x * blockDim.x) {
    f128 e = ld(suffix + y);
    f128 acc = mk(0, 0);
    uint64_t lo = e.lo, hi = e.hi;
    while (lo) {
      acc = gadd(acc, w[__ffsll((long long)lo) - 1]);
      lo &= lo - 1;
    }
    while (hi) {
      acc = gadd(acc, w[64 + __ffsll((long long)hi) - 1]);
      hi &= hi - 1;
    }
    if (eq_ood) acc = gadd(acc, gmul(coef, ld(eq_ood + y)));
    st(basis + y, acc);
  }
}

// sum_y a[y] * b[y], XOR-reduced into acc[0..2).
__global__ void k_dot(const f128 *__restrict__ a, const f128 *__restrict__ b, size_t n,
                      unsigned long long *acc, Publish pub) {
  wide s = wzero();
  for (size_t y = blockIdx.x * (size_t)blockDim.x + threadIdx.x; y < n;
       y += (size_t)gridDim.x * blockDim.x)
    wacc(s, gmul_wide(ld(a + y), ld(b + y)));
  f128 r = greduce(s);
  uint64_t v[2] = {r.lo, r.hi};
  block_xor_publish<2>(v, acc, pub);
}

__global__ void k_axpy(f128 *__restrict__ y, f128 a, const f128 *__restrict__ x, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    st(y + i, gadd(ld(y + i), gmul(a, ld(x + i))));
}

void axpy(f128 *y, f128 a, const f128 *x, size_t n, cudaStream_t s) {
  k_axpy<<<grid_for(n), kThreads, 0, s>>>(y, a, x, n);
  BZ_LAUNCH_CHECK();
}

void ring_claims(const f128 *f, const f128 *suffix, size_t n, unsigned long long *claims,
                 cudaStream_t s) {
  int blocks = (int)((n + 63) / 64);
  if (blocks > kSMs * 4) blocks = kSMs * 4;
  k_ring_claims<<<blocks, 128, 0, s>>>(f, suffix, n, claims);
  BZ_LAUNCH_CHECK();
}

void packed_basis(const f128 *suffix, size_t n, const f128 *bw, const f128 *eq_ood, f128 coef,
                  f128 *basis, cudaStream_t s) {
  k_packed_basis<<<grid_for(n), kThreads, 0, s>>>(suffix, n, bw, eq_ood, coef, basis);
  BZ_LAUNCH_CHECK();
}

void dot(const f128 *a, const f128 *b, size_t n, unsigned long long *acc, Publish pub,
         cudaStream_t s) {
  k_dot<<<grid_for(n), kThreads, 0, s>>>(a, b, n, acc, pub);
  BZ_LAUNCH_CHECK();
}

// ----------------------------------------------------- Reed-Solomon encode
//
// The codeword is 2^d rows of 2^k columns (row-major, 16-byte entries); the
// message is its first 2^l rows, repeated across the 2^(d-l) row blocks
// before the additive FFT's levels t = l-1 .. 0 run. Level t takes rows q
// and q + 2^t of each 2^(t+1)-row block based at q0 to
// (u + lam w, u + (lam + 1) w), lam = Wh_t(x_q0), the sum of the basis
// table's wh[t][sb] = Wh_t(X^sb) over the set bits sb > t of the row index.

// lam of level t for a row whose bits above t are those of `row`; wt is
// level t's row of the basis table (wt[sb] = Wh_t(X^sb)).
__device__ __forceinline__ f128 rs_lambda(const f128 *wt, int t, int d, size_t row) {
  f128 lam = mk(0, 0);
  for (int sb = t + 1; sb < d; sb++)
    if ((row >> sb) & 1) lam = gadd(lam, wt[sb]);
  return lam;
}

// Levels [s, s + r) of the FFT, top down, on a shared-memory tile of 2^r rows
// (row y of the tile is codeword row ((z0 + y) << s) | lo) by C = 2^cshift
// columns; whs holds the basis table's rows s .. s + r - 1 (kMaxRsDim each).
__device__ __forceinline__ void rs_tile_levels(f128 *tile, int s, int r, int cshift, int d,
                                               size_t z0, size_t lo, const f128 *whs) {
  const int pairs = 1 << (r - 1 + cshift);
  const int cmask = (1 << cshift) - 1;
  for (int t = s + r - 1; t >= s; t--) {
    const int ht = t - s;  // the level's half-distance in tile rows: 2^ht
    for (int q = threadIdx.x; q < pairs; q += blockDim.x) {
      const int c = q & cmask, p = q >> cshift;
      const int yu = ((p >> ht) << (ht + 1)) | (p & ((1 << ht) - 1));
      const int yw = yu + (1 << ht);
      const f128 lam = rs_lambda(whs + (t - s) * kMaxRsDim, t, d, ((z0 + (size_t)yu) << s) | lo);
      const f128 u = tile[(yu << cshift) + c], w = tile[(yw << cshift) + c];
      const f128 u2 = gadd(u, gmul(lam, w));
      tile[(yu << cshift) + c] = u2;
      tile[(yw << cshift) + c] = gadd(u2, w);
    }
    __syncthreads();
  }
}

// One pass of the FFT over levels [s, s + r), one tile per block: the tile
// (the 2^r rows whose row bits [s, s + r) vary, the others fixed, by C
// columns) arrives by one TMA tensor copy, its r levels run in shared memory
// and it leaves by one TMA tensor copy. Tensor maps see a codeword of 2^rows
// rows as (u64 words of a row, row bits below s, row bits from s up); a box
// is (2C, 1, 2^r). The first pass (`first`) reads the message (rows = l) and
// writes repetition `rep` of the codeword (its row bits from l up), so the
// spread costs no pass of its own; later passes read and write the codeword.
// A copy that has not landed within its time limit sets *err and the block
// returns.
constexpr int kRsTileEntries = 1024;  // 16 KiB tiles
constexpr int kRsPassLevels = 6;      // levels per pass at most
__global__ void __launch_bounds__(512) k_rs_pass(const __grid_constant__ CUtensorMap src,
                                                 const __grid_constant__ CUtensorMap dst, int d,
                                                 int l, int s, int r, int cshift, int ncc,
                                                 int first, const f128 *__restrict__ wh,
                                                 unsigned int *err) {
  __shared__ __align__(128) f128 tile[kRsTileEntries];
  __shared__ f128 whs[kRsPassLevels * kMaxRsDim];
  __shared__ uint64_t bar;
  const int src_rows = first ? l : d;
  // block -> (column chunk, row bits below s, row bits above s + r, repetition)
  unsigned b = blockIdx.x;
  const int cc = (int)(b % (unsigned)ncc);
  b /= (unsigned)ncc;
  const size_t lo = b & (((size_t)1 << s) - 1);
  b >>= s;
  const size_t nhi = (size_t)1 << (src_rows - s - r);
  const size_t hi = b % nhi;
  const size_t rep = b / nhi;
  const int x = 2 * (cc << cshift);
  const size_t zs = hi << r;                            // tile's first row group, source
  const size_t zd = (first ? rep << (l - s) : 0) + zs;  // and destination
  const uint32_t bytes = (uint32_t)(16u << (r + cshift));
  if (threadIdx.x == 0) {
    mbar_init(&bar);
    mbar_expect(&bar, bytes);
    tensor_load_3d(tile, &src, x, (int)lo, (int)zs, &bar);
  }
  // the pass's rows of the basis table while the tile is in flight
  for (int i = threadIdx.x; i < r * d; i += blockDim.x)
    whs[(i / d) * kMaxRsDim + i % d] = wh[(s + i / d) * kMaxRsDim + i % d];
  __syncthreads();
  if (!mbar_wait(&bar, 0)) {
    if (threadIdx.x == 0) {
      if (err) *reinterpret_cast<volatile unsigned int *>(err) = 1u;
      mbar_wait(&bar, 0);  // the copy may still land: give it one more limit
    }
    return;
  }
  rs_tile_levels(tile, s, r, cshift, d, zd, lo, whs);
  fence_async_shared();
  __syncthreads();
  if (threadIdx.x == 0) {
    tensor_store_3d(&dst, x, (int)lo, (int)zd, tile);
    bulk_store_drain();
  }
}

// The whole encode of a small codeword (at most 2^10 entries) in one block:
// the message arrives by one bulk copy, is repeated across the row blocks in
// shared memory, every level runs in place and the codeword leaves by one
// bulk copy. Larger codewords go through k_rs_pass, whose tiles spread a
// level over 128 or more blocks.
constexpr int kRsBlockThreads = 1024;
constexpr int kRsBlockLog = 10;
constexpr size_t kRsBlockMax = (size_t)1 << kRsBlockLog;  // 16 KiB of shared memory
__global__ void __launch_bounds__(kRsBlockThreads) k_rs_encode_block(const f128 *__restrict__ msg,
                                                                     int k, int l, int d,
                                                                     const f128 *__restrict__ wh,
                                                                     f128 *__restrict__ cw,
                                                                     unsigned int *err) {
  __shared__ __align__(128) f128 sm[kRsBlockMax];
  __shared__ f128 whs[kRsBlockLog * kRsBlockLog];
  __shared__ uint64_t bar;
  const size_t total = (size_t)1 << (d + k);
  const size_t mlen = (size_t)1 << (l + k);
  if (threadIdx.x == 0) {
    mbar_init(&bar);
    mbar_expect(&bar, (uint32_t)(mlen * sizeof(f128)));
    bulk_load(sm, msg, (uint32_t)(mlen * sizeof(f128)), &bar);
  }
  // the basis table's rows t < l, columns sb < d, while the message is in flight
  for (int i = threadIdx.x; i < l * d; i += blockDim.x)
    whs[(i / d) * kRsBlockLog + i % d] = wh[(i / d) * kMaxRsDim + i % d];
  __syncthreads();
  if (!mbar_wait(&bar, 0)) {
    if (threadIdx.x == 0) {
      if (err) *reinterpret_cast<volatile unsigned int *>(err) = 1u;
      mbar_wait(&bar, 0);
    }
    return;
  }
  for (size_t i = mlen + threadIdx.x; i < total; i += blockDim.x) sm[i] = sm[i & (mlen - 1)];
  __syncthreads();
  const size_t cmask = ((size_t)1 << k) - 1;
  for (int t = l - 1; t >= 0; t--) {
    const size_t half = (size_t)1 << t;
    for (size_t i = threadIdx.x; i < total / 2; i += blockDim.x) {
      const size_t c = i & cmask, p = i >> k;
      const size_t base = (p >> t) << (t + 1);
      const size_t j = p & (half - 1);
      const f128 lam = rs_lambda(whs + t * kRsBlockLog, t, d, base);
      const size_t iu = ((base + j) << k) + c, iw = ((base + half + j) << k) + c;
      const f128 u = sm[iu], w = sm[iw];
      const f128 u2 = gadd(u, gmul(lam, w));
      sm[iu] = u2;
      sm[iw] = gadd(u2, w);
    }
    __syncthreads();
  }
  fence_async_shared();
  __syncthreads();
  if (threadIdx.x == 0) {
    bulk_store(cw, sm, (uint32_t)(total * sizeof(f128)));
    bulk_store_drain();
  }
}

namespace {

PFN_cuTensorMapEncodeTiled tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled fn = [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    BZ_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
    if (!p || q != cudaDriverEntryPointSuccess)
      throw CudaError("cuTensorMapEncodeTiled is not available");
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled>(p);
  }();
  return fn;
}

// The 3-D view of a codeword of 2^rows rows x 2^k columns that k_rs_pass
// copies: (2^(k+1) u64 words of a row, 2^s rows below bit s, 2^(rows-s) row
// groups), box (2C, 1, 2^r).
CUtensorMap rows_map(const f128 *base, int rows, int k, int s, int r, int cshift) {
  CUtensorMap m;
  const cuuint64_t row_bytes = (cuuint64_t)16 << k;
  const cuuint64_t dim[3] = {(cuuint64_t)2 << k, (cuuint64_t)1 << s, (cuuint64_t)1 << (rows - s)};
  const cuuint64_t stride[2] = {row_bytes, row_bytes << s};
  const cuuint32_t box[3] = {(cuuint32_t)2 << cshift, 1, (cuuint32_t)1 << r};
  const cuuint32_t estride[3] = {1, 1, 1};
  const CUresult rc = tensor_map_encoder()(
      &m, CU_TENSOR_MAP_DATA_TYPE_UINT64, 3, const_cast<f128 *>(base), dim, stride, box, estride,
      CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
      CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (rc != CUDA_SUCCESS) throw CudaError("cuTensorMapEncodeTiled failed for a codeword view");
  return m;
}

}  // namespace

void rs_encode(const f128 *msg, int log_n, int k, int rate, const f128 *wh, f128 *cw,
               unsigned int *err, cudaStream_t s) {
  const int l = log_n - k, d = l + rate;
  const size_t total = (size_t)1 << (d + k);
  if (total <= kRsBlockMax) {
    k_rs_encode_block<<<1, kRsBlockThreads, 0, s>>>(msg, k, l, d, wh, cw, err);
    BZ_LAUNCH_CHECK();
    return;
  }
  if (l < 1) throw CudaError("rs_encode: a codeword of one message row");
  // the levels split into passes of at most 6, top down, the first from the
  // message; a pass of r levels takes tiles of 2^r rows by C = 2^cshift
  // columns, C as wide as keeps 128 or more tiles (blocks) per pass and a
  // tile within kRsTileEntries (a pass has 2^(d + k - r - cshift) tiles)
  const int npass = (l + kRsPassLevels - 1) / kRsPassLevels;
  int top = l;  // levels [0, top) remain
  bool first = true;
  for (int pass = 0; pass < npass; pass++) {
    const int r = (top + (npass - pass) - 1) / (npass - pass);
    const int sb = top - r;
    int cshift = std::min(std::min(k, 6), 10 - r);
    cshift = std::max(0, std::min(cshift, d + k - 7 - r));
    const int ncc = 1 << (k - cshift);
    const int src_rows = first ? l : d;
    const CUtensorMap src = rows_map(first ? msg : cw, src_rows, k, sb, r, cshift);
    const CUtensorMap dst = rows_map(cw, d, k, sb, r, cshift);
    const size_t blocks = (size_t)ncc << (src_rows - r) << (first ? d - l : 0);
    const int threads = std::min(512, 1 << (r - 1 + cshift));
    k_rs_pass<<<(unsigned)blocks, threads, 0, s>>>(src, dst, d, l, sb, r, cshift, ncc,
                                                   first ? 1 : 0, wh, err);
    BZ_LAUNCH_CHECK();
    top = sb;
    first = false;
  }
}

// ------------------------------------------------------------------ Merkle

// Leaf i = BLAKE3 of codeword row i (2^k elements, at most 1 KiB: one chunk).
__global__ void k_merkle_leaves(const f128 *__restrict__ cw, size_t rows, int k,
                                uint32_t *__restrict__ nodes) {
  const uint32_t IV[8] = {0x6A09E667, 0xBB67AE85, 0x3C6EF372, 0xA54FF53A,
                          0x510E527F, 0x9B05688C, 0x1F83D9AB, 0x5BE0CD19};
  int nbytes = 16 << k;
  int nblk = (nbytes + 63) / 64;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < rows;
       i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t *p = reinterpret_cast<const uint32_t *>(cw + (i << k));
    uint32_t cv[8];
    for (int j = 0; j < 8; j++) cv[j] = IV[j];
    for (int b = 0; b < nblk; b++) {
      uint32_t m[16];
      int len = nbytes - 64 * b < 64 ? nbytes - 64 * b : 64;
      for (int j = 0; j < 16; j++) m[j] = 4 * j < len ? p[16 * b + j] : 0;
      uint32_t fl = (b == 0 ? B3_CHUNK_START : 0) | (b == nblk - 1 ? B3_CHUNK_END | B3_ROOT : 0);
      b3_compress(cv, m, 0, (uint32_t)len, fl, cv);
    }
    for (int j = 0; j < 8; j++) nodes[8 * (rows + i) + j] = cv[j];
  }
}

// Parents lo..hi-1: node i = BLAKE3(node 2i || node 2i+1).
__global__ void k_merkle_parents(uint32_t *nodes, size_t lo, size_t hi) {
  const uint32_t IV[8] = {0x6A09E667, 0xBB67AE85, 0x3C6EF372, 0xA54FF53A,
                          0x510E527F, 0x9B05688C, 0x1F83D9AB, 0x5BE0CD19};
  for (size_t i = lo + blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < hi;
       i += (size_t)gridDim.x * blockDim.x) {
    uint32_t m[16], cv[8];
    for (int j = 0; j < 16; j++) m[j] = nodes[16 * i + j];
    b3_compress(IV, m, 0, 64, B3_CHUNK_START | B3_CHUNK_END | B3_ROOT, cv);
    for (int j = 0; j < 8; j++) nodes[8 * i + j] = cv[j];
  }
}

void merkle_build(const f128 *cw, size_t rows, int k, uint32_t *nodes, cudaStream_t s) {
  k_merkle_leaves<<<grid_for(rows), kThreads, 0, s>>>(cw, rows, k, nodes);
  BZ_LAUNCH_CHECK();
  for (size_t lo = rows / 2; lo >= 1; lo /= 2) {
    k_merkle_parents<<<grid_for(lo), kThreads, 0, s>>>(nodes, lo, 2 * lo);
    BZ_LAUNCH_CHECK();
  }
}

// A small tree in one block: the leaves (unless leaves_done: a grid launch
// hashed them already), then each level of parents after a block barrier (the
// nodes stay in global memory, which the block's barrier orders), and the
// root (node 1) posted as four mailbox words.
constexpr int kMerkleBlockThreads = 512;
__global__ void __launch_bounds__(kMerkleBlockThreads) k_merkle_block(
    const f128 *__restrict__ cw, size_t rows, int k, uint32_t *nodes, Publish pub,
    int leaves_done) {
  const uint32_t IV[8] = {0x6A09E667, 0xBB67AE85, 0x3C6EF372, 0xA54FF53A,
                          0x510E527F, 0x9B05688C, 0x1F83D9AB, 0x5BE0CD19};
  const int nbytes = 16 << k;
  const int nblk = (nbytes + 63) / 64;
  for (size_t i = threadIdx.x; i < rows && !leaves_done; i += blockDim.x) {
    const uint32_t *p = reinterpret_cast<const uint32_t *>(cw + (i << k));
    uint32_t cv[8];
    for (int j = 0; j < 8; j++) cv[j] = IV[j];
    for (int b = 0; b < nblk; b++) {
      uint32_t m[16];
      const int len = nbytes - 64 * b < 64 ? nbytes - 64 * b : 64;
      for (int j = 0; j < 16; j++) m[j] = 4 * j < len ? p[16 * b + j] : 0;
      const uint32_t fl =
          (b == 0 ? B3_CHUNK_START : 0) | (b == nblk - 1 ? B3_CHUNK_END | B3_ROOT : 0);
      b3_compress(cv, m, 0, (uint32_t)len, fl, cv);
    }
    for (int j = 0; j < 8; j++) nodes[8 * (rows + i) + j] = cv[j];
  }
  __syncthreads();
  for (size_t lo = rows / 2; lo >= 1; lo /= 2) {
    for (size_t i = lo + threadIdx.x; i < 2 * lo; i += blockDim.x) {
      uint32_t m[16], cv[8];
      for (int j = 0; j < 16; j++) m[j] = nodes[16 * i + j];
      b3_compress(IV, m, 0, 64, B3_CHUNK_START | B3_CHUNK_END | B3_ROOT, cv);
      for (int j = 0; j < 8; j++) nodes[8 * i + j] = cv[j];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0 && pub.counter)
    for (int w = 0; w < 4; w++)
      mailbox_post(pub.mailbox, pub.seq, w,
                   (unsigned long long)nodes[8 + 2 * w] |
                       ((unsigned long long)nodes[8 + 2 * w + 1] << 32));
}

bool merkle_build_posted(const f128 *cw, size_t rows, int k, uint32_t *nodes, Publish pub,
                         cudaStream_t s) {
  if (rows > kMerkleBlockMaxRows || !pub.counter) return false;
  // many leaf compressions: the leaves over the whole GPU first, then the
  // parents and the post in one block
  const size_t leaf_compressions = rows * (size_t)(((16 << k) + 63) / 64);
  const int split = leaf_compressions > 2 * (size_t)kMerkleBlockThreads;
  if (split) {
    k_merkle_leaves<<<grid_for(rows), kThreads, 0, s>>>(cw, rows, k, nodes);
    BZ_LAUNCH_CHECK();
  }
  k_merkle_block<<<1, kMerkleBlockThreads, 0, s>>>(cw, rows, k, nodes, pub, split);
  BZ_LAUNCH_CHECK();
  return true;
}

// ----------------------------------------------------- Ligerito query glue

// basis[j] += sum_q s_q prod_{t in j} w[q][t]: block q builds its tensor table
// in shared memory by doubling and XORs it into the basis. The factors are
// the subspace polynomials at the queried row: w[q][t] = Wh_t(x_q) = the sum
// of Wh_t(X^s) over the set bits s >= t of idx[q] (wh is that table, t-major
// with kMaxRsDim entries per t), formed by the block's first threads.
__global__ void k_query_basis(const uint64_t *__restrict__ idx, const f128 *__restrict__ wh,
                              const f128 *__restrict__ scale, int l,
                              unsigned long long *basis) {
  extern __shared__ f128 tab[];
  __shared__ f128 w[kMaxRsDim];
  const int q = blockIdx.x;
  if (threadIdx.x < l) {
    const int t = threadIdx.x;
    f128 v = mk(0, 0);
    // row indices stay below 2^kMaxRsDim; the mask keeps every read in wh
    for (uint64_t bits = (idx[q] >> t) & ((1ull << (kMaxRsDim - t)) - 1); bits; bits &= bits - 1)
      v = gadd(v, ld(wh + t * kMaxRsDim + t + __ffsll((long long)bits) - 1));
    w[t] = v;
  }
  if (threadIdx.x == 0) tab[0] = scale[q];
  __syncthreads();
  for (int t = 0; t < l; t++) {
    int h = 1 << t;
    const f128 wt = w[t];
    for (int j = threadIdx.x; j < h; j += blockDim.x) tab[h + j] = gmul(tab[j], wt);
    __syncthreads();
  }
  for (int j = threadIdx.x; j < (1 << l); j += blockDim.x) {
    f128 v = tab[j];
    if (v.lo) atomicXor(basis + 2 * j, (unsigned long long)v.lo);
    if (v.hi) atomicXor(basis + 2 * j + 1, (unsigned long long)v.hi);
  }
}

void query_basis(const uint64_t *idx, const f128 *wh, const f128 *scale, int nq, int l,
                 f128 *basis, cudaStream_t s) {
  if (l > kMaxRsDim || l > kThreads) throw CudaError("query basis dimension out of range");
  size_t smem = sizeof(f128) << l;
  if (smem > 48 * 1024 - sizeof(f128) * kMaxRsDim)
    BZ_CUDA(cudaFuncSetAttribute(k_query_basis, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
  k_query_basis<<<nq, kThreads, smem, s>>>(idx, wh, scale, l, (unsigned long long *)basis);
  BZ_LAUNCH_CHECK();
}

// The opened rows and their Merkle paths, in proof order: per query the row
// (width entries of 16 bytes), then the sibling of every node from the leaf
// (rows + idx) up to the root's children (32 bytes each). One block per query.
__global__ void k_gather_openings(const f128 *__restrict__ cw, const uint32_t *__restrict__ nodes,
                                  size_t rows, int width, int depth,
                                  const uint64_t *__restrict__ idx, f128 *__restrict__ out) {
  const size_t stride = (size_t)width + 2 * (size_t)depth;  // in 16-byte units
  f128 *o = out + blockIdx.x * stride;
  const uint64_t id = idx[blockIdx.x];
  for (int c = threadIdx.x; c < width; c += blockDim.x) st(o + c, ld(cw + id * width + c));
  for (int k = threadIdx.x; k < 2 * depth; k += blockDim.x) {
    const int d = k >> 1, half = k & 1;
    const size_t sib = ((rows + id) >> d) ^ 1;
    st(o + width + k, ld(reinterpret_cast<const f128 *>(nodes + 8 * sib) + half));
  }
}

void gather_openings(const f128 *cw, const uint32_t *nodes, size_t rows, int width, int depth,
                     const uint64_t *idx, int nq, f128 *out, cudaStream_t s) {
  k_gather_openings<<<nq, 64, 0, s>>>(cw, nodes, rows, width, depth, idx, out);
  BZ_LAUNCH_CHECK();
}

// Every kernel of this file, loaded when the process's first lane on a device
// is made (lane_bootstrap, context.cpp).
void preload_pcs_kernels() {
  load_kernels({(const void *)k_fold_columns,
                (const void *)k_comb_pow,
                (const void *)k_mt_transpose,
                (const void *)k_mt_col0,
                (const void *)k_mt_dense,
                (const void *)k_mt_gather,
                (const void *)k_b3_chunks,
                (const void *)k_b3_parents,
                (const void *)k_b3_top,
                (const void *)k_ring_claims,
                (const void *)k_packed_basis,
                (const void *)k_dot,
                (const void *)k_axpy,
                (const void *)k_rs_pass,
                (const void *)k_rs_encode_block,
                (const void *)k_merkle_leaves,
                (const void *)k_merkle_parents,
                (const void *)k_merkle_block,
                (const void *)k_query_basis,
                (const void *)k_gather_openings});
}

}  // namespace bz
