// Spartan's outer and inner sumchecks and the matrix bind over the
// transcript-drawn prime (crates/spartan/src/piop.rs:67-113,
// sumcheck.rs:252-553, matrix.rs:336-467).
//
// Tables hold Montgomery residues. Each round is one launch that folds the
// previous round's challenge into every table and accumulates the next
// round's coefficients from the folded values in registers (the reference's
// fold/round fusion, sumcheck.rs:963-1026), then one single-block launch adds
// the per-block partial sums; 48 (outer) or 32 (inner) bytes go to the host.
#include "device.cuh"
#include "context.hpp"
#include "spartan.hpp"

#include <chrono>
#include <cstdio>

namespace bz {

// Both factor tables in one launch: block 0 the low a coordinates, block 1
// the high b.
__global__ void k_fp_eq_factor(FpPoint p, int a, int b, FpCtx c, fp *lo, fp *hi) {
  const int first = blockIdx.x == 0 ? 0 : a, n = blockIdx.x == 0 ? a : b;
  fp *out = blockIdx.x == 0 ? lo : hi;
  if (threadIdx.x == 0) out[0] = c.one;
  __syncthreads();
  for (int i = 0; i < n; i++) {
    fp z = p.c[first + i];
    int half = 1 << i;
    for (int k = threadIdx.x; k < half; k += blockDim.x) {
      fp par = out[k];
      fp one = fp_mul(par, z, c);
      out[k] = fp_sub(par, one, c);
      out[k + half] = one;
    }
    __syncthreads();
  }
}

__global__ void k_fp_eq_expand(const fp *__restrict__ lo, int a, const fp *__restrict__ hi,
                               FpCtx c, fp *__restrict__ out, size_t total) {
  size_t mask = ((size_t)1 << a) - 1;
  for (size_t x = blockIdx.x * (size_t)blockDim.x + threadIdx.x; x < total;
       x += (size_t)gridDim.x * blockDim.x)
    out[x] = fp_mul(lo[x & mask], hi[x >> a], c);
}

void fp_eq_table(const fp *point, int n, const FpCtx &c, fp *out, fp *scratch, cudaStream_t s) {
  FpPoint p;
  for (int i = 0; i < n; i++) p.c[i] = point[i];
  int a = n / 2, b = n - a;
  fp *lo = scratch, *hi = scratch + ((size_t)1 << a);
  k_fp_eq_factor<<<2, kThreads, 0, s>>>(p, a, b, c, lo, hi);
  BZ_LAUNCH_CHECK();
  size_t total = (size_t)1 << n;
  k_fp_eq_expand<<<grid_for(total), kThreads, 0, s>>>(lo, a, hi, c, out, total);
  BZ_LAUNCH_CHECK();
}

__device__ __forceinline__ fp fp_from_i64(int64_t v, const FpCtx &c) {
  fp x;
  if (v >= 0) {
    x = fp{(uint64_t)v, 0};
  } else {
    uint64_t m = (uint64_t)(-(v + 1)) + 1;  // |v|, which is below q
    x.lo = c.q0 - m;
    x.hi = c.q1 - (c.q0 < m);
  }
  return fp_mul(x, c.r2, c);
}

// build_product_mles (matrix.rs:336-370): A h, B h, C h mod q, zero padded.
__global__ void k_products_to_fp(const int64_t *__restrict__ prod, size_t rows, size_t padded,
                                 FpCtx c, fp *__restrict__ A, fp *__restrict__ B,
                                 fp *__restrict__ C) {
  for (size_t r = blockIdx.x * (size_t)blockDim.x + threadIdx.x; r < padded;
       r += (size_t)gridDim.x * blockDim.x) {
    if (r < rows) {
      A[r] = fp_from_i64(prod[r], c);
      B[r] = fp_from_i64(prod[rows + r], c);
      C[r] = fp_from_i64(prod[2 * rows + r], c);
    } else {
      A[r] = B[r] = C[r] = fp_zero();
    }
  }
}

BZ_HD fp interp(fp a, fp b, fp r, const FpCtx &c) {
  return fp_add(a, fp_mul(r, fp_sub(b, a, c), c), c);
}

// cubic_contribution (sumcheck.rs:724-746): [e0 r0, e0 rq + ed rl, ed rq]
BZ_HD void cubic(fp e0, fp e1, fp a0, fp a1, fp b0, fp b1, fp c0, fp c1, const FpCtx &c,
                 fp (&acc)[3]) {
  fp ed = fp_sub(e1, e0, c), ad = fp_sub(a1, a0, c), bd = fp_sub(b1, b0, c), cd = fp_sub(c1, c0, c);
  fp r0 = fp_sub(fp_mul(a0, b0, c), c0, c);
  fp rl = fp_sub(fp_add(fp_mul(a0, bd, c), fp_mul(ad, b0, c), c), cd, c);
  fp rq = fp_mul(ad, bd, c);
  acc[0] = fp_add(acc[0], fp_mul(e0, r0, c), c);
  acc[1] = fp_add(acc[1], fp_add(fp_mul(e0, rq, c), fp_mul(ed, rl, c), c), c);
  acc[2] = fp_add(acc[2], fp_mul(ed, rq, c), c);
}

// The round's message from the blocks' partial sums (block_fp_sum<N> left
// them at partial[block * N + k], written by thread 0): the last block to
// count itself in `counter` adds every block's partials (mod q, in any order)
// and posts the N totals as words 2k (low half) and 2k + 1 (high half) of
// publication seq. Every thread calls it; true in the last block (whose
// threads are still together), false in the others.
template <int N>
__device__ bool fp_last_block_post(const fp *partial, const FpCtx &c, unsigned int *counter,
                                   Mailbox *mb, unsigned long long seq) {
  static_assert(2 * N <= kMailboxWords, "mailbox too small");
  __shared__ int last_s;
  __shared__ fp red[N][kThreads / 32];
  if (threadIdx.x == 0) {
    __threadfence();
    last_s = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last_s) return false;
  __threadfence();
  fp v[N];
#pragma unroll
  for (int k = 0; k < N; k++) v[k] = fp_zero();
  for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x)
#pragma unroll
    for (int k = 0; k < N; k++) {
      const ulonglong2 w = __ldcg(reinterpret_cast<const ulonglong2 *>(partial + b * N + k));
      v[k] = fp_add(v[k], fp{w.x, w.y}, c);
    }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < N; k++) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      fp o;
      o.lo = __shfl_xor_sync(0xffffffffu, v[k].lo, off);
      o.hi = __shfl_xor_sync(0xffffffffu, v[k].hi, off);
      v[k] = fp_add(v[k], o, c);
    }
    if (lane == 0) red[k][warp] = v[k];
  }
  __syncthreads();
  if (threadIdx.x == 0)
    for (int k = 0; k < N; k++) {
      fp x = red[k][0];
      for (int w = 1; w < (int)(blockDim.x >> 5); w++) x = fp_add(x, red[k][w], c);
      mailbox_post(mb, seq, 2 * k, x.lo);
      mailbox_post(mb, seq, 2 * k + 1, x.hi);
    }
  return true;
}

// fp_last_block_post through the lane's shared counter (reset by the last
// block), then the last block fetches the next challenge for the round link.
template <int N>
__device__ void fp_round_end(const fp *partial, const FpCtx &c, const Publish &p,
                             const RoundLink &lk) {
  if (!fp_last_block_post<N>(partial, c, p.counter, p.mailbox, p.seq)) return;
  if (threadIdx.x == 0) {
    *p.counter = 0;
    link_fetch(lk);
  }
}

// One outer round. fold = 0: sums over the pairs of the tables as they are.
// fold = 1: fold every table at r (output at half length) and sum over the
// folded pairs. emit = 0 only folds (the last fold).
__global__ void k_outer_round(const fp *E, const fp *A, const fp *B, const fp *C, fp *E2, fp *A2,
                              fp *B2, fp *C2, size_t n, int fold, int emit, fp r, FpCtx c,
                              fp *partial, Publish pub, RoundLink lk) {
  if (lk.in) {
    unsigned long long w0, w1;
    if (!link_begin(lk, w0, w1)) return;
    r = fp{w0, w1};
  }
  fp acc[3] = {fp_zero(), fp_zero(), fp_zero()};
  size_t npairs = fold ? (n / 2 + 1) / 2 : n / 2;
  for (size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x; j < npairs;
       j += (size_t)gridDim.x * blockDim.x) {
    fp e[2], a[2], b[2], cc[2];
    if (fold) {
      for (int t = 0; t < 2; t++) {
        size_t o = 2 * j + t;
        if (o >= n / 2) {
          e[t] = a[t] = b[t] = cc[t] = fp_zero();
          continue;
        }
        e[t] = interp(E[2 * o], E[2 * o + 1], r, c);
        a[t] = interp(A[2 * o], A[2 * o + 1], r, c);
        b[t] = interp(B[2 * o], B[2 * o + 1], r, c);
        cc[t] = interp(C[2 * o], C[2 * o + 1], r, c);
        E2[o] = e[t];
        A2[o] = a[t];
        B2[o] = b[t];
        C2[o] = cc[t];
      }
    } else {
      for (int t = 0; t < 2; t++) {
        e[t] = E[2 * j + t];
        a[t] = A[2 * j + t];
        b[t] = B[2 * j + t];
        cc[t] = C[2 * j + t];
      }
    }
    if (emit) cubic(e[0], e[1], a[0], a[1], b[0], b[1], cc[0], cc[1], c, acc);
  }
  if (emit) {
    block_fp_sum<3>(acc, c, partial);
    if (pub.counter) fp_round_end<3>(partial, c, pub, lk);
  }
}

// One inner round over D and the assignment W. W is read from the packed h
// bits while w_bits is set (round 0, and the input of round 1's fold).
__global__ void k_inner_round(const fp *D, const fp *W, const uint32_t *hbits, int w_bits, fp *D2,
                              fp *W2, size_t n, int fold, int emit, fp r, FpCtx c, fp *partial,
                              Publish pub, RoundLink lk) {
  if (lk.in) {
    unsigned long long w0, w1;
    if (!link_begin(lk, w0, w1)) return;
    r = fp{w0, w1};
  }
  fp acc[2] = {fp_zero(), fp_zero()};
  size_t npairs = fold ? (n / 2 + 1) / 2 : n / 2;
  for (size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x; j < npairs;
       j += (size_t)gridDim.x * blockDim.x) {
    fp d[2], w[2];
    for (int t = 0; t < 2; t++) {
      size_t o = 2 * j + t;
      if (fold) {
        if (o >= n / 2) {
          d[t] = w[t] = fp_zero();
          continue;
        }
        fp w0, w1;
        if (w_bits) {
          size_t i0 = 2 * o;
          w0 = ((hbits[i0 >> 5] >> (i0 & 31)) & 1) ? c.one : fp_zero();
          w1 = ((hbits[(i0 + 1) >> 5] >> ((i0 + 1) & 31)) & 1) ? c.one : fp_zero();
        } else {
          w0 = W[2 * o];
          w1 = W[2 * o + 1];
        }
        d[t] = interp(D[2 * o], D[2 * o + 1], r, c);
        w[t] = interp(w0, w1, r, c);
        D2[o] = d[t];
        W2[o] = w[t];
      } else {
        d[t] = D[o];
        w[t] = ((hbits[o >> 5] >> (o & 31)) & 1) ? c.one : fp_zero();
      }
    }
    if (emit) {
      acc[0] = fp_add(acc[0], fp_mul(d[0], w[0], c), c);
      acc[1] = fp_add(acc[1], fp_mul(fp_sub(d[1], d[0], c), fp_sub(w[1], w[0], c), c), c);
    }
  }
  if (emit) {
    block_fp_sum<2>(acc, c, partial);
    if (pub.counter) fp_round_end<2>(partial, c, pub, lk);
  }
}

// One block adds the per-block partials; the totals go to out and, when
// publishing, to the mailbox (written by the thread that wrote out).
template <int N>
__global__ void k_fp_finalize(const fp *partial, int nblocks, FpCtx c, fp *out, Publish pub) {
  fp acc[N];
  for (int k = 0; k < N; k++) acc[k] = fp_zero();
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
    for (int k = 0; k < N; k++) acc[k] = fp_add(acc[k], partial[b * N + k], c);
  block_fp_sum<N>(acc, c, out);
  static_assert(2 * N <= kMailboxWords, "mailbox too small");
  if (pub.counter && threadIdx.x == 0) {
    for (int k = 0; k < N; k++) {
      mailbox_post(pub.mailbox, pub.seq, 2 * k, out[k].lo);
      mailbox_post(pub.mailbox, pub.seq, 2 * k + 1, out[k].hi);
    }
  }
}

// The coefficient table of the bind: scale_k * coefficient for every distinct
// (matrix, coefficient) pair.
__global__ void k_bind_table(const int64_t *__restrict__ vals, const uint8_t *__restrict__ which,
                             int n, fp rho, fp rho2, FpCtx c, fp *tab) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  fp v = fp_from_i64(vals[i], c);
  fp s = which[i] == 0 ? c.one : which[i] == 1 ? rho : rho2;
  tab[i] = fp_mul(v, s, c);
}

// bind_and_batch (matrix.rs:429-467) as a gather over the column-major copy of
// A, B and C: D(y) = sum over column y's entries of eq(r_x, row) * table[idx].
// Column 0 (the constant, one entry per round constant and bit constraint)
// is left to k_bind_col0, which spreads it over a whole grid.
__global__ void k_bind(const uint32_t *__restrict__ off, const uint32_t *__restrict__ row,
                       const uint16_t *__restrict__ idx, const fp *__restrict__ tab,
                       const fp *__restrict__ eq, size_t cols, size_t padded, FpCtx c, fp *D) {
  for (size_t y = blockIdx.x * (size_t)blockDim.x + threadIdx.x; y < padded;
       y += (size_t)gridDim.x * blockDim.x) {
    fp acc = fp_zero();
    if (y > 0 && y < cols)
      for (uint32_t e = off[y]; e < off[y + 1]; e++) acc = fp_add(acc, fp_mul(eq[row[e]], tab[idx[e]], c), c);
    D[y] = acc;
  }
}

// Column 0's entries [0, n) split across blocks, and with them the
// statement-dependent part of C on column 0: the bit constraints whose
// expected value is one put rho^2 eq(r_x, row) there (each thread scales its
// share of those rows, which sums to the same total mod q). Per-block
// partial sums.
__global__ void k_bind_col0(const uint32_t *__restrict__ row, const uint16_t *__restrict__ idx,
                            const fp *__restrict__ tab, const fp *__restrict__ eq, uint32_t n,
                            const uint32_t *__restrict__ bit_rows, int n_bits, fp rho2, FpCtx c,
                            fp *partial) {
  fp acc[1] = {fp_zero()};
  for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x)
    acc[0] = fp_add(acc[0], fp_mul(eq[row[e]], tab[idx[e]], c), c);
  fp bits = fp_zero();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_bits; i += gridDim.x * blockDim.x)
    bits = fp_add(bits, eq[bit_rows[i]], c);
  acc[0] = fp_add(acc[0], fp_mul(bits, rho2, c), c);
  block_fp_sum<1>(acc, c, partial);
}

// D[0] = the column-0 partial sums.
__global__ void k_bind_col0_finish(const fp *partial, int nblocks, FpCtx c, fp *D) {
  fp acc[1] = {fp_zero()};
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) acc[0] = fp_add(acc[0], partial[b], c);
  __shared__ fp out[1];
  block_fp_sum<1>(acc, c, out);
  __syncthreads();
  if (threadIdx.x == 0) D[0] = out[0];
}


// The last rounds of each sumcheck in one resident block, fed through the
// lane's downbox (bounded waits; a missing challenge ends the kernel without
// a post). The tables (at most kSpTailN entries each) sit in shared memory.
// Each round folds at the previous round's challenge (when `fold`), sums the
// round's coefficients and posts them; after the last round the final fold's
// single entries are posted.
constexpr int kSpTailN = 512;
constexpr unsigned long long kSpWaitNs = 2000000000ull;

// Folds T tables of len entries in place at r (all reads, then all writes).
template <int T>
__device__ __forceinline__ int sp_fold(fp (*tab)[kSpTailN], int len, fp r, const FpCtx &c) {
  const int nout = len / 2;
  fp f[T][2];
  int cnt = 0;
  for (int o = threadIdx.x; o < nout; o += blockDim.x, cnt++)
    for (int t = 0; t < T; t++) f[t][cnt] = interp(tab[t][2 * o], tab[t][2 * o + 1], r, c);
  __syncthreads();
  cnt = 0;
  for (int o = threadIdx.x; o < nout; o += blockDim.x, cnt++)
    for (int t = 0; t < T; t++) tab[t][o] = f[t][cnt];
  __syncthreads();
  return nout;
}

__device__ __forceinline__ bool sp_challenge(const Mailbox *down, unsigned long long dseq,
                                             const FpCtx &c, fp &r) {
  __shared__ unsigned long long chal[2];
  __shared__ int ok;
  if (threadIdx.x == 0) ok = mailbox_wait_device(down, dseq, 2, chal, kSpWaitNs);
  __syncthreads();
  r = fp{chal[0], chal[1]};
  bool good = ok;
  __syncthreads();
  return good;
}

// The T tables (len entries each, one after another) as handover
// publication seq: the host runs the sumcheck's remaining rounds.
template <int T>
__device__ __forceinline__ void sp_handover(fp (*tab)[kSpTailN], int len,
                                            unsigned long long *handover,
                                            unsigned long long seq) {
  for (int k = threadIdx.x; k < T * len; k += blockDim.x) {
    const fp v = tab[k / len][k % len];
    handover_post(handover, seq, 2 * k, v.lo);
    handover_post(handover, seq, 2 * k + 1, v.hi);
  }
}

template <int N>
__device__ __forceinline__ void sp_post(fp (&acc)[N], const FpCtx &c, Mailbox *mb,
                                        unsigned long long seq) {
  __shared__ fp red[N];
  block_fp_sum<N>(acc, c, red);
  if (threadIdx.x == 0)
    for (int k = 0; k < N; k++) {
      mailbox_post(mb, seq, 2 * k, red[k].lo);
      mailbox_post(mb, seq, 2 * k + 1, red[k].hi);
    }
  __syncthreads();
}

// Outer rounds round0 .. rounds-1 over E, A, B, C (len0 entries each).
__global__ void __launch_bounds__(kThreads) sp_outer_tail(const fp *E, const fp *A, const fp *B,
                                                          const fp *C, int len0, int fold0,
                                                          int nrounds, FpCtx c, Mailbox *mb,
                                                          unsigned long long seq0,
                                                          const Mailbox *down,
                                                          unsigned long long dseq0,
                                                          int hand_round,
                                                          unsigned long long *handover,
                                                          unsigned long long hseq) {
  __shared__ fp tab[4][kSpTailN];
  for (int k = threadIdx.x; k < len0; k += blockDim.x) {
    tab[0][k] = E[k];
    tab[1][k] = A[k];
    tab[2][k] = B[k];
    tab[3][k] = C[k];
  }
  __syncthreads();
  int len = len0, nd = 0, np = 0;
  for (int round = 0; round < nrounds; round++) {
    if (round == hand_round) {  // the remaining rounds run on the host
      sp_handover<4>(tab, len, handover, hseq);
      return;
    }
    if (round > 0 || fold0) {
      fp r;
      if (!sp_challenge(down, dseq0 + nd++, c, r)) return;
      len = sp_fold<4>(tab, len, r, c);
    }
    fp acc[3] = {fp_zero(), fp_zero(), fp_zero()};
    for (int j = threadIdx.x; j < len / 2; j += blockDim.x)
      cubic(tab[0][2 * j], tab[0][2 * j + 1], tab[1][2 * j], tab[1][2 * j + 1], tab[2][2 * j],
            tab[2][2 * j + 1], tab[3][2 * j], tab[3][2 * j + 1], c, acc);
    sp_post<3>(acc, c, mb, seq0 + np++);
  }
  fp r;
  if (!sp_challenge(down, dseq0 + nd, c, r)) return;
  sp_fold<4>(tab, len, r, c);
  if (threadIdx.x == 0)
    for (int k = 0; k < 3; k++) {
      mailbox_post(mb, seq0 + np, 2 * k, tab[k + 1][0].lo);
      mailbox_post(mb, seq0 + np, 2 * k + 1, tab[k + 1][0].hi);
    }
}

// Inner rounds over D and W (W from the packed h bits when w_bits).
__global__ void __launch_bounds__(kThreads) sp_inner_tail(const fp *D, const fp *W,
                                                          const uint32_t *hbits, int w_bits,
                                                          int len0, int fold0, int nrounds,
                                                          FpCtx c, Mailbox *mb,
                                                          unsigned long long seq0,
                                                          const Mailbox *down,
                                                          unsigned long long dseq0,
                                                          int hand_round,
                                                          unsigned long long *handover,
                                                          unsigned long long hseq) {
  __shared__ fp tab[2][kSpTailN];
  for (int k = threadIdx.x; k < len0; k += blockDim.x) {
    tab[0][k] = D[k];
    tab[1][k] = w_bits ? (((hbits[k >> 5] >> (k & 31)) & 1) ? c.one : fp_zero()) : W[k];
  }
  __syncthreads();
  int len = len0, nd = 0, np = 0;
  for (int round = 0; round < nrounds; round++) {
    if (round == hand_round) {  // the remaining rounds run on the host
      sp_handover<2>(tab, len, handover, hseq);
      return;
    }
    if (round > 0 || fold0) {
      fp r;
      if (!sp_challenge(down, dseq0 + nd++, c, r)) return;
      len = sp_fold<2>(tab, len, r, c);
    }
    fp acc[2] = {fp_zero(), fp_zero()};
    for (int j = threadIdx.x; j < len / 2; j += blockDim.x) {
      fp d0 = tab[0][2 * j], d1 = tab[0][2 * j + 1], w0 = tab[1][2 * j], w1 = tab[1][2 * j + 1];
      acc[0] = fp_add(acc[0], fp_mul(d0, w0, c), c);
      acc[1] = fp_add(acc[1], fp_mul(fp_sub(d1, d0, c), fp_sub(w1, w0, c), c), c);
    }
    sp_post<2>(acc, c, mb, seq0 + np++);
  }
  fp r;
  if (!sp_challenge(down, dseq0 + nd, c, r)) return;
  sp_fold<2>(tab, len, r, c);
  if (threadIdx.x == 0) {
    mailbox_post(mb, seq0 + np, 0, tab[0][0].lo);
    mailbox_post(mb, seq0 + np, 1, tab[0][0].hi);
    mailbox_post(mb, seq0 + np, 2, tab[1][0].lo);
    mailbox_post(mb, seq0 + np, 3, tab[1][0].hi);
  }
}

// ------------------------------------------------------------------- host

// The tail hands its tables to the host at the first round whose input is at
// most this long; each round after that costs the host a few microseconds,
// against a PCIe round trip and a device step.
constexpr size_t kSpHostLen = 64;

// The first round (at or after the tail's first, t0) whose input of
// n0 >> (k - 1) entries (n0 at k = 0) is at most kSpHostLen; -1 without a
// handover area or a round that small.
static int sp_host_round(const RoundChannel *ch, size_t n0, int t0, int nrounds) {
  if (!ch->handover_host) return -1;
  for (int k = t0; k < nrounds; k++)
    if ((k == 0 ? n0 : n0 >> (k - 1)) <= kSpHostLen) return k;
  return -1;
}

// The handover's T tables of len entries each.
static void sp_take_handover(RoundChannel *ch, cudaStream_t s, unsigned long long seq, int T,
                             size_t len, std::vector<fp> *tab) {
  std::vector<uint64_t> w(2 * T * len);
  ch->wait_handover(s, seq, w.data(), (int)w.size());
  for (int t = 0; t < T; t++) {
    tab[t].resize(len);
    for (size_t k = 0; k < len; k++)
      tab[t][k] = fp{w[2 * (t * len + k)], w[2 * (t * len + k) + 1]};
  }
}

// sp_fold on the host: each table folded at r in place (entry o from 2o and
// 2o + 1, read before it is overwritten).
static void host_sp_fold(std::vector<fp> *tab, int T, fp r, const FpCtx &c) {
  for (int t = 0; t < T; t++) {
    const size_t n = tab[t].size() / 2;
    for (size_t o = 0; o < n; o++) tab[t][o] = interp(tab[t][2 * o], tab[t][2 * o + 1], r, c);
    tab[t].resize(n);
  }
}

// The outer and inner rounds' sums, as the tail kernels form them.
static void host_outer_sums(const std::vector<fp> *tab, const FpCtx &c, fp *out) {
  fp acc[3] = {fp_zero(), fp_zero(), fp_zero()};
  for (size_t j = 0; j < tab[0].size() / 2; j++)
    cubic(tab[0][2 * j], tab[0][2 * j + 1], tab[1][2 * j], tab[1][2 * j + 1], tab[2][2 * j],
          tab[2][2 * j + 1], tab[3][2 * j], tab[3][2 * j + 1], c, acc);
  for (int k = 0; k < 3; k++) out[k] = acc[k];
}

static void host_inner_sums(const std::vector<fp> *tab, const FpCtx &c, fp *out) {
  fp acc[2] = {fp_zero(), fp_zero()};
  for (size_t j = 0; j < tab[0].size() / 2; j++) {
    const fp d0 = tab[0][2 * j], d1 = tab[0][2 * j + 1], w0 = tab[1][2 * j], w1 = tab[1][2 * j + 1];
    acc[0] = fp_add(acc[0], fp_mul(d0, w0, c), c);
    acc[1] = fp_add(acc[1], fp_mul(fp_sub(d1, d0, c), fp_sub(w1, w0, c), c), c);
  }
  out[0] = acc[0];
  out[1] = acc[1];
}

static fp host_partial_sum(const fp *d_partial, int nblocks, int N, fp *d_out, fp *h_out,
                           const FpCtx &c, cudaStream_t s, RoundChannel *ch) {
  Publish pub = ch ? ch->arm() : Publish{nullptr, nullptr, 0};
  KernelProbe &probe = KernelProbe::get();
  const bool probed = probe.on("k_fp_finalize");
  if (probed) probe.before(s);
  if (N == 3)
    k_fp_finalize<3><<<1, kThreads, 0, s>>>(d_partial, nblocks, c, d_out, pub);
  else
    k_fp_finalize<2><<<1, kThreads, 0, s>>>(d_partial, nblocks, c, d_out, pub);
  BZ_LAUNCH_CHECK();
  if (probed) probe.after(s, "k_fp_finalize", 16.0 * N * (nblocks + 1));
  if (ch) {
    ch->wait(s, reinterpret_cast<uint64_t *>(h_out), 2 * N);
  } else {
    BZ_CUDA(cudaMemcpyAsync(h_out, d_out, N * sizeof(fp), cudaMemcpyDeviceToHost, s));
    BZ_CUDA(stream_wait(s));
  }
  return h_out[0];
}

static void put_canonical(uint8_t *b, fp mont, const FpCtx &c) {
  fp v = fp_mul(mont, fp{1, 0}, c);
  memcpy(b, &v.lo, 8);
  memcpy(b + 8, &v.hi, 8);
}

// recover_full_round_polynomial_and_sample_next_challenge (sumcheck.rs:787-811)
static fp round_message(Transcript &ts, const FpCtx &c, fp &claim, const fp *wl, int ncoef,
                        u128 q, fp *coefs_out) {
  fp co[4];
  co[0] = wl[0];
  co[1] = fp_zero();
  for (int i = 2; i < ncoef; i++) co[i] = wl[i - 1];
  fp at_one = fp_zero();
  for (int i = 0; i < ncoef; i++) at_one = fp_add(at_one, co[i], c);
  co[1] = fp_sub(fp_sub(claim, co[0], c), at_one, c);
  uint8_t msg[64];
  for (int i = 0; i < ncoef; i++) put_canonical(msg + 16 * i, co[i], c);
  ts.public_message(msg, 16 * (size_t)ncoef);
  u128 rc = ts.challenge_fp(q);
  fp r = fp_mul(fp{(uint64_t)rc, (uint64_t)(rc >> 64)}, c.r2, c);
  fp v = fp_zero();
  for (int i = ncoef - 1; i >= 0; i--) v = fp_add(fp_mul(v, r, c), co[i], c);
  claim = v;
  for (int i = 0; i < ncoef; i++) coefs_out[i] = co[i];
  return r;
}

// The grid rounds k0 .. k1-1 of a sumcheck (outer: T = 4 tables E, A, B, C
// and the cubic message, N = 3; inner: T = 2 tables D, W and N = 2) in one
// cooperative launch that stays resident. Tables fold on their low
// coordinate (pairs 2o, 2o + 1), so block b owns the contiguous chunk [b m,
// (b + 1) m) of each input table (m = n_in / kSpMidBlocks) and, after each
// fold, the first half of what it held: the chunk stays in the block's shared
// memory from the first round to the last, and blocks share nothing but the
// challenge (block 0 reads r_{k-1} from the downbox as publication
// d0 + k - 1 and relays it through ctl[k - 1]) and the message (per-block
// partial sums; the last block through round k, counted in ctl[k].done, adds
// them and posts publication p0 + k). At the end each block writes its chunk
// to `out` for the tail kernel. All blocks are resident together
// (cooperative launch), so the relay waits end; each is bounded all the same.
constexpr int kSpMidBlocks = 128;     // a lane proving alone
constexpr int kSpMidPoolBlocks = 32;  // a pooled lane, sharing the GPU with others
constexpr size_t kSpMidMaxChunk = 2048;  // entries per table per block
struct SpTabs {
  fp *t[4];
};

template <int T, int N>
__global__ void __launch_bounds__(kThreads) sp_mid(SpTabs in, SpTabs out, size_t n_in, int k0,
                                                   int k1, FpCtx c, fp *partial, Mailbox *mb,
                                                   unsigned long long p0, const Mailbox *down,
                                                   unsigned long long d0, RoundCtl *ctl) {
  extern __shared__ fp chunk[];
  const size_t m = n_in / gridDim.x;
  fp *tab[T];
#pragma unroll
  for (int t = 0; t < T; t++) tab[t] = chunk + t * m;
  const size_t base = (size_t)blockIdx.x * m;
  for (size_t i = threadIdx.x; i < m; i += blockDim.x)
#pragma unroll
    for (int t = 0; t < T; t++) tab[t][i] = in.t[t][base + i];
  __syncthreads();
  size_t len = m;
  for (int k = k0; k < k1; k++) {
    if (k > 0) {
      unsigned long long rw[2];
      if (!resident_challenge(down, d0 + (k - 1), ctl + (k - 1), rw)) return;
      const fp r = fp{rw[0], rw[1]};
      // fold in place: every read of the level, then every write
      constexpr int kPer = (int)(kSpMidMaxChunk / 2 / kThreads);
      fp f[T][kPer];
      const size_t nout = len / 2;
#pragma unroll
      for (int q = 0; q < kPer; q++) {
        const size_t o = threadIdx.x + (size_t)q * kThreads;
        if (o < nout)
#pragma unroll
          for (int t = 0; t < T; t++) f[t][q] = interp(tab[t][2 * o], tab[t][2 * o + 1], r, c);
      }
      __syncthreads();
#pragma unroll
      for (int q = 0; q < kPer; q++) {
        const size_t o = threadIdx.x + (size_t)q * kThreads;
        if (o < nout)
#pragma unroll
          for (int t = 0; t < T; t++) tab[t][o] = f[t][q];
      }
      __syncthreads();
      len = nout;
    }
    fp acc[N];
#pragma unroll
    for (int q = 0; q < N; q++) acc[q] = fp_zero();
    for (size_t j = threadIdx.x; j < len / 2; j += blockDim.x) {
      if constexpr (T == 4) {
        cubic(tab[0][2 * j], tab[0][2 * j + 1], tab[1][2 * j], tab[1][2 * j + 1], tab[2][2 * j],
              tab[2][2 * j + 1], tab[3][2 * j], tab[3][2 * j + 1], c, acc);
      } else {
        const fp d0v = tab[0][2 * j], d1v = tab[0][2 * j + 1];
        const fp w0v = tab[1][2 * j], w1v = tab[1][2 * j + 1];
        acc[0] = fp_add(acc[0], fp_mul(d0v, w0v, c), c);
        acc[1] = fp_add(acc[1], fp_mul(fp_sub(d1v, d0v, c), fp_sub(w1v, w0v, c), c), c);
      }
    }
    block_fp_sum<N>(acc, c, partial);
    fp_last_block_post<N>(partial, c, &ctl[k].done, mb, p0 + k);
    __syncthreads();  // the chunk's reads of this round before the next fold
  }
  const size_t ob = (size_t)blockIdx.x * len;
  for (size_t i = threadIdx.x; i < len; i += blockDim.x)
#pragma unroll
    for (int t = 0; t < T; t++) out.t[t][ob + i] = tab[t][i];
}

// sp_mid over rounds k0 .. k1-1 as a cooperative launch of sc.mid_blocks
// blocks; n_in entries per input table.
template <int T, int N>
static void launch_sp_mid(const SpTabs &in, const SpTabs &out, size_t n_in, int k0, int k1,
                          const FpCtx &c, const SpartanScratch &sc, unsigned long long p0,
                          unsigned long long d0, cudaStream_t s) {
  const int nb = sc.mid_blocks;
  const size_t smem = T * (n_in / nb) * sizeof(fp);
  static const int capacity = [] {
    int dev = 0, sms = 0, per_sm = 0;
    const size_t most = T * kSpMidMaxChunk * sizeof(fp);
    BZ_CUDA(cudaGetDevice(&dev));
    BZ_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    BZ_CUDA(cudaFuncSetAttribute(sp_mid<T, N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)most));
    BZ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sp_mid<T, N>, kThreads, most));
    return sms * per_sm;
  }();
  if (nb < 1 || nb > kSpMidBlocks || capacity < nb)
    throw CudaError("sp_mid: the blocks do not fit resident together");
  RoundChannel *ch = sc.channel;
  SpTabs a = in, b = out;
  FpCtx cc = c;
  fp *partial = sc.partial;
  Mailbox *mb = ch->dev;
  const Mailbox *down = ch->down_dev;
  RoundCtl *ctl = sc.ctl;
  void *args[] = {&a, &b, &n_in, &k0, &k1, &cc, &partial, &mb, &p0, &down, &d0, &ctl};
  BZ_CUDA(cudaLaunchCooperativeKernel((const void *)sp_mid<T, N>, dim3(nb), dim3(kThreads), args,
                                      smem, s));
  BZ_LAUNCH_CHECK();
}

// The first round (>= kmin) from which sp_mid can run the rounds up to t0:
// its input fits the blocks' chunks, and the last resident round still sums
// whole pairs in every block. t0 when there is none.
static int sp_mid_start(size_t n0, int kmin, int t0, int nb) {
  if (nb <= 0) return t0;
  for (int k = kmin; k < t0; k++) {
    const size_t n_in = k == 0 ? n0 : n0 >> (k - 1);
    const size_t last = (n0 >> (t0 - 1)) / nb;  // per block after the last fold
    if (n_in % nb == 0 && n_in / nb <= kSpMidMaxChunk && last >= 2) return k;
  }
  return t0;
}

// Grid of the resident grid rounds for a lane: kSpMidBlocks for a lane proving
// alone; for a pooled lane none, or kSpMidPoolBlocks with BITZ_POOL_MID=1 (as
// for the GKR middle rounds, gkr.cu).
int sp_mid_blocks(bool alone) {
  if (alone) return kSpMidBlocks;
  static const bool pool = [] {
    const char *e = getenv("BITZ_POOL_MID");
    return e && e[0] == '1';
  }();
  return pool ? kSpMidPoolBlocks : 0;
}

void spartan_prove(const SpartanArgs &a, Transcript &ts, SpartanScratch &sc, cudaStream_t s,
                   SpartanOut &out) {
  const FpCtx &c = a.ctx;
  const int nr = a.num_row_vars, nc = a.num_col_vars;
  const size_t R = (size_t)1 << nr, Cn = (size_t)1 << nc;
  ts.public_message(a.digest, 32);
  fp tau[kMaxFpPoint];
  for (int i = 0; i < nr; i++) {
    u128 t = ts.challenge_fp(a.q);
    tau[i] = fp_mul(fp{(uint64_t)t, (uint64_t)(t >> 64)}, c.r2, c);
  }
  fp *E = sc.t[0], *A = sc.t[1], *B = sc.t[2], *C = sc.t[3];
  fp *E2 = sc.t[4], *A2 = sc.t[5], *B2 = sc.t[6], *C2 = sc.t[7];
  fp_eq_table(tau, nr, c, E, sc.eq_scratch, s);
  k_products_to_fp<<<grid_for(R), kThreads, 0, s>>>(a.prod, a.rows, R, c, A, B, C);
  BZ_LAUNCH_CHECK();
  fp claim = fp_zero();
  out.outer.resize(4 * (size_t)nr);
  out.rx.resize(nr);
  size_t len = R;
  fp r = fp_zero();
  RoundChannel *ch = sc.channel;
  const bool resident = resident_rounds_enabled();
  bool tail = false;  // a resident tail kernel runs the remaining rounds
  // no other thread's device allocation while a tail kernel waits for this one
  ResidentScope gate(ch && resident);
  auto send_r = [&](fp x) {
    const uint64_t w[2] = {x.lo, x.hi};
    ch->send(w, 2);
  };
  // BITZ_ROUND_TRACE=1 prints the host time between consecutive round results
  static const bool trace = getenv("BITZ_ROUND_TRACE") != nullptr;
  auto t_prev = std::chrono::steady_clock::now();
  auto trace_round = [&](const char *what, int round, bool queued_kernel) {
    if (!trace) return;
    const auto now = std::chrono::steady_clock::now();
    fprintf(stderr, "[spartan] %s round %2d %s %7.2f us\n", what, round,
            queued_kernel ? "grid" : "tail",
            std::chrono::duration<double, std::micro>(now - t_prev).count());
    t_prev = now;
  };
  fp fin[3];
  // Queued mode: every outer round is queued now, then the tail. Round k > 0
  // folds at r_{k-1}, which the host posts as downbox publication d0 + k - 1
  // and the round before fetches into ctl[k-1] (the tail reads its first
  // challenge from the downbox itself); round k posts its message as
  // publication p0 + k.
  const bool queued = ch && resident && sc.ctl;
  try {
  if (queued) {
    int t0 = 0;  // the tail's first round: its table fits in shared memory
    while (t0 < nr && (t0 == 0 ? R : R >> (t0 - 1)) > (size_t)kSpTailN) t0++;
    const unsigned long long p0 = ch->next + 1, d0 = ch->down_next + 1;
    tail = true;  // from here a kernel of the lane may wait for this thread
    fp *set[2][4] = {{E, A, B, C}, {E2, A2, B2, C2}};
    // rounds km .. t0-1 resident (sp_mid, a grid of sc.mid_blocks blocks) when
    // a round's input fits the blocks' shared memory; the rounds before them
    // are queued launches
    const int km = sp_mid_start(R, 0, t0, sc.mid_blocks);
    BZ_CUDA(cudaMemsetAsync(sc.ctl, 0, sizeof(RoundCtl) * (nr + 1), s));
    for (int k = 0; k < km; k++) {
      const int fold = k > 0;
      const size_t n = k == 0 ? R : R >> (k - 1);
      fp *const *in = set[fold ? (k - 1) % 2 : 0];
      fp *const *to = set[k % 2];
      const size_t npairs = fold ? (n / 2 + 1) / 2 : n / 2;
      RoundLink lk{fold ? sc.ctl + (k - 1) : nullptr, k + 1 < km ? sc.ctl + k : nullptr,
                   ch->down_dev, d0 + k};
      k_outer_round<<<grid_for(npairs), kThreads, 0, s>>>(
          in[0], in[1], in[2], in[3], to[0], to[1], to[2], to[3], n, fold, 1, fp_zero(), c,
          sc.partial, Publish{ch->counter, ch->dev, p0 + k}, lk);
      BZ_LAUNCH_CHECK();
    }
    int cur_set = t0 > 0 ? (t0 - 1) % 2 : 0;
    if (km < t0) {
      const int si = km > 0 ? (km - 1) % 2 : 0;
      const size_t n_in = km == 0 ? R : R >> (km - 1);
      launch_sp_mid<4, 3>(SpTabs{{set[si][0], set[si][1], set[si][2], set[si][3]}},
                          SpTabs{{set[1 - si][0], set[1 - si][1], set[1 - si][2], set[1 - si][3]}},
                          n_in, km, t0, c, sc, p0, d0, s);
      cur_set = 1 - si;
    }
    // rounds kh .. nr-1 on the host, from the tail's handover
    const int kh = sp_host_round(ch, R, t0, nr);
    const unsigned long long hseq = p0 + (kh >= 0 ? kh : 0);
    std::vector<fp> host_tab[4];
    {
      fp *const *cur = set[cur_set];
      const size_t n = t0 == 0 ? R : R >> (t0 - 1);
      sp_outer_tail<<<1, kThreads, 0, s>>>(cur[0], cur[1], cur[2], cur[3], (int)n, t0 > 0,
                                           nr - t0, c, ch->dev, p0 + t0, ch->down_dev,
                                           d0 + (t0 > 0 ? t0 - 1 : 0), kh >= 0 ? kh - t0 : -1,
                                           ch->handover_dev, hseq);
      BZ_LAUNCH_CHECK();
      tail = true;
    }
    for (int round = 0; round < nr; round++) {
      if (kh >= 0 && round >= kh) {
        if (round == kh) {
          sp_take_handover(ch, s, hseq, 4, round == 0 ? R : R >> (round - 1), host_tab);
          tail = false;  // the tail kernel ends after the handover
        }
        if (round > 0) host_sp_fold(host_tab, 4, r, c);
        host_outer_sums(host_tab, c, sc.host);
        ch->arm();  // publication numbering as if the device had posted
      } else {
        if (round > 0) send_r(r);
        ch->arm();
        ch->wait(s, reinterpret_cast<uint64_t *>(sc.host), 6);
      }
      trace_round("outer", round, round < t0);
      fp co[4];
      r = round_message(ts, c, claim, sc.host, 4, a.q, co);
      for (int i = 0; i < 4; i++) out.outer[4 * round + i] = co[i];
      out.rx[round] = r;
    }
    if (kh >= 0) {  // the last fold leaves one entry per table
      host_sp_fold(host_tab, 4, r, c);
      for (int k = 0; k < 3; k++) fin[k] = host_tab[k + 1][0];
      ch->arm();
    } else {
      // the tail's last publication: the single entries of A, B and C
      send_r(r);
      ch->arm();
      ch->wait(s, reinterpret_cast<uint64_t *>(fin), 6);
    }
  } else {
  for (int round = 0; round < nr; round++) {
    int fold = round > 0;
    if (!tail && ch && resident && len <= (size_t)kSpTailN) {
      sp_outer_tail<<<1, kThreads, 0, s>>>(E, A, B, C, (int)len, fold, nr - round, c, ch->dev,
                                           ch->next + 1, ch->down_dev, ch->down_next + 1, -1,
                                           nullptr, 0);
      BZ_LAUNCH_CHECK();
      tail = true;
    }
    if (tail) {
      if (fold) {
        send_r(r);
        len /= 2;
      }
      ch->arm();
      ch->wait(s, reinterpret_cast<uint64_t *>(sc.host), 6);
    } else {
      size_t npairs = fold ? (len / 2 + 1) / 2 : len / 2;
      int g = grid_for(npairs);
      KernelProbe &probe = KernelProbe::get();
      const bool probed = probe.on("k_outer_round");
      if (probed) probe.before(s);
      k_outer_round<<<g, kThreads, 0, s>>>(E, A, B, C, E2, A2, B2, C2, len, fold, 1, r, c,
                                           sc.partial, Publish{nullptr, nullptr, 0},
                                           RoundLink{nullptr, nullptr, nullptr, 0});
      BZ_LAUNCH_CHECK();
      // four tables of 16-byte residues: read whole, written folded to half
      if (probed) probe.after(s, "k_outer_round", 16.0 * 4 * (double)len * (fold ? 1.5 : 1.0));
      host_partial_sum(sc.partial, g, 3, sc.sums, sc.host, c, s, sc.channel);
      if (fold) {
        std::swap(E, E2);
        std::swap(A, A2);
        std::swap(B, B2);
        std::swap(C, C2);
        len /= 2;
      }
    }
    fp co[4];
    r = round_message(ts, c, claim, sc.host, 4, a.q, co);
    for (int i = 0; i < 4; i++) out.outer[4 * round + i] = co[i];
    out.rx[round] = r;
  }
  if (tail) {
    // the tail's last publication: the single entries of A, B and C
    send_r(r);
    ch->arm();
    ch->wait(s, reinterpret_cast<uint64_t *>(fin), 6);
  } else {
    // the last fold leaves one entry per table
    k_outer_round<<<1, kThreads, 0, s>>>(E, A, B, C, E2, A2, B2, C2, len, 1, 0, r, c, sc.partial,
                                         Publish{nullptr, nullptr, 0},
                                         RoundLink{nullptr, nullptr, nullptr, 0});
    BZ_LAUNCH_CHECK();
    BZ_CUDA(cudaMemcpyAsync(&fin[0], A2, sizeof(fp), cudaMemcpyDeviceToHost, s));
    BZ_CUDA(cudaMemcpyAsync(&fin[1], B2, sizeof(fp), cudaMemcpyDeviceToHost, s));
    BZ_CUDA(cudaMemcpyAsync(&fin[2], C2, sizeof(fp), cudaMemcpyDeviceToHost, s));
    BZ_CUDA(stream_wait(s));
  }
  }
  } catch (...) {
    if (tail) {  // release the waiting kernel before the lane is reused
      ch->abort();
      stream_wait(s);
      ch->clear_down();
    }
    throw;
  }
  tail = false;
  uint8_t msg[48];
  for (int k = 0; k < 3; k++) {
    out.abc[k] = fin[k];
    put_canonical(msg + 16 * k, fin[k], c);
  }
  ts.public_message(msg, 48);
  u128 rhoc = ts.challenge_fp(a.q);
  fp rho = fp_mul(fp{(uint64_t)rhoc, (uint64_t)(rhoc >> 64)}, c.r2, c);
  fp rho2 = fp_mul(rho, rho, c);
  claim = fp_add(fp_add(fin[0], fp_mul(rho, fin[1], c), c), fp_mul(rho2, fin[2], c), c);
  // bind: eq(r_x) over the rows, then the column gather
  fp *eq = sc.t[0];
  fp_eq_table(out.rx.data(), nr, c, eq, sc.eq_scratch, s);
  k_bind_table<<<(a.ntab + 127) / 128, 128, 0, s>>>(a.tab_vals, a.tab_which, a.ntab, rho, rho2, c,
                                                     sc.tab);
  BZ_LAUNCH_CHECK();
  fp *D = sc.d[0], *W = sc.d[1], *D2 = sc.d[2], *W2 = sc.d[3];
  k_bind<<<grid_for(Cn), kThreads, 0, s>>>(a.csc_off, a.csc_row, a.csc_idx, sc.tab, eq, a.cols, Cn,
                                           c, D);
  BZ_LAUNCH_CHECK();
  {
    int g = grid_for(std::max<size_t>(a.col0_nnz, (size_t)a.n_bit_rows));
    k_bind_col0<<<g, kThreads, 0, s>>>(a.csc_row, a.csc_idx, sc.tab, eq, a.col0_nnz, a.bit_rows,
                                       a.n_bit_rows, rho2, c, sc.partial);
    BZ_LAUNCH_CHECK();
    k_bind_col0_finish<<<1, kThreads, 0, s>>>(sc.partial, g, c, D);
    BZ_LAUNCH_CHECK();
  }
  // inner sumcheck
  out.inner.resize(3 * (size_t)nc);
  out.ry.resize(nc);
  len = Cn;
  int w_bits = 1;
  fp dw[2];
  try {
  if (queued) {
    // as the outer rounds: round k > 0 folds at r_{k-1} (downbox publication
    // d0 + k - 1, fetched into ctl[k-1] by round k - 1) and posts p0 + k; W
    // comes from the packed bits of h until round 1 has folded them
    int t0 = 0;
    while (t0 < nc && (t0 == 0 ? Cn : Cn >> (t0 - 1)) > (size_t)kSpTailN) t0++;
    const unsigned long long p0 = ch->next + 1, d0 = ch->down_next + 1;
    tail = true;  // from here a kernel of the lane may wait for this thread
    fp *set[2][2] = {{D, W}, {D2, W2}};
    // W is read from the packed bits of h through round 1: resident rounds
    // start at 2 at the earliest
    const int km = sp_mid_start(Cn, 2, t0, sc.mid_blocks);
    BZ_CUDA(cudaMemsetAsync(sc.ctl, 0, sizeof(RoundCtl) * (nc + 1), s));
    for (int k = 0; k < km; k++) {
      const int fold = k > 0;
      const size_t n = k == 0 ? Cn : Cn >> (k - 1);
      fp *const *in = set[fold ? (k - 1) % 2 : 0];
      fp *const *to = set[k % 2];
      const size_t npairs = fold ? (n / 2 + 1) / 2 : n / 2;
      RoundLink lk{fold ? sc.ctl + (k - 1) : nullptr, k + 1 < km ? sc.ctl + k : nullptr,
                   ch->down_dev, d0 + k};
      k_inner_round<<<grid_for(npairs), kThreads, 0, s>>>(
          in[0], in[1], a.hbits, k <= 1 ? 1 : 0, to[0], to[1], n, fold, 1, fp_zero(), c,
          sc.partial, Publish{ch->counter, ch->dev, p0 + k}, lk);
      BZ_LAUNCH_CHECK();
    }
    int cur_set = t0 > 0 ? (t0 - 1) % 2 : 0;
    if (km < t0) {
      const int si = (km - 1) % 2;
      launch_sp_mid<2, 2>(SpTabs{{set[si][0], set[si][1], nullptr, nullptr}},
                          SpTabs{{set[1 - si][0], set[1 - si][1], nullptr, nullptr}},
                          Cn >> (km - 1), km, t0, c, sc, p0, d0, s);
      cur_set = 1 - si;
    }
    // rounds kh .. nc-1 on the host, from the tail's handover
    const int kh = sp_host_round(ch, Cn, t0, nc);
    const unsigned long long hseq = p0 + (kh >= 0 ? kh : 0);
    std::vector<fp> host_tab[2];
    {
      fp *const *cur = set[cur_set];
      const size_t n = t0 == 0 ? Cn : Cn >> (t0 - 1);
      sp_inner_tail<<<1, kThreads, 0, s>>>(cur[0], cur[1], a.hbits, t0 <= 1 ? 1 : 0, (int)n,
                                           t0 > 0, nc - t0, c, ch->dev, p0 + t0, ch->down_dev,
                                           d0 + (t0 > 0 ? t0 - 1 : 0), kh >= 0 ? kh - t0 : -1,
                                           ch->handover_dev, hseq);
      BZ_LAUNCH_CHECK();
      tail = true;
    }
    for (int round = 0; round < nc; round++) {
      if (kh >= 0 && round >= kh) {
        if (round == kh) {
          sp_take_handover(ch, s, hseq, 2, round == 0 ? Cn : Cn >> (round - 1), host_tab);
          tail = false;  // the tail kernel ends after the handover
        }
        if (round > 0) host_sp_fold(host_tab, 2, r, c);
        host_inner_sums(host_tab, c, sc.host);
        ch->arm();  // publication numbering as if the device had posted
      } else {
        if (round > 0) send_r(r);
        ch->arm();
        ch->wait(s, reinterpret_cast<uint64_t *>(sc.host), 4);
      }
      trace_round("inner", round, round < t0);
      fp co[3];
      r = round_message(ts, c, claim, sc.host, 3, a.q, co);
      for (int i = 0; i < 3; i++) out.inner[3 * round + i] = co[i];
      out.ry[round] = r;
    }
    if (kh >= 0) {  // the last fold leaves one entry per table
      host_sp_fold(host_tab, 2, r, c);
      dw[0] = host_tab[0][0];
      dw[1] = host_tab[1][0];
      ch->arm();
    } else {
      send_r(r);
      ch->arm();
      ch->wait(s, reinterpret_cast<uint64_t *>(dw), 4);
    }
  } else {
  for (int round = 0; round < nc; round++) {
    int fold = round > 0;
    if (!tail && ch && resident && len <= (size_t)kSpTailN) {
      sp_inner_tail<<<1, kThreads, 0, s>>>(D, W, a.hbits, w_bits, (int)len, fold, nc - round, c,
                                           ch->dev, ch->next + 1, ch->down_dev,
                                           ch->down_next + 1, -1, nullptr, 0);
      BZ_LAUNCH_CHECK();
      tail = true;
    }
    if (tail) {
      if (fold) {
        send_r(r);
        len /= 2;
      }
      ch->arm();
      ch->wait(s, reinterpret_cast<uint64_t *>(sc.host), 4);
    } else {
      size_t npairs = fold ? (len / 2 + 1) / 2 : len / 2;
      int g = grid_for(npairs);
      KernelProbe &probe = KernelProbe::get();
      const bool probed = probe.on("k_inner_round");
      if (probed) probe.before(s);
      k_inner_round<<<g, kThreads, 0, s>>>(D, W, a.hbits, w_bits, D2, W2, len, fold, 1, r, c,
                                           sc.partial, Publish{nullptr, nullptr, 0},
                                           RoundLink{nullptr, nullptr, nullptr, 0});
      BZ_LAUNCH_CHECK();
      // D (16-byte residues) and W (16-byte residues, or bits while w_bits is
      // set): read whole, written folded to half
      if (probed) {
        const double wbytes = w_bits ? (double)len / 8.0 : 16.0 * (double)len;
        probe.after(s, "k_inner_round",
                    16.0 * (double)len + wbytes + (fold ? 16.0 * (double)len : 0.0));
      }
      host_partial_sum(sc.partial, g, 2, sc.sums, sc.host, c, s, sc.channel);
      if (fold) {
        std::swap(D, D2);
        std::swap(W, W2);
        len /= 2;
        w_bits = 0;
      }
    }
    fp co[3];
    r = round_message(ts, c, claim, sc.host, 3, a.q, co);
    for (int i = 0; i < 3; i++) out.inner[3 * round + i] = co[i];
    out.ry[round] = r;
  }
  if (tail) {
    send_r(r);
    ch->arm();
    ch->wait(s, reinterpret_cast<uint64_t *>(dw), 4);
  } else {
    k_inner_round<<<1, kThreads, 0, s>>>(D, W, a.hbits, w_bits, D2, W2, len, 1, 0, r, c,
                                         sc.partial, Publish{nullptr, nullptr, 0},
                                         RoundLink{nullptr, nullptr, nullptr, 0});
    BZ_LAUNCH_CHECK();
    BZ_CUDA(cudaMemcpyAsync(&dw[0], D2, sizeof(fp), cudaMemcpyDeviceToHost, s));
    BZ_CUDA(cudaMemcpyAsync(&dw[1], W2, sizeof(fp), cudaMemcpyDeviceToHost, s));
    BZ_CUDA(stream_wait(s));
  }
  }
  } catch (...) {
    if (tail) {
      ch->abort();
      stream_wait(s);
      ch->clear_down();
    }
    throw;
  }
  out.d_at_ry = dw[0];
  out.final_claim = claim;
  out.ok = fp_mul(dw[0], dw[1], c).lo == claim.lo && fp_mul(dw[0], dw[1], c).hi == claim.hi;
}

// Per-block partial sums of D[y] * E[y] over n entries (mod q).
__global__ void k_fp_dot(const fp *__restrict__ D, const fp *__restrict__ E, size_t n, FpCtx c,
                         fp *partial) {
  fp acc[1] = {fp_zero()};
  for (size_t y = blockIdx.x * (size_t)blockDim.x + threadIdx.x; y < n;
       y += (size_t)gridDim.x * blockDim.x)
    acc[0] = fp_add(acc[0], fp_mul(D[y], E[y], c), c);
  block_fp_sum<1>(acc, c, partial);
}

fp spartan_matrix_eval(const SpartanArgs &a, const fp *rx, fp rho, const fp *ry,
                       SpartanScratch &sc, cudaStream_t s) {
  const FpCtx &c = a.ctx;
  const int nr = a.num_row_vars, nc = a.num_col_vars;
  const size_t Cn = (size_t)1 << nc;
  const fp rho2 = fp_mul(rho, rho, c);
  // the prover's bind at (r_x, rho): D(y) for every column y
  fp *eq = sc.t[0];
  fp_eq_table(rx, nr, c, eq, sc.eq_scratch, s);
  k_bind_table<<<(a.ntab + 127) / 128, 128, 0, s>>>(a.tab_vals, a.tab_which, a.ntab, rho, rho2, c,
                                                     sc.tab);
  BZ_LAUNCH_CHECK();
  fp *D = sc.d[0], *EY = sc.d[1];
  k_bind<<<grid_for(Cn), kThreads, 0, s>>>(a.csc_off, a.csc_row, a.csc_idx, sc.tab, eq, a.cols, Cn,
                                           c, D);
  BZ_LAUNCH_CHECK();
  {
    int g = grid_for(std::max<size_t>(a.col0_nnz, (size_t)a.n_bit_rows));
    k_bind_col0<<<g, kThreads, 0, s>>>(a.csc_row, a.csc_idx, sc.tab, eq, a.col0_nnz, a.bit_rows,
                                       a.n_bit_rows, rho2, c, sc.partial);
    BZ_LAUNCH_CHECK();
    k_bind_col0_finish<<<1, kThreads, 0, s>>>(sc.partial, g, c, D);
    BZ_LAUNCH_CHECK();
  }
  // then sum_y D(y) eq(r_y, y)
  fp_eq_table(ry, nc, c, EY, sc.eq_scratch, s);
  const int g = grid_for(Cn);
  k_fp_dot<<<g, kThreads, 0, s>>>(D, EY, Cn, c, sc.partial);
  BZ_LAUNCH_CHECK();
  k_fp_finalize<1><<<1, kThreads, 0, s>>>(sc.partial, g, c, sc.sums, Publish{nullptr, nullptr, 0});
  BZ_LAUNCH_CHECK();
  BZ_CUDA(cudaMemcpyAsync(sc.host, sc.sums, sizeof(fp), cudaMemcpyDeviceToHost, s));
  BZ_CUDA(stream_wait(s));
  return sc.host[0];
}

FpCtx make_fp_ctx(u128 q) {
  FpCtx c;
  c.q0 = (uint64_t)q;
  c.q1 = (uint64_t)(q >> 64);
  // -q^{-1} mod 2^64 by Newton iteration on the odd low word
  uint64_t inv = 1;
  for (int i = 0; i < 7; i++) inv *= 2 - c.q0 * inv;
  c.qinv = (uint64_t)0 - inv;
  u128 one = ((~(u128)0) % q + 1) % q;  // 2^128 mod q
  c.one = fp{(uint64_t)one, (uint64_t)(one >> 64)};
  u128 x = one;
  for (int i = 0; i < 128; i++) {
    x <<= 1;  // x < q < 2^126: no overflow
    if (x >= q) x -= q;
  }
  c.r2 = fp{(uint64_t)x, (uint64_t)(x >> 64)};
  return c;
}

u128 fp_canonical(fp mont, const FpCtx &c) {
  fp v = fp_mul(mont, fp{1, 0}, c);
  return (u128)v.lo | ((u128)v.hi << 64);
}

// Montgomery residues to canonical values (the 16-byte little-endian codec of
// crates/field/src/codec.rs:69-73), one thread per element.
__global__ void k_fp_canonical(const fp *__restrict__ in, size_t n, FpCtx c, fp *__restrict__ out) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
       k += (size_t)gridDim.x * blockDim.x)
    out[k] = fp_mul(in[k], fp{1, 0}, c);
}

void fp_canonical_device(const fp *in, size_t n, const FpCtx &c, fp *out, cudaStream_t s) {
  k_fp_canonical<<<grid_for(n), kThreads, 0, s>>>(in, n, c, out);
  BZ_LAUNCH_CHECK();
}

fp fp_to_mont(u128 v, const FpCtx &c) { return fp_mul(fp{(uint64_t)v, (uint64_t)(v >> 64)}, c.r2, c); }

// Every kernel of this file, loaded when the process's first lane on a device
// is made (lane_bootstrap, context.cpp).
void preload_spartan_kernels() {
  load_kernels({(const void *)k_fp_eq_factor,
                (const void *)k_fp_eq_expand,
                (const void *)k_products_to_fp,
                (const void *)k_outer_round,
                (const void *)k_inner_round,
                (const void *)k_fp_finalize<1>,
                (const void *)k_fp_finalize<2>,
                (const void *)k_fp_finalize<3>,
                (const void *)k_bind_table,
                (const void *)k_bind,
                (const void *)k_bind_col0,
                (const void *)k_bind_col0_finish,
                (const void *)sp_outer_tail,
                (const void *)sp_inner_tail,
                (const void *)sp_mid<4, 3>,
                (const void *)sp_mid<2, 2>,
                (const void *)k_fp_dot,
                (const void *)k_fp_canonical});
}

}  // namespace bz
