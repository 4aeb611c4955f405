// The post-GKR sumcheck (crates/post_gkr/src/lib.rs:121-148, sumcheck.rs:98-215):
// from the inner-product claim <rows (x) cols, f> = target over the committed
// bits f to an evaluation claim MLE[f](rho) = v.
//
// Device layout: the packed bits stay as the committed F128 words; the two
// tables of the quadratic rounds (weights W and values V) live in two
// ping-pong buffers of 2^(m-1) F128 each. Every round is one launch that
// folds both tables at the previous challenge and, from the freshly folded
// values still in registers, accumulates the next round's (a0, a2); the two
// sums leave the device as 32 bytes. Round 1 reads the bits directly: its
// coefficients are XOR sums of weights with no multiplication
// (lib.rs:189-239).
#include <vector>

#include "device.cuh"
#include "context.hpp"
#include "post_gkr.hpp"

namespace bz {

// One pair's share of the next round's (a0, a2) = (w0 v0, (w0 + w1)(v0 + v1)).
// A product whose V factor is zero is skipped: it adds nothing, and the
// committed bits past the witness's last one are zero padding (most of f for
// small statements), so whole stretches of V stay zero round after round.
__device__ __forceinline__ void pair_sums(wide &a0, wide &a2, f128 w0, f128 w1, f128 v0,
                                          f128 v1) {
  if (!gis_zero(v0)) wacc(a0, gmul_wide(w0, v0));
  const f128 dv = gadd(v0, v1);
  if (!gis_zero(dv)) wacc(a2, gmul_wide(gadd(w0, w1), dv));
}

// Round 1 message and the claim check, one warp per packed element: lane l
// owns bit pairs l and l + 32, so the warp reads the element's 128 row
// weights as one contiguous 2 KiB run.
__global__ void pg_first_message(const f128 *__restrict__ rows, int log_rows,
                                 const f128 *__restrict__ cols, const f128 *__restrict__ packed,
                                 size_t npacked, unsigned long long *acc, Publish pub) {
  const int lane = threadIdx.x & 31;
  const size_t warp = (blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5;
  const size_t nwarps = (gridDim.x * (size_t)blockDim.x) >> 5;
  const int shift = log_rows - 7;
  const size_t per_col_mask = ((size_t)1 << shift) - 1;
  wide a0 = wzero(), a2 = wzero(), ws = wzero();
  for (size_t e = warp; e < npacked; e += nwarps) {
    f128 word = ld(packed + e);
    if (gis_zero(word)) continue;  // no set bit: nothing to add (the warp's whole element)
    const f128 *rw = rows + ((e & per_col_mask) << 7);
    f128 s0 = mk(0, 0), s2 = mk(0, 0), sw = mk(0, 0);
    // Branch-free: each lane's two bits become all-ones / all-zero masks.
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int p = lane + 32 * h;
      const uint64_t w = h == 0 ? word.lo : word.hi;
      const int sh = 2 * lane;
      const uint64_t m0 = 0 - ((w >> sh) & 1ull);
      const uint64_t m1 = 0 - ((w >> (sh + 1)) & 1ull);
      const f128 w0 = ld(rw + 2 * p), w1 = ld(rw + 2 * p + 1);
      s0.lo ^= w0.lo & m0;
      s0.hi ^= w0.hi & m0;
      sw.lo ^= (w0.lo & m0) ^ (w1.lo & m1);
      sw.hi ^= (w0.hi & m0) ^ (w1.hi & m1);
      s2.lo ^= (w0.lo ^ w1.lo) & (m0 ^ m1);
      s2.hi ^= (w0.hi ^ w1.hi) & (m0 ^ m1);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      s0.lo ^= __shfl_xor_sync(0xffffffffu, s0.lo, off);
      s0.hi ^= __shfl_xor_sync(0xffffffffu, s0.hi, off);
      s2.lo ^= __shfl_xor_sync(0xffffffffu, s2.lo, off);
      s2.hi ^= __shfl_xor_sync(0xffffffffu, s2.hi, off);
      sw.lo ^= __shfl_xor_sync(0xffffffffu, sw.lo, off);
      sw.hi ^= __shfl_xor_sync(0xffffffffu, sw.hi, off);
    }
    if (lane == 0) {
      f128 c = ld(cols + (e >> shift));
      wacc(a0, gmul_wide(c, s0));
      wacc(a2, gmul_wide(c, s2));
      wacc(ws, gmul_wide(c, sw));
    }
  }
  f128 r0 = greduce(a0), r2 = greduce(a2), rw = greduce(ws);
  uint64_t v[6] = {r0.lo, r0.hi, r2.lo, r2.hi, rw.lo, rw.hi};
  block_xor_publish<6>(v, acc, pub);
}

// Round 1's fold: W'[c * R/2 + k] = cols[c] * fold(rows)[k] and V' the bound
// bit pairs {0, 1+r, r, 1} (lib.rs:241-283), fused with round 2's sums.
// Thread j writes the new pair (2j, 2j+1) of both tables.
__global__ void pg_first_fold(const f128 *__restrict__ rows, int log_rows,
                              const f128 *__restrict__ cols, const f128 *__restrict__ packed,
                              f128 r, f128 *__restrict__ w_out, f128 *__restrict__ v_out,
                              size_t npairs_out, unsigned long long *acc, Publish pub,
                              RoundLink lk) {
  __shared__ MulTable T;  // products by r through r's window table
  mul_table_build(T, r);
  const size_t half_rows = (size_t)1 << (log_rows - 1);
  // the bound bit pair (t = b0 + 2 b1) -> {0, 1 + r, r, 1}, by selects (no local array)
  auto bound_pair = [&](int t) {
    return t == 0 ? mk(0, 0) : t == 1 ? mk(r.lo ^ 1, r.hi) : t == 2 ? r : mk(1, 0);
  };
  wide a0 = wzero(), a2 = wzero();
  for (size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x; j < npairs_out;
       j += (size_t)gridDim.x * blockDim.x) {
    size_t i0 = 2 * j;
    size_t c = i0 / half_rows, k = i0 % half_rows;
    f128 col = ld(cols + c);
    f128 x0 = ld(rows + 2 * k), x1 = ld(rows + 2 * k + 1);
    f128 x2 = ld(rows + 2 * k + 2), x3 = ld(rows + 2 * k + 3);
    f128 w0 = gmul(col, gadd(x0, mul_table(T, gadd(x0, x1))));
    f128 w1 = gmul(col, gadd(x2, mul_table(T, gadd(x2, x3))));
    f128 word = ld(packed + (i0 >> 6));
    int p = (int)(i0 & 63);
    int t0 = bit128(word, 2 * p) | (bit128(word, 2 * p + 1) << 1);
    int t1 = bit128(word, 2 * p + 2) | (bit128(word, 2 * p + 3) << 1);
    f128 v0 = bound_pair(t0), v1 = bound_pair(t1);
    st(w_out + i0, w0);
    st(w_out + i0 + 1, w1);
    st(v_out + i0, v0);
    st(v_out + i0 + 1, v1);
    pair_sums(a0, a2, w0, w1, v0, v1);
  }
  f128 r0 = greduce(a0), r2 = greduce(a2);
  uint64_t v[4] = {r0.lo, r0.hi, r2.lo, r2.hi};
  block_xor_atomic<4>(v, acc);
  publish_link<4>(acc, pub, lk);
}

// A quadratic round (sumcheck.rs:63-95,198-215): fold W and V at r (entry =
// t0 + r (t0 + t1)) and accumulate the next round's (a0, a2) over the folded
// pairs. With emit == 0 only the fold runs (the last round).
__global__ void pg_round(const f128 *__restrict__ w_in, const f128 *__restrict__ v_in, f128 r,
                         f128 *__restrict__ w_out, f128 *__restrict__ v_out, size_t nout,
                         int emit, unsigned long long *acc, Publish pub, RoundLink lk) {
  if (lk.in) {  // a queued round: the challenge left by the kernel before
    unsigned long long w0, w1;
    if (!link_begin(lk, w0, w1)) return;
    r = mk(w0, w1);
  }
  __shared__ MulTable T;  // products by r through r's window table
  mul_table_build(T, r);
  wide a0 = wzero(), a2 = wzero();
  const size_t npairs = (nout + 1) / 2;
  for (size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x; j < npairs;
       j += (size_t)gridDim.x * blockDim.x) {
    size_t o = 2 * j;
    f128 w0 = ld(w_in + 2 * o), w1 = ld(w_in + 2 * o + 1);
    f128 v0 = ld(v_in + 2 * o), v1 = ld(v_in + 2 * o + 1);
    f128 fw0 = gadd(w0, mul_table(T, gadd(w0, w1)));
    f128 fv0 = gadd(v0, mul_table(T, gadd(v0, v1)));
    st(w_out + o, fw0);
    st(v_out + o, fv0);
    if (o + 1 < nout) {
      f128 w2 = ld(w_in + 2 * o + 2), w3 = ld(w_in + 2 * o + 3);
      f128 v2 = ld(v_in + 2 * o + 2), v3 = ld(v_in + 2 * o + 3);
      f128 fw1 = gadd(w2, mul_table(T, gadd(w2, w3)));
      f128 fv1 = gadd(v2, mul_table(T, gadd(v2, v3)));
      st(w_out + o + 1, fw1);
      st(v_out + o + 1, fv1);
      if (emit) pair_sums(a0, a2, fw0, fw1, fv0, fv1);
    }
  }
  if (emit) {
    f128 r0 = greduce(a0), r2 = greduce(a2);
    uint64_t v[4] = {r0.lo, r0.hi, r2.lo, r2.hi};
    block_xor_atomic<4>(v, acc);
    publish_link<4>(acc, pub, lk);
  }
}

// (a0, a2) over the pairs of W and V as they are (no fold).
__global__ void pg_sums(const f128 *__restrict__ w, const f128 *__restrict__ v, size_t n,
                        unsigned long long *acc, Publish pub) {
  wide a0 = wzero(), a2 = wzero();
  for (size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x; j < n / 2;
       j += (size_t)gridDim.x * blockDim.x) {
    f128 w0 = ld(w + 2 * j), w1 = ld(w + 2 * j + 1), v0 = ld(v + 2 * j), v1 = ld(v + 2 * j + 1);
    pair_sums(a0, a2, w0, w1, v0, v1);
  }
  f128 r0 = greduce(a0), r2 = greduce(a2);
  uint64_t o[4] = {r0.lo, r0.hi, r2.lo, r2.hi};
  block_xor_publish<4>(o, acc, pub);
}

void quad_sums(const f128 *w, const f128 *v, size_t n, unsigned long long *acc, Publish pub,
               cudaStream_t s) {
  pg_sums<<<grid_for(n / 2), kThreads, 0, s>>>(w, v, n, acc, pub);
  BZ_LAUNCH_CHECK();
}

// pg_round's algorithmic work for `nout` folded entries: each reads two
// entries of W and of V and writes one of each (96 B), binds both by r through
// r's window table, and each pair of them adds two wide products to the sums.
static void probe_pg_round(KernelProbe &probe, bool on, cudaStream_t s, size_t nout, int emit) {
  if (on)
    probe.after(s, "pg_round", 96.0 * (double)nout, 0.0,
                emit ? (double)(nout & ~(size_t)1) : 0.0, 2.0 * (double)nout);
}

void quad_fold(const f128 *w, const f128 *v, f128 r, f128 *w2, f128 *v2, size_t n, int emit,
               unsigned long long *acc, Publish pub, cudaStream_t s) {
  size_t nout = n / 2;
  KernelProbe &probe = KernelProbe::get();
  const bool probed = probe.on("pg_round");
  if (probed) probe.before(s);
  pg_round<<<grid_for((nout + 1) / 2), kThreads, 0, s>>>(w, v, r, w2, v2, nout, emit && nout >= 2,
                                                         acc, pub,
                                                         RoundLink{nullptr, nullptr, nullptr, 0});
  BZ_LAUNCH_CHECK();
  probe_pg_round(probe, probed, s, nout, emit && nout >= 2);
}

// h' = p(rho) with a1 = h + a2 (lib.rs:320-323).
static f128 advance(f128 claim, f128 a0, f128 a2, f128 r) {
  return gadd(a0, gmul(r, gadd(gadd(claim, a2), gmul(r, a2))));
}

// A round's result words: through the mailbox when the scratch has a
// channel, else by a copy and a stream sync.
// The tail hands its tables to the host at the first round whose input is at
// most this long (the host then folds and sums in a few microseconds a round).
constexpr size_t kPgHostLen = 64;

// One pg_tail round on the host: fold W and V at r (entry o = t0 + r (t0 +
// t1)); then the next round's (a0, a2) into sums, or, once one entry is left,
// the closing pair into pair. Returns true when the pair is formed.
static bool host_pg_round(std::vector<f128> &W, std::vector<f128> &V, f128 r, f128 sums[2],
                          f128 pair[2]) {
  const size_t n = W.size() / 2;
  for (size_t o = 0; o < n; o++) {
    W[o] = gadd(W[2 * o], gmul(r, gadd(W[2 * o], W[2 * o + 1])));
    V[o] = gadd(V[2 * o], gmul(r, gadd(V[2 * o], V[2 * o + 1])));
  }
  W.resize(n);
  V.resize(n);
  if (n == 1) {
    pair[0] = W[0];
    pair[1] = V[0];
    return true;
  }
  f128 a0 = mk(0, 0), a2 = mk(0, 0);
  for (size_t j = 0; j < n / 2; j++) {
    a0 = gadd(a0, gmul(W[2 * j], V[2 * j]));
    a2 = gadd(a2, gmul(gadd(W[2 * j], W[2 * j + 1]), gadd(V[2 * j], V[2 * j + 1])));
  }
  sums[0] = a0;
  sums[1] = a2;
  return false;
}

// The last rounds in one resident block, fed through the lane's downbox like
// the GKR tail: the tables (at most 2 * kPgTailN entries each) sit in shared
// memory; each round waits (bounded) for the host's challenge, folds both
// tables at it and posts the next round's (a0, a2), or, after the last fold,
// the closing pair (w, v). A missing challenge ends the kernel without a post.
constexpr int kPgTailN = 512;  // entries after the first fold
constexpr unsigned long long kPgWaitNs = 2000000000ull;

__global__ void __launch_bounds__(kThreads) pg_tail(const f128 *__restrict__ w_in,
                                                    const f128 *__restrict__ v_in, int len0,
                                                    Mailbox *mb, unsigned long long seq0,
                                                    const Mailbox *down, unsigned long long dseq0,
                                                    int hand_round, unsigned long long *handover,
                                                    unsigned long long hseq) {
  __shared__ f128 W[2 * kPgTailN], V[2 * kPgTailN];
  __shared__ unsigned long long chal[2];
  __shared__ int ok;
  for (int k = threadIdx.x; k < len0; k += blockDim.x) {
    W[k] = ld(w_in + k);
    V[k] = ld(v_in + k);
  }
  int len = len0;
  for (int round = 0; len > 1; round++) {
    if (round == hand_round) {  // the remaining rounds run on the host: W, then V
      __syncthreads();
      for (int k = threadIdx.x; k < 2 * len; k += blockDim.x) {
        const f128 x = k < len ? W[k] : V[k - len];
        handover_post(handover, hseq, 2 * k, x.lo);
        handover_post(handover, hseq, 2 * k + 1, x.hi);
      }
      return;
    }
    if (threadIdx.x == 0) ok = mailbox_wait_device(down, dseq0 + round, 2, chal, kPgWaitNs);
    __syncthreads();
    if (!ok) return;
    const f128 r = mk(chal[0], chal[1]);
    const unsigned long long seq = seq0 + round;
    const int nout = len / 2;
    // fold: read every pair first, then write (the halves overlap in place)
    f128 fw[2], fv[2];
    int cnt = 0;
    for (int o = threadIdx.x; o < nout; o += blockDim.x, cnt++) {
      fw[cnt] = gadd(W[2 * o], gmul(r, gadd(W[2 * o], W[2 * o + 1])));
      fv[cnt] = gadd(V[2 * o], gmul(r, gadd(V[2 * o], V[2 * o + 1])));
    }
    __syncthreads();
    cnt = 0;
    for (int o = threadIdx.x; o < nout; o += blockDim.x, cnt++) {
      W[o] = fw[cnt];
      V[o] = fv[cnt];
    }
    __syncthreads();
    len = nout;
    if (len == 1) {
      if (threadIdx.x == 0) {
        mailbox_post(mb, seq, 0, W[0].lo);
        mailbox_post(mb, seq, 1, W[0].hi);
        mailbox_post(mb, seq, 2, V[0].lo);
        mailbox_post(mb, seq, 3, V[0].hi);
      }
      return;
    }
    wide a0 = wzero(), a2 = wzero();
    for (int j = threadIdx.x; j < len / 2; j += blockDim.x) {
      f128 w0 = W[2 * j], w1 = W[2 * j + 1], v0 = V[2 * j], v1 = V[2 * j + 1];
      pair_sums(a0, a2, w0, w1, v0, v1);
    }
    f128 s0 = greduce(a0), s2 = greduce(a2);
    uint64_t vv[4] = {s0.lo, s0.hi, s2.lo, s2.hi};
    block_xor_reduce<4>(vv);
    if (threadIdx.x == 0)
      for (int k = 0; k < 4; k++) mailbox_post(mb, seq, k, vv[k]);
  }
}

static Publish arm(PostGkrScratch &sc) {
  return sc.channel ? sc.channel->arm() : Publish{nullptr, nullptr, 0};
}

static void round_read(PostGkrScratch &sc, const unsigned long long *d_acc, int words,
                       cudaStream_t s) {
  if (sc.channel) {
    sc.channel->wait(s, sc.host, words);
    return;
  }
  BZ_CUDA(cudaMemcpyAsync(sc.host, d_acc, words * 8, cudaMemcpyDeviceToHost, s));
  BZ_CUDA(stream_wait(s));
}

// The post-GKR rounds km .. t0-1 in one cooperative launch that stays
// resident (a lone lane). Tables fold on their low coordinate (pairs 2o,
// 2o + 1), so block b owns the contiguous chunk [b m, (b + 1) m) of W and V
// (m = n_in / kPgMidBlocks) and, after each fold, the first half of what it
// held: the chunk stays in shared memory across rounds. Round k folds at r_k,
// which block 0 reads from the downbox (publication d0 + k) and relays
// through ctl[k]; each block XORs its share of the next message into
// acc + 8 (k + acc_off) and the last block through the round (counted in
// ctl[k].done) posts it as publication p0 + k + 1 (the last round only with
// emit_last; the Ligerito levels run their folds here too). At the end each block
// writes its chunk to (w_out, v_out) for pg_tail. All blocks are resident
// together (cooperative launch), so the relay waits end; each is bounded all
// the same.
constexpr int kPgMidBlocks = 128;     // a lane proving alone
constexpr int kPgMidPoolBlocks = 32;  // a pooled lane, sharing the GPU with others
constexpr size_t kPgMidMaxChunk = 2048;  // entries per table per block

__global__ void __launch_bounds__(kThreads) pg_mid(const f128 *__restrict__ w_in,
                                                   const f128 *__restrict__ v_in, size_t n_in,
                                                   int km, int t0, int emit_last, int acc_off,
                                                   f128 *__restrict__ w_out,
                                                   f128 *__restrict__ v_out,
                                                   unsigned long long *acc, Mailbox *mb,
                                                   unsigned long long p0, const Mailbox *down,
                                                   unsigned long long d0, RoundCtl *ctl) {
  extern __shared__ f128 pgm[];
  __shared__ MulTable T;
  const size_t m = n_in / gridDim.x;
  f128 *W = pgm, *V = pgm + m;
  const size_t base = (size_t)blockIdx.x * m;
  for (size_t i = threadIdx.x; i < m; i += blockDim.x) {
    W[i] = ld(w_in + base + i);
    V[i] = ld(v_in + base + i);
  }
  __syncthreads();
  size_t len = m;
  for (int k = km; k < t0; k++) {
    unsigned long long rw[2];
    if (!resident_challenge(down, d0 + k, ctl + k, rw)) return;
    mul_table_build(T, mk(rw[0], rw[1]));
    // fold in place: every read, then every write
    constexpr int kPer = (int)(kPgMidMaxChunk / 2 / kThreads);
    f128 fw[kPer], fv[kPer];
    const size_t nout = len / 2;
#pragma unroll
    for (int q = 0; q < kPer; q++) {
      const size_t o = threadIdx.x + (size_t)q * kThreads;
      if (o < nout) {
        const f128 w0 = W[2 * o], w1 = W[2 * o + 1], v0 = V[2 * o], v1 = V[2 * o + 1];
        fw[q] = gadd(w0, mul_table(T, gadd(w0, w1)));
        fv[q] = gadd(v0, mul_table(T, gadd(v0, v1)));
      }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < kPer; q++) {
      const size_t o = threadIdx.x + (size_t)q * kThreads;
      if (o < nout) {
        W[o] = fw[q];
        V[o] = fv[q];
      }
    }
    __syncthreads();
    len = nout;
    if (k + 1 == t0 && !emit_last) break;  // the last fold: no message after it
    // the next message over the folded pairs
    wide a0 = wzero(), a2 = wzero();
    for (size_t j = threadIdx.x; j < len / 2; j += blockDim.x) {
      const f128 w0 = W[2 * j], w1 = W[2 * j + 1], v0 = V[2 * j], v1 = V[2 * j + 1];
      pair_sums(a0, a2, w0, w1, v0, v1);
    }
    const f128 r0 = greduce(a0), r2 = greduce(a2);
    uint64_t v[4] = {r0.lo, r0.hi, r2.lo, r2.hi};
    unsigned long long *ak = acc + 8 * (k + acc_off);
    block_xor_atomic<4>(v, ak);
    if (threadIdx.x == 0) {
      __threadfence();
      if (atomicAdd(&ctl[k].done, 1u) == gridDim.x - 1) {
        __threadfence();
#pragma unroll
        for (int q = 0; q < 4; q++) mailbox_post(mb, p0 + k + 1, q, atomicExch(ak + q, 0ull));
      }
    }
    __syncthreads();  // the chunk's reads of this round before the next fold
  }
  const size_t ob = (size_t)blockIdx.x * len;
  for (size_t i = threadIdx.x; i < len; i += blockDim.x) {
    st(w_out + ob + i, W[i]);
    st(v_out + ob + i, V[i]);
  }
}

// The first round pg_mid can start at: its input fits the blocks' chunks and
// the last resident round still sums whole pairs in every block; t0 when
// there is none.
bool pg_mid_fits_folds(size_t n, int rounds, int nb) {
  // a fold whose output is still summed needs two entries per block after it
  return nb > 0 && rounds >= 1 && n % nb == 0 && n / nb <= kPgMidMaxChunk &&
         (rounds < 2 || (n >> (rounds - 1)) / nb >= 2);
}

int pg_mid_start(size_t n1, int t0, int nb) {
  if (nb <= 0) return t0;
  for (int k = 0; k < t0; k++) {
    const size_t n_in = n1 >> k;
    if (n_in % nb == 0 && n_in / nb <= kPgMidMaxChunk && (n1 >> t0) / nb >= 2) return k;
  }
  return t0;
}

int pg_mid_blocks(bool alone) {
  if (alone) return kPgMidBlocks;
  static const bool pool = [] {
    const char *e = getenv("BITZ_POOL_MID");
    return e && e[0] == '1';
  }();
  return pool ? kPgMidPoolBlocks : 0;
}

void launch_pg_mid(const f128 *w_in, const f128 *v_in, size_t n_in, int km, int t0,
                   int emit_last, int acc_off, f128 *w_out, f128 *v_out, unsigned long long *acc,
                   RoundChannel *ch, unsigned long long p0, unsigned long long d0, RoundCtl *ctl,
                   int nb, cudaStream_t s) {
  static const int capacity = [] {
    int dev = 0, sms = 0, per_sm = 0;
    const size_t most = 2 * kPgMidMaxChunk * sizeof(f128);
    BZ_CUDA(cudaGetDevice(&dev));
    BZ_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    BZ_CUDA(cudaFuncSetAttribute(pg_mid, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)most));
    BZ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pg_mid, kThreads, most));
    return sms * per_sm;
  }();
  if (nb < 1 || nb > kPgMidBlocks || capacity < nb)
    throw CudaError("pg_mid: the blocks do not fit resident together");
  const size_t smem = 2 * (n_in / nb) * sizeof(f128);
  Mailbox *mb = ch->dev;
  const Mailbox *down = ch->down_dev;
  void *args[] = {&w_in, &v_in, &n_in, &km, &t0, &emit_last, &acc_off, &w_out,
                  &v_out, &acc, &mb,   &p0,   &down, &d0, &ctl};
  BZ_CUDA(cudaLaunchCooperativeKernel((const void *)pg_mid, dim3(nb), dim3(kThreads), args, smem,
                                      s));
  BZ_LAUNCH_CHECK();
}

int post_gkr_prove(const PostGkrArgs &a, Transcript &ts, PostGkrScratch &sc, cudaStream_t s,
                   f128 *point_out, f128 *value_out) {
  const int log_rows = a.log_rows, log_cols = a.log_cols;
  const size_t npacked = ((size_t)1 << (log_rows - 7)) << log_cols;
  const int m = log_rows + log_cols;
  const size_t n1 = (size_t)1 << (m - 1);  // table length after round 1
  if (sc.capacity < n1) return BZ_ERR_SCRATCH;
  unsigned long long *acc = sc.acc;
  BZ_CUDA(cudaMemsetAsync(acc, 0, sizeof(unsigned long long) * 8 * (m + 2), s));

  pg_first_message<<<grid_for(npacked * 32), kThreads, 0, s>>>(a.rows, log_rows, a.cols,
                                                                 a.packed, npacked, acc, arm(sc));
  BZ_LAUNCH_CHECK();
  round_read(sc, acc, 6, s);
  f128 a0 = mk(sc.host[0], sc.host[1]), a2 = mk(sc.host[2], sc.host[3]);
  f128 wsum = mk(sc.host[4], sc.host[5]);
  if (!geq(wsum, a.target)) {
    sc.claim_seen = wsum;
    return BZ_ERR_CLAIM;
  }

  uint64_t msg[4] = {a0.lo, a0.hi, a2.lo, a2.hi};
  ts.prover_message(msg, 32);
  ts.grind("bitz/pcs/sumcheck/v1", a.grind_bits);
  f128 r = ts.challenge_f128();
  f128 claim = advance(a.target, a0, a2, r);
  point_out[0] = r;

  // Round 1's fold fused with round 2's message.
  f128 *w = sc.w0, *v = sc.v0, *w2 = sc.w1, *v2 = sc.v1;
  const int rounds = m - 1;
  size_t len = n1;
  RoundChannel *ch = sc.channel;
  bool tail = false;  // pg_tail is resident and runs the remaining rounds
  const bool resident = resident_rounds_enabled();
  // Queued mode: the rounds above the tail are launched now behind the first
  // fold, then the tail. Loop iteration k folds at r_k (point_out[1 + k]),
  // which the host posts as downbox publication d0 + k; the kernel before
  // the k-th queued fold fetches it into ctl[k] (the tail reads its first
  // challenge itself), and the k-th fold posts publication p0 + k + 1.
  const bool queued = ch && resident && sc.ctl && rounds >= 1;
  int t0 = 0;  // the loop iteration at which the tail takes over
  while (t0 < rounds && (n1 >> t0) > (size_t)2 * kPgTailN) t0++;
  int kh = -1;                   // queued: the host runs iterations kh .. rounds-1
  unsigned long long hseq = 0;   // the tail's handover publication
  bool host_fin = false;         // the closing pair came from the host's rounds
  f128 fin_host[2] = {mk(0, 0), mk(0, 0)};
  // no other thread's device allocation while a round kernel waits for this one
  ResidentScope gate(ch && resident);
  try {
  {
    unsigned long long *acc1 = acc + 8;
    size_t npairs = n1 / 2;
    if (rounds >= 1) {
      const unsigned long long d0 = queued ? ch->down_next + 1 : 0;
      // rounds km .. t0-1 resident (pg_mid) when the lane proves alone; the
      // rounds before them are queued launches
      const int km = queued ? pg_mid_start(n1, t0, sc.mid_blocks) : t0;
      if (queued) BZ_CUDA(cudaMemsetAsync(sc.ctl, 0, sizeof(RoundCtl) * (rounds + 1), s));
      RoundLink lk{nullptr, queued && km > 0 ? sc.ctl : nullptr, queued ? ch->down_dev : nullptr,
                   d0};
      tail = queued;  // from here a kernel of the lane may wait for this thread
      pg_first_fold<<<grid_for(npairs), kThreads, 0, s>>>(a.rows, log_rows, a.cols, a.packed, r,
                                                          w, v, npairs, acc1, arm(sc), lk);
      BZ_LAUNCH_CHECK();
      if (queued) {
        const unsigned long long p0 = ch->next;  // the first fold's publication
        f128 *set[2][2] = {{sc.w0, sc.v0}, {sc.w1, sc.v1}};
        for (int k = 0; k < km; k++) {
          const size_t nout = (n1 >> k) / 2;
          f128 *const *in = set[k % 2];
          f128 *const *to = set[(k + 1) % 2];
          RoundLink lk2{sc.ctl + k, k + 1 < km ? sc.ctl + k + 1 : nullptr, ch->down_dev,
                        d0 + k + 1};
          pg_round<<<grid_for((nout + 1) / 2), kThreads, 0, s>>>(
              in[0], in[1], mk(0, 0), to[0], to[1], nout, 1, acc + 8 * (k + 2),
              Publish{ch->counter, ch->dev, p0 + k + 1}, lk2);
          BZ_LAUNCH_CHECK();
        }
        int cur_set = t0 % 2;
        if (km < t0) {
          f128 *const *in = set[km % 2];
          f128 *const *to = set[(km + 1) % 2];
          launch_pg_mid(in[0], in[1], n1 >> km, km, t0, 1, 2, to[0], to[1], acc, ch, p0, d0, sc.ctl,
                        sc.mid_blocks, s);
          cur_set = (km + 1) % 2;
        }
        f128 *const *cur = set[cur_set];
        // iterations kh .. rounds-1 on the host, from the tail's handover
        for (int k = t0; k < rounds && kh < 0 && ch->handover_host; k++)
          if ((n1 >> k) <= kPgHostLen) kh = k;
        hseq = p0 + (kh >= 0 ? kh : 0) + 1;
        pg_tail<<<1, kThreads, 0, s>>>(cur[0], cur[1], (int)(n1 >> t0), ch->dev, p0 + t0 + 1,
                                       ch->down_dev, d0 + t0, kh >= 0 ? kh - t0 : -1,
                                       ch->handover_dev, hseq);
        BZ_LAUNCH_CHECK();
      }
    }
  }
  if (queued) {
    std::vector<f128> HW, HV;
    f128 hsums[2];
    for (int k = 0; k < rounds; k++) {
      if (kh >= 0 && k > kh) {  // the host's own round
        sc.host[0] = hsums[0].lo;
        sc.host[1] = hsums[0].hi;
        sc.host[2] = hsums[1].lo;
        sc.host[3] = hsums[1].hi;
      } else {
        round_read(sc, nullptr, 4, s);
      }
      f128 m0 = mk(sc.host[0], sc.host[1]), m2 = mk(sc.host[2], sc.host[3]);
      uint64_t mm[4] = {m0.lo, m0.hi, m2.lo, m2.hi};
      ts.prover_message(mm, 32);
      ts.grind("bitz/pcs/sumcheck/v1", a.grind_bits);
      f128 rr = ts.challenge_f128();
      claim = advance(claim, m0, m2, rr);
      point_out[1 + k] = rr;
      if (kh >= 0 && k >= kh) {
        if (k == kh) {  // the tail's W and V as they stood before folding at rr
          const size_t len = n1 >> k;
          std::vector<uint64_t> words(4 * len);
          ch->wait_handover(s, hseq, words.data(), (int)words.size());
          tail = false;  // the tail kernel ends after the handover
          HW.resize(len);
          HV.resize(len);
          for (size_t i = 0; i < len; i++) {
            HW[i] = mk(words[2 * i], words[2 * i + 1]);
            HV[i] = mk(words[2 * (len + i)], words[2 * (len + i) + 1]);
          }
        }
        host_fin = host_pg_round(HW, HV, rr, hsums, fin_host);
        ch->arm();  // publication numbering as if the device had posted
        continue;
      }
      const uint64_t rw[2] = {rr.lo, rr.hi};
      ch->send(rw, 2);
      ch->arm();
    }
  } else {
  for (int k = 0; k < rounds; k++) {
    unsigned long long *ak = acc + 8 * (k + 1);
    round_read(sc, ak, 4, s);
    f128 m0 = mk(sc.host[0], sc.host[1]), m2 = mk(sc.host[2], sc.host[3]);
    uint64_t mm[4] = {m0.lo, m0.hi, m2.lo, m2.hi};
    ts.prover_message(mm, 32);
    ts.grind("bitz/pcs/sumcheck/v1", a.grind_bits);
    f128 rr = ts.challenge_f128();
    claim = advance(claim, m0, m2, rr);
    point_out[1 + k] = rr;
    if (!tail && ch && resident && len <= (size_t)2 * kPgTailN) {
      pg_tail<<<1, kThreads, 0, s>>>(w, v, (int)len, ch->dev, ch->next + 1, ch->down_dev,
                                     ch->down_next + 1, -1, nullptr, 0);
      BZ_LAUNCH_CHECK();
      tail = true;
    }
    if (tail) {
      const uint64_t rw[2] = {rr.lo, rr.hi};
      ch->send(rw, 2);
      ch->arm();
      len /= 2;
      continue;
    }
    size_t nout = len / 2;
    int emit = nout >= 2;
    KernelProbe &probe = KernelProbe::get();
    const bool probed = probe.on("pg_round");
    if (probed) probe.before(s);
    pg_round<<<grid_for((nout + 1) / 2), kThreads, 0, s>>>(w, v, rr, w2, v2, nout, emit,
                                                           acc + 8 * (k + 2),
                                                           emit ? arm(sc) : Publish{nullptr, nullptr, 0},
                                                           RoundLink{nullptr, nullptr, nullptr, 0});
    BZ_LAUNCH_CHECK();
    probe_pg_round(probe, probed, s, nout, emit);
    f128 *t = w;
    w = w2;
    w2 = t;
    t = v;
    v = v2;
    v2 = t;
    len = nout;
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
  f128 fin[2];
  if (host_fin) {
    fin[0] = fin_host[0];
    fin[1] = fin_host[1];
  } else if (tail) {
    // the tail's last publication is the closing pair
    ch->wait(s, sc.host, 4);
    fin[0] = mk(sc.host[0], sc.host[1]);
    fin[1] = mk(sc.host[2], sc.host[3]);
  } else {
    BZ_CUDA(cudaMemcpyAsync(fin, w, 16, cudaMemcpyDeviceToHost, s));
    BZ_CUDA(cudaMemcpyAsync(fin + 1, v, 16, cudaMemcpyDeviceToHost, s));
    BZ_CUDA(stream_wait(s));
  }
  *value_out = fin[1];
  ts.prover_f128(fin[1]);
  return geq(gmul(fin[0], fin[1]), claim) ? BZ_OK : BZ_ERR_INTERNAL;
}

// Every kernel of this file, loaded when the process's first lane on a device
// is made (lane_bootstrap, context.cpp).
void preload_post_gkr_kernels() {
  load_kernels({(const void *)pg_first_message,
                (const void *)pg_first_fold,
                (const void *)pg_round,
                (const void *)pg_sums,
                (const void *)pg_tail,
                (const void *)pg_mid});
}

}  // namespace bz
