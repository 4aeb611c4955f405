// The grand-product GKR (crates/gkr/src/lib.rs:24-81,88-240,785-897).
//
// Leaf (b << s) | c of the product tree is the row image b where column c has
// bit b set, one elsewhere (crates/prover/src/reduce.rs:1-5); node k of each
// layer multiplies nodes k and k + half of the layer below. The reference
// keeps layers 0-2 in 16-entry lookup tables to save CPU memory traffic;
// here every layer is a dense device table (2^(7+s) leaves at most, 512 MiB
// at s = 18), built by one pass per layer. Round messages are exact field
// values, so the dense sums equal the reference's bucketed ones bit for bit.
//
// A layer sumcheck binds its point's top coordinate first. Round i splits
// the children into L = C[0, 2^n) and R = C[2^n, 2^(n+1)), each into halves
// at 2^i. One launch per round binds round i+1 in place, sums the eq table
// down to round i's (eq_i[x] = eq_{i+1}[x] + eq_{i+1}[x + 2^i], summing out
// coordinate i), and accumulates round i's two sums from the freshly bound
// values; 32 bytes leave the device per round.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <vector>

#include "context.hpp"
#include "eq.cuh"
#include "gkr.hpp"

namespace bz {

__global__ void gkr_leaves(const f128 *__restrict__ cols, int s, const f128 *__restrict__ images,
                           f128 *__restrict__ out) {
  const size_t total = (size_t)128 << s;
  const size_t cmask = ((size_t)1 << s) - 1;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < total;
       k += (size_t)gridDim.x * blockDim.x) {
    size_t c = k & cmask;
    int b = (int)(k >> s);
    f128 word = ld(cols + c);
    st(out + k, bit128(word, b) ? ld(images + b) : mk(1, 0));
  }
}

// Padding: the low s bits of every layer index are the column, and a column at
// or beyond `live` has only one-valued nodes. Whenever entry x of a half is
// such a column, so are x + h and x + 2h (same column, or a higher one below
// 2^s), so a thread whose x is padded binds nothing (1 + r (1 + 1) = 1) and
// adds e * 1 * 1 = e to the first sum and e * 0 * 0 = 0 to the second.
__device__ __forceinline__ bool padded(size_t x, size_t colmask, size_t live) {
  return (x & colmask) >= live;
}

__global__ void gkr_parent(const f128 *__restrict__ child, size_t half, f128 *__restrict__ out,
                           size_t colmask, size_t live) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < half;
       k += (size_t)gridDim.x * blockDim.x)
    st(out + k, padded(k, colmask, live) ? mk(1, 0) : gmul(ld(child + k), ld(child + half + k)));
}

// Queued rounds (the round link in device.cuh): every bind round of a layer
// is queued at the layer's start, so no round waits for a launch from the
// host.

// Every thread calls it; false when the chain has stopped (the block returns).
__device__ __forceinline__ bool round_begin(const RoundLink &lk, f128 r_arg, f128 &r) {
  if (!lk.in) {
    r = r_arg;
    return true;
  }
  unsigned long long w0, w1;
  const bool ok = link_begin(lk, w0, w1);
  r = mk(w0, w1);
  return ok;
}

// publish<4>, then the last block fetches the next challenge for `out`.
__device__ __forceinline__ void round_end(unsigned long long *acc, const Publish &p,
                                          const RoundLink &lk) {
  publish_link<4>(acc, p, lk);
}

// A layer's start. The eq table over the n - 1 coordinates below the top one
// is the product of two factor tables, lo over the first a coordinates and
// hi over the other b: block 0 builds lo and clears the layer's round
// accumulators, block 1 builds hi and clears the round controls; the top
// sums kernel multiplies the factors out as it reads them.
__global__ void __launch_bounds__(kThreads) gkr_layer_setup(Point p, int a, int b, f128 *lo,
                                                            f128 *hi, unsigned long long *acc,
                                                            int acc_words, RoundCtl *ctl,
                                                            int nctl) {
  __shared__ MulTable T;
  if (blockIdx.x == 0) {
    for (int k = threadIdx.x; k < acc_words; k += blockDim.x) acc[k] = 0;
    eq_factor_block(p, 0, a, lo, T);
  } else {
    for (int k = threadIdx.x; k < nctl; k += blockDim.x) ctl[k] = RoundCtl{0, 0, 0, 0, 0};
    eq_factor_block(p, a, b, hi, T);
  }
}

// Round i's sums (round_sums, lib.rs:164-216) before any bind: the top round.
// Entry x of the eq table is lo[x mod 2^a] * hi[x >> a]; it is stored for the
// bind rounds as it is formed.
__global__ void gkr_top_sums(const f128 *__restrict__ c, size_t n_half, size_t h,
                             const f128 *__restrict__ lo, int a, const f128 *__restrict__ hi,
                             f128 *__restrict__ eq, int at_one, unsigned long long *acc,
                             Publish pub, RoundLink lk, size_t colmask, size_t live) {
  const f128 *L = c, *R = c + n_half;
  const size_t amask = ((size_t)1 << a) - 1;
  wide sb = wzero(), si = wzero();
  for (size_t x = blockIdx.x * (size_t)blockDim.x + threadIdx.x; x < h;
       x += (size_t)gridDim.x * blockDim.x) {
    const f128 e = gmul(ld(lo + (x & amask)), ld(hi + (x >> a)));
    st(eq + x, e);
    if (padded(x, colmask, live)) {
      sb.w0 ^= e.lo;
      sb.w1 ^= e.hi;
      continue;
    }
    f128 l0 = ld(L + x), l1 = ld(L + h + x), r0 = ld(R + x), r1 = ld(R + h + x);
    f128 lb = at_one ? l1 : l0, rb = at_one ? r1 : r0;
    wacc(sb, gmul_wide(gmul(e, lb), rb));
    wacc(si, gmul_wide(gmul(e, gadd(l1, l0)), gadd(r1, r0)));
  }
  f128 sa = greduce(sb), sbb = greduce(si);
  uint64_t v[4] = {sa.lo, sa.hi, sbb.lo, sbb.hi};
  block_xor_atomic<4>(v, acc);
  round_end(acc, pub, lk);
}

// Bind round i+1 at r (halves of 2^(i+1)), derive eq_i in place, and sum
// round i (halves of 2^i). Thread x < 2^i owns entries x and x + 2^i.
__global__ void gkr_bind_sums(f128 *__restrict__ c, size_t n_half, size_t h, f128 r_arg,
                              f128 *__restrict__ eq, int at_one, unsigned long long *acc,
                              Publish pub, RoundLink lk, size_t colmask, size_t live) {
  f128 r;
  if (!round_begin(lk, r_arg, r)) return;
  __shared__ MulTable T;  // the binds by r through r's window table
  mul_table_build(T, r);
  f128 *L = c, *R = c + n_half;
  const size_t h2 = 2 * h;
  wide sb = wzero(), si = wzero();
  for (size_t x = blockIdx.x * (size_t)blockDim.x + threadIdx.x; x < h;
       x += (size_t)gridDim.x * blockDim.x) {
    if (padded(x, colmask, live)) {
      f128 e = gadd(ld(eq + x), ld(eq + x + h));
      st(eq + x, e);
      sb.w0 ^= e.lo;
      sb.w1 ^= e.hi;
      continue;
    }
    f128 a0 = ld(L + x), a1 = ld(L + x + h2), b0 = ld(L + x + h), b1 = ld(L + x + h + h2);
    f128 l0 = gadd(a0, mul_table(T, gadd(a1, a0)));
    f128 l1 = gadd(b0, mul_table(T, gadd(b1, b0)));
    f128 c0 = ld(R + x), c1 = ld(R + x + h2), d0 = ld(R + x + h), d1 = ld(R + x + h + h2);
    f128 r0 = gadd(c0, mul_table(T, gadd(c1, c0)));
    f128 r1 = gadd(d0, mul_table(T, gadd(d1, d0)));
    st(L + x, l0);
    st(L + x + h, l1);
    st(R + x, r0);
    st(R + x + h, r1);
    f128 e = gadd(ld(eq + x), ld(eq + x + h));
    st(eq + x, e);
    f128 lb = at_one ? l1 : l0, rb = at_one ? r1 : r0;
    wacc(sb, gmul_wide(gmul(e, lb), rb));
    wacc(si, gmul_wide(gmul(e, gadd(l1, l0)), gadd(r1, r0)));
  }
  f128 a = greduce(sb), b = greduce(si);
  uint64_t v[4] = {a.lo, a.hi, b.lo, b.hi};
  block_xor_atomic<4>(v, acc);
  round_end(acc, pub, lk);
}

// gkr_bind_sums by tiles, for rounds where few elements leave each thread's
// chain of eight products (four binds, two with e, two wide) as the round's
// latency. A block takes a tile of kMidTile elements and works it in three
// levels, each product of a level on its own thread: the 4 * kMidTile binds
// by r through the block's window table (2 per thread), then the
// 2 * kMidTile products with e, then the 2 * kMidTile wide products. Same
// values, same sums as gkr_bind_sums.
constexpr int kTailH = 256;  // gkr_tail's first round binds at most 4 kTailH entries per half
constexpr int kMidThreads = 256;
constexpr int kMidTile = 128;
constexpr size_t kMidMaxH = (size_t)1 << 15;  // larger rounds are issue bound: gkr_bind_sums
static_assert(kMidThreads == 2 * kMidTile && kMidThreads == kThreads, "one product per thread");

// Shared memory of one tile: the window table of r, the tile's bound
// entries L[x], L[x+h], R[x], R[x+h], its eq entries and the products with e.
struct TileShared {
  MulTable T;
  f128 B[4][kMidTile];
  f128 E[kMidTile], P[kMidTile], Q[kMidTile];
};

// L2 loads: a resident kernel reads entries that other blocks wrote in its
// previous round, which this SM's L1 may hold stale.
__device__ __forceinline__ f128 ld_cg(const f128 *p) {
  const ulonglong2 v = __ldcg(reinterpret_cast<const ulonglong2 *>(p));
  return mk(v.x, v.y);
}

// Elements [x0, x0 + kMidTile) of a bind round with S.T built for r: the
// three levels, the tile's share of the first message summed by even
// threads into acc_w, of the second by odd ones. Every thread calls it; it
// ends with the block synchronised.
__device__ __forceinline__ void bind_tile(TileShared &S, f128 *L, f128 *R, f128 *eq, size_t h,
                                          size_t x0, int at_one, size_t colmask, size_t live,
                                          wide &acc_w) {
  const size_t h2 = 2 * h;
  const int t = threadIdx.x;
  // level 1: entry (k, q) of the tile is L[x], L[x+h], R[x], R[x+h] for q = 0..3
#pragma unroll
  for (int it = 0; it < 4 * kMidTile / kMidThreads; it++) {
    const int u = t + it * kMidThreads;
    const int k = u >> 2, q = u & 3;
    const size_t x = x0 + k;
    if (x >= h) continue;
    if (q == 0) {
      const f128 e = gadd(ld_cg(eq + x), ld_cg(eq + x + h));
      st(eq + x, e);
      S.E[k] = e;
    }
    f128 v = mk(1, 0);  // a padded column stays one
    if (!padded(x, colmask, live)) {
      f128 *tab = q < 2 ? L : R;
      const size_t at = x + (q & 1) * h;
      const f128 a0 = ld_cg(tab + at), a1 = ld_cg(tab + at + h2);
      v = gadd(a0, mul_table(S.T, gadd(a1, a0)));
      st(tab + at, v);
    }
    S.B[q][k] = v;
  }
  __syncthreads();
  // level 2: P = e * L_b, Q = e * (L_1 + L_0)
  {
    const int k = t >> 1;
    const size_t x = x0 + k;
    if (x < h) {
      const f128 e = S.E[k];
      if (padded(x, colmask, live)) {  // e * 1 and e * 0
        if (t & 1)
          S.Q[k] = mk(0, 0);
        else
          S.P[k] = e;
      } else if (t & 1) {
        S.Q[k] = gmul(e, gadd(S.B[1][k], S.B[0][k]));
      } else {
        S.P[k] = gmul(e, at_one ? S.B[1][k] : S.B[0][k]);
      }
    }
  }
  __syncthreads();
  // level 3: P * R_b into the first sum, Q * (R_1 + R_0) into the second
  {
    const int k = t >> 1;
    const size_t x = x0 + k;
    if (x < h) {
      if (padded(x, colmask, live)) {  // P * 1 and Q * 0
        if (!(t & 1)) {
          acc_w.w0 ^= S.P[k].lo;
          acc_w.w1 ^= S.P[k].hi;
        }
      } else if (t & 1) {
        wacc(acc_w, gmul_wide(S.Q[k], gadd(S.B[3][k], S.B[2][k])));
      } else {
        wacc(acc_w, gmul_wide(S.P[k], at_one ? S.B[3][k] : S.B[2][k]));
      }
    }
  }
  __syncthreads();  // the tile's tables before the next tile overwrites them
}

// The block's four words of the round's sums (even threads hold the first
// message, odd ones the second).
__device__ __forceinline__ void tile_words(const wide &acc_w, uint64_t (&v)[4]) {
  const f128 s = greduce(acc_w);
  const bool odd = threadIdx.x & 1;
  v[0] = odd ? 0 : s.lo;
  v[1] = odd ? 0 : s.hi;
  v[2] = odd ? s.lo : 0;
  v[3] = odd ? s.hi : 0;
}

__global__ void __launch_bounds__(kMidThreads) gkr_round(
    f128 *__restrict__ c, size_t n_half, size_t h, f128 r_arg, f128 *__restrict__ eq, int at_one,
    unsigned long long *acc, Publish pub, RoundLink lk, size_t colmask, size_t live) {
  f128 r;
  if (!round_begin(lk, r_arg, r)) return;
  __shared__ TileShared S;
  mul_table_build(S.T, r);
  wide acc_w = wzero();
  for (size_t x0 = (size_t)blockIdx.x * kMidTile; x0 < h; x0 += (size_t)gridDim.x * kMidTile)
    bind_tile(S, c, c + n_half, eq, h, x0, at_one, colmask, live, acc_w);
  uint64_t v[4];
  tile_words(acc_w, v);
  block_xor_atomic<4>(v, acc);
  round_end(acc, pub, lk);
}

// The middle rounds of a layer (bind r_i for i = i_hi .. i_lo) in one
// cooperative launch of B blocks that stays resident, with the layer's live
// entries in shared memory from the first round to the last. With the period
// P = B kMidRuns, block b owns the positions whose residue mod P lies in
// [b kMidRuns, (b + 1) kMidRuns); slot m of the block is position
// P (m / kMidRuns) + b kMidRuns + m % kMidRuns. Every h of these rounds is a
// multiple of P, so positions y, y + h, y + 2h, y + 3h belong to one block and
// sit at slots m, m + E, m + 2E, m + 3E (E = h / B elements per block): each
// round binds slot m < 2E from slots m and m + 2E in place and sums elements
// j < E from slots j and j + E. Blocks share nothing but the challenge and the
// sums: block 0 reads r_i from the downbox (publication d0 + n - 1 - i) and
// relays it through ctl; each block adds its share of the sums into acc and
// the last one through the round posts them as publication p0 + n - i. The
// entries the tail kernel reads are written back at the end. All blocks are
// resident together (cooperative launch), so the relay waits end; each is
// bounded all the same. A lane proving alone uses kMidBlocks blocks; a pooled
// lane, which shares the GPU with other lanes' kernels, kMidPoolBlocks (each
// block then holds four times the entries, 192 KB of shared memory at the
// largest round).
constexpr int kMidBlocks = 128;      // a lane proving alone
constexpr int kMidPoolBlocks = 32;   // a pooled lane, sharing the GPU with others
constexpr int kMidRuns = 4;
static_assert((size_t)kMidBlocks * kMidRuns <= 2 * (size_t)kTailH,
              "the tail starts below the middle rounds");

// The period is gridDim.x kMidRuns positions: the grid is kMidBlocks blocks
// or fewer.
__device__ __forceinline__ size_t mid_pos(size_t m) {
  const size_t period = (size_t)gridDim.x * kMidRuns;
  return period * (m / kMidRuns) + (size_t)blockIdx.x * kMidRuns + m % kMidRuns;
}

// Dynamic shared memory for e0 elements: L and R at slots < 2 e0 (lo) and
// [2 e0, 4 e0) (hi), eq at slots < 2 e0, and the products with e.
__host__ __device__ constexpr size_t mid_smem_bytes(size_t e0) { return 12 * e0 * sizeof(f128); }

__global__ void __launch_bounds__(kMidThreads) gkr_mid(
    f128 *__restrict__ c, size_t n_half, int n, int i_hi, int i_lo, f128 *__restrict__ eq,
    unsigned long long at_one_mask, unsigned long long *acc_base, Mailbox *mb,
    unsigned long long p0, const Mailbox *down, unsigned long long d0, RoundCtl *ctl,
    size_t colmask, size_t live) {
  extern __shared__ f128 dyn[];
  __shared__ MulTable T;
  const int t = threadIdx.x;
  const size_t e0 = ((size_t)1 << (i_hi - 1)) / gridDim.x;
  f128 *SL = dyn, *SL1 = dyn + 2 * e0, *SR = dyn + 4 * e0, *SR1 = dyn + 6 * e0;
  f128 *EQ = dyn + 8 * e0, *P = dyn + 10 * e0, *Q = dyn + 11 * e0;
  f128 *L = c, *R = c + n_half;
  {
    const size_t h0 = (size_t)1 << (i_hi - 1);
    for (size_t m = t; m < 2 * e0; m += kMidThreads) {
      const size_t y = mid_pos(m);
      SL[m] = ld(L + y);
      SL1[m] = ld(L + y + 2 * h0);
      SR[m] = ld(R + y);
      SR1[m] = ld(R + y + 2 * h0);
      EQ[m] = ld(eq + y);
    }
  }
  for (int i = i_hi; i >= i_lo; i--) {
    RoundCtl *cl = ctl + (n - 1 - i);
    unsigned long long rw[2];
    if (!resident_challenge(down, d0 + (n - 1 - i), cl, rw)) return;
    mul_table_build(T, mk(rw[0], rw[1]));
    const size_t e = ((size_t)1 << (i - 1)) / gridDim.x;
    const int at_one = (int)((at_one_mask >> (i - 1)) & 1);
    // the upper half of the live slots: separate arrays in the first round,
    // slots [2e, 4e) of the lower ones after it
    const f128 *hl = i == i_hi ? SL1 : SL + 2 * e, *hr = i == i_hi ? SR1 : SR + 2 * e;
    // level 1: the 2e slots of L and of R bound at r; the eq table summed down
    for (size_t u = t; u < 4 * e; u += kMidThreads) {
      const bool right = u >= 2 * e;
      const size_t m = right ? u - 2 * e : u;
      if (padded(mid_pos(m), colmask, live)) continue;  // stays one
      f128 *lo = right ? SR : SL;
      const f128 a0 = lo[m];
      lo[m] = gadd(a0, mul_table(T, gadd((right ? hr : hl)[m], a0)));
    }
    for (size_t j = t; j < e; j += kMidThreads) EQ[j] = gadd(EQ[j], EQ[j + e]);
    __syncthreads();
    // level 2: P = e * L_b, Q = e * (L_1 + L_0) for the e elements
    for (size_t u = t; u < 2 * e; u += kMidThreads) {
      const size_t j = u >> 1;
      const f128 ev = EQ[j];
      if (padded(mid_pos(j), colmask, live)) {  // e * 1 and e * 0
        if (u & 1)
          Q[j] = mk(0, 0);
        else
          P[j] = ev;
      } else if (u & 1) {
        Q[j] = gmul(ev, gadd(SL[j + e], SL[j]));
      } else {
        P[j] = gmul(ev, at_one ? SL[j + e] : SL[j]);
      }
    }
    __syncthreads();
    // level 3: P * R_b into the first sum, Q * (R_1 + R_0) into the second
    wide acc_w = wzero();
    for (size_t u = t; u < 2 * e; u += kMidThreads) {
      const size_t j = u >> 1;
      if (padded(mid_pos(j), colmask, live)) {  // P * 1 and Q * 0
        if (!(u & 1)) {
          acc_w.w0 ^= P[j].lo;
          acc_w.w1 ^= P[j].hi;
        }
      } else if (u & 1) {
        wacc(acc_w, gmul_wide(Q[j], gadd(SR[j + e], SR[j])));
      } else {
        wacc(acc_w, gmul_wide(P[j], at_one ? SR[j + e] : SR[j]));
      }
    }
    uint64_t v[4];
    tile_words(acc_w, v);  // kMidThreads is even: thread parity = u parity
    unsigned long long *acc = acc_base + 4 * (n - i);
    block_xor_atomic<4>(v, acc);  // synchronises the block: P, Q, SL, SR free again
    if (t == 0) {
      __threadfence();
      const unsigned int prev = atomicAdd(&cl->done, 1u);
      if (prev == gridDim.x - 1) {
        __threadfence();
#pragma unroll
        for (int k = 0; k < 4; k++) mailbox_post(mb, p0 + (n - i), k, atomicExch(acc + k, 0ull));
      }
    }
  }
  // the live entries after round i_lo: L and R below 2 h, eq below h
  const size_t e = ((size_t)1 << (i_lo - 1)) / gridDim.x;
  for (size_t m = t; m < 2 * e; m += kMidThreads) {
    const size_t y = mid_pos(m);
    st(L + y, SL[m]);
    st(R + y, SR[m]);
  }
  for (size_t j = t; j < e; j += kMidThreads) st(eq + mid_pos(j), EQ[j]);
}

// The bind after round 0: one pair left in each half. Delivered through the
// mailbox when publishing, else to out[0..2).
__global__ void gkr_final_bind(const f128 *__restrict__ c, size_t n_half, f128 r, f128 *out,
                               Publish pub) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    f128 l0 = ld(c), l1 = ld(c + 1), r0 = ld(c + n_half), r1 = ld(c + n_half + 1);
    f128 lr = gadd(l0, gmul(r, gadd(l1, l0)));
    f128 rr = gadd(r0, gmul(r, gadd(r1, r0)));
    if (pub.counter) {
      mailbox_post(pub.mailbox, pub.seq, 0, lr.lo);
      mailbox_post(pub.mailbox, pub.seq, 1, lr.hi);
      mailbox_post(pub.mailbox, pub.seq, 2, rr.lo);
      mailbox_post(pub.mailbox, pub.seq, 3, rr.hi);
    } else {
      st(out, lr);
      st(out + 1, rr);
    }
  }
}

// The last rounds of a layer in one resident block. From iteration i0 (where
// the live halves hold 4h0 = 2^(i0+1) entries, h0 <= kTailH) down to 0 the
// block keeps both halves and the eq table in shared memory; each iteration
// waits for the host's challenge r_i in the lane's downbox (bounded), binds
// and sums exactly as gkr_bind_sums / gkr_final_bind, and posts the round's
// four words to the mailbox (publication seq0 + i0 - i). A missing challenge
// ends the kernel without a post, which the host reads as a failed round.
// At iteration i_host (-1: none) the block hands its tables to the host
// instead and ends: rounds whose tables are that small cost the host about a
// microsecond each, against a PCIe round trip and a device step per round.
//
// A round is a chain of three dependent products per element (the bind,
// e * L, then * R); with few elements one thread per element leaves the
// block idle behind that chain, so the round is spread by product instead:
// the 4h binds (and the eq update) across the block, then the 2h products
// with e, then the 2h wide products, each level one product per thread.
constexpr int kTailThreads = 512;
constexpr unsigned long long kTailWaitNs = 2000000000ull;  // 2 s per challenge

__global__ void __launch_bounds__(kTailThreads) gkr_tail(const f128 *__restrict__ c,
                                                         size_t n_half, int i0,
                                                         const f128 *__restrict__ eq,
                                                         uint32_t at_one_mask, Mailbox *mb,
                                                         unsigned long long seq0,
                                                         const Mailbox *down,
                                                         unsigned long long dseq0, size_t colmask,
                                                         size_t live_cols, int i_host,
                                                         unsigned long long *handover,
                                                         unsigned long long hseq) {
  __shared__ f128 L[4 * kTailH], R[4 * kTailH], E[2 * kTailH];
  __shared__ uint64_t red[4][kTailThreads / 32];
  __shared__ unsigned long long chal[2];
  __shared__ int ok;
  const int h0 = i0 > 0 ? 1 << (i0 - 1) : 1;
  const int live = i0 > 0 ? 4 * h0 : 2;
  for (int k = threadIdx.x; k < live; k += blockDim.x) {
    L[k] = ld(c + k);
    R[k] = ld(c + n_half + k);
  }
  for (int k = threadIdx.x; k < 2 * h0 && i0 > 0; k += blockDim.x) E[k] = ld(eq + k);
  for (int i = i0; i >= 0; i--) {
    if (i == i_host) {
      // the layer's last rounds run on the host: the tables as they stand
      // before r_i's bind (L and R: 4h entries each, then E: 2h) go out as
      // handover publication hseq, two words per entry, and the block ends
      const int h = 1 << (i - 1), nl = 4 * h;
      __syncthreads();  // the tables as loaded (a first iteration has no barrier yet)
      for (int k = threadIdx.x; k < 2 * nl + 2 * h; k += blockDim.x) {
        const f128 v = k < nl ? L[k] : k < 2 * nl ? R[k - nl] : E[k - 2 * nl];
        handover_post(handover, hseq, 2 * k, v.lo);
        handover_post(handover, hseq, 2 * k + 1, v.hi);
      }
      return;
    }
    if (threadIdx.x == 0) ok = mailbox_wait_device(down, dseq0 + (i0 - i), 2, chal, kTailWaitNs);
    __syncthreads();
    if (!ok) return;
    const f128 r = mk(chal[0], chal[1]);
    const unsigned long long seq = seq0 + (i0 - i);
    if (i == 0) {
      if (threadIdx.x == 0) {
        f128 lr = gadd(L[0], gmul(r, gadd(L[1], L[0])));
        f128 rr = gadd(R[0], gmul(r, gadd(R[1], R[0])));
        mailbox_post(mb, seq, 0, lr.lo);
        mailbox_post(mb, seq, 1, lr.hi);
        mailbox_post(mb, seq, 2, rr.lo);
        mailbox_post(mb, seq, 3, rr.hi);
      }
      return;
    }
    const int h = 1 << (i - 1), h2 = 2 * h;
    const int at_one = (at_one_mask >> (i - 1)) & 1;
    // level 1: the binds of round i+1 at r; entry (x, q) is L[x], L[x+h],
    // R[x], R[x+h] for q = 0..3, each read and written by one thread only;
    // the q = 0 thread also sums the eq table down
    for (int t = threadIdx.x; t < 4 * h; t += blockDim.x) {
      const int x = t >> 2, q = t & 3;
      if (q == 0) E[x] = gadd(E[x], E[x + h]);
      if (padded((size_t)x, colmask, live_cols)) continue;  // stays one
      f128 *T = q < 2 ? L : R;
      const int at = x + (q & 1) * h;
      T[at] = gadd(T[at], gmul(r, gadd(T[at + h2], T[at])));
    }
    __syncthreads();
    // level 2: P = e * L_b, Q = e * (L_1 + L_0), kept in the halves' upper
    // quarters [2h, 3h), which the binds above have consumed
    f128 *P = L + h2, *Q = R + h2;
    for (int t = threadIdx.x; t < 2 * h; t += blockDim.x) {
      const int x = t >> 1;
      const f128 e = E[x];
      if (padded((size_t)x, colmask, live_cols)) {  // e * 1 and e * 0
        if (t & 1)
          Q[x] = mk(0, 0);
        else
          P[x] = e;
        continue;
      }
      if (t & 1)
        Q[x] = gmul(e, gadd(L[x + h], L[x]));
      else
        P[x] = gmul(e, at_one ? L[x + h] : L[x]);
    }
    __syncthreads();
    // level 3: P * R_b into the first sum, Q * (R_1 + R_0) into the second
    uint64_t v[4] = {0, 0, 0, 0};
    for (int t = threadIdx.x; t < 2 * h; t += blockDim.x) {
      const int x = t >> 1;
      if (padded((size_t)x, colmask, live_cols)) {  // P * 1 and Q * 0
        if (!(t & 1)) {
          v[0] ^= P[x].lo;
          v[1] ^= P[x].hi;
        }
        continue;
      }
      if (t & 1) {
        f128 p = gmul(Q[x], gadd(R[x + h], R[x]));
        v[2] ^= p.lo;
        v[3] ^= p.hi;
      } else {
        f128 p = gmul(P[x], at_one ? R[x + h] : R[x]);
        v[0] ^= p.lo;
        v[1] ^= p.hi;
      }
    }
    // block XOR-reduction of the four words; thread 0 posts
#pragma unroll
    for (int k = 0; k < 4; k++)
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) v[k] ^= __shfl_xor_sync(0xffffffffu, v[k], off);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0)
      for (int k = 0; k < 4; k++) red[k][warp] = v[k];
    __syncthreads();
    if (warp == 0) {
      const int nw = blockDim.x >> 5;
      for (int k = 0; k < 4; k++) {
        uint64_t x = lane < nw ? red[k][lane] : 0;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) x ^= __shfl_xor_sync(0xffffffffu, x, off);
        v[k] = x;
      }
      if (lane == 0)
        for (int k = 0; k < 4; k++) mailbox_post(mb, seq, k, v[k]);
    }
    __syncthreads();  // this round's tables before the next round's reads
  }
}

static Publish arm(GkrScratch &sc) {
  return sc.channel ? sc.channel->arm() : Publish{nullptr, nullptr, 0};
}

// The round's four words, from the mailbox or by a copy of `src`.
static void round_read(GkrScratch &sc, const void *src, cudaStream_t s) {
  if (sc.channel) {
    sc.channel->wait(s, sc.host, 4);
    return;
  }
  BZ_CUDA(cudaMemcpyAsync(sc.host, src, 32, cudaMemcpyDeviceToHost, s));
  BZ_CUDA(stream_wait(s));
}

void gkr_build(const f128 *cols, int s, const f128 *images, GkrScratch &sc, cudaStream_t st_) {
  size_t total = (size_t)128 << s;
  if (sc.capacity < total) throw CudaError("gkr_build: scratch too small");
  gkr_leaves<<<grid_for(total), kThreads, 0, st_>>>(cols, s, images, sc.layer[0]);
  BZ_LAUNCH_CHECK();
  size_t len = total;
  const size_t colmask = ((size_t)1 << s) - 1;
  const size_t live = sc.live_cols ? sc.live_cols : colmask + 1;
  for (int j = 0; j < 7; j++) {
    gkr_parent<<<grid_for(len / 2), kThreads, 0, st_>>>(sc.layer[j], len / 2, sc.layer[j + 1],
                                                         colmask, live);
    BZ_LAUNCH_CHECK();
    len /= 2;
  }
}

static f128 eq_factor(f128 r, f128 z) { return gadd(gadd(mk(1, 0), r), z); }

// One bind round of hh elements per half: by tiles up to kMidMaxH, one
// element per thread above (issue bound there).
// Grid of the resident middle rounds for a lane: kMidBlocks for a lane proving
// alone; for a pooled lane none (every middle round a queued launch), or
// kMidPoolBlocks with BITZ_POOL_MID=1. On the batched mix the pooled grids cut
// a proof's launches from 189 to 130 but not its time: at 24 lanes and more
// the cooperative grids of different lanes compete for SMs and the mix ran
// 10-20 % slower, so they are off by default.
int gkr_mid_blocks(bool alone) {
  if (alone) return kMidBlocks;
  static const bool pool = [] {
    const char *e = getenv("BITZ_POOL_MID");
    return e && e[0] == '1';
  }();
  return pool ? kMidPoolBlocks : 0;
}

// Elements below h whose packed column holds bits of h (the rest are padding).
static double live_threads(size_t h, size_t colmask, size_t live) {
  return h > colmask ? (double)(h / (colmask + 1)) * (double)live : (double)std::min(h, live);
}

static void launch_bind(f128 *c, size_t n_half, size_t hh, f128 r, f128 *eq, int at_one,
                        unsigned long long *acc, const Publish &pub, const RoundLink &lk,
                        size_t colmask, size_t live, cudaStream_t st) {
  if (hh <= kMidMaxH)
    gkr_round<<<(unsigned)((hh + kMidTile - 1) / kMidTile), kMidThreads, 0, st>>>(
        c, n_half, hh, r, eq, at_one, acc, pub, lk, colmask, live);
  else
    gkr_bind_sums<<<grid_for(hh), kThreads, 0, st>>>(c, n_half, hh, r, eq, at_one, acc, pub, lk,
                                                      colmask, live);
  BZ_LAUNCH_CHECK();
}

// gkr_mid over bind rounds i_hi .. i_lo as a cooperative launch of
// sc.mid_blocks blocks (every block must be resident together).
static void launch_mid(f128 *c, size_t n_half, int n, int i_hi, int i_lo, const f128 *point,
                       GkrScratch &sc, unsigned long long p0, unsigned long long d0,
                       size_t colmask, size_t live, cudaStream_t st) {
  const int nb = sc.mid_blocks;
  const size_t e0 = ((size_t)1 << (i_hi - 1)) / nb;
  const size_t smem = mid_smem_bytes(e0);
  // residency for the largest rounds of each grid size (the kernel's shared
  // memory limit raised once to the largest, the pooled grid's)
  static const int capacity[2] = {[] {
    int dev = 0, sms = 0, per_sm = 0;
    BZ_CUDA(cudaGetDevice(&dev));
    BZ_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    BZ_CUDA(cudaFuncSetAttribute(gkr_mid, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)mid_smem_bytes(kMidMaxH / kMidPoolBlocks)));
    BZ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gkr_mid, kMidThreads,
                                                          mid_smem_bytes(kMidMaxH / kMidBlocks)));
    return sms * per_sm;
  }(), [] {
    int dev = 0, sms = 0, per_sm = 0;
    BZ_CUDA(cudaGetDevice(&dev));
    BZ_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    BZ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm, gkr_mid, kMidThreads, mid_smem_bytes(kMidMaxH / kMidPoolBlocks)));
    return sms * per_sm;
  }()};
  if (nb != kMidBlocks && nb != kMidPoolBlocks) throw CudaError("gkr_mid: unsupported grid");
  if (capacity[nb == kMidBlocks ? 0 : 1] < nb)
    throw CudaError("gkr_mid: the blocks do not fit resident together");
  if (((size_t)1 << (i_lo - 1)) < (size_t)nb * kMidRuns || ((size_t)1 << (i_hi - 1)) > kMidMaxH)
    throw CudaError("gkr_mid: round sizes outside the resident range");
  unsigned long long mask = 0;
  for (int i = i_lo; i <= i_hi; i++) mask |= (unsigned long long)gis_zero(point[i - 1]) << (i - 1);
  RoundChannel *ch = sc.channel;
  f128 *eq = sc.eq;
  unsigned long long *acc = sc.acc;
  Mailbox *mb = ch->dev;
  const Mailbox *down = ch->down_dev;
  RoundCtl *ctl = sc.ctl;
  void *args[] = {&c,  &n_half, &n,    &i_hi, &i_lo, &eq,      &mask,  &acc,
                  &mb, &p0,     &down, &d0,   &ctl,  &colmask, &live};
  BZ_CUDA(cudaLaunchCooperativeKernel((const void *)gkr_mid, dim3(nb), dim3(kMidThreads), args,
                                      smem, st));
  BZ_LAUNCH_CHECK();
}

// The rounds from this iteration down run on the host once gkr_tail has
// handed over its tables (h <= 2^(kHostTailI - 1) = 64 pairs).
constexpr int kHostTailI = 7;

// One iteration of gkr_tail on the host, with the same arithmetic: bind the
// tables (L, R: 4h entries, E: 2h, h = 2^(i-1)) at r and leave the sums of
// the next round in out, or, at i == 0, the bound pair (lr, rr).
static void host_tail_round(std::vector<f128> &L, std::vector<f128> &R, std::vector<f128> &E,
                            int i, f128 r, uint32_t at_one_mask, size_t colmask, size_t live,
                            f128 out[2]) {
  if (i == 0) {
    out[0] = gadd(L[0], gmul(r, gadd(L[1], L[0])));
    out[1] = gadd(R[0], gmul(r, gadd(R[1], R[0])));
    return;
  }
  const size_t h = (size_t)1 << (i - 1), h2 = 2 * h;
  const bool at_one = (at_one_mask >> (i - 1)) & 1;
  for (size_t x = 0; x < h; x++) {
    E[x] = gadd(E[x], E[x + h]);
    if ((x & colmask) >= live) continue;  // a padded column stays one
    for (int q = 0; q < 4; q++) {
      std::vector<f128> &T = q < 2 ? L : R;
      const size_t at = x + (q & 1) * h;
      T[at] = gadd(T[at], gmul(r, gadd(T[at + h2], T[at])));
    }
  }
  f128 s0 = mk(0, 0), s1 = mk(0, 0);
  for (size_t x = 0; x < h; x++) {
    const f128 e = E[x];
    if ((x & colmask) >= live) {  // e * 1 * 1 and e * 0 * 0
      s0 = gadd(s0, e);
      continue;
    }
    const f128 p = gmul(e, at_one ? L[x + h] : L[x]);
    const f128 q = gmul(e, gadd(L[x + h], L[x]));
    s0 = gadd(s0, gmul(p, at_one ? R[x + h] : R[x]));
    s1 = gadd(s1, gmul(q, gadd(R[x + h], R[x])));
  }
  out[0] = s0;
  out[1] = s1;
}

f128 gkr_prove(int s, const f128 *zeta, uint32_t grind_bits, Transcript &ts, GkrScratch &sc,
               cudaStream_t st_, f128 *point_out) {
  f128 point[kMaxPoint], next[kMaxPoint];
  for (int i = 0; i < s; i++) point[i] = zeta[i];
  int n = s;
  const size_t colmask = ((size_t)1 << s) - 1;
  const size_t live = sc.live_cols ? sc.live_cols : colmask + 1;
  f128 claim = mk(0, 0);
  KernelProbe &probe = KernelProbe::get();
  RoundChannel *ch = sc.channel;
  bool tail = false;  // a tail kernel of this layer is resident and waiting
  // without resident rounds every round is its own launch (same results)
  const bool resident = resident_rounds_enabled();
  // BITZ_ROUND_TRACE=1 prints the host time between consecutive round results
  static const bool trace = getenv("BITZ_ROUND_TRACE") != nullptr;
  auto t_prev = std::chrono::steady_clock::now();
  // no other thread's device allocation while a round kernel waits for this one
  ResidentScope gate(ch && resident);
  try {
  for (int j = 6; j >= 0; j--) {
    f128 *c = sc.layer[j];
    size_t n_half = (size_t)1 << n;
    int rounds = n;
    // eq over the coordinates below the top one (2^(n-1) entries) as the
    // factors over the lower a and the upper b of them; the accumulators and
    // round controls of the layer cleared
    const int a = (n - 1) / 2, b = (n - 1) - a;
    f128 *lo = sc.eq_scratch, *hi = sc.eq_scratch + ((size_t)1 << a);
    {
      Point pt;
      pt.n = n - 1;
      for (int k = 0; k < n - 1; k++) pt.c[k] = point[k];
      gkr_layer_setup<<<2, kThreads, 0, st_>>>(pt, a, b, lo, hi, sc.acc, 4 * (rounds + 1),
                                               sc.ctl, rounds);
      BZ_LAUNCH_CHECK();
    }
    size_t h = n_half / 2;
    // Queued mode: the bind rounds above the tail's first (h <= kTailH) and
    // the tail itself are all queued behind the top sums, each round's
    // challenge fetched on the device. Publication p0 + (n - i) carries the
    // sums after binding r_i, which the host posts as downbox publication
    // d0 + (n - 1 - i). The kernel probe times kernels alone, so it runs
    // every round as its own launch.
    const bool queued = ch && resident;
    int i_tail = n - 1;
    while (i_tail > 0 && ((size_t)1 << (i_tail - 1)) > (size_t)kTailH) i_tail--;
    const Publish top = arm(sc);
    const unsigned long long p0 = top.seq, d0 = ch ? ch->down_next + 1 : 0;
    // Queued mode: the tail hands its tables over at iteration i_host and the
    // host runs the rounds from there down (handover publication hseq).
    const int i_host =
        queued && ch->handover_host && i_tail >= 1 ? std::min(kHostTailI, i_tail) : -1;
    const unsigned long long hseq = p0 + (n - i_host);
    uint32_t tail_mask = 0;
    for (int k = 1; k <= i_tail; k++) tail_mask |= (uint32_t)gis_zero(point[k - 1]) << (k - 1);
    std::vector<f128> HL, HR, HE;
    f128 host_out[2] = {mk(0, 0), mk(0, 0)};  // sums (or the pair) the host computed
    RoundLink none{nullptr, nullptr, nullptr, 0};
    // Bind round i > i_tail runs in gkr_mid (which reads r_i from the downbox
    // itself) when the lane keeps the middle rounds resident and 2^(i-1) <=
    // kMidMaxH; otherwise as a queued launch that reads r_i from ctl, left
    // there by the kernel before it.
    auto in_mid = [&](int i) {
      return sc.mid_blocks > 0 && ((size_t)1 << (i - 1)) <= kMidMaxH;
    };
    auto link_for = [&](int i) {  // where the kernel before bind round i leaves r_i
      return queued && i > i_tail && !in_mid(i) ? sc.ctl + (n - 1 - i) : nullptr;
    };
    RoundLink top_link = none;
    if (queued && n - 1 > i_tail) top_link = RoundLink{nullptr, link_for(n - 1), ch->down_dev, d0};
    if (queued) tail = true;  // from here a kernel of the lane may wait for this thread
    const bool probe_top = probe.on("gkr_top_sums");
    if (probe_top) probe.before(st_);
    gkr_top_sums<<<grid_for(h), kThreads, 0, st_>>>(c, n_half, h, lo, a, hi, sc.eq,
                                                    gis_zero(point[n - 1]), sc.acc, top, top_link,
                                                    colmask, live);
    BZ_LAUNCH_CHECK();
    if (probe_top) {
      // each thread forms e = lo * hi and writes it; a live one also reads its
      // four child entries and multiplies e by two of them and the results by two more
      const double nl = live_threads(h, colmask, live);
      probe.after(st_, "gkr_top_sums", 16.0 * (double)h + 64.0 * nl, (double)h + 2.0 * nl,
                  2.0 * nl);
    }
    if (queued) {
      int i = n - 1;
      for (; i > i_tail && !in_mid(i); i--) {
        const size_t hh = (size_t)1 << (i - 1);
        RoundLink lk{sc.ctl + (n - 1 - i), link_for(i - 1), ch->down_dev, d0 + (n - i)};
        const Publish pub{ch->counter, ch->dev, p0 + (n - i)};
        launch_bind(c, n_half, hh, mk(0, 0), sc.eq, gis_zero(point[i - 1]),
                    sc.acc + 4 * (n - i), pub, lk, colmask, live, st_);
      }
      if (i > i_tail) launch_mid(c, n_half, n, i, i_tail + 1, point, sc, p0, d0, colmask, live, st_);
      gkr_tail<<<1, kTailThreads, 0, st_>>>(c, n_half, i_tail, sc.eq, tail_mask, ch->dev,
                                            p0 + (n - i_tail), ch->down_dev,
                                            d0 + (n - 1 - i_tail), colmask, live, i_host,
                                            ch->handover_dev, hseq);
      BZ_LAUNCH_CHECK();
      tail = true;
    }
    f128 eq_bound = mk(1, 0);
    for (int i = n - 1; i >= 0; i--) {
      unsigned long long *acc = sc.acc + 4 * (n - 1 - i);
      if (i_host >= 0 && i < i_host) {  // the host's own round
        sc.host[0] = host_out[0].lo;
        sc.host[1] = host_out[0].hi;
        sc.host[2] = host_out[1].lo;
        sc.host[3] = host_out[1].hi;
      } else {
        round_read(sc, acc, st_);
      }
      if (trace) {
        const auto now = std::chrono::steady_clock::now();
        fprintf(stderr, "[gkr] layer %d round %2d h %8zu %s %7.2f us\n", j, i, (size_t)1 << i,
                i == n - 1 ? "top " : (queued && i < i_tail) ? "tail" : "bind",
                std::chrono::duration<double, std::micro>(now - t_prev).count());
        t_prev = now;
      }
      f128 sb = mk(sc.host[0], sc.host[1]), si = mk(sc.host[2], sc.host[3]);
      f128 msg[2] = {gmul(eq_bound, sb), gmul(eq_bound, si)};
      ts.prover_message(msg, 32);
      ts.grind("gkr/cubic/v1", grind_bits);
      f128 r = ts.challenge_f128();
      next[i] = r;
      eq_bound = gmul(eq_bound, eq_factor(r, point[i]));
      const uint64_t rw[2] = {r.lo, r.hi};
      if (queued && i_host >= 0 && i <= i_host) {
        if (i == i_host) {  // the tail's tables, as it stood before binding r_i
          const int h = 1 << (i - 1), nl = 4 * h;
          std::vector<uint64_t> w(2 * (2 * nl + 2 * h));
          ch->wait_handover(st_, hseq, w.data(), (int)w.size());
          tail = false;  // the tail kernel ends after the handover
          auto take = [&](std::vector<f128> &v, int at, int cnt) {
            v.resize(cnt);
            for (int k = 0; k < cnt; k++) v[k] = mk(w[2 * (at + k)], w[2 * (at + k) + 1]);
          };
          take(HL, 0, nl);
          take(HR, nl, nl);
          take(HE, 2 * nl, 2 * h);
        }
        host_tail_round(HL, HR, HE, i, r, tail_mask, colmask, live, host_out);
        ch->arm();  // publication numbering as if the device had posted
      } else if (queued) {
        ch->send(rw, 2);
        ch->arm();
      } else if (i > 0) {
        size_t hh = (size_t)1 << (i - 1);
        const char *name = hh <= kMidMaxH ? "gkr_round" : "gkr_bind_sums";
        const bool probed = probe.on(name);
        if (probed) probe.before(st_);
        launch_bind(c, n_half, hh, r, sc.eq, gis_zero(point[i - 1]), acc + 4, arm(sc), none,
                    colmask, live, st_);
        if (probed) {
          // a live element reads 8 child and 2 eq entries and writes 4 and 1
          // (240 B), binds four entries by r through r's window table and
          // makes four general products (two by e, two wide); a padded one
          // moves the eq table's 3 entries (48 B)
          const double nl = live_threads(hh, colmask, live);
          probe.after(st_, name, 240.0 * nl + 48.0 * ((double)hh - nl), 2.0 * nl, 2.0 * nl,
                      4.0 * nl);
        }
      } else {
        gkr_final_bind<<<1, 32, 0, st_>>>(c, n_half, r, sc.pair, arm(sc));
        BZ_LAUNCH_CHECK();
      }
    }
    f128 lr[2];
    if (i_host >= 0) {
      lr[0] = host_out[0];
      lr[1] = host_out[1];
    } else {
      round_read(sc, sc.pair, st_);
      tail = false;  // the tail kernel ends after posting the pair
      memcpy(lr, sc.host, 32);
    }
    ts.prover_message(lr, 32);
    f128 t = ts.challenge_f128();
    next[n] = t;
    claim = gadd(lr[0], gmul(t, gadd(lr[1], lr[0])));
    n++;
    for (int i = 0; i < n; i++) point[i] = next[i];
  }
  } catch (...) {
    if (tail) {  // release the waiting kernel before the lane is reused
      ch->abort();
      stream_wait(st_);
      ch->clear_down();
    }
    throw;
  }
  for (int i = 0; i < n; i++) point_out[i] = point[i];
  return claim;
}

// Every kernel of this file, loaded when the process's first lane on a device
// is made (lane_bootstrap, context.cpp).
void preload_gkr_kernels() {
  load_kernels({(const void *)gkr_leaves,
                (const void *)gkr_parent,
                (const void *)gkr_layer_setup,
                (const void *)gkr_top_sums,
                (const void *)gkr_bind_sums,
                (const void *)gkr_round,
                (const void *)gkr_mid,
                (const void *)gkr_final_bind,
                (const void *)gkr_tail});
}

}  // namespace bz
