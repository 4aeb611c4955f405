// Witness generation on the device (tooling/cli/src/end_to_end.rs:215-243).
//
// f = inputs || per compression the hint bits of sha256.rs:228-316 in
// allocation order; h = M (1 || f) (crates/circuit/src/witgen.rs:438-446);
// the exact products A h, B h, C h and the integer satisfiability check
// (crates/circuit/src/matrix_products.rs:482-495). Both bit vectors are packed
// little-endian into 32-bit words, which is also the packed F128 layout the
// commitment and the BitZ table read (end_to_end.rs:499-507).
#include "device.cuh"
#include "witness.hpp"
#include "context.hpp"

namespace bz {

__constant__ uint32_t c_sha_k[64] = {
    0x428a2f98, 0x71374491, 0xb5c0fbcf, 0xe9b5dba5, 0x3956c25b, 0x59f111f1, 0x923f82a4, 0xab1c5ed5,
    0xd807aa98, 0x12835b01, 0x243185be, 0x550c7dc3, 0x72be5d74, 0x80deb1fe, 0x9bdc06a7, 0xc19bf174,
    0xe49b69c1, 0xefbe4786, 0x0fc19dc6, 0x240ca1cc, 0x2de92c6f, 0x4a7484aa, 0x5cb0a9dc, 0x76f988da,
    0x983e5152, 0xa831c66d, 0xb00327c8, 0xbf597fc7, 0xc6e00bf3, 0xd5a79147, 0x06ca6351, 0x14292967,
    0x27b70a85, 0x2e1b2138, 0x4d2c6dfc, 0x53380d13, 0x650a7354, 0x766a0abb, 0x81c2c92e, 0x92722c85,
    0xa2bfe8a1, 0xa81a664b, 0xc24b8b70, 0xc76c51a3, 0xd192e819, 0xd6990624, 0xf40e3585, 0x106aa070,
    0x19a4c116, 0x1e376c08, 0x2748774c, 0x34b0bcb5, 0x391c0cb3, 0x4ed8aa4a, 0x5b9cca4f, 0x682e6ff3,
    0x748f82ee, 0x78a5636f, 0x84c87814, 0x8cc70208, 0x90befffa, 0xa4506ceb, 0xbef9a3f7, 0xc67178f2};

__device__ __forceinline__ uint32_t ror32(uint32_t x, int n) { return __funnelshift_r(x, x, n); }

// ORs the low `width` bits of v into the bit array at bit offset `pos`.
__device__ __forceinline__ void put_bits(uint32_t *f, uint64_t pos, uint64_t v, int width) {
  while (width > 0) {
    uint64_t w = pos >> 5;
    int sh = (int)(pos & 31);
    int take = 32 - sh < width ? 32 - sh : width;
    uint32_t chunk = (uint32_t)(v & ((1ull << take) - 1)) << sh;
    if (chunk) atomicOr(f + w, chunk);
    v >>= take;
    pos += (uint64_t)take;
    width -= take;
  }
}

// One warp per compression: the schedule sums (34 bits), each round's e and
// a sums before truncation (35 bits: the doubled-Ch/Maj quotient), and the
// eight feed-forward sums (33 bits), in that order from the compression's
// bit offset. Lane 0 runs the compression and keeps the 184 values in shared
// memory; the warp's lanes then OR them into f.
constexpr int kShaWarps = 4;  // compressions per block
constexpr int kShaVals = 48 + 128 + 8;
__global__ void __launch_bounds__(32 * kShaWarps) k_sha_hints(const uint32_t *__restrict__ states,
                                                              const uint32_t *__restrict__ msgs,
                                                              const uint64_t *__restrict__ offsets,
                                                              int nblocks, uint32_t *f) {
  __shared__ uint64_t vals[kShaWarps][kShaVals];
  const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int blk = blockIdx.x * kShaWarps + wib;
  if (blk >= nblocks) return;  // the whole warp
  uint64_t *v = vals[wib];
  if (lane == 0) {
    uint32_t w[64];
    for (int i = 0; i < 16; i++) w[i] = msgs[16 * blk + i];
    for (int i = 16; i < 64; i++) {
      uint64_t s = (uint64_t)w[i - 16] +
                   (ror32(w[i - 15], 7) ^ ror32(w[i - 15], 18) ^ (w[i - 15] >> 3)) +
                   (uint64_t)w[i - 7] +
                   (ror32(w[i - 2], 17) ^ ror32(w[i - 2], 19) ^ (w[i - 2] >> 10));
      v[i - 16] = s;
      w[i] = (uint32_t)s;
    }
    uint32_t st[8];
    for (int i = 0; i < 8; i++) st[i] = states[8 * blk + i];
    uint32_t a = st[0], b = st[1], c = st[2], d = st[3], e = st[4], ff = st[5], g = st[6],
             h = st[7];
    for (int i = 0; i < 64; i++) {
      uint64_t s1 = ror32(e, 6) ^ ror32(e, 11) ^ ror32(e, 25);
      uint64_t ch = (e & ff) ^ (~e & g);
      uint64_t s0 = ror32(a, 2) ^ ror32(a, 13) ^ ror32(a, 22);
      uint64_t mj = (a & b) ^ (a & c) ^ (b & c);
      uint64_t base = (uint64_t)h + s1 + c_sha_k[i] + w[i] + ch;
      uint64_t ne = base + d;
      uint64_t na = base + s0 + mj;
      v[48 + 2 * i] = ne;
      v[49 + 2 * i] = na;
      h = g;
      g = ff;
      ff = e;
      e = (uint32_t)ne;
      d = c;
      c = b;
      b = a;
      a = (uint32_t)na;
    }
    const uint32_t work[8] = {a, b, c, d, e, ff, g, h};
    for (int i = 0; i < 8; i++) v[176 + i] = (uint64_t)st[i] + work[i];
  }
  __syncwarp();
  const uint64_t pos = offsets[blk];
  for (int k = lane; k < kShaVals; k += 32) {
    uint64_t off;
    int width;
    if (k < 48) {
      off = 34ull * k;
      width = 34;
    } else if (k < 176) {
      off = 1632 + 35ull * (k - 48);
      width = 35;
    } else {
      off = 1632 + 4480 + 33ull * (k - 176);
      width = 33;
    }
    put_bits(f, pos + off, v[k], width);
  }
}

__device__ __forceinline__ int fbit(const uint32_t *f, uint32_t p) {
  // position 0 is the constant one, position p >= 1 is f bit p - 1
  if (p == 0) return 1;
  uint32_t q = p - 1;
  return (f[q >> 5] >> (q & 31)) & 1;
}

// h = M (1 || f), 32 rows per warp, one word per ballot.
__global__ void k_hbits(const uint32_t *__restrict__ off, const uint32_t *__restrict__ pos,
                        size_t h_len, const uint32_t *__restrict__ f, uint32_t *h) {
  size_t nwords = (h_len + 31) / 32;
  size_t warp = (blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5;
  size_t nwarps = (gridDim.x * (size_t)blockDim.x) >> 5;
  int lane = threadIdx.x & 31;
  for (size_t wd = warp; wd < nwords; wd += nwarps) {
    size_t r = wd * 32 + lane;
    int bit = 0;
    if (r < h_len)
      for (uint32_t e = off[r]; e < off[r + 1]; e++) bit ^= fbit(f, pos[e]);
    unsigned m = __ballot_sync(0xffffffffu, bit);
    if (lane == 0) h[wd] = m;
  }
}

__device__ __forceinline__ int hbit(const uint32_t *h, uint32_t c) { return (h[c >> 5] >> (c & 31)) & 1; }

// Exact products per R1CS row and the integer satisfiability check. The bit
// constraints' C constant is the statement's expected value (bit_c). One warp
// per row: the lanes stride over the row's nonzeros of A, B and C (coalesced
// loads of the columns and coefficients) and the warp adds the three sums with
// shuffles. Two's-complement addition wraps the same in any order, so the
// sums equal a row-serial loop's.
__device__ __forceinline__ int64_t warp_sum64(int64_t v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

__global__ void k_products(const uint32_t *__restrict__ aoff, const uint32_t *__restrict__ acol,
                           const int64_t *__restrict__ acoef, const uint32_t *__restrict__ boff,
                           const uint32_t *__restrict__ bcol, const int64_t *__restrict__ bcoef,
                           const uint32_t *__restrict__ coff, const uint32_t *__restrict__ ccol,
                           const int64_t *__restrict__ ccoef, const uint32_t *__restrict__ h,
                           size_t rows, size_t n_in, const uint8_t *__restrict__ bit_c,
                           int64_t *prod, int *unsat) {
  const int lane = threadIdx.x & 31;
  const size_t warps = ((size_t)gridDim.x * blockDim.x) >> 5;
  for (size_t r = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < rows; r += warps) {
    int64_t a = 0, b = 0, c = 0;
    for (uint32_t e = aoff[r] + lane; e < aoff[r + 1]; e += 32) a += hbit(h, acol[e]) ? acoef[e] : 0;
    for (uint32_t e = boff[r] + lane; e < boff[r + 1]; e += 32) b += hbit(h, bcol[e]) ? bcoef[e] : 0;
    for (uint32_t e = coff[r] + lane; e < coff[r + 1]; e += 32) c += hbit(h, ccol[e]) ? ccoef[e] : 0;
    a = warp_sum64(a);
    b = warp_sum64(b);
    c = warp_sum64(c);
    if (lane == 0) {
      if (r < n_in) c += bit_c[r];
      if (r >= rows - 256) c += bit_c[n_in + (r - (rows - 256))];
      prod[r] = a;
      prod[rows + r] = b;
      prod[2 * rows + r] = c;
      if ((__int128)a * b != (__int128)c) atomicExch(unsat, 1);
    }
  }
}

void witness_generate(const WitnessArgs &a, cudaStream_t s) {
  k_sha_hints<<<(a.nblocks + kShaWarps - 1) / kShaWarps, 32 * kShaWarps, 0, s>>>(
      a.states, a.msgs, a.offsets, a.nblocks, a.f);
  BZ_LAUNCH_CHECK();
  size_t words = (a.h_len + 31) / 32;
  k_hbits<<<grid_for(words * 32), kThreads, 0, s>>>(a.m_off, a.m_pos, a.h_len, a.f, a.h);
  BZ_LAUNCH_CHECK();
  k_products<<<grid_for(a.rows * 32), kThreads, 0, s>>>(
      a.abc_off[0], a.abc_col[0], a.abc_coef[0], a.abc_off[1], a.abc_col[1], a.abc_coef[1],
      a.abc_off[2], a.abc_col[2], a.abc_coef[2], a.h, a.rows, a.n_inputs, a.bit_c, a.prod,
      a.unsat);
  BZ_LAUNCH_CHECK();
}

// Every kernel of this file, loaded when the process's first lane on a device
// is made (lane_bootstrap, context.cpp).
void preload_witness_kernels() {
  load_kernels({(const void *)k_sha_hints,
                (const void *)k_hbits,
                (const void *)k_products});
}

}  // namespace bz
