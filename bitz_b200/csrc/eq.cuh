// Equality tables eq(r, x) = prod_i (x_i ? r_i : 1 + r_i) over GF(2^128)
// (crates/poly/src/eq.rs:63-98, variable i = index bit i).
//
// A table over n coordinates is formed as the tensor product of two factor
// tables over the low and high halves of the point (eq.rs:107-115 splits the
// same way): each factor is built by doubling inside one thread block's
// shared memory, and the expansion writes every entry with one multiply.
#pragma once
#include <cuda_runtime.h>

#include "device.cuh"

namespace bz {

constexpr int kMaxPoint = 48;

struct Point {
  f128 c[kMaxPoint];
  int n;
};

#if defined(__CUDACC__)
// Builds eq over coordinates first .. first + n - 1 of p into out[0, 2^n) by
// doubling, every thread of the block taking part (the block's barriers order
// the global-memory levels). Each level multiplies every entry by the same
// coordinate z, through z's window table once the level is wide enough to
// repay building it.
__device__ __forceinline__ void eq_factor_block(const Point &p, int first, int n, f128 *out,
                                                MulTable &T) {
  if (threadIdx.x == 0) out[0] = mk(1, 0);
  __syncthreads();
  for (int i = 0; i < n; i++) {
    const f128 z = p.c[first + i];
    const int half = 1 << i;
    const bool tab = half >= 64;  // uniform across the block
    if (tab) mul_table_build(T, z);
    for (int k = threadIdx.x; k < half; k += blockDim.x) {
      const f128 par = out[k];
      const f128 one = tab ? mul_table(T, par) : gmul(par, z);
      out[k] = gadd(par, one);
      out[k + half] = one;
    }
    __syncthreads();
  }
}
#endif

void eq_table_device(const f128 *point, int n, f128 *out, f128 *scratch, cudaStream_t s);
// Scratch entries eq_table_device needs for an n-coordinate table.
inline size_t eq_scratch_entries(int n) {
  int a = n / 2, b = n - a;
  return ((size_t)1 << a) + ((size_t)1 << b);
}

}  // namespace bz
