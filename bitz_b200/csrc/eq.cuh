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

void eq_table_device(const f128 *point, int n, f128 *out, f128 *scratch, cudaStream_t s);
// Scratch entries eq_table_device needs for an n-coordinate table.
inline size_t eq_scratch_entries(int n) {
  int a = n / 2, b = n - a;
  return ((size_t)1 << a) + ((size_t)1 << b);
}

}  // namespace bz
