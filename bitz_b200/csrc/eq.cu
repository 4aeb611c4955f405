#include "eq.cuh"

#include "context.hpp"

namespace bz {

// Both factor tables in one launch: block 0 the low a coordinates, block 1
// the high b.
__global__ void __launch_bounds__(kThreads) eq_factors_kernel(Point p, int a, int b, f128 *lo,
                                                              f128 *hi) {
  __shared__ MulTable T;
  if (blockIdx.x == 0)
    eq_factor_block(p, 0, a, lo, T);
  else
    eq_factor_block(p, a, b, hi, T);
}

__global__ void eq_expand_kernel(const f128 *__restrict__ lo, int a, const f128 *__restrict__ hi,
                                 f128 *__restrict__ out, size_t total) {
  size_t mask = ((size_t)1 << a) - 1;
  for (size_t x = blockIdx.x * (size_t)blockDim.x + threadIdx.x; x < total;
       x += (size_t)gridDim.x * blockDim.x)
    st(out + x, gmul(ld(lo + (x & mask)), ld(hi + (x >> a))));
}

void eq_table_device(const f128 *point, int n, f128 *out, f128 *scratch, cudaStream_t s) {
  if (n > kMaxPoint) throw CudaError("eq_table_device: point too long");
  Point p;
  p.n = n;
  for (int i = 0; i < n; i++) p.c[i] = point[i];
  int a = n / 2, b = n - a;
  f128 *lo = scratch, *hi = scratch + ((size_t)1 << a);
  eq_factors_kernel<<<2, kThreads, 0, s>>>(p, a, b, lo, hi);
  BZ_LAUNCH_CHECK();
  size_t total = (size_t)1 << n;
  eq_expand_kernel<<<grid_for(total), kThreads, 0, s>>>(lo, a, hi, out, total);
  BZ_LAUNCH_CHECK();
}

// Every kernel of this file, loaded when the process's first lane on a device
// is made (lane_bootstrap, context.cpp).
void preload_eq_kernels() {
  load_kernels({(const void *)eq_factors_kernel,
                (const void *)eq_expand_kernel});
}

}  // namespace bz
