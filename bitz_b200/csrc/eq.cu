#include "eq.cuh"

namespace bz {

// Builds eq over `n` coordinates of `p` starting at `first` into out[0, 2^n)
// by doubling; one block of threads, whose __syncthreads() orders the
// global-memory writes of one level before the reads of the next.
__global__ void eq_factor_kernel(Point p, int first, int n, f128 *out) {
  if (threadIdx.x == 0) out[0] = mk(1, 0);
  __syncthreads();
  for (int i = 0; i < n; i++) {
    f128 z = p.c[first + i];
    int half = 1 << i;
    for (int k = threadIdx.x; k < half; k += blockDim.x) {
      f128 par = out[k];
      f128 one = gmul(par, z);
      out[k] = gadd(par, one);
      out[k + half] = one;
    }
    __syncthreads();
  }
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
  eq_factor_kernel<<<1, kThreads, 0, s>>>(p, 0, a, lo);
  BZ_LAUNCH_CHECK();
  eq_factor_kernel<<<1, kThreads, 0, s>>>(p, a, b, hi);
  BZ_LAUNCH_CHECK();
  size_t total = (size_t)1 << n;
  eq_expand_kernel<<<grid_for(total), kThreads, 0, s>>>(lo, a, hi, out, total);
  BZ_LAUNCH_CHECK();
}

}  // namespace bz
