#include "context.hpp"

#include <immintrin.h>

#include <atomic>
#include <chrono>

namespace bz {

void RoundChannel::wait(cudaStream_t s, uint64_t *out, int n) {
  const unsigned long long want = next;
  auto t0 = std::chrono::steady_clock::now();
  uint64_t spins = 0;
  while (host->seq != want) {
    if ((++spins & 0x3ff) == 0) {
      cudaError_t e = cudaStreamQuery(s);
      if (e != cudaSuccess && e != cudaErrorNotReady)
        throw CudaError(std::string("round kernel failed: ") + cudaGetErrorString(e));
      if (e == cudaSuccess && host->seq != want)
        throw CudaError("round kernel finished without publishing its result");
      if (std::chrono::steady_clock::now() - t0 > std::chrono::seconds(30))
        throw CudaError("timed out waiting for a round result");
    }
    _mm_pause();
  }
  std::atomic_thread_fence(std::memory_order_acquire);
  const volatile unsigned long long *p = host->payload;
  for (int k = 0; k < n; k++) out[k] = p[k];
}

Context::Context() {
  BZ_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
  acc_.resize(8 * 128);
  BZ_CUDA(cudaMallocHost(&host_, 64 * sizeof(uint64_t)));
  pg_.acc = acc_.get();
  pg_.host = host_;
  gk_pair_.resize(2);
  gk_.acc = acc_.get();
  gk_.host = host_;
  gk_.pair = gk_pair_.get();
  // the round mailbox: one mapped pinned page and a device block counter
  void *mb = nullptr;
  BZ_CUDA(cudaHostAlloc(&mb, 4096, cudaHostAllocMapped));
  memset(mb, 0, 4096);
  channel_.host = (Mailbox *)mb;
  void *mbd = nullptr;
  BZ_CUDA(cudaHostGetDevicePointer(&mbd, mb, 0));
  channel_.dev = (Mailbox *)mbd;
  counter_.resize(1);
  BZ_CUDA(cudaMemset(counter_.get(), 0, sizeof(unsigned int)));
  channel_.counter = counter_.get();
  pg_.channel = &channel_;
  gk_.channel = &channel_;
}

unsigned long long &launch_counter() {
  static unsigned long long n = 0;
  return n;
}

Context &Context::get() {
  // One context per process, created on first use on the current device.
  static Context *ctx = new Context();
  return *ctx;
}

}  // namespace bz
