#include "context.hpp"

namespace bz {

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
