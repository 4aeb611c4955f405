// Measurement aids: the round-trip floor of the two ways a round's result
// reaches the host and its challenge reaches the device. Not on the proving
// path; exported through bitz_diag_round_trip.
#include <chrono>

#include "context.hpp"

namespace bz {

// One launch per round: a single thread posts the round's word.
__global__ void k_post_once(Mailbox *mb, unsigned long long seq, unsigned long long v) {
  if (threadIdx.x == 0 && blockIdx.x == 0) mailbox_post(mb, seq, 0, v);
}

// One resident kernel for all rounds: wait for the host's word, post it back.
__global__ void k_ping_pong(Mailbox *mb, unsigned long long seq0, const Mailbox *down,
                            unsigned long long dseq0, int rounds) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int i = 0; i < rounds; i++) {
    unsigned long long v;
    if (!mailbox_wait_device(down, dseq0 + i, 1, &v, 2000000000ull)) return;
    mailbox_post(mb, seq0 + i, 0, v + 1);
  }
}

// One thread waits up to limit_ns for the host's word (downbox publication
// dseq) and posts it back plus one as publication seq, or zero when the word
// never came while the kernel ran.
__global__ void k_host_echo(Mailbox *mb, unsigned long long seq, const Mailbox *down,
                            unsigned long long dseq, unsigned long long limit_ns) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  unsigned long long v = 0;
  const bool got = mailbox_wait_device(down, dseq, 1, &v, limit_ns);
  mailbox_post(mb, seq, 0, got ? v + 1 : 0);
}

// Whether this host thread can talk to a kernel while the kernel runs: false
// under a tool that holds the host at every launch until the kernel has
// finished (a kernel profiler), where every kernel that waits for the host
// would sit out its time limit. Costs one round trip, 100 ms at most.
bool host_reaches_running_kernel(Context &lane) {
  cudaStream_t s = lane.stream();
  RoundChannel *ch = lane.channel();
  const uint64_t word = 0x5eedull;
  const Publish p = ch->arm();
  k_host_echo<<<1, 32, 0, s>>>(p.mailbox, p.seq, ch->down_dev, ch->down_next + 1, 100000000ull);
  BZ_LAUNCH_CHECK();
  ch->send(&word, 1);
  uint64_t out = 0;
  ch->wait(s, &out, 1);
  BZ_CUDA(cudaStreamSynchronize(s));
  ch->clear_down();
  return out == word + 1;
}

// Mean microseconds per round over `rounds` rounds: mode 0 launches one
// kernel per round, mode 1 runs one resident kernel that waits for the host.
double diag_round_trip(int mode, int rounds) {
  Context &lane = Context::get();
  cudaStream_t s = lane.stream();
  RoundChannel *ch = lane.channel();
  uint64_t out = 0;
  auto t0 = std::chrono::steady_clock::now();
  if (mode == 0) {
    for (int i = 0; i < rounds; i++) {
      Publish p = ch->arm();
      k_post_once<<<1, 32, 0, s>>>(p.mailbox, p.seq, (unsigned long long)i);
      BZ_LAUNCH_CHECK();
      ch->wait(s, &out, 1);
      if (out != (uint64_t)i) throw CudaError("round trip returned a wrong word");
    }
  } else {
    k_ping_pong<<<1, 32, 0, s>>>(ch->dev, ch->next + 1, ch->down_dev, ch->down_next + 1, rounds);
    BZ_LAUNCH_CHECK();
    try {
      for (int i = 0; i < rounds; i++) {
        uint64_t w = (uint64_t)i;
        ch->send(&w, 1);
        ch->arm();
        ch->wait(s, &out, 1);
        if (out != (uint64_t)i + 1) throw CudaError("round trip returned a wrong word");
      }
    } catch (...) {
      ch->abort();
      cudaStreamSynchronize(s);
      ch->clear_down();
      throw;
    }
  }
  BZ_CUDA(cudaStreamSynchronize(s));
  double us = std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now() - t0).count();
  return us / rounds;
}

// The GPU's GF(2^128) product throughput, the ceiling of the integer-bound
// kernels: every thread runs kChains independent chains of `iters` products
// of one kind (0 reduced general products, 1 unreduced ones folded into an
// accumulator, 2 products by one factor through its window table in shared
// memory). The chains' values are XORed into `sink` so none is dead code.
// The time is that of one launch of blocks_per_sm waves of blocks per SM.
constexpr int kPeakChains = 4;

template <int kKind>
__global__ void __launch_bounds__(kThreads) k_gf_peak(int iters, f128 y, f128 *sink) {
  __shared__ MulTable T;
  if (kKind == 2) mul_table_build(T, y);
  f128 x[kPeakChains];
  for (int k = 0; k < kPeakChains; k++)
    x[k] = mk(0x9e3779b97f4a7c15ull * (blockIdx.x * blockDim.x + threadIdx.x + 1) + k,
              0xc2b2ae3d27d4eb4full ^ (uint64_t)k);
  wide acc = wzero();
  for (int i = 0; i < iters; i++)
#pragma unroll
    for (int k = 0; k < kPeakChains; k++) {
      if (kKind == 0) {
        x[k] = gmul(x[k], y);
      } else if (kKind == 1) {
        const wide w = gmul_wide(x[k], y);
        wacc(acc, w);
        x[k] = mk(w.w0 ^ w.w2, w.w1 ^ w.w3);  // the next operand depends on the product
      } else {
        x[k] = mul_table(T, x[k]);
      }
    }
  f128 r = greduce(acc);
  for (int k = 0; k < kPeakChains; k++) r = gadd(r, x[k]);
  if (gis_zero(r)) st(sink, r);  // practically never; keeps the chains live
}

template <int kKind>
static float time_gf_peak(int blocks, int iters, f128 y, f128 *sink, cudaStream_t s) {
  cudaEvent_t e0, e1;
  BZ_CUDA(cudaEventCreate(&e0));
  BZ_CUDA(cudaEventCreate(&e1));
  k_gf_peak<kKind><<<blocks, kThreads, 0, s>>>(16, y, sink);  // warm-up
  BZ_LAUNCH_CHECK();
  BZ_CUDA(cudaEventRecord(e0, s));
  k_gf_peak<kKind><<<blocks, kThreads, 0, s>>>(iters, y, sink);
  BZ_LAUNCH_CHECK();
  BZ_CUDA(cudaEventRecord(e1, s));
  BZ_CUDA(cudaEventSynchronize(e1));
  float ms = 0;
  BZ_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return ms;
}

// Products per second of `kind` over a grid of `blocks_per_sm` blocks per SM.
double diag_gf_peak(int kind, int blocks_per_sm) {
  Context &lane = Context::get();
  cudaStream_t s = lane.stream();
  int dev = 0, sms = 0;
  BZ_CUDA(cudaGetDevice(&dev));
  BZ_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  DeviceBuffer<f128> sink(1);
  const int blocks = sms * blocks_per_sm, iters = kind == 2 ? 4096 : 1024;
  const f128 y = mk(0x0123456789abcdefull, 0xfedcba9876543210ull);
  const float ms = kind == 0   ? time_gf_peak<0>(blocks, iters, y, sink.get(), s)
                   : kind == 1 ? time_gf_peak<1>(blocks, iters, y, sink.get(), s)
                               : time_gf_peak<2>(blocks, iters, y, sink.get(), s);
  return (double)blocks * kThreads * kPeakChains * iters / (ms * 1e-3);
}

// Every kernel of this file, loaded when the process's first lane on a device
// is made (lane_bootstrap, context.cpp).
void preload_diag_kernels() {
  load_kernels({(const void *)k_post_once,
                (const void *)k_ping_pong,
                (const void *)k_host_echo,
                (const void *)k_gf_peak<0>,
                (const void *)k_gf_peak<1>,
                (const void *)k_gf_peak<2>});
}

}  // namespace bz
