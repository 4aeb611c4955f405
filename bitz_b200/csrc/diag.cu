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

}  // namespace bz
