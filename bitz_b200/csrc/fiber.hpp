// Cooperative fibers: several prover lanes on one host thread.
//
// A proof's host thread spends most of a round waiting for the device (the
// round result, a stream to drain). With a host thread per lane, lanes beyond
// the host's cores spin against each other. A FiberLoop runs several lanes'
// host work on one thread instead: each lane is a fiber with its own stack,
// and wherever it would wait for the device it yields (fiber_yield), so the
// thread works on another lane's transcript meanwhile. Fibers never migrate
// between threads; a fiber that blocks in a call the loop does not see blocks
// the whole thread, so every wait on the proving path goes through the
// helpers below.
#pragma once
#include <cuda_runtime.h>

#include <functional>
#include <memory>
#include <vector>

namespace bz {

struct Fiber;

// Per-fiber (or, outside fibers, per-thread) counters of the device gate's
// scopes (context.cpp).
struct GateDepth {
  int resident = 0, alloc = 0;
};

class FiberLoop {
 public:
  explicit FiberLoop(size_t stack_bytes = (size_t)1 << 20);
  ~FiberLoop();
  FiberLoop(const FiberLoop &) = delete;
  FiberLoop &operator=(const FiberLoop &) = delete;
  // Adds a fiber that runs fn to its end. fn must not let an exception out.
  void add(std::function<void()> fn);
  // Runs the fibers round robin on the calling thread until all have ended.
  void run();

 private:
  size_t stack_bytes_;
  std::vector<std::unique_ptr<Fiber>> fibers_;
};

// True inside a fiber of a running FiberLoop.
bool in_fiber();
// Lets the thread's other fibers run; returns when this one is resumed. A
// no-op outside fibers.
void fiber_yield();
// The gate counters of the current fiber, or of the thread outside fibers.
GateDepth &gate_depth();

// Waits for all work in the stream (cudaStreamSynchronize), yielding to other
// fibers while it runs. Returns the stream's status.
cudaError_t stream_wait(cudaStream_t s);
// Waits for the event (cudaEventSynchronize), yielding likewise.
cudaError_t event_wait(cudaEvent_t e);

// A CPU-only self-test of the fiber runtime (no GPU): `threads` threads each
// run `fibers` fibers that interleave `yields` yields, throw and catch an
// exception on their own stacks and check their gate counters stay their own.
// Returns a checksum over the order of the work, and sets *ok.
unsigned long long fiber_selftest(int threads, int fibers, int yields, bool *ok);

}  // namespace bz
