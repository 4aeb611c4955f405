// Cooperative fibers (fiber.hpp): a round-robin loop per host thread and a
// stack switch that saves the callee-saved registers of the System V x86-64
// ABI (rbx, rbp, r12-r15, the SSE control word MXCSR and the x87 control
// word) on the outgoing stack and restores them from the incoming one.
#include "fiber.hpp"

#include <immintrin.h>
#include <stdint.h>
#include <sys/mman.h>
#include <unistd.h>

#include <stdexcept>
#include <thread>

#include "device.cuh"

extern "C" void bz_fiber_swap(void **save_sp, void *load_sp);

#if !defined(__CUDA_ARCH__)
__asm__(
    ".text\n"
    ".globl bz_fiber_swap\n"
    ".type bz_fiber_swap,@function\n"
    "bz_fiber_swap:\n"
    "  pushq %rbp\n"
    "  pushq %rbx\n"
    "  pushq %r12\n"
    "  pushq %r13\n"
    "  pushq %r14\n"
    "  pushq %r15\n"
    "  subq $8, %rsp\n"
    "  stmxcsr (%rsp)\n"
    "  fnstcw 4(%rsp)\n"
    "  movq %rsp, (%rdi)\n"
    "  movq %rsi, %rsp\n"
    "  ldmxcsr (%rsp)\n"
    "  fldcw 4(%rsp)\n"
    "  addq $8, %rsp\n"
    "  popq %r15\n"
    "  popq %r14\n"
    "  popq %r13\n"
    "  popq %r12\n"
    "  popq %rbx\n"
    "  popq %rbp\n"
    "  ret\n"
    ".size bz_fiber_swap, .-bz_fiber_swap\n");
#endif

namespace bz {

struct Fiber {
  std::function<void()> fn;
  void *sp = nullptr;
  void *mem = nullptr;
  size_t mem_bytes = 0;
  bool done = false;
  GateDepth depth;
};

namespace {
thread_local Fiber *t_current = nullptr;
thread_local void *t_loop_sp = nullptr;  // the loop's stack while a fiber runs
thread_local GateDepth t_depth;

// First frame of every fiber: runs its function, then returns to the loop for
// good (the loop never resumes a finished fiber).
void fiber_entry() {
  Fiber *f = t_current;
  f->fn();
  f->done = true;
  bz_fiber_swap(&f->sp, t_loop_sp);
  __builtin_trap();  // unreachable: a finished fiber is never resumed
}
}  // namespace

FiberLoop::FiberLoop(size_t stack_bytes) : stack_bytes_(stack_bytes) {}

FiberLoop::~FiberLoop() {
  for (auto &f : fibers_)
    if (f->mem) munmap(f->mem, f->mem_bytes);
}

void FiberLoop::add(std::function<void()> fn) {
  auto f = std::make_unique<Fiber>();
  f->fn = std::move(fn);
  const size_t page = (size_t)sysconf(_SC_PAGESIZE);
  const size_t bytes = (stack_bytes_ + page - 1) / page * page + page;  // + a guard page
  void *mem = mmap(nullptr, bytes, PROT_READ | PROT_WRITE, MAP_PRIVATE | MAP_ANONYMOUS, -1, 0);
  if (mem == MAP_FAILED) throw std::runtime_error("fiber stack allocation failed");
  mprotect(mem, page, PROT_NONE);  // an overflow faults instead of corrupting memory
  f->mem = mem;
  f->mem_bytes = bytes;
  // The stack as bz_fiber_swap leaves it: the control words, six registers,
  // then fiber_entry as the return address, entered with rsp = 8 mod 16 as
  // after a call.
  uint64_t *p = (uint64_t *)(((uintptr_t)mem + bytes) & ~(uintptr_t)15);
  *--p = 0;                                   // fiber_entry's own return address (never used)
  *--p = (uint64_t)(uintptr_t)&fiber_entry;   // where the first switch returns to
  for (int i = 0; i < 6; i++) *--p = 0;       // r15 .. rbp
  *--p = 0x0000037F00001F80ull;               // MXCSR 0x1F80, x87 control word 0x037F
  f->sp = p;
  fibers_.push_back(std::move(f));
}

void FiberLoop::run() {
  if (t_current) throw std::runtime_error("a fiber loop cannot run inside a fiber");
  size_t live = fibers_.size();
  while (live) {
    live = 0;
    for (auto &f : fibers_) {
      if (f->done) continue;
      t_current = f.get();
      bz_fiber_swap(&t_loop_sp, f->sp);
      t_current = nullptr;
      if (!f->done) live++;
    }
    if (live == 1) _mm_pause();  // one lane left polling: as a lone thread would
  }
}

bool in_fiber() { return t_current != nullptr; }

void fiber_yield() {
  Fiber *f = t_current;
  if (!f) return;
  bz_fiber_swap(&f->sp, t_loop_sp);
}

GateDepth &gate_depth() { return t_current ? t_current->depth : t_depth; }

cudaError_t stream_wait(cudaStream_t s) {
  if (!in_fiber()) return cudaStreamSynchronize(s);
  for (;;) {
    const cudaError_t e = cudaStreamQuery(s);
    if (e != cudaErrorNotReady) return e;
    fiber_yield();
  }
}

cudaError_t event_wait(cudaEvent_t ev) {
  if (!in_fiber()) return cudaEventSynchronize(ev);
  for (;;) {
    const cudaError_t e = cudaEventQuery(ev);
    if (e != cudaErrorNotReady) return e;
    fiber_yield();
  }
}

unsigned long long fiber_selftest(int threads, int fibers, int yields, bool *ok) {
  std::vector<unsigned long long> sums(threads, 0);
  std::vector<int> good(threads, 1);
  auto thread_main = [&](int t) {
    FiberLoop loop((size_t)64 << 10);
    std::vector<int> finished(fibers, 0);
    unsigned long long h = 1469598103934665603ull;
    for (int i = 0; i < fibers; i++) {
      loop.add([&, i] {
        for (int k = 0; k < yields; k++) {
          gate_depth().resident += i + 1;
          h = (h ^ (unsigned long long)(i * 1000003 + k)) * 1099511628211ull;
          fiber_yield();
          if (gate_depth().resident != i + 1) good[t] = 0;  // another fiber's count leaked in
          gate_depth().resident -= i + 1;
          if (k == yields / 2) {
            try {
              volatile double x = 1.0 / (k + 3);
              fiber_yield();
              throw std::runtime_error(std::to_string(x));
            } catch (const std::exception &e) {
              if (e.what()[0] == 0) good[t] = 0;
            }
          }
        }
        finished[i] = 1;
      });
    }
    loop.run();
    for (int v : finished) good[t] &= v;
    if (gate_depth().resident != 0) good[t] = 0;  // the thread's own counter untouched
    sums[t] = h;
  };
  std::vector<std::thread> ts;
  for (int t = 1; t < threads; t++) ts.emplace_back(thread_main, t);
  thread_main(0);
  for (auto &x : ts) x.join();
  unsigned long long out = 0;
  bool all = true;
  for (int t = 0; t < threads; t++) {
    out = out * 31 + sums[t];
    all &= good[t] != 0;
  }
  *ok = all;
  return out;
}

}  // namespace bz
