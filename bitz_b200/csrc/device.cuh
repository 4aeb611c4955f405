// Device-side helpers shared by the kernels: block reductions of GF(2^128)
// and prime-field partial sums, launch sizing and error checks.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include <atomic>
#include <condition_variable>
#include <mutex>
#include <stdexcept>
#include <string>

#include "fiber.hpp"
#include "field.cuh"

namespace bz {

struct CudaError : std::runtime_error {
  explicit CudaError(const std::string &s) : std::runtime_error(s) {}
};

#define BZ_CUDA(call)                                                                          \
  do {                                                                                         \
    cudaError_t e_ = (call);                                                                   \
    if (e_ != cudaSuccess)                                                                     \
      throw ::bz::CudaError(std::string(#call) + ": " + cudaGetErrorString(e_) + " at " +     \
                            __FILE__ + ":" + std::to_string(__LINE__));                        \
  } while (0)

// Every launch site ends in BZ_LAUNCH_CHECK(), which also counts the launch
// (read through bitz_launch_count()).
std::atomic<unsigned long long> &launch_counter();
#define BZ_LAUNCH_CHECK()           \
  do {                              \
    ++::bz::launch_counter();       \
    BZ_CUDA(cudaGetLastError());    \
  } while (0)

constexpr int kThreads = 256;
// 148 SMs on B200; grids are sized in multiples of the SM count and walked
// with grid-stride loops, so one launch shape serves every table size.
constexpr int kSMs = 148;

inline int grid_for(size_t work, int per_block = kThreads, int max_blocks = kSMs * 8) {
  size_t b = (work + per_block - 1) / per_block;
  if (b < 1) b = 1;
  if (b > (size_t)max_blocks) b = max_blocks;
  return (int)b;
}

// A round's result delivered without a copy or a stream sync: the last block
// of the kernel writes the accumulated words into host-mapped pinned memory.
// Every 64-bit slot carries 32 data bits under a 32-bit tag (the round's
// sequence number); naturally aligned 8-byte writes are single-copy atomic,
// so the host accepts the result once every slot shows the current tag, and
// the device needs no system-scope fence to order data before a flag.
constexpr int kMailboxWords = 8;  // 64-bit data words per publication
constexpr int kHandoverWords = 1280;  // 64-bit data words of a handover
struct Mailbox {
  unsigned long long slot[2 * kMailboxWords];
};

#if defined(__CUDACC__)
// One 16-byte store per word: both tagged halves leave in one transaction.
__device__ __forceinline__ void mailbox_post(Mailbox *mb, unsigned long long seq, int k,
                                             unsigned long long v) {
  const unsigned long long tag = seq << 32;
  unsigned long long *p = mb->slot + 2 * k;
  asm volatile("st.volatile.global.v2.u64 [%0], {%1, %2};" ::"l"(p),
               "l"(tag | (v & 0xffffffffull)), "l"(tag | (v >> 32))
               : "memory");
}

// Word k of a handover (tagged like a mailbox word) into the mapped area.
__device__ __forceinline__ void handover_post(unsigned long long *slots, unsigned long long seq,
                                              int k, unsigned long long v) {
  const unsigned long long tag = seq << 32;
  asm volatile("st.volatile.global.v2.u64 [%0], {%1, %2};" ::"l"(slots + 2 * k),
               "l"(tag | (v & 0xffffffffull)), "l"(tag | (v >> 32))
               : "memory");
}
#endif

// Where a round kernel publishes: counter counts finished blocks (reset by
// the last one); a null counter disables publishing.
struct Publish {
  unsigned int *counter;
  Mailbox *mailbox;  // device view of the mapped mailbox
  unsigned long long seq;
};

#if defined(__CUDACC__)
// Called by every thread after the block's atomics (issued by thread 0):
// the last block to finish reads and clears the N accumulator words and
// posts them, tagged, to the mailbox.
template <int N>
__device__ __forceinline__ void publish(unsigned long long *acc, const Publish &p) {
  static_assert(N <= kMailboxWords, "mailbox too small");
  if (!p.counter) return;
  if (threadIdx.x == 0) {
    __threadfence();
    unsigned int prev = atomicAdd(p.counter, 1u);
    if (prev == gridDim.x - 1) {
      __threadfence();
#pragma unroll
      for (int k = 0; k < N; k++) mailbox_post(p.mailbox, p.seq, k, atomicExch(acc + k, 0ull));
      *p.counter = 0;
    }
  }
}

// XOR-reduce `n` 64-bit words across the block and fold the block's result
// into `acc` with atomicXor. XOR is associative and commutative, so the total
// is the same whatever the order the blocks land in.
template <int N>
__device__ __forceinline__ void block_xor_atomic(uint64_t (&v)[N], unsigned long long *acc) {
  __shared__ uint64_t sm[N][kThreads / 32];
#pragma unroll
  for (int k = 0; k < N; k++) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v[k] ^= __shfl_xor_sync(0xffffffffu, v[k], off);
  }
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < N; k++) sm[k][warp] = v[k];
  }
  __syncthreads();
  if (warp == 0) {
    int nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < N; k++) {
      uint64_t x = lane < nw ? sm[k][lane] : 0;
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) x ^= __shfl_xor_sync(0xffffffffu, x, off);
      if (lane == 0 && x) atomicXor(acc + k, (unsigned long long)x);
    }
  }
}

// XOR-reduce `n` 64-bit words across the block; thread 0 ends with the
// totals in v. Every thread must call it (it synchronises the block twice).
template <int N>
__device__ __forceinline__ void block_xor_reduce(uint64_t (&v)[N]) {
  __shared__ uint64_t sm[N][kThreads / 32];
#pragma unroll
  for (int k = 0; k < N; k++) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v[k] ^= __shfl_xor_sync(0xffffffffu, v[k], off);
  }
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < N; k++) sm[k][warp] = v[k];
  }
  __syncthreads();
  if (warp == 0) {
    int nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < N; k++) {
      uint64_t x = lane < nw ? sm[k][lane] : 0;
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) x ^= __shfl_xor_sync(0xffffffffu, x, off);
      v[k] = x;
    }
  }
  __syncthreads();
}

// block_xor_atomic, then publish the totals when this is the last block.
template <int N>
__device__ __forceinline__ void block_xor_publish(uint64_t (&v)[N], unsigned long long *acc,
                                                  const Publish &p) {
  block_xor_atomic<N>(v, acc);
  publish<N>(acc, p);
}

// Sum `N` prime-field values across the block (mod q) and write the block's
// partial sums to out[blockIdx.x * N + k]; the host (or a second pass) adds
// the per-block partials. Modular addition is exact in any order.
template <int N>
__device__ __forceinline__ void block_fp_sum(fp (&v)[N], const FpCtx &c, fp *out) {
  __shared__ fp sm[N][kThreads / 32];
#pragma unroll
  for (int k = 0; k < N; k++) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      fp o;
      o.lo = __shfl_xor_sync(0xffffffffu, v[k].lo, off);
      o.hi = __shfl_xor_sync(0xffffffffu, v[k].hi, off);
      v[k] = fp_add(v[k], o, c);
    }
  }
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < N; k++) sm[k][warp] = v[k];
  }
  __syncthreads();
  if (warp == 0) {
    int nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < N; k++) {
      fp x = lane < nw ? sm[k][lane] : fp_zero();
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        fp o;
        o.lo = __shfl_xor_sync(0xffffffffu, x.lo, off);
        o.hi = __shfl_xor_sync(0xffffffffu, x.hi, off);
        x = fp_add(x, o, c);
      }
      if (lane == 0) out[blockIdx.x * N + k] = x;
    }
  }
}

#endif

// Host side of a mailbox: one mapped pinned page, a device counter, and the
// next sequence number. wait() polls with a time limit and surfaces any
// stream error instead of spinning on a failed kernel.
struct RoundChannel {
  Mailbox *host = nullptr;  // host view
  Mailbox *dev = nullptr;   // device view
  unsigned int *counter = nullptr;
  unsigned long long next = 0;
  // The reverse direction, for kernels that run several rounds and wait for
  // the host's challenge between them: same tagged format, host to device.
  Mailbox *down_host = nullptr, *down_dev = nullptr;
  unsigned long long down_next = 0;
  // host time spent inside wait() and the number of waits (phase timer)
  unsigned long long wait_ns = 0, waits = 0;
  // A word in the same mapped page that the lane's kernels set when a bounded
  // wait of theirs ran out (a TMA copy that did not land); check_device_error
  // throws (and clears it) when it is set.
  unsigned int *err_host = nullptr, *err_dev = nullptr;
  void check_device_error(const char *stage);
  // A larger tagged area in the same mapped allocation (kHandoverWords words,
  // one 16-byte slot each as in the mailbox) for a kernel that hands a
  // sumcheck's last small tables to the host instead of waiting for its
  // challenges; wait_handover reads publication `seq` of n words.
  unsigned long long *handover_host = nullptr, *handover_dev = nullptr;
  void wait_handover(cudaStream_t s, unsigned long long seq, uint64_t *out, int n);
  Publish arm() { return Publish{counter, dev, ++next}; }
  // Waits for the publication armed last; copies n payload words.
  void wait(cudaStream_t s, uint64_t *out, int n);
  // Posts n words to the device as publication down_next + 1.
  void send(const uint64_t *words, int n);
  // Posts an abort marker that a waiting kernel reads as "stop"; clear_down
  // empties the downbox again once no kernel can be waiting.
  void abort();
  void clear_down();
};

// Queued sumcheck rounds. With the host's challenges delivered to the
// device, the rounds of a sumcheck can all be queued at its start, so no
// round waits for a launch from the host: the last block of each round
// kernel posts the round's message, then waits (bounded) for the next
// challenge in the lane's downbox and leaves it in `out` for the next kernel
// in the stream, which reads it from `in`. Only that one block waits; the
// next kernel starts when it has left. A missing challenge (time limit or
// the host's abort marker) leaves flag 2, and every later kernel of the chain
// passes it on and does no work.
//
// RoundCtl: one challenge in device memory (flag 1: valid, 2: the chain
// stopped); `done` counts the blocks of a resident kernel through a round.
struct RoundCtl {
  unsigned long long r_lo, r_hi;
  unsigned int flag, done;
  unsigned long long pad;
};

struct RoundLink {
  const RoundCtl *in;       // this round's challenge; null: the launch argument
  RoundCtl *out;            // the next challenge; null: no wait
  const Mailbox *down;      // the host's downbox
  unsigned long long dseq;  // the host's publication of the next challenge
};
constexpr unsigned long long kRoundWaitNs = 2000000000ull;  // 2 s per challenge

// Whether kernels that wait for their lane's host thread may run (resident
// tails, queued rounds, the resident middle rounds). BITZ_RESIDENT_ROUNDS=0
// turns them off and =1 on. Otherwise they are off when a CUDA injection tool
// announces itself (CUDA_INJECTION64_PATH), or when the process's first lane
// found that its host thread cannot reach a running kernel (a kernel that
// waits up to 100 ms for one word from the host got none): a kernel profiler
// holds the host at every launch until the kernel has finished, so a kernel
// that waits for the host would sit out its time limit. The proof bytes are
// the same either way.
bool resident_rounds_enabled();

// Kernels that wait for their lane's host thread, and calls that wait for the
// whole device. Such a kernel must never be in flight while another thread
// is inside cudaFree, cudaFreeHost, cudaMalloc, cudaMallocHost or
// cudaHostAlloc: the call waits for the kernel, the driver can hold the
// lane's host thread (its next launch or stream query) behind the call, and
// neither moves until the kernel's time limit ends the proof. A lane holds a
// ResidentScope from before it launches the first such kernel of a stretch
// until the stretch has ended; those calls run under an AllocScope, which
// waits until no ResidentScope is held and holds new ones back meanwhile.
// Scopes nest within a thread; an allocation inside a ResidentScope of its
// own thread is a bug and throws.
class DeviceGate {
 public:
  static DeviceGate &get();
  void enter_resident();
  void leave_resident();
  void enter_alloc();
  void leave_alloc();
  // Since the process started: allocation stretches and the nanoseconds they
  // waited for the gate, resident stretches and the nanoseconds they waited.
  void stats(unsigned long long out[4]) const;

 private:
  std::mutex mu_;
  std::condition_variable cv_;
  int residents_ = 0, allocs_waiting_ = 0;
  bool alloc_ = false;
  std::atomic<unsigned long long> alloc_n_{0}, alloc_wait_ns_{0}, resident_n_{0},
      resident_wait_ns_{0};
};

class ResidentScope {
 public:
  explicit ResidentScope(bool on = true);
  ~ResidentScope();
  ResidentScope(const ResidentScope &) = delete;
  ResidentScope &operator=(const ResidentScope &) = delete;

 private:
  bool on_;
};

class AllocScope {
 public:
  // `strict`: throw when this thread holds a ResidentScope (false in
  // destructors, which must not throw and then free without the gate).
  explicit AllocScope(bool strict = true);
  ~AllocScope();
  AllocScope(const AllocScope &) = delete;
  AllocScope &operator=(const AllocScope &) = delete;

 private:
  bool on_ = false;
};

#if defined(__CUDACC__)
// The host's abort marker: every slot tagged 0xffffffff.
constexpr unsigned long long kDownAbortTag = 0xffffffffull;

__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Thread-level wait for host publication `seq` (n words) in a device-view
// mailbox. Bounded by time: returns false after `limit_ns` or on the host's
// abort marker, so a kernel never spins forever on a host that went away.
__device__ __forceinline__ bool mailbox_wait_device(const Mailbox *mb, unsigned long long seq,
                                                    int n, unsigned long long *out,
                                                    unsigned long long limit_ns) {
  // Every poll issues all of its 16-byte loads before looking at any, so one
  // poll costs one round trip to host memory, and the words of a successful
  // poll are used as read.
  const unsigned long long *s = mb->slot;
  const unsigned long long tag = seq & 0xffffffffull;
  const unsigned long long t0 = globaltimer_ns();
  for (;;) {
    unsigned long long x[kMailboxWords], y[kMailboxWords];
#pragma unroll
    for (int k = 0; k < kMailboxWords; k++)
      if (k < n)
        asm volatile("ld.volatile.global.v2.u64 {%0, %1}, [%2];"
                     : "=l"(x[k]), "=l"(y[k])
                     : "l"(s + 2 * k)
                     : "memory");
    bool ready = true, aborted = false;
#pragma unroll
    for (int k = 0; k < kMailboxWords; k++)
      if (k < n) {
        const unsigned long long tx = x[k] >> 32, ty = y[k] >> 32;
        aborted |= tx == kDownAbortTag || ty == kDownAbortTag;
        ready &= tx == tag && ty == tag;
      }
    if (aborted) return false;
    if (ready) {
#pragma unroll
      for (int k = 0; k < kMailboxWords; k++)
        if (k < n) out[k] = (x[k] & 0xffffffffull) | (y[k] << 32);
      return true;
    }
    if (globaltimer_ns() - t0 > limit_ns) return false;
    __nanosleep(32);
  }
}

// Every thread calls it: the challenge words from lk.in (lk.in not null);
// false when the chain has stopped, which block 0 passes on to lk.out.
__device__ __forceinline__ bool link_begin(const RoundLink &lk, unsigned long long &w0,
                                           unsigned long long &w1) {
  __shared__ unsigned long long s[3];
  if (threadIdx.x == 0) {
    s[0] = lk.in->r_lo;
    s[1] = lk.in->r_hi;
    s[2] = lk.in->flag;
  }
  __syncthreads();
  w0 = s[0];
  w1 = s[1];
  if (s[2] == 1) return true;
  if (blockIdx.x == 0 && threadIdx.x == 0 && lk.out) lk.out->flag = 2;
  return false;
}

// One thread of a round's last block, after its post: the next challenge
// from the downbox into lk.out (nothing without lk.out).
__device__ __forceinline__ void link_fetch(const RoundLink &lk) {
  if (!lk.out) return;
  unsigned long long w[2] = {0, 0};
  const bool ok = mailbox_wait_device(lk.down, lk.dseq, 2, w, kRoundWaitNs);
  lk.out->r_lo = w[0];
  lk.out->r_hi = w[1];
  lk.out->flag = ok ? 1u : 2u;
}

// Block 0's relay of a challenge to the other blocks of a resident kernel:
// flag written last with release semantics, read with acquire (bounded).
__device__ __forceinline__ void relay_post(RoundCtl *cl, const unsigned long long w[2], bool ok) {
  cl->r_lo = w[0];
  cl->r_hi = w[1];
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(&cl->flag), "r"(ok ? 1u : 2u)
               : "memory");
}

__device__ __forceinline__ bool relay_wait(const RoundCtl *cl, unsigned long long w[2]) {
  const unsigned long long t0 = globaltimer_ns();
  for (;;) {
    unsigned int f;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(f) : "l"(&cl->flag) : "memory");
    if (f == 1) {
      asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(w[0]) : "l"(&cl->r_lo) : "memory");
      asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(w[1]) : "l"(&cl->r_hi) : "memory");
      return true;
    }
    if (f == 2 || globaltimer_ns() - t0 > kRoundWaitNs) return false;
    __nanosleep(64);
  }
}

// Every thread of every block of a resident kernel calls it: block 0 waits
// for host publication dseq in the downbox and relays it through cl; the
// other blocks read the relay. The challenge words land in w (every thread);
// false when it did not come (time limit or abort marker).
__device__ __forceinline__ bool resident_challenge(const Mailbox *down, unsigned long long dseq,
                                                   RoundCtl *cl, unsigned long long w[2]) {
  __shared__ unsigned long long rs[2];
  __shared__ int ok_s;
  if (threadIdx.x == 0) {
    unsigned long long v[2] = {0, 0};
    bool ok;
    if (blockIdx.x == 0) {
      ok = mailbox_wait_device(down, dseq, 2, v, kRoundWaitNs);
      relay_post(cl, v, ok);
    } else {
      ok = relay_wait(cl, v);
    }
    rs[0] = v[0];
    rs[1] = v[1];
    ok_s = ok;
  }
  __syncthreads();
  w[0] = rs[0];
  w[1] = rs[1];
  const bool ok = ok_s;
  __syncthreads();
  return ok;
}

// publish<N> (after the block's atomics), then the last block fetches the
// next challenge for the round link.
template <int N>
__device__ __forceinline__ void publish_link(unsigned long long *acc, const Publish &p,
                                             const RoundLink &lk) {
  static_assert(N <= kMailboxWords, "mailbox too small");
  if (!p.counter) return;
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned int prev = atomicAdd(p.counter, 1u);
    if (prev == gridDim.x - 1) {
      __threadfence();
#pragma unroll
      for (int k = 0; k < N; k++) mailbox_post(p.mailbox, p.seq, k, atomicExch(acc + k, 0ull));
      *p.counter = 0;
      link_fetch(lk);
    }
  }
}
#endif

#if defined(__CUDACC__)
// Products by one fixed element r through 4-bit windows: b = sum over j of
// v_j X^(4j) (v_j the j-th nibble of b), so r b = XOR over j of the entry
// r v_j X^(4j). The 32 x 16 entries live in shared memory as separate low and
// high 64-bit words: a row of 16 words spans the 32 banks once, so the lanes
// of a half-warp never conflict, whatever nibbles they look up. A product is
// 32 independent lookups instead of about 550 dependent integer instructions.
struct MulTable {
  uint64_t lo[32][16], hi[32][16];
};

// Every thread of the block calls it; it synchronises the block twice.
__device__ __forceinline__ void mul_table_build(MulTable &T, f128 r) {
  for (int k = threadIdx.x; k < 128; k += blockDim.x) {
    const f128 b = gmul_xk(r, k);  // r X^k: the single-bit entry of window k / 4
    T.lo[k >> 2][1 << (k & 3)] = b.lo;
    T.hi[k >> 2][1 << (k & 3)] = b.hi;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < 512; e += blockDim.x) {
    const int j = e >> 4, v = e & 15;
    if (v != 0 && (v & (v - 1)) == 0) continue;  // written above
    uint64_t lo = 0, hi = 0;
#pragma unroll
    for (int b = 0; b < 4; b++)
      if ((v >> b) & 1) {
        lo ^= T.lo[j][1 << b];
        hi ^= T.hi[j][1 << b];
      }
    T.lo[j][v] = lo;
    T.hi[j][v] = hi;
  }
  __syncthreads();
}

__device__ __forceinline__ f128 mul_table(const MulTable &T, f128 b) {
  const uint32_t w[4] = {(uint32_t)b.lo, (uint32_t)(b.lo >> 32), (uint32_t)b.hi,
                         (uint32_t)(b.hi >> 32)};
  uint64_t lo = 0, hi = 0;
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int n = 0; n < 8; n++) {
      const uint32_t v = (w[i] >> (4 * n)) & 15u;
      lo ^= T.lo[8 * i + n][v];
      hi ^= T.hi[8 * i + n][v];
    }
  return mk(lo, hi);
}

__device__ __forceinline__ f128 ld(const f128 *p) {
  ulonglong2 v = *reinterpret_cast<const ulonglong2 *>(p);
  return mk(v.x, v.y);
}
__device__ __forceinline__ void st(f128 *p, f128 v) {
  *reinterpret_cast<ulonglong2 *>(p) = make_ulonglong2(v.lo, v.hi);
}
__device__ __forceinline__ int bit128(f128 e, int v) {
  return v < 64 ? (int)((e.lo >> v) & 1) : (int)((e.hi >> (v - 64)) & 1);
}
#endif

}  // namespace bz
