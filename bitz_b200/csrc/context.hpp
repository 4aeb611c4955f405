// Per-process device context: one stream and the scratch buffers the stage
// kernels reuse across calls, grown on demand and kept resident in HBM.
#pragma once
#include <cuda_runtime.h>

#include <initializer_list>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "device.cuh"
#include "eq.cuh"
#include "gkr.hpp"
#include "spartan.hpp"
#include "post_gkr.hpp"

namespace bz {

constexpr int kMaxPointGkr = 64;

template <class T>
class DeviceBuffer {
 public:
  DeviceBuffer() = default;
  explicit DeviceBuffer(size_t n) { resize(n); }
  ~DeviceBuffer() { release(); }
  DeviceBuffer(const DeviceBuffer &) = delete;
  DeviceBuffer &operator=(const DeviceBuffer &) = delete;
  DeviceBuffer(DeviceBuffer &&o) noexcept : p_(o.p_), n_(o.n_) {
    o.p_ = nullptr;
    o.n_ = 0;
  }
  void resize(size_t n) {
    if (n <= n_) return;
    AllocScope gate;
    release();
    BZ_CUDA(cudaMalloc(&p_, (n ? n : 1) * sizeof(T)));
    n_ = n;
  }
  void release() {
    if (p_) {
      AllocScope gate(false);
      cudaFree(p_);
    }
    p_ = nullptr;
    n_ = 0;
  }
  void upload(const T *h, size_t n, cudaStream_t s) {
    resize(n);
    BZ_CUDA(cudaMemcpyAsync(p_, h, n * sizeof(T), cudaMemcpyHostToDevice, s));
  }
  void download(T *h, size_t n, cudaStream_t s) const {
    BZ_CUDA(cudaMemcpyAsync(h, p_, n * sizeof(T), cudaMemcpyDeviceToHost, s));
  }
  T *get() const { return p_; }
  size_t size() const { return n_; }

 private:
  T *p_ = nullptr;
  size_t n_ = 0;
};

// Page-locked host memory, grown on demand (for asynchronous copies).
template <class T>
class PinnedBuffer {
 public:
  PinnedBuffer() = default;
  ~PinnedBuffer() {
    if (p_) {
      AllocScope gate(false);
      cudaFreeHost(p_);
    }
  }
  PinnedBuffer(const PinnedBuffer &) = delete;
  PinnedBuffer &operator=(const PinnedBuffer &) = delete;
  T *get(size_t n) {
    if (n > n_) {
      AllocScope gate;
      if (p_) cudaFreeHost(p_);
      p_ = nullptr;
      n_ = 0;
      BZ_CUDA(cudaMallocHost(&p_, (n ? n : 1) * sizeof(T)));
      n_ = n;
    }
    return p_;
  }

 private:
  T *p_ = nullptr;
  size_t n_ = 0;
};

struct Workspace;  // the end-to-end prover's reusable buffers (prover.cpp)

// A prover lane: one stream, one round mailbox and the scratch buffers that a
// proof running on the stream reuses. Independent lanes prove concurrently;
// one lane runs one proof at a time.
class Context {
 public:
  Context();
  ~Context();
  Context(const Context &) = delete;
  Context &operator=(const Context &) = delete;

  // The process-wide default lane, created on first use on the current device.
  static Context &get();

  cudaStream_t stream() const { return stream_; }
  RoundChannel *channel() { return &channel_; }
  // The lane's round controls (kMaxPointGkr entries), used by one phase at a time.
  RoundCtl *round_ctl() { return gk_ctl_.get(); }
  // Grid of the resident Spartan grid rounds on this lane (0: none).
  int sp_mid_blocks() const { return sp_mid_blocks_; }
  // Grid of the resident post-GKR and Ligerito folds on this lane (0: none).
  int pg_mid_blocks() const { return pg_.mid_blocks; }
  // Prover workspace slot, owned by the lane (created by the prover).
  std::shared_ptr<Workspace> workspace;

  PostGkrScratch &post_gkr_scratch(size_t entries) {
    if (pg_.capacity < entries) {
      pg_w0_.resize(entries);
      pg_v0_.resize(entries);
      pg_w1_.resize(entries);
      pg_v1_.resize(entries);
      pg_.w0 = pg_w0_.get();
      pg_.v0 = pg_v0_.get();
      pg_.w1 = pg_w1_.get();
      pg_.v1 = pg_v1_.get();
      pg_.capacity = entries;
    }
    return pg_;
  }

  GkrScratch &gkr_scratch(int s) {
    size_t leaves = (size_t)128 << s;
    if (gk_.capacity < leaves) {
      size_t total = 0;
      for (int j = 0; j < 8; j++) total += leaves >> j;
      gk_layers_.resize(total);
      size_t off = 0;
      for (int j = 0; j < 8; j++) {
        gk_.layer[j] = gk_layers_.get() + off;
        off += leaves >> j;
      }
      gk_eq_.resize(leaves / 4);
      gk_eq_scratch_.resize(eq_scratch_entries(6 + s));
      gk_.eq = gk_eq_.get();
      gk_.eq_scratch = gk_eq_scratch_.get();
      gk_.capacity = leaves;
    }
    return gk_;
  }

 private:
  cudaStream_t stream_ = nullptr;
  PostGkrScratch pg_;
  DeviceBuffer<f128> pg_w0_, pg_v0_, pg_w1_, pg_v1_;
  DeviceBuffer<unsigned long long> acc_;
  uint64_t *host_ = nullptr;
  GkrScratch gk_;
  DeviceBuffer<f128> gk_layers_, gk_eq_, gk_eq_scratch_, gk_pair_;
  DeviceBuffer<RoundCtl> gk_ctl_;
  RoundChannel channel_;
  DeviceBuffer<unsigned int> counter_;
  int sp_mid_blocks_ = 0;
};

// Loads kernels now (cudaFuncGetAttributes), so no kernel is loaded on its
// first launch while a kernel that waits for a host thread is in flight: a
// load may wait for the running kernels to finish.
void load_kernels(std::initializer_list<const void *> kernels);

// A lane held for one proof: the process's default lane when no other proof
// holds it, else one from the process's lane pool (given back when the lease
// ends). Defined with the C ABI (capi_stages.cpp).
class LaneLease {
 public:
  LaneLease();
  ~LaneLease();
  LaneLease(const LaneLease &) = delete;
  LaneLease &operator=(const LaneLease &) = delete;
  Context *lane() const { return lane_; }

 private:
  Context *lane_ = nullptr;
  std::unique_ptr<Context> pool_;
  int device_ = 0;
  bool default_ = false;
};

// Optional CUDA-event timing of every launch of the probed kernels, with the
// algorithmic bytes each launch moves and the GF(2^128) products it computes
// (a measurement aid; off by default). Events are recorded on the launching
// stream; totals are collected once the stream has synchronised. While the
// probe is on, every sumcheck round runs as its own launch (as under a kernel
// profiler), so each probed launch is timed alone.
class KernelProbe {
 public:
  static KernelProbe &get();
  // "" or null: off; "*": every probed launch site; else a comma-separated
  // list of kernel names. Enabling resets the totals.
  void enable(const char *spec);
  bool active() const { return active_; }
  bool on(const char *name) const;
  void before(cudaStream_t s);
  // GF(2^128) products of the launch: `gmuls` reduced general products,
  // `wides` unreduced ones (reduced once per sum), `tables` products by one
  // fixed factor (the round's challenge) through its window table
  void after(cudaStream_t s, const char *name, double bytes, double gmuls = 0, double wides = 0,
             double tables = 0);
  void collect();  // adds the finished launches' times to the totals
  // Totals of one kernel (zeros if it never ran).
  // out: ms, bytes, gmuls, wides, tables
  void read(const char *name, double out[5], unsigned long long *launches);
  // Names of the kernels with at least one collected launch, comma-separated.
  std::string names();

 private:
  struct Totals {
    double v[5] = {0, 0, 0, 0, 0};  // ms, bytes, gmuls, wides, tables
    unsigned long long launches = 0;
  };
  struct Pending {
    std::string name;
    double work[4];  // bytes, gmuls, wides, tables
  };
  void collect_locked_full();
  mutable std::mutex mu_;
  bool active_ = false, all_ = false;
  std::vector<std::string> targets_;
  std::vector<cudaEvent_t> ev_;
  std::vector<Pending> pending_;
  size_t used_ = 0;
  std::map<std::string, Totals> totals_;
};

}  // namespace bz
