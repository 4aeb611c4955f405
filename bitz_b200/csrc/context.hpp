// Per-process device context: one stream and the scratch buffers the stage
// kernels reuse across calls, grown on demand and kept resident in HBM.
#pragma once
#include <cuda_runtime.h>

#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "device.cuh"
#include "eq.cuh"
#include "gkr.hpp"
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
  // The lane proves alone: sumcheck middle rounds may run in resident kernels.
  bool resident_middle() const { return gk_.resident_middle; }
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
};

// Optional CUDA-event timing of every launch of one named kernel, with the
// algorithmic bytes each launch moves (a measurement aid; off by default).
// Events are recorded on the launching stream; totals are collected once the
// stream has synchronised.
class KernelProbe {
 public:
  static KernelProbe &get();
  void enable(const char *name);  // null or "" turns the probe off
  bool on(const char *name) const { return active_ && target_ == name; }
  void before(cudaStream_t s);
  void after(cudaStream_t s, double bytes);
  void collect();  // adds the finished launches' times to the totals
  void read(double *ms, double *bytes, unsigned long long *launches);

 private:
  void collect_locked_full();
  std::mutex mu_;
  bool active_ = false;
  std::string target_;
  std::vector<cudaEvent_t> ev_;
  std::vector<double> pending_bytes_;
  size_t used_ = 0;
  double ms_ = 0, bytes_ = 0;
  unsigned long long launches_ = 0;
};

}  // namespace bz
