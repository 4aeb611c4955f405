#include "context.hpp"

#include "fiber.hpp"

#include <immintrin.h>

#include <atomic>
#include <mutex>
#include <set>
#include <chrono>
#include <thread>

namespace bz {

// True once the first 2n slots all carry the tag of publication `want`.
static bool slots_ready(const unsigned long long *slots, unsigned long long want, int n) {
  const volatile unsigned long long *s = slots;
  const unsigned long long tag = (want << 32) >> 32;
  for (int k = 0; k < 2 * n; k++)
    if ((s[k] >> 32) != tag) return false;
  return true;
}

// Waits until n tagged words of publication `want` are in `slots`, surfacing
// a failed or finished stream instead of spinning; copies the payload.
static void wait_slots(RoundChannel &ch, cudaStream_t s, const unsigned long long *slots,
                       unsigned long long want, uint64_t *out, int n) {
  auto t0 = std::chrono::steady_clock::now();
  uint64_t spins = 0;
  while (!slots_ready(slots, want, n)) {
    if ((++spins & 0x3ff) == 0) {
      cudaError_t e = cudaStreamQuery(s);
      if (e != cudaSuccess && e != cudaErrorNotReady)
        throw CudaError(std::string("round kernel failed: ") + cudaGetErrorString(e));
      if (e == cudaSuccess && !slots_ready(slots, want, n)) {
        // the stream is idle: its writes land within microseconds
        std::this_thread::sleep_for(std::chrono::milliseconds(2));
        if (!slots_ready(slots, want, n))
          throw CudaError("round kernel finished without publishing its result");
      }
      if (std::chrono::steady_clock::now() - t0 > std::chrono::seconds(30))
        throw CudaError("timed out waiting for a round result");
    }
    // on a fiber, let the thread's other lanes run; else spin briefly, then
    // give the core to other lanes' host threads
    if (in_fiber())
      fiber_yield();
    else if (spins < 4096)
      _mm_pause();
    else
      std::this_thread::yield();
  }
  std::atomic_thread_fence(std::memory_order_acquire);
  const volatile unsigned long long *p = slots;
  for (int k = 0; k < n; k++) out[k] = (p[2 * k] & 0xffffffffull) | (p[2 * k + 1] << 32);
  ch.wait_ns += (unsigned long long)std::chrono::duration_cast<std::chrono::nanoseconds>(
                    std::chrono::steady_clock::now() - t0)
                    .count();
  ch.waits++;
}

void RoundChannel::wait(cudaStream_t s, uint64_t *out, int n) {
  if (n > kMailboxWords) throw CudaError("mailbox read too long");
  wait_slots(*this, s, host->slot, next, out, n);
}

void RoundChannel::wait_handover(cudaStream_t s, unsigned long long seq, uint64_t *out, int n) {
  if (!handover_host || n > kHandoverWords) throw CudaError("handover read too long");
  wait_slots(*this, s, handover_host, seq, out, n);
}

void RoundChannel::send(const uint64_t *words, int n) {
  if (n > kMailboxWords) throw CudaError("downbox write too long");
  const unsigned long long tag = (++down_next & 0xffffffffull) << 32;
  // one aligned 16-byte store per word, so a device poll sees both halves
  unsigned long long *s = down_host->slot;
  for (int k = 0; k < n; k++) {
    __m128i v = _mm_set_epi64x((long long)(tag | (words[k] >> 32)),
                               (long long)(tag | (words[k] & 0xffffffffull)));
    _mm_store_si128(reinterpret_cast<__m128i *>(s + 2 * k), v);
  }
  std::atomic_thread_fence(std::memory_order_release);
}

void RoundChannel::check_device_error(const char *stage) {
  if (!err_host) return;
  volatile unsigned int *e = err_host;
  if (*e) {
    *e = 0;
    throw CudaError(std::string(stage) + ": a TMA copy did not land within its time limit");
  }
}

void RoundChannel::abort() {
  volatile unsigned long long *s = down_host->slot;
  for (int k = 0; k < 2 * kMailboxWords; k++) s[k] = 0xffffffffull << 32;
  std::atomic_thread_fence(std::memory_order_release);
}

void RoundChannel::clear_down() {
  volatile unsigned long long *s = down_host->slot;
  for (int k = 0; k < 2 * kMailboxWords; k++) s[k] = 0;
}

// The probe's result, set when the process's first lane is made: -1 not
// yet probed, 0 the host cannot reach a running kernel, 1 it can.
static std::atomic<int> g_host_reaches_kernel{-1};

bool resident_rounds_enabled() {
  static const int forced = [] {
    const char *e = getenv("BITZ_RESIDENT_ROUNDS");
    if (e && e[0] == '0') return 0;
    if (e && e[0] == '1') return 1;
    const char *inj = getenv("CUDA_INJECTION64_PATH");
    return (inj && inj[0]) ? 0 : -1;
  }();
  const bool on = forced >= 0 ? forced == 1 : g_host_reaches_kernel.load() != 0;
  // probed launches are timed one by one, each its own round
  return on && !KernelProbe::get().active();
}

void load_kernels(std::initializer_list<const void *> kernels) {
  cudaFuncAttributes a;
  for (const void *k : kernels) BZ_CUDA(cudaFuncGetAttributes(&a, k));
}

void preload_pcs_kernels();
void preload_eq_kernels();
void preload_gkr_kernels();
void preload_post_gkr_kernels();
void preload_spartan_kernels();
void preload_witness_kernels();
void preload_diag_kernels();
bool host_reaches_running_kernel(Context &lane);

// Once per device, when its first lane is made: every kernel of the library
// is loaded; and once per process, whether this host can reach a running
// kernel is probed on that lane (a tool that holds the host at every launch
// cannot run the kernels that wait for the host).
static void lane_bootstrap(Context &lane) {
  static std::mutex mu;
  static std::set<int> loaded;
  std::lock_guard<std::mutex> lk(mu);
  int dev = 0;
  BZ_CUDA(cudaGetDevice(&dev));
  if (loaded.insert(dev).second) {
    preload_pcs_kernels();
    preload_eq_kernels();
    preload_gkr_kernels();
    preload_post_gkr_kernels();
    preload_spartan_kernels();
    preload_witness_kernels();
    preload_diag_kernels();
  }
  if (g_host_reaches_kernel.load() < 0)
    g_host_reaches_kernel.store(host_reaches_running_kernel(lane) ? 1 : 0);
}

// ------------------------------------------------------------ DeviceGate

DeviceGate &DeviceGate::get() {
  static DeviceGate *g = new DeviceGate();
  return *g;
}

// A fiber must not block its thread in the gate: the thread's other fibers
// may hold the scopes it waits for. It polls and yields instead.
static unsigned long long ns_since(std::chrono::steady_clock::time_point t0) {
  return (unsigned long long)std::chrono::duration_cast<std::chrono::nanoseconds>(
             std::chrono::steady_clock::now() - t0)
      .count();
}

void DeviceGate::enter_resident() {
  std::unique_lock<std::mutex> lk(mu_);
  resident_n_++;
  if (alloc_ || allocs_waiting_ != 0) {
    const auto t0 = std::chrono::steady_clock::now();
    if (in_fiber()) {
      while (alloc_ || allocs_waiting_ != 0) {
        lk.unlock();
        fiber_yield();
        lk.lock();
      }
    } else {
      cv_.wait(lk, [&] { return !alloc_ && allocs_waiting_ == 0; });
    }
    resident_wait_ns_ += ns_since(t0);
  }
  residents_++;
}

void DeviceGate::leave_resident() {
  std::lock_guard<std::mutex> lk(mu_);
  if (--residents_ == 0) cv_.notify_all();
}

void DeviceGate::enter_alloc() {
  std::unique_lock<std::mutex> lk(mu_);
  alloc_n_++;
  allocs_waiting_++;
  if (alloc_ || residents_ != 0) {
    const auto t0 = std::chrono::steady_clock::now();
    if (in_fiber()) {
      while (alloc_ || residents_ != 0) {
        lk.unlock();
        fiber_yield();
        lk.lock();
      }
    } else {
      cv_.wait(lk, [&] { return !alloc_ && residents_ == 0; });
    }
    alloc_wait_ns_ += ns_since(t0);
  }
  allocs_waiting_--;
  alloc_ = true;
}

void DeviceGate::leave_alloc() {
  std::lock_guard<std::mutex> lk(mu_);
  alloc_ = false;
  cv_.notify_all();
}

void DeviceGate::stats(unsigned long long out[4]) const {
  out[0] = alloc_n_.load();
  out[1] = alloc_wait_ns_.load();
  out[2] = resident_n_.load();
  out[3] = resident_wait_ns_.load();
}

ResidentScope::ResidentScope(bool on) : on_(on) {
  if (on_ && gate_depth().resident++ == 0) DeviceGate::get().enter_resident();
}

ResidentScope::~ResidentScope() {
  if (on_ && --gate_depth().resident == 0) DeviceGate::get().leave_resident();
}

AllocScope::AllocScope(bool strict) {
  if (gate_depth().resident > 0) {
    if (strict) throw CudaError("device allocation while a round kernel of this lane may wait");
    return;  // unwinding out of a resident stretch: free without the gate
  }
  on_ = true;
  if (gate_depth().alloc++ == 0) DeviceGate::get().enter_alloc();
}

AllocScope::~AllocScope() {
  if (on_ && --gate_depth().alloc == 0) DeviceGate::get().leave_alloc();
}

Context::Context() {
  AllocScope gate;
  BZ_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
  acc_.resize(8 * 128);
  BZ_CUDA(cudaMallocHost(&host_, 64 * sizeof(uint64_t)));
  pg_.acc = acc_.get();
  pg_.host = host_;
  gk_pair_.resize(2);
  gk_.acc = acc_.get();
  gk_.host = host_;
  gk_.pair = gk_pair_.get();
  gk_ctl_.resize(kMaxPointGkr);
  gk_.ctl = gk_ctl_.get();
  // the round mailbox: one mapped pinned page and a device block counter
  void *mb = nullptr;
  // one mapped allocation: mailbox (0), downbox (512), error word (1024),
  // handover area (4096, 16 bytes per word)
  const size_t mapped = 4096 + 16 * (size_t)kHandoverWords;
  BZ_CUDA(cudaHostAlloc(&mb, mapped, cudaHostAllocMapped));
  memset(mb, 0, mapped);
  channel_.host = (Mailbox *)mb;
  void *mbd = nullptr;
  BZ_CUDA(cudaHostGetDevicePointer(&mbd, mb, 0));
  channel_.dev = (Mailbox *)mbd;
  channel_.down_host = (Mailbox *)((char *)mb + 512);
  channel_.down_dev = (Mailbox *)((char *)mbd + 512);
  channel_.err_host = (unsigned int *)((char *)mb + 1024);
  channel_.err_dev = (unsigned int *)((char *)mbd + 1024);
  channel_.handover_host = (unsigned long long *)((char *)mb + 4096);
  channel_.handover_dev = (unsigned long long *)((char *)mbd + 4096);
  counter_.resize(1);
  BZ_CUDA(cudaMemset(counter_.get(), 0, sizeof(unsigned int)));
  channel_.counter = counter_.get();
  pg_.channel = &channel_;
  pg_.ctl = gk_ctl_.get();
  gk_.channel = &channel_;
  gk_.mid_blocks = gkr_mid_blocks(false);
  sp_mid_blocks_ = ::bz::sp_mid_blocks(false);
  pg_.mid_blocks = ::bz::pg_mid_blocks(false);
  lane_bootstrap(*this);
}

Context::~Context() {
  if (stream_) cudaStreamSynchronize(stream_);
  workspace.reset();
  AllocScope gate(false);
  if (channel_.host) cudaFreeHost(channel_.host);
  if (host_) cudaFreeHost(host_);
  if (stream_) cudaStreamDestroy(stream_);
}

std::atomic<unsigned long long> &launch_counter() {
  static std::atomic<unsigned long long> n{0};
  return n;
}

Context &Context::get() {
  // One default lane per process, created on first use on the current device.
  // It proves one statement at a time with the GPU to itself, so its resident
  // middle rounds (GKR, Spartan, post-GKR and Ligerito) use grids of 128
  // blocks; pool lanes, which share the GPU, run those rounds as queued
  // launches (or 32-block grids with BITZ_POOL_MID=1).
  static Context *ctx = [] {
    Context *c = new Context();
    c->gk_.mid_blocks = gkr_mid_blocks(true);
    c->sp_mid_blocks_ = ::bz::sp_mid_blocks(true);
    c->pg_.mid_blocks = ::bz::pg_mid_blocks(true);
    return c;
  }();
  return *ctx;
}

// ------------------------------------------------------------ KernelProbe

KernelProbe &KernelProbe::get() {
  static KernelProbe *p = new KernelProbe();
  return *p;
}

void KernelProbe::enable(const char *spec) {
  std::lock_guard<std::mutex> lk(mu_);
  const std::string sp = spec ? spec : "";
  targets_.clear();
  size_t at = 0;
  while (at <= sp.size() && !sp.empty()) {
    size_t comma = sp.find(',', at);
    if (comma == std::string::npos) comma = sp.size();
    if (comma > at) targets_.push_back(sp.substr(at, comma - at));
    at = comma + 1;
  }
  all_ = sp == "*";
  active_ = !targets_.empty();
  totals_.clear();
  used_ = 0;
  pending_.clear();
  if (active_ && ev_.empty()) {
    ev_.resize(2 * 4096);
    for (auto &e : ev_) BZ_CUDA(cudaEventCreate(&e));
  }
}

bool KernelProbe::on(const char *name) const {
  if (!active_) return false;
  if (all_) return true;
  std::lock_guard<std::mutex> lk(mu_);
  for (const auto &t : targets_)
    if (t == name) return true;
  return false;
}

void KernelProbe::before(cudaStream_t s) {
  std::lock_guard<std::mutex> lk(mu_);
  if (2 * used_ + 1 >= ev_.size()) collect_locked_full();
  BZ_CUDA(cudaEventRecord(ev_[2 * used_], s));
}

void KernelProbe::after(cudaStream_t s, const char *name, double bytes, double gmuls,
                        double wides, double tables) {
  std::lock_guard<std::mutex> lk(mu_);
  BZ_CUDA(cudaEventRecord(ev_[2 * used_ + 1], s));
  pending_.push_back(Pending{name, {bytes, gmuls, wides, tables}});
  used_++;
}

void KernelProbe::collect() {
  std::lock_guard<std::mutex> lk(mu_);
  collect_locked_full();
}

void KernelProbe::collect_locked_full() {
  for (size_t i = 0; i < used_; i++) {
    BZ_CUDA(cudaEventSynchronize(ev_[2 * i + 1]));
    float ms = 0;
    BZ_CUDA(cudaEventElapsedTime(&ms, ev_[2 * i], ev_[2 * i + 1]));
    Totals &t = totals_[pending_[i].name];
    t.v[0] += ms;
    for (int k = 0; k < 4; k++) t.v[1 + k] += pending_[i].work[k];
    t.launches++;
  }
  used_ = 0;
  pending_.clear();
}

void KernelProbe::read(const char *name, double out[5], unsigned long long *launches) {
  std::lock_guard<std::mutex> lk(mu_);
  Totals t;
  auto it = totals_.find(name ? name : "");
  if (it != totals_.end()) t = it->second;
  for (int k = 0; k < 5; k++) out[k] = t.v[k];
  if (launches) *launches = t.launches;
}

std::string KernelProbe::names() {
  std::lock_guard<std::mutex> lk(mu_);
  std::string out;
  for (const auto &kv : totals_) {
    if (!out.empty()) out += ",";
    out += kv.first;
  }
  return out;
}

}  // namespace bz
