// The post-GKR sumcheck without any allocation: the ping-pong tables and the
// round accumulators live in file-scope device arrays of a fixed maximum
// size, for callers that cannot allocate device memory.
//
// Who needs this: processes whose device memory is owned by another
// allocator or by a fixed budget reserved up front (cudaMalloc would take
// memory the budget does not have), and embedders that forbid allocation on
// their request path (an allocation can block behind work on the whole
// device). They pass device pointers to the inputs and host pointers for the
// outputs, and nothing else is needed. The call is not for stream capture:
// every round copies its message to the host and synchronises the stream so
// that the host transcript can draw the next challenge, and neither is
// allowed while a stream is being captured.
//
// The arrays take the same device memory in every process that loads this
// library, on every GPU it touches, until the process exits. Every call
// shares them: two calls whose work overlaps on the GPU (different streams,
// or different host threads) race and corrupt each other; serialise them.
// The arrays' device addresses are looked up on the first call on a device
// and again whenever the device's context has changed since (after
// cudaDeviceReset the module is loaded anew, at new addresses).
#include <mutex>

#include "device.cuh"
#include "post_gkr.hpp"

namespace bz {

// Largest claim served: 2^20 bits (log_rows + log_cols <= 20), so four tables
// of 2^19 F128 each (32 MiB) and round accumulators for up to 64 rounds.
constexpr int kNoAllocMaxLogBits = 20;
constexpr size_t kNoAllocTable = (size_t)1 << (kNoAllocMaxLogBits - 1);

static __device__ __align__(256) f128 g_noalloc_tables[4 * kNoAllocTable];
static __device__ __align__(256) unsigned long long g_noalloc_acc[8 * 64];

constexpr int kMaxDevices = 64;
static f128 *s_tables[kMaxDevices];
static unsigned long long *s_acc[kMaxDevices];
static void *s_context[kMaxDevices];  // the context the addresses belong to
static std::mutex s_setup_mu;

// The calling thread's current context (the device's primary context once
// the runtime has set it up), read through the driver entry point so the
// library needs no link against the driver library. nullptr if unavailable.
static void *current_context() {
  typedef int (*CtxGetCurrent)(void **);
  static const CtxGetCurrent fn = [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return (CtxGetCurrent) nullptr;
    return (CtxGetCurrent)p;
  }();
  void *ctx = nullptr;
  if (fn && fn(&ctx) != 0) ctx = nullptr;
  return ctx;
}

// Host code cannot use the arrays' names as device addresses: look them up
// with the device current, once per device and context.
static int noalloc_setup(int device, std::string &err) {
  std::lock_guard<std::mutex> lk(s_setup_mu);
  if (device < 0 || device >= kMaxDevices) {
    err = "device index out of range";
    return BZ_ERR_ARGUMENT;
  }
  void *ctx = current_context();
  if (s_tables[device] && ctx && ctx == s_context[device]) return BZ_OK;
  void *t = nullptr, *a = nullptr;
  cudaError_t e1 = cudaGetSymbolAddress(&t, g_noalloc_tables);
  if (e1 != cudaSuccess) {
    err = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e1);
    return BZ_ERR_CUDA;
  }
  cudaError_t e2 = cudaGetSymbolAddress(&a, g_noalloc_acc);
  if (e2 != cudaSuccess) {
    err = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e2);
    return BZ_ERR_CUDA;
  }
  s_acc[device] = (unsigned long long *)a;
  s_tables[device] = (f128 *)t;
  // the lookup made the context current if it was not yet
  s_context[device] = ctx ? ctx : current_context();
  return BZ_OK;
}

int post_gkr_prove_noalloc(const PostGkrArgs &a, Transcript &ts, cudaStream_t s, f128 *point_out,
                           f128 *value_out, std::string &err) {
  if (a.log_rows + a.log_cols > kNoAllocMaxLogBits) {
    err = "claim larger than the fixed scratch: log_rows + log_cols must be at most 20";
    return BZ_ERR_SCRATCH;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    err = cudaGetErrorString(e);
    return BZ_ERR_CUDA;
  }
  int rc = noalloc_setup(dev, err);
  if (rc) return rc;
  uint64_t host[8];  // pageable: the round messages copy back synchronously
  PostGkrScratch sc;
  sc.capacity = kNoAllocTable;
  sc.w0 = s_tables[dev];
  sc.v0 = s_tables[dev] + kNoAllocTable;
  sc.w1 = s_tables[dev] + 2 * kNoAllocTable;
  sc.v1 = s_tables[dev] + 3 * kNoAllocTable;
  sc.acc = s_acc[dev];  // zeroed by post_gkr_prove before its first round
  sc.host = host;
  return post_gkr_prove(a, ts, sc, s, point_out, value_out);
}

}  // namespace bz
