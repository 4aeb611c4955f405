// Batched and served proving across prover lanes, and the measurement aids.
//
// A lane (Context) is one CUDA stream with its own round mailbox and scratch;
// each lane is driven by one host thread, which runs the proof's transcript.
// Proofs on different lanes overlap on the device: while one proof's host
// thread absorbs a round message, the kernels of the others run. Lanes are
// pooled per process, so their scratch stays resident in HBM across calls.
#include <cuda_runtime.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/bitz_b200.h"
#include "fiber.hpp"
#include "prover.hpp"
#include "status.hpp"

struct bitz_system {
  bz::ProofSystem *ps;
};

namespace bz {
int capi_fail(int code, const std::string &msg);
int check_statement(int circuit_kind, const uint8_t *input_bits, size_t n_inputs,
                    const uint8_t *output_bits, uint32_t security_bits);
double diag_round_trip(int mode, int rounds);
double diag_gf_peak(int kind, int blocks_per_sm);

namespace {

constexpr int kMaxLanes = 64;

// Process-wide pool of idle lanes (per device), grown on demand.
class LanePool {
 public:
  static LanePool &get() {
    static LanePool *p = new LanePool();
    return *p;
  }
  std::vector<std::unique_ptr<Context>> take(int device, int n) {
    std::vector<std::unique_ptr<Context>> out;
    {
      std::lock_guard<std::mutex> lk(mu_);
      auto &idle = idle_[device];
      while ((int)out.size() < n && !idle.empty()) {
        out.push_back(std::move(idle.back()));
        idle.pop_back();
      }
    }
    while ((int)out.size() < n) out.push_back(std::make_unique<Context>());
    return out;
  }
  void give(int device, std::vector<std::unique_ptr<Context>> &lanes) {
    std::lock_guard<std::mutex> lk(mu_);
    for (auto &l : lanes) idle_[device].push_back(std::move(l));
    lanes.clear();
  }

 private:
  std::mutex mu_;
  std::unordered_map<int, std::vector<std::unique_ptr<Context>>> idle_;
};

// Host threads for `lanes` lanes: one per lane up to the host's hardware
// threads (BITZ_LANE_THREADS overrides the cap); beyond that, lanes share
// threads as fibers.
int lane_threads(int lanes) {
  static const int cap = [] {
    const char *e = getenv("BITZ_LANE_THREADS");
    if (e && atoi(e) > 0) return atoi(e);
    const unsigned hw = std::thread::hardware_concurrency();
    return (int)std::max(1u, hw);
  }();
  return std::max(1, std::min(lanes, cap));
}

double ms_between(std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

// Runs one proof on a lane; the status, message and bytes come back.
int prove_on(ProofSystem &ps, Context &lane, std::vector<uint8_t> &proof, std::string &err) {
  try {
    int rc = ps.prove(proof, nullptr, true, &lane);
    if (rc) err = ps.error;
    return rc;
  } catch (const CudaError &e) {
    err = e.what();
    return BZ_ERR_CUDA;
  } catch (const std::exception &e) {
    err = e.what();
    return BZ_ERR_INTERNAL;
  }
}

uint8_t *copy_out(const std::vector<uint8_t> &p) {
  uint8_t *b = (uint8_t *)malloc(std::max<size_t>(p.size(), 1));
  if (b) memcpy(b, p.data(), p.size());
  return b;
}

}  // namespace

// One lane from the pool for a caller that holds it across calls (the staged
// witness/commit/prove calls), and its return.
std::unique_ptr<Context> take_lane(int device) {
  auto v = LanePool::get().take(device, 1);
  return std::move(v[0]);
}

void give_lane(int device, std::unique_ptr<Context> lane) {
  std::vector<std::unique_ptr<Context>> v;
  v.push_back(std::move(lane));
  LanePool::get().give(device, v);
}

}  // namespace bz

using namespace bz;

// ------------------------------------------------------------------ server

struct ServeRequest {
  uint64_t ticket = 0;
  int kind = 0;
  std::vector<uint8_t> inputs, outputs;
  uint64_t footprint = 0;
  std::chrono::steady_clock::time_point submitted;
  std::unique_ptr<ProofSystem> ps;  // the prepared statement
  bool done = false;
  int status = BZ_OK;
  std::string error;
  std::vector<uint8_t> proof;
  double latency_ms = 0;
};

// Two stages: preparer threads build each request's statement (the circuit
// shape from the cache, the statement's matrix digest, the staged inputs: host
// work), prover lanes prove prepared requests. A lane never idles on host-only
// set-up while prepared work waits.
struct bitz_server {
  int device = 0;
  uint32_t security = 100;
  uint64_t budget = 0;
  std::vector<std::unique_ptr<Context>> lanes, prep_lanes;
  std::vector<std::thread> workers;
  std::mutex mu;
  std::condition_variable prep_cv, work_cv, done_cv;
  std::deque<std::shared_ptr<ServeRequest>> queue;           // submitted, not prepared
  std::map<uint64_t, std::shared_ptr<ServeRequest>> ready;   // prepared, by ticket
  std::unordered_map<uint64_t, std::shared_ptr<ServeRequest>> tickets;
  uint64_t next_ticket = 1, submitted = 0, finished = 0, in_flight = 0, in_flight_bytes = 0,
           peak_in_flight = 0;
  bool stopping = false;

  // Admission: oldest prepared request first, a free lane, and its footprint
  // fits the budget beside the requests in flight (always when none is).
  bool admissible() const {
    if (ready.empty()) return false;
    uint64_t need = ready.begin()->second->footprint;
    return in_flight == 0 || in_flight_bytes + need <= budget;
  }

  void finish(const std::shared_ptr<ServeRequest> &rq, int rc, std::string err,
              std::vector<uint8_t> proof) {
    auto t = std::chrono::steady_clock::now();
    {
      std::lock_guard<std::mutex> lk(mu);
      rq->status = rc;
      rq->error = std::move(err);
      rq->proof = std::move(proof);
      rq->latency_ms = ms_between(rq->submitted, t);
      rq->ps.reset();
      rq->done = true;
      finished++;
    }
    done_cv.notify_all();
  }

  void prepare(Context *lane) {
    cudaSetDevice(device);
    for (;;) {
      std::shared_ptr<ServeRequest> rq;
      {
        std::unique_lock<std::mutex> lk(mu);
        prep_cv.wait(lk, [&] { return stopping || !queue.empty(); });
        if (stopping) return;
        rq = queue.front();
        queue.pop_front();
      }
      try {
        rq->ps.reset(new ProofSystem(rq->kind, rq->inputs.data(), rq->inputs.size(),
                                     rq->outputs.data(), (int)security, lane));
      } catch (const CudaError &e) {
        finish(rq, BZ_ERR_CUDA, e.what(), {});
        continue;
      } catch (const std::exception &e) {
        finish(rq, BZ_ERR_CONFIG, e.what(), {});
        continue;
      }
      {
        std::lock_guard<std::mutex> lk(mu);
        ready[rq->ticket] = rq;
      }
      work_cv.notify_one();
    }
  }

  void run(Context *lane) {
    cudaSetDevice(device);
    for (;;) {
      std::shared_ptr<ServeRequest> rq;
      {
        std::unique_lock<std::mutex> lk(mu);
        work_cv.wait(lk, [&] { return stopping || admissible(); });
        if (stopping) return;
        rq = ready.begin()->second;
        ready.erase(ready.begin());
        in_flight++;
        in_flight_bytes += rq->footprint;
        peak_in_flight = std::max(peak_in_flight, in_flight);
      }
      std::vector<uint8_t> proof;
      std::string err;
      // the statement was staged on the device when it was prepared
      int rc;
      try {
        rc = rq->ps->prove(proof, nullptr, false, lane);
        if (rc) err = rq->ps->error;
      } catch (const CudaError &e) {
        rc = BZ_ERR_CUDA;
        err = e.what();
      } catch (const std::exception &e) {
        rc = BZ_ERR_INTERNAL;
        err = e.what();
      }
      {
        std::lock_guard<std::mutex> lk(mu);
        in_flight--;
        in_flight_bytes -= rq->footprint;
      }
      finish(rq, rc, std::move(err), std::move(proof));
      work_cv.notify_all();
    }
  }
};

extern "C" {

int bitz_batch_prove(bitz_system *const *systems, size_t n, int lanes, uint8_t **proofs,
                     size_t *proof_lens, double *latency_ms) {
  if ((!systems || !proofs || !proof_lens) && n) return capi_fail(BZ_ERR_ARGUMENT, "null argument");
  if (lanes < 1 || lanes > kMaxLanes) return capi_fail(BZ_ERR_ARGUMENT, "lanes must be 1..64");
  for (size_t i = 0; i < n; i++) {
    if (!systems[i]) return capi_fail(BZ_ERR_ARGUMENT, "null system");
    proofs[i] = nullptr;
    proof_lens[i] = 0;
  }
  if (n == 0) return BZ_OK;
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) return capi_fail(BZ_ERR_NO_DEVICE, "no CUDA device");
  int nl = (int)std::min<size_t>((size_t)lanes, n);
  std::vector<std::unique_ptr<Context>> pool;
  try {
    pool = LanePool::get().take(device, nl);
  } catch (const std::exception &e) {
    return capi_fail(BZ_ERR_CUDA, e.what());
  }
  // Largest statements first. A lane's first proof is then the largest it
  // proves in the batch, so its scratch grows at most once per batch (a
  // growth allocation waits until no lane has a kernel waiting for its host
  // thread and holds every lane back meanwhile), and the batch ends on its
  // shortest proofs. The proofs come back in the callers' order.
  std::vector<size_t> order(n);
  std::iota(order.begin(), order.end(), (size_t)0);
  {
    std::vector<std::pair<uint64_t, size_t>> key(n);
    for (size_t i = 0; i < n; i++) {
      const ProofSystem &ps = *systems[i]->ps;
      key[i] = {ProofSystem::footprint_bytes(ps.kind(), ps.n_inputs()), ps.n_inputs()};
    }
    std::stable_sort(order.begin(), order.end(),
                     [&](size_t a, size_t b) { return key[a] > key[b]; });
  }
  std::atomic<size_t> next{0};
  std::vector<int> status(n, BZ_OK);
  std::vector<std::string> errors(n);
  auto worker = [&](Context *lane) {
    for (size_t k; (k = next.fetch_add(1)) < n;) {
      const size_t i = order[k];
      std::vector<uint8_t> proof;
      auto ts = std::chrono::steady_clock::now();
      status[i] = prove_on(*systems[i]->ps, *lane, proof, errors[i]);
      if (latency_ms) latency_ms[i] = ms_between(ts, std::chrono::steady_clock::now());
      if (status[i] == BZ_OK) {
        proofs[i] = copy_out(proof);
        proof_lens[i] = proof.size();
        if (!proofs[i]) {
          status[i] = BZ_ERR_INTERNAL;
          errors[i] = "out of host memory";
        }
      }
    }
  };
  // lane k runs on host thread k mod nt; a thread with several lanes runs
  // each as a fiber that yields wherever it waits for the device
  const int nt = lane_threads(nl);
  auto thread_main = [&](int t) {
    cudaSetDevice(device);
    std::vector<Context *> mine;
    for (int k = t; k < nl; k += nt) mine.push_back(pool[k].get());
    if (mine.size() == 1) {
      worker(mine[0]);
      return;
    }
    FiberLoop loop;
    for (Context *c : mine) loop.add([&worker, c] { worker(c); });
    loop.run();
  };
  std::vector<std::thread> threads;
  for (int t = 1; t < nt; t++) threads.emplace_back(thread_main, t);
  thread_main(0);
  for (auto &t : threads) t.join();
  LanePool::get().give(device, pool);
  for (size_t i = 0; i < n; i++)
    if (status[i]) return capi_fail(status[i], "proof " + std::to_string(i) + ": " + errors[i]);
  return BZ_OK;
}

int bitz_server_start(int lanes, uint64_t hbm_budget_bytes, uint32_t security_bits,
                      bitz_server **out) {
  if (!out) return capi_fail(BZ_ERR_ARGUMENT, "null argument");
  *out = nullptr;
  if (lanes < 1 || lanes > kMaxLanes) return capi_fail(BZ_ERR_ARGUMENT, "lanes must be 1..64");
  if (security_bits != 100 && security_bits != 128)
    return capi_fail(BZ_ERR_ARGUMENT, "security_bits must be 100 or 128");
  auto *srv = new bitz_server();
  if (cudaGetDevice(&srv->device) != cudaSuccess) {
    delete srv;
    return capi_fail(BZ_ERR_NO_DEVICE, "no CUDA device");
  }
  srv->security = security_bits;
  srv->budget = hbm_budget_bytes;
  try {
    srv->lanes = LanePool::get().take(srv->device, lanes);
    unsigned hw = std::thread::hardware_concurrency();
    srv->prep_lanes = LanePool::get().take(srv->device, (int)std::max(2u, hw / 2));
  } catch (const std::exception &e) {
    delete srv;
    return capi_fail(BZ_ERR_CUDA, e.what());
  }
  for (auto &l : srv->lanes) srv->workers.emplace_back(&bitz_server::run, srv, l.get());
  for (auto &l : srv->prep_lanes) srv->workers.emplace_back(&bitz_server::prepare, srv, l.get());
  *out = srv;
  return BZ_OK;
}

int bitz_server_submit(bitz_server *srv, int circuit_kind, const uint8_t *input_bits,
                       size_t n_inputs, const uint8_t *output_bits, uint64_t *ticket) {
  if (!srv || !ticket) return capi_fail(BZ_ERR_ARGUMENT, "null argument");
  int rc = check_statement(circuit_kind, input_bits, n_inputs, output_bits, srv->security);
  if (rc) return rc;
  auto rq = std::make_shared<ServeRequest>();
  rq->kind = circuit_kind;
  rq->inputs.assign(input_bits, input_bits + n_inputs);
  rq->outputs.assign(output_bits, output_bits + 256);
  rq->footprint = ProofSystem::footprint_bytes(circuit_kind, n_inputs);
  rq->submitted = std::chrono::steady_clock::now();
  {
    std::lock_guard<std::mutex> lk(srv->mu);
    if (srv->stopping) return capi_fail(BZ_ERR_ARGUMENT, "server is stopping");
    rq->ticket = srv->next_ticket++;
    srv->tickets[rq->ticket] = rq;
    srv->queue.push_back(rq);
    srv->submitted++;
    *ticket = rq->ticket;
  }
  srv->prep_cv.notify_one();
  return BZ_OK;
}

int bitz_server_poll(bitz_server *srv, uint64_t ticket, int wait_ms, uint8_t **proof,
                     size_t *proof_len, double *latency_ms) {
  if (!srv || !proof || !proof_len) return capi_fail(BZ_ERR_ARGUMENT, "null argument");
  *proof = nullptr;
  *proof_len = 0;
  std::unique_lock<std::mutex> lk(srv->mu);
  auto it = srv->tickets.find(ticket);
  if (it == srv->tickets.end()) return capi_fail(BZ_ERR_ARGUMENT, "unknown ticket");
  std::shared_ptr<ServeRequest> rq = it->second;
  if (!rq->done && wait_ms > 0)
    srv->done_cv.wait_for(lk, std::chrono::milliseconds(wait_ms), [&] { return rq->done; });
  if (!rq->done) return BZ_PENDING;
  srv->tickets.erase(it);
  if (latency_ms) *latency_ms = rq->latency_ms;
  if (rq->status) return capi_fail(rq->status, rq->error);
  *proof = copy_out(rq->proof);
  if (!*proof) return capi_fail(BZ_ERR_INTERNAL, "out of host memory");
  *proof_len = rq->proof.size();
  return BZ_OK;
}

int bitz_server_stats(bitz_server *srv, uint64_t out[6]) {
  if (!srv || !out) return capi_fail(BZ_ERR_ARGUMENT, "null argument");
  std::lock_guard<std::mutex> lk(srv->mu);
  out[0] = srv->submitted;
  out[1] = srv->finished;
  out[2] = srv->in_flight;
  out[3] = srv->queue.size() + srv->ready.size();
  out[4] = srv->in_flight_bytes;
  out[5] = srv->peak_in_flight;
  return BZ_OK;
}

int bitz_server_stop(bitz_server *srv) {
  if (!srv) return capi_fail(BZ_ERR_ARGUMENT, "null argument");
  {
    std::lock_guard<std::mutex> lk(srv->mu);
    srv->stopping = true;
    srv->queue.clear();
    srv->ready.clear();
  }
  srv->work_cv.notify_all();
  srv->prep_cv.notify_all();
  for (auto &t : srv->workers) t.join();
  LanePool::get().give(srv->device, srv->lanes);
  LanePool::get().give(srv->device, srv->prep_lanes);
  delete srv;
  return BZ_OK;
}

int bitz_probe_kernel(const char *name) {
  try {
    KernelProbe::get().enable(name);
    return BZ_OK;
  } catch (const std::exception &e) {
    return capi_fail(BZ_ERR_CUDA, e.what());
  }
}

int bitz_probe_read(const char *kernel, double out[5], unsigned long long *launches) {
  if (!kernel || !out) return capi_fail(BZ_ERR_ARGUMENT, "null argument");
  try {
    KernelProbe::get().collect();
    KernelProbe::get().read(kernel, out, launches);
    return BZ_OK;
  } catch (const std::exception &e) {
    return capi_fail(BZ_ERR_CUDA, e.what());
  }
}

size_t bitz_probe_kernels(char *out, size_t cap) {
  try {
    KernelProbe::get().collect();
    const std::string n = KernelProbe::get().names();
    if (out && cap) {
      const size_t k = std::min(cap - 1, n.size());
      memcpy(out, n.data(), k);
      out[k] = 0;
    }
    return n.size();
  } catch (const std::exception &e) {
    capi_fail(BZ_ERR_CUDA, e.what());
    return 0;
  }
}

int bitz_diag_round_trip(int mode, int rounds, double *us_per_round) {
  if (!us_per_round || rounds < 1 || (mode != 0 && mode != 1))
    return capi_fail(BZ_ERR_ARGUMENT, "bad argument");
  try {
    *us_per_round = diag_round_trip(mode, rounds);
    return BZ_OK;
  } catch (const std::exception &e) {
    return capi_fail(BZ_ERR_CUDA, e.what());
  }
}

int bitz_diag_fibers(int threads, int fibers, int yields, unsigned long long *checksum) {
  if (!checksum || threads < 1 || threads > 64 || fibers < 1 || fibers > 256 || yields < 2)
    return capi_fail(BZ_ERR_ARGUMENT, "bad argument");
  try {
    bool ok = false;
    *checksum = fiber_selftest(threads, fibers, yields, &ok);
    return ok ? BZ_OK : capi_fail(BZ_ERR_INTERNAL, "fiber self-test failed");
  } catch (const std::exception &e) {
    return capi_fail(BZ_ERR_INTERNAL, e.what());
  }
}

int bitz_diag_gf_peak(int kind, double *products_per_s) {
  if (!products_per_s || kind < 0 || kind > 2) return capi_fail(BZ_ERR_ARGUMENT, "bad argument");
  try {
    *products_per_s = diag_gf_peak(kind, 4);
    return BZ_OK;
  } catch (const std::exception &e) {
    return capi_fail(BZ_ERR_CUDA, e.what());
  }
}

int bitz_l2_flush(void) {
  static std::mutex mu;
  static void *buf = nullptr;
  const size_t bytes = (size_t)256 << 20;
  std::lock_guard<std::mutex> lk(mu);
  try {
    cudaStream_t s = Context::get().stream();
    if (!buf) {
      AllocScope gate;
      BZ_CUDA(cudaMalloc(&buf, bytes));
    }
    static unsigned char v = 0;
    BZ_CUDA(cudaMemsetAsync(buf, ++v, bytes, s));
    BZ_CUDA(cudaStreamSynchronize(s));
    return BZ_OK;
  } catch (const std::exception &e) {
    return capi_fail(BZ_ERR_CUDA, e.what());
  }
}

}  // extern "C"
