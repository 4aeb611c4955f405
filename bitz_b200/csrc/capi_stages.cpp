// C ABI of the reference's separate stages: CircuitProofSystem::witness,
// commit and prove (tooling/cli/src/end_to_end.rs:215-336).
//
// The witness and its commitment stay on the device between the calls, in
// the buffers of the lane that computed them, so a staged proof holds that
// lane from bitz_witness until bitz_prove consumes it (or a handle is freed).
// The lane is the process's default lane when no other staged proof or
// single-call proof holds it (it keeps the middle sumcheck rounds resident),
// else one from the lane pool.
#include <stdlib.h>
#include <string.h>

#include <atomic>
#include <memory>
#include <string>

#include "../../include/bitz_b200.h"
#include "hash.cuh"
#include "prover.hpp"
#include "status.hpp"

struct bitz_system {
  bz::ProofSystem *ps;
};

namespace bz {
int capi_fail(int code, const std::string &msg);
std::unique_ptr<Context> take_lane(int device);
void give_lane(int device, std::unique_ptr<Context> lane);

static std::atomic<bool> g_default_lane_held{false};

// A lane for one proof: the default lane if nobody holds it, else a pool lane.
LaneLease::LaneLease() {
  bool expect = false;
  if (g_default_lane_held.compare_exchange_strong(expect, true)) {
    default_ = true;
    lane_ = &Context::get();
    return;
  }
  BZ_CUDA(cudaGetDevice(&device_));
  pool_ = take_lane(device_);
  lane_ = pool_.get();
}

LaneLease::~LaneLease() {
  if (default_) g_default_lane_held.store(false);
  if (pool_) give_lane(device_, std::move(pool_));
}

// One staged proof: its system, its lane, and whether it is still running.
struct StagedProof {
  bitz_system *sys = nullptr;
  std::unique_ptr<LaneLease> lease;
  bool live = false;
  ~StagedProof() {
    if (live && sys) sys->ps->split_drop();
  }
};
}  // namespace bz

using namespace bz;

struct bitz_witness_handle {
  std::shared_ptr<StagedProof> sp;
};
struct bitz_committed_witness {
  std::shared_ptr<StagedProof> sp;
};

namespace {
int staged_error(int rc, ProofSystem *ps) { return capi_fail(rc, ps->error); }

// Ends a staged proof that a handle gives up: nothing can use its lane any more.
void end_staged(StagedProof &sp) {
  if (sp.live) {
    sp.sys->ps->split_drop();
    sp.live = false;
  }
  sp.lease.reset();
}
}  // namespace

extern "C" {

int bitz_witness(bitz_system *sys, const uint8_t *input_bits, size_t n_inputs,
                 bitz_witness_handle **out) {
  if (!sys || !out || (!input_bits && n_inputs)) return capi_fail(BZ_ERR_ARGUMENT, "null argument");
  *out = nullptr;
  try {
    auto sp = std::make_shared<StagedProof>();
    sp->sys = sys;
    sp->lease = std::make_unique<LaneLease>();
    int rc = sys->ps->split_witness(input_bits, n_inputs, sp->lease->lane());
    if (rc) return staged_error(rc, sys->ps);
    sp->live = true;
    *out = new bitz_witness_handle{sp};
    return BZ_OK;
  } catch (const CudaError &e) {
    sys->ps->split_drop();
    return capi_fail(BZ_ERR_CUDA, e.what());
  } catch (const std::exception &e) {
    sys->ps->split_drop();
    return capi_fail(BZ_ERR_INTERNAL, e.what());
  }
}

int bitz_commit(bitz_system *sys, const bitz_witness_handle *wit, bitz_committed_witness **out) {
  if (!sys || !wit || !out) return capi_fail(BZ_ERR_ARGUMENT, "null argument");
  *out = nullptr;
  StagedProof &sp = *wit->sp;
  if (sp.sys != sys) return capi_fail(BZ_ERR_ARGUMENT, "the witness belongs to another system");
  if (!sp.live) return capi_fail(BZ_ERR_ARGUMENT, "the witness was already used or dropped");
  try {
    int rc = sys->ps->split_commit();
    if (rc) return staged_error(rc, sys->ps);
    *out = new bitz_committed_witness{wit->sp};
    return BZ_OK;
  } catch (const CudaError &e) {
    end_staged(sp);
    return capi_fail(BZ_ERR_CUDA, e.what());
  } catch (const std::exception &e) {
    end_staged(sp);
    return capi_fail(BZ_ERR_INTERNAL, e.what());
  }
}

int bitz_prove(bitz_system *sys, bitz_witness_handle *wit, bitz_committed_witness *com,
               uint8_t **proof, size_t *proof_len) {
  // both handles are consumed on every return, as prove takes them by value
  std::unique_ptr<bitz_witness_handle> w(wit);
  std::unique_ptr<bitz_committed_witness> c(com);
  if (proof) *proof = nullptr;
  if (proof_len) *proof_len = 0;
  if (!sys || !wit || !com || !proof || !proof_len)
    return capi_fail(BZ_ERR_ARGUMENT, "null argument");
  if (w->sp != c->sp) return capi_fail(BZ_ERR_ARGUMENT, "the commitment is of another witness");
  StagedProof &sp = *w->sp;
  if (sp.sys != sys) return capi_fail(BZ_ERR_ARGUMENT, "the witness belongs to another system");
  if (!sp.live) return capi_fail(BZ_ERR_ARGUMENT, "the witness was already used or dropped");
  try {
    std::vector<uint8_t> p;
    sp.live = false;  // split_prove ends the staged proof whatever it returns
    int rc = sys->ps->split_prove(p);
    sp.lease.reset();
    if (rc) return staged_error(rc, sys->ps);
    *proof = (uint8_t *)malloc(p.size());
    if (!*proof) return capi_fail(BZ_ERR_INTERNAL, "out of host memory");
    memcpy(*proof, p.data(), p.size());
    *proof_len = p.size();
    return BZ_OK;
  } catch (const CudaError &e) {
    end_staged(sp);
    return capi_fail(BZ_ERR_CUDA, e.what());
  } catch (const std::exception &e) {
    end_staged(sp);
    return capi_fail(BZ_ERR_INTERNAL, e.what());
  }
}

int bitz_verify(bitz_system *sys, const uint8_t *proof, size_t proof_len) {
  if (!sys || (!proof && proof_len)) return capi_fail(BZ_ERR_ARGUMENT, "null argument");
  try {
    LaneLease lease;
    int rc = sys->ps->verify(proof, proof_len, lease.lane());
    if (rc) return capi_fail(rc, sys->ps->error);
    return BZ_OK;
  } catch (const CudaError &e) {
    return capi_fail(BZ_ERR_CUDA, e.what());
  } catch (const std::exception &e) {
    return capi_fail(BZ_ERR_INTERNAL, e.what());
  }
}

int bitz_wire_decode(const uint8_t *bytes, size_t len, uint64_t out[4]) {
  if (!out) return capi_fail(BZ_ERR_ARGUMENT, "null argument");
  WireView w;
  std::string err;
  int rc = wire_decode(bytes, len, w, err);
  if (rc) return capi_fail(rc, err);
  out[0] = 32;
  out[1] = w.narg_len;
  out[2] = 32 + w.narg_len;
  out[3] = w.hints_len;
  return BZ_OK;
}

int bitz_blake3(const char *derive_key_context, const uint8_t *in, size_t len, uint8_t out[32]) {
  if ((!in && len) || !out) return capi_fail(BZ_ERR_ARGUMENT, "null argument");
  Blake3 h = derive_key_context ? Blake3::derive_key(derive_key_context) : Blake3();
  h.update(in, len);
  h.finalize(out);
  return BZ_OK;
}

void bitz_witness_free(bitz_witness_handle *wit) {
  if (!wit) return;
  end_staged(*wit->sp);
  delete wit;
}

void bitz_committed_witness_free(bitz_committed_witness *com) {
  if (!com) return;
  end_staged(*com->sp);
  delete com;
}

}  // extern "C"
