// The end-to-end prover: CircuitProofSystem's setup, witness, commit and
// prove (tooling/cli/src/end_to_end.rs:161-336) on one device stream.
#pragma once
#include <cuda_runtime.h>

#include <memory>
#include <string>
#include <vector>

#include "circuit.hpp"
#include "context.hpp"
#include "spartan.hpp"
#include "transcript.hpp"

namespace bz {

// One Ligerito level (crates/pcs/src/profiles.rs:66-126).
struct PcsLevel {
  int k, log_inv_rate, log_msg_cols, queries, fold_grinding, grinding, ood_samples;
};

struct PcsConfig {
  int m = 0, log_n = 0, security = 0, nlevels = 0, final_log_n = 0;
  PcsLevel levels[8];
};

bool pcs_config(int m, int security_bits, PcsConfig &cfg);

// Device copies of one circuit's setup, shared by every statement of that
// circuit and size.
struct DeviceSetup {
  std::shared_ptr<CircuitSetup> host;
  DeviceBuffer<uint32_t> m_off, m_pos, csc_off, csc_row;
  DeviceBuffer<uint32_t> abc_off[3], abc_col[3];
  DeviceBuffer<int64_t> abc_coef[3];
  // column-major copy of A, B, C for the Spartan bind
  DeviceBuffer<uint32_t> sp_off, sp_row;
  DeviceBuffer<uint16_t> sp_idx;
  DeviceBuffer<int64_t> tab_vals;
  DeviceBuffer<uint8_t> tab_which;
  int ntab = 0;
  uint32_t col0_nnz = 0;
};

// The two streams of a proof's bitzPCS wire container.
struct WireView {
  const uint8_t *narg = nullptr, *hints = nullptr;
  size_t narg_len = 0, hints_len = 0;
};
// WireProof::from_bytes (crates/host/src/wire_proof.rs:109-140): strict;
// BZ_ERR_MALFORMED with the reference's error variant named in err.
int wire_decode(const uint8_t *bytes, size_t len, WireView &out, std::string &err);

struct StageTimes {
  double witness_ms = 0, commit_ms = 0, prove_ms = 0;
  double device_ms = 0;  // CUDA-event span on the prover's stream, first to last launch
};

class ProofSystem {
 public:
  // CircuitProofSystem::new (end_to_end.rs:161-197): one statement (its input
  // and expected output bits, one byte each) at a PCS security level.
  // Staging runs on `lane` (the default lane when null).
  ProofSystem(int kind, const uint8_t *inputs, size_t n_inputs, const uint8_t *outputs,
              int security_bits, Context *lane = nullptr);
  // Device bytes a proof of this statement keeps in its lane's scratch at
  // most (the padded tables of the largest stages), for admission control.
  static uint64_t footprint_bytes(int kind, size_t n_inputs);
  ~ProofSystem();
  ProofSystem(const ProofSystem &) = delete;
  ProofSystem &operator=(const ProofSystem &) = delete;

  // witness + commit + prove (benchmark.rs:28-79), returning the proof bytes:
  // root || Spartan section || bitzPCS wire container. With restage set the
  // statement (input bits, chaining values, message words) is copied from
  // host memory first; otherwise the copy made at construction is reused.
  // The proof runs on `lane` (the process default lane when null); a system
  // proves on one lane at a time, distinct systems on distinct lanes run
  // concurrently.
  int prove(std::vector<uint8_t> &proof, StageTimes *times, bool restage = true,
            Context *lane = nullptr);

  // The reference's stages as separate calls (CircuitProofSystem::witness,
  // commit and prove, end_to_end.rs:215-336), on one lane from the witness to
  // the proof: the witness stays in the lane's device buffers and the
  // commitment (codeword, Merkle tree, transcript) with it. A system holds at
  // most one such proof at a time, and prove() refuses while it does.
  // split_witness takes the witness's input bits (one byte each; the same
  // count as the statement's, else BZ_ERR_ARGUMENT) and returns
  // BZ_ERR_UNSATISFIED when they do not satisfy the statement.
  int split_witness(const uint8_t *inputs, size_t n_inputs, Context *lane);
  int split_commit();
  // Runs the prove stage and ends the split proof (also on failure).
  int split_prove(std::vector<uint8_t> &proof);
  // Ends a split proof at any stage without proving.
  void split_drop();
  int split_stage() const { return split_; }  // 0 none, 1 witnessed, 2 committed

  const CircuitSetup &setup() const { return *dev_->host; }
  int security() const { return security_; }
  int kind() const { return kind_; }
  size_t n_inputs() const { return inputs_.size(); }
  std::string error;

  // CircuitProofSystem::verify (end_to_end.rs:339-377) on proof bytes (root
  // || Spartan section || wire container), on `lane` (the default lane when
  // null): BZ_OK when every check passes, BZ_ERR_MALFORMED when the bytes do
  // not parse, BZ_ERR_VERIFY naming the failed check otherwise.
  int verify(const uint8_t *proof, size_t proof_len, Context *lane = nullptr);

  // Witness-stage products for inspection (valid after prove()).
  void download_witness(std::vector<uint32_t> &f, std::vector<uint32_t> &h,
                        std::vector<int64_t> &prod);

 private:
  void stage_statement(cudaStream_t s);
  int witness(cudaStream_t s);
  int commit(cudaStream_t s);
  int prove_after_commit(cudaStream_t s, std::vector<uint8_t> &proof);
  std::vector<uint8_t> ligerito(cudaStream_t s, f128 target);

  void bind_lane(Context *lane);
  Context *lane_ = nullptr;  // the lane of the proof in progress
  int split_ = 0;            // stage of a split proof (split_stage)
  int kind_, security_;
  std::vector<uint8_t> inputs_, outputs_;
  std::shared_ptr<DeviceSetup> dev_;
  PcsConfig pcs_;
  uint8_t matrix_digest_[32];
  std::vector<uint8_t> public_bytes_, pcs_enc_;
  std::vector<uint32_t> bit_rows_;  // bit constraints whose expected value is one
  f128 generator_;

  // the statement in host memory: chaining values, message words, hint
  // offsets, the packed input bits and every bit constraint's expected value
  std::vector<uint32_t> states_h_, msgs_h_, fin_h_;
  std::vector<uint8_t> bitc_h_;
  uint64_t serial_;  // identifies the statement staged in a lane's buffers
  cudaEvent_t ev_start_ = nullptr, ev_stop_ = nullptr;

  // the proof's device state, in the buffers of the lane running it (bound
  // at the start of prove())
  DeviceBuffer<uint32_t> *states_ = nullptr, *msgs_ = nullptr, *fin_ = nullptr;
  DeviceBuffer<uint64_t> *offsets_ = nullptr;
  DeviceBuffer<uint32_t> *f_ = nullptr, *h_ = nullptr;
  DeviceBuffer<int64_t> *prod_ = nullptr;
  DeviceBuffer<uint8_t> *bit_c_ = nullptr;
  DeviceBuffer<uint32_t> *d_bit_rows_ = nullptr;
  DeviceBuffer<f128> *codeword0_ = nullptr;
  DeviceBuffer<uint32_t> *nodes0_ = nullptr;
  std::unique_ptr<Transcript> ts_;
  uint8_t root_[32];
  std::vector<f128> ood_point_;
  f128 ood_value_;
};

}  // namespace bz
