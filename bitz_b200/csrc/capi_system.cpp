// C ABI of the end-to-end prover (CircuitProofSystem, end_to_end.rs:150-336).
#include <cuda_runtime.h>
#include <stdlib.h>
#include <string.h>

#include <string>

#include "../../include/bitz_b200.h"
#include "prover.hpp"
#include "status.hpp"

using namespace bz;

struct bitz_system {
  ProofSystem *ps;
};

namespace bz {
int capi_fail(int code, const std::string &msg);

// integer_matrix_digest with the statement's bit constants (circuit.cpp)
void matrix_digest(const CircuitSetup &S, const std::vector<int64_t> &expected_c, uint8_t out[32]);

// Input checks of CircuitProofSystem::new (circuits.rs:58-210 dimensions).
int check_statement(int circuit_kind, const uint8_t *input_bits, size_t n_inputs,
                    const uint8_t *output_bits, uint32_t security_bits) {
  if (circuit_kind < 0 || circuit_kind > 3) return capi_fail(BZ_ERR_ARGUMENT, "unknown circuit");
  if (security_bits != 100 && security_bits != 128)
    return capi_fail(BZ_ERR_ARGUMENT, "security_bits must be 100 or 128");
  if ((!input_bits && n_inputs) || !output_bits) return capi_fail(BZ_ERR_ARGUMENT, "null argument");
  bool ok = false;
  switch (circuit_kind) {
    case kCompression: ok = n_inputs == 768; break;
    case kChain: ok = n_inputs > 0 && n_inputs % 512 == 0; break;
    case kBlockAligned: ok = n_inputs % 512 == 0; break;
    case k2kb: ok = n_inputs == 2048 * 8; break;
  }
  if (!ok) return capi_fail(BZ_ERR_ARGUMENT, "invalid circuit input/output dimensions");
  for (size_t i = 0; i < n_inputs; i++)
    if (input_bits[i] > 1) return capi_fail(BZ_ERR_ARGUMENT, "input bits must be 0 or 1");
  for (int i = 0; i < 256; i++)
    if (output_bits[i] > 1) return capi_fail(BZ_ERR_ARGUMENT, "output bits must be 0 or 1");
  return BZ_OK;
}
}  // namespace bz

extern "C" {

int bitz_system_new(int circuit_kind, const uint8_t *input_bits, size_t n_inputs,
                    const uint8_t *output_bits, uint32_t security_bits, bitz_system **out) {
  if (!input_bits || !output_bits || !out) return capi_fail(BZ_ERR_ARGUMENT, "null argument");
  *out = nullptr;
  int rc = check_statement(circuit_kind, input_bits, n_inputs, output_bits, security_bits);
  if (rc) return rc;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0)
    return capi_fail(BZ_ERR_NO_DEVICE, "no CUDA device");
  try {
    *out = new bitz_system{
        new ProofSystem(circuit_kind, input_bits, n_inputs, output_bits, (int)security_bits)};
    return BZ_OK;
  } catch (const CudaError &e) {
    return capi_fail(BZ_ERR_CUDA, e.what());
  } catch (const std::exception &e) {
    return capi_fail(BZ_ERR_CONFIG, e.what());
  }
}

void bitz_system_free(bitz_system *sys) {
  if (!sys) return;
  delete sys->ps;
  delete sys;
}

int bitz_system_stats(const bitz_system *sys, uint64_t out[8]) {
  if (!sys || !out) return capi_fail(BZ_ERR_ARGUMENT, "null argument");
  const CircuitSetup &S = sys->ps->setup();
  out[0] = S.rows;
  out[1] = S.h_len;
  out[2] = S.f_bits;
  out[3] = (uint64_t)1 << S.committed_m;
  out[4] = 121;
  out[5] = (uint64_t)sys->ps->security();
  out[6] = (uint64_t)S.claim_log_cols;
  out[7] = S.n_blocks;
  return BZ_OK;
}

int bitz_system_prove(bitz_system *sys, uint8_t **proof, size_t *proof_len, double times_ms[4]) {
  return bitz_system_prove_ex(sys, 1, proof, proof_len, times_ms);
}

int bitz_system_prove_ex(bitz_system *sys, int restage, uint8_t **proof, size_t *proof_len,
                         double times_ms[4]) {
  if (!sys || !proof || !proof_len) return capi_fail(BZ_ERR_ARGUMENT, "null argument");
  *proof = nullptr;
  *proof_len = 0;
  try {
    std::vector<uint8_t> p;
    StageTimes t;
    LaneLease lease;  // the default lane unless a staged proof holds it
    int rc = sys->ps->prove(p, &t, restage != 0, lease.lane());
    if (rc) return capi_fail(rc, sys->ps->error);
    *proof = (uint8_t *)malloc(p.size());
    if (!*proof) return capi_fail(BZ_ERR_INTERNAL, "out of host memory");
    memcpy(*proof, p.data(), p.size());
    *proof_len = p.size();
    if (times_ms) {
      times_ms[0] = t.witness_ms;
      times_ms[1] = t.commit_ms;
      times_ms[2] = t.prove_ms;
      times_ms[3] = t.device_ms;
    }
    return BZ_OK;
  } catch (const CudaError &e) {
    return capi_fail(BZ_ERR_CUDA, e.what());
  } catch (const std::exception &e) {
    return capi_fail(BZ_ERR_INTERNAL, e.what());
  }
}

void bitz_free(void *p) { free(p); }

unsigned long long bitz_launch_count(void) { return launch_counter(); }

int bitz_resident_rounds(void) { return resident_rounds_enabled() ? 1 : 0; }

int bitz_round_wait_stats(unsigned long long out[2]) {
  if (!out) return capi_fail(BZ_ERR_ARGUMENT, "null argument");
  try {
    RoundChannel *ch = Context::get().channel();
    out[0] = ch->wait_ns;
    out[1] = ch->waits;
    return BZ_OK;
  } catch (const std::exception &e) {
    return capi_fail(BZ_ERR_CUDA, e.what());
  }
}

int bitz_gate_stats(unsigned long long out[4]) {
  if (!out) return capi_fail(BZ_ERR_ARGUMENT, "null argument");
  DeviceGate::get().stats(out);
  return BZ_OK;
}

int bitz_system_witness(bitz_system *sys, uint32_t *f_words, size_t f_cap, uint32_t *h_words,
                        size_t h_cap, int64_t *products, size_t prod_cap) {
  if (!sys) return capi_fail(BZ_ERR_ARGUMENT, "null argument");
  try {
    std::vector<uint32_t> f, h;
    std::vector<int64_t> pr;
    sys->ps->download_witness(f, h, pr);
    if (f_cap < f.size() || h_cap < h.size() || prod_cap < pr.size())
      return capi_fail(BZ_ERR_ARGUMENT, "output buffers too small");
    memcpy(f_words, f.data(), f.size() * 4);
    memcpy(h_words, h.data(), h.size() * 4);
    memcpy(products, pr.data(), pr.size() * 8);
    return BZ_OK;
  } catch (const std::exception &e) {
    return capi_fail(BZ_ERR_CUDA, e.what());
  }
}

int bitz_circuit_layout(int circuit_kind, size_t n_inputs, uint64_t sizes[8],
                        uint8_t map_digest[32], uint32_t *m_off, uint32_t *m_pos,
                        uint32_t *c_off, uint32_t *c_col, int64_t *c_coef) {
  if (!sizes || !map_digest) return capi_fail(BZ_ERR_ARGUMENT, "null argument");
  if (circuit_kind < 0 || circuit_kind > 3) return capi_fail(BZ_ERR_ARGUMENT, "unknown circuit");
  try {
    CircuitSetup S;
    build_circuit_setup(circuit_kind, n_inputs, S);
    sizes[0] = S.f_bits;
    sizes[1] = S.h_len;
    sizes[2] = S.rows;
    sizes[3] = S.m_pos.size();
    sizes[4] = S.abc[2].col.size();
    sizes[5] = S.n_blocks;
    sizes[6] = (uint64_t)S.claim_log_cols;
    sizes[7] = (uint64_t)S.committed_m;
    memcpy(map_digest, S.map_digest, 32);
    if (m_off) memcpy(m_off, S.m_off.data(), S.m_off.size() * 4);
    if (m_pos) memcpy(m_pos, S.m_pos.data(), S.m_pos.size() * 4);
    if (c_off) memcpy(c_off, S.abc[2].off.data(), S.abc[2].off.size() * 4);
    if (c_col) memcpy(c_col, S.abc[2].col.data(), S.abc[2].col.size() * 4);
    if (c_coef) memcpy(c_coef, S.abc[2].coef.data(), S.abc[2].coef.size() * 8);
    return BZ_OK;
  } catch (const std::exception &e) {
    return capi_fail(BZ_ERR_INTERNAL, e.what());
  }
}

int bitz_statement_digest(int circuit_kind, const uint8_t *input_bits, size_t n_inputs,
                          const uint8_t *output_bits, uint8_t digest[32]) {
  if (!digest) return capi_fail(BZ_ERR_ARGUMENT, "null argument");
  int rc = check_statement(circuit_kind, input_bits, n_inputs, output_bits, 100);
  if (rc) return rc;
  try {
    CircuitSetup S;
    build_circuit_setup(circuit_kind, n_inputs, S);
    std::vector<int64_t> ex(n_inputs + 256);
    for (size_t i = 0; i < n_inputs; i++) ex[i] = input_bits[i];
    for (int i = 0; i < 256; i++) ex[n_inputs + i] = output_bits[i];
    matrix_digest(S, ex, digest);
    return BZ_OK;
  } catch (const std::exception &e) {
    return capi_fail(BZ_ERR_INTERNAL, e.what());
  }
}

}  // extern "C"
