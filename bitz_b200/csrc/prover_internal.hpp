// Internals shared by the prover and the verifier (prover.cpp, verifier.cpp):
// the per-lane device workspace, the process-wide tables and byte helpers.
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "context.hpp"
#include "prover.hpp"

namespace bz {

inline void put_u64(std::vector<uint8_t> &b, uint64_t v) {
  for (int i = 0; i < 8; i++) b.push_back((uint8_t)(v >> (8 * i)));
}
inline void put_u128(std::vector<uint8_t> &b, u128 v) {
  for (int i = 0; i < 16; i++) b.push_back((uint8_t)(v >> (8 * i)));
}
inline int ceil_log2(size_t n) {
  int l = 0;
  while (((size_t)1 << l) < n) l++;
  return l;
}

// Process-wide tables: the generator's comb and the additive-FFT subspace
// table, built once.
struct Tables {
  f128 generator;
  DeviceBuffer<f128> comb, wh;
  std::vector<f128> wh_host;
};
Tables &tables(cudaStream_t s);

// Slots of Workspace::pin_small, the page-locked home of the small
// device-to-host reads (16-byte units).
constexpr size_t kPinFlag = 0, kPinRoot = 1, kPinLevelRoot = 3, kPinW0 = 5, kPinOne = 6,
                 kPinClaims = 8, kPinSmall = 8 + 128;

// Per-lane device workspace, grown on demand.
struct Workspace {
  DeviceBuffer<int> flag;
  DeviceBuffer<fp> sp_t, sp_d, sp_eqs, sp_part, sp_sums, sp_tab;
  DeviceBuffer<fp> cols_fp;
  DeviceBuffer<u128> exps, folds;
  DeviceBuffer<f128> images, u1, u2, weights, w0, ones, eq, eqs, suffix, basis, eq_ood, lf, lb,
      lf2, lb2, qs, level_cw, bw;
  DeviceBuffer<uint32_t> b3, level_nodes;
  DeviceBuffer<unsigned long long> acc;
  fp *host_fp = nullptr;
  uint64_t *host_acc = nullptr;
  // the claim's canonical column weights and the column folds, copied back
  // while the host absorbs earlier messages
  DeviceBuffer<fp> cols_canon;
  PinnedBuffer<u128> host_cols, host_folds;
  // Ligerito: the next levels' codewords and trees, the query indices and the
  // gathered openings, with their host copies
  DeviceBuffer<f128> lig_cw[2], openings;
  DeviceBuffer<uint32_t> lig_nodes[2];
  DeviceBuffer<uint64_t> qidx;
  PinnedBuffer<uint64_t> pin_idx;
  PinnedBuffer<f128> pin_open, pin_f, pin_b, pin_qw, pin_small;
  // the proof's own state: the staged statement, the witness, the level-0
  // codeword and tree
  DeviceBuffer<uint32_t> states, msgs, fin, f, h, bit_rows, nodes0;
  DeviceBuffer<uint64_t> offsets;
  DeviceBuffer<int64_t> prod;
  DeviceBuffer<uint8_t> bit_c;
  DeviceBuffer<f128> codeword0;
  DeviceBuffer<f128> mt_dense;  // the rows' eq table for the M^T gather
  uint64_t staged_serial = 0;  // the system whose statement these hold
  cudaEvent_t ev_cols = nullptr, ev_folds = nullptr;
  Workspace() {
    AllocScope gate;
    BZ_CUDA(cudaMallocHost(&host_fp, 8 * sizeof(fp)));
    BZ_CUDA(cudaMallocHost(&host_acc, 512 * sizeof(uint64_t)));
    BZ_CUDA(cudaEventCreateWithFlags(&ev_cols, cudaEventDisableTiming));
    BZ_CUDA(cudaEventCreateWithFlags(&ev_folds, cudaEventDisableTiming));
  }
  ~Workspace() {
    AllocScope gate(false);
    if (host_fp) cudaFreeHost(host_fp);
    if (host_acc) cudaFreeHost(host_acc);
    if (ev_cols) cudaEventDestroy(ev_cols);
    if (ev_folds) cudaEventDestroy(ev_folds);
  }
};

Workspace &workspace(Context &lane);

}  // namespace bz
