// Host interface of the Spartan kernels.
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "device.cuh"
#include "transcript.hpp"

namespace bz {

constexpr int kMaxFpPoint = 40;
struct FpPoint {
  fp c[kMaxFpPoint];
};

struct SpartanArgs {
  FpCtx ctx;
  u128 q;
  int num_row_vars, num_col_vars;
  size_t rows, cols;      // logical R1CS rows and assignment entries
  const int64_t *prod;    // device: rows x 3 exact products
  const uint32_t *hbits;  // device: packed assignment bits
  const uint8_t *digest;  // host: the matrix statement digest
  // column-major A, B, C: entries (row, coefficient-table index)
  const uint32_t *csc_off, *csc_row;
  const uint16_t *csc_idx;
  uint32_t col0_nnz;  // entries of column 0 (the first col0_nnz of csc_row/csc_idx)
  const int64_t *tab_vals;    // device: distinct coefficients
  const uint8_t *tab_which;   // device: 0 = A, 1 = B, 2 = C
  int ntab;
  const uint32_t *bit_rows;   // device: bit constraints with expected value one
  int n_bit_rows;
};

struct SpartanScratch {
  fp *t[8];        // outer tables: E, A, B, C and their fold targets (2^rows each)
  fp *d[4];        // inner tables: D, W and fold targets (2^cols each)
  fp *eq_scratch;  // factor tables
  fp *partial;     // per-block partial sums
  fp *sums;        // device, 3 entries
  fp *tab;         // coefficient table, ntab entries
  fp *host;        // pinned, 4 entries
  RoundChannel *channel = nullptr;  // mailbox for round results; null: copy + sync
  RoundCtl *ctl = nullptr;          // the lane's round controls (queued rounds)
  // blocks of the cooperative kernel that runs the grid rounds resident (128
  // for a lane proving alone, fewer for a pooled lane); 0: queued launches
  int mid_blocks = 0;
};

struct SpartanOut {
  std::vector<fp> outer, inner, rx, ry;  // Montgomery
  fp abc[3];
  fp d_at_ry, final_claim;
  bool ok = false;
};

// The grid of a lane's resident Spartan rounds (SpartanScratch::mid_blocks).
int sp_mid_blocks(bool alone);
FpCtx make_fp_ctx(u128 q);
u128 fp_canonical(fp mont, const FpCtx &c);
// out[k] = canonical value of in[k] (as two LE words), on the device.
void fp_canonical_device(const fp *in, size_t n, const FpCtx &c, fp *out, cudaStream_t s);
fp fp_to_mont(u128 v, const FpCtx &c);
void fp_eq_table(const fp *point, int n, const FpCtx &c, fp *out, fp *scratch, cudaStream_t s);

void spartan_prove(const SpartanArgs &a, Transcript &ts, SpartanScratch &sc, cudaStream_t s,
                   SpartanOut &out);
// The verifier's matrix evaluation: sum over the entries of A + rho B +
// rho^2 C (with the statement's bit constants in C) of eq(r_x, row) eq(r_y,
// col) times the entry, on the device through the prover's bind (the dense
// D(y) over the columns) and a dot product with eq(r_y). Montgomery in and
// out; uses sc.t[0], sc.d[0..1], eq_scratch, partial, sums, tab and host.
fp spartan_matrix_eval(const SpartanArgs &a, const fp *rx, fp rho, const fp *ry,
                       SpartanScratch &sc, cudaStream_t s);

}  // namespace bz
