// Host interface of the witness kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace bz {

struct WitnessArgs {
  // per compression: chaining value (8 words), message block (16 words), and
  // the f bit offset of its first hint
  const uint32_t *states, *msgs;
  const uint64_t *offsets;
  int nblocks;
  uint32_t *f;  // packed bits, inputs already written, the rest zero
  size_t h_len;
  const uint32_t *m_off, *m_pos;  // M rows over (1 || f)
  uint32_t *h;                    // packed output bits, zero-initialised
  size_t rows, n_inputs;
  const uint32_t *abc_off[3], *abc_col[3];
  const int64_t *abc_coef[3];
  const uint8_t *bit_c;  // expected value of every bit constraint (inputs, outputs)
  int64_t *prod;         // rows x 3: A h, B h, C h
  int *unsat;            // set to 1 if some row has (A h)(B h) != C h
};

void witness_generate(const WitnessArgs &a, cudaStream_t s);

}  // namespace bz
