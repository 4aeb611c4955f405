// Setup of the SHA-256 circuits: the symbolic replay that yields the
// constraint matrices, the virtual map M and their digests, once per
// (circuit, size). Mirrors tooling/cli/src/end_to_end.rs:161-197 (setup),
// crates/circuit/src/constraints.rs:678-880 (ConstraintGenerator),
// crates/circuit/src/matrix_transpose.rs:475-560 (MTransposeGenerator) over the
// gadgets of crates/circuit/src/sha256.rs:187-504.
#pragma once
#include <stdint.h>

#include <string>
#include <memory>
#include <mutex>
#include <vector>

namespace bz {

enum CircuitKind { kCompression = 0, kChain = 1, kBlockAligned = 2, k2kb = 3 };
const char *circuit_name(int kind);

// The per-compression witness layout (sha256.rs:45, 344-456): hint bits are
// allocated as 48 schedule sums of 34 bits, 64 rounds of two 35-bit sums
// (e then a), and 8 final sums of 33 bits.
constexpr int kHintBitsPerBlock = 48 * 34 + 64 * 70 + 8 * 33;  // 6376
constexpr int kLiftsPerBlock = 20456;
constexpr int kRowsPerBlock = 184;

struct Matrix {  // CSR with integer coefficients
  std::vector<uint32_t> off, col;
  std::vector<int64_t> coef;
};

struct CircuitSetup {
  int kind = 0;
  size_t n_inputs = 0;
  size_t n_blocks = 0;     // compressions, padding block included
  size_t f_bits = 0;       // committed witness bits (inputs then hints)
  size_t h_len = 0;        // integer witness entries, the constant included
  size_t rows = 0;         // R1CS rows
  std::vector<uint32_t> m_off, m_pos;    // M rows over (1 || f)
  std::vector<uint32_t> csc_off, csc_row;  // M^T
  Matrix abc[3];
  std::vector<uint64_t> block_f_offset;  // first hint bit of each compression
  uint8_t map_digest[32];
  uint8_t matrix_digest[32];
  int claim_log_cols = 0;  // s of the claim shape (7 row bits)
  int committed_m = 0;     // log2 of committed bits after padding
  // the integer-matrix digest's hash state after its statement-independent
  // prefix, computed on first use
  std::shared_ptr<std::once_flag> digest_prefix_once = std::make_shared<std::once_flag>();
  mutable uint8_t digest_prefix_state[160];
};

// Builds everything that does not depend on the witness. n_inputs is the
// statement's input bit count (768 for compression, 512 n otherwise).
void build_circuit_setup(int kind, size_t n_inputs, CircuitSetup &out);

void sha256_host(const uint8_t *in, size_t len, uint8_t out[32]);
void sha256_compress_host(uint32_t state[8], const uint32_t block[16]);

}  // namespace bz
