// The verifier: CircuitProofSystem::verify (tooling/cli/src/end_to_end.rs:
// 339-377) on proof bytes, replayed message by message through this
// library's own transcript, with the bulk steps on the device through the
// prover's kernels: the Spartan matrix evaluation (the prover's bind, then a
// dot product with eq(r_y)), the column images (the comb), the transposed
// query and its weight digest, the weights' evaluation, the ring-switch basis
// and the Ligerito basis folds and query glue. The checks follow
// crates/spartan/src/piop.rs (verify side), crates/verifier/src/{fold,reduce,
// verify}.rs, crates/gkr/src/lib.rs:717-772, crates/post_gkr/src/{lib,
// sumcheck}.rs, crates/pcs/src/{commitment,opening,ood,mle}.rs and this
// library's Ligerito construction (prover.cpp, ProofSystem::ligerito).
#include <string.h>

#include <string>
#include <vector>

#include "bitz_kernels.hpp"
#include "eq.cuh"
#include "hash.cuh"
#include "post_gkr.hpp"
#include "prover.hpp"
#include "prover_internal.hpp"
#include "spartan.hpp"
#include "status.hpp"

namespace bz {

// ------------------------------------------------------------ wire format

// WireProof::from_bytes (crates/host/src/wire_proof.rs:109-140): a 32-byte
// header (magic "bitzPCS\0", version 1, header length 32, flags 0, the two
// stream lengths), then exactly the declared narg and hint bytes.
int wire_decode(const uint8_t *bytes, size_t len, WireView &out, std::string &err) {
  auto le = [&](size_t at, int n) {
    uint64_t v = 0;
    for (int i = n - 1; i >= 0; i--) v = (v << 8) | bytes[at + i];
    return v;
  };
  if (!bytes || len < 32) {
    err = "OutOfInput: proof is too short";
    return BZ_ERR_MALFORMED;
  }
  static const uint8_t kMagic[8] = {'b', 'i', 't', 'z', 'P', 'C', 'S', 0};
  if (memcmp(bytes, kMagic, 8) != 0) {
    err = "BadMagic: the first eight bytes are not bitzPCS\\0";
    return BZ_ERR_MALFORMED;
  }
  if (le(8, 2) != 1) {
    err = "UnsupportedVersion(" + std::to_string(le(8, 2)) + ")";
    return BZ_ERR_MALFORMED;
  }
  if (le(10, 2) != 32) {
    err = "BadHeaderLen(" + std::to_string(le(10, 2)) + ")";
    return BZ_ERR_MALFORMED;
  }
  if (le(12, 4) != 0) {
    err = "ReservedFlagsSet(" + std::to_string(le(12, 4)) + ")";
    return BZ_ERR_MALFORMED;
  }
  const uint64_t narg = le(16, 8), hints = le(24, 8);
  if (narg > UINT64_MAX - 32 || hints > UINT64_MAX - 32 - narg) {
    err = "LengthOverflow: the declared lengths do not fit the address space";
    return BZ_ERR_MALFORMED;
  }
  if (32 + narg + hints != (uint64_t)len) {
    err = "LengthMismatch: declared " + std::to_string(32 + narg + hints) + ", was " +
          std::to_string(len);
    return BZ_ERR_MALFORMED;
  }
  out.narg = bytes + 32;
  out.narg_len = (size_t)narg;
  out.hints = bytes + 32 + narg;
  out.hints_len = (size_t)hints;
  return BZ_OK;
}

namespace {

const f128 kOne = {1, 0};

// The narg stream: each prover message is read and absorbed as the prover
// absorbed it; reading past the end marks the proof short (zeros are
// returned so the replay can run to its first failed check).
struct Narg {
  Transcript &t;
  const uint8_t *p;
  size_t len, pos = 0;
  bool short_read = false;
  void take(void *out, size_t n) {
    if (pos + n > len) {
      short_read = true;
      memset(out, 0, n);
      pos = len;
      return;
    }
    memcpy(out, p + pos, n);
    pos += n;
    t.public_message(out, n);
  }
  f128 f() {
    f128 v;
    take(&v, 16);
    return v;
  }
  uint64_t u64() {
    uint8_t b[8];
    take(b, 8);
    uint64_t v = 0;
    for (int i = 7; i >= 0; i--) v = (v << 8) | b[i];
    return v;
  }
  // Transcript::grind's verifier side (crates/transcript/src/pow.rs:21-50):
  // the header, the seed, and the prover's nonce checked.
  bool grind(const char *label, uint32_t bits) {
    if (bits == 0) return true;
    const size_t ll = strlen(label);
    t.public_message("bitz-transcript-pow-v1", 22);
    t.public_u64((uint64_t)ll);
    t.public_message(label, ll);
    uint8_t b4[4];
    for (int i = 0; i < 4; i++) b4[i] = (uint8_t)(bits >> (8 * i));
    t.public_message(b4, 4);
    uint8_t seed[16];
    t.squeeze(seed, 16);
    const uint64_t nonce = u64();
    return !short_read && pow_valid(seed, nonce, bits);
  }
};

// The hint stream (never absorbed).
struct Hints {
  const uint8_t *p;
  size_t len, pos = 0;
  const uint8_t *take(size_t n) {
    if (n > len - pos) return nullptr;
    const uint8_t *q = p + pos;
    pos += n;
    return q;
  }
};

u128 get_u128(const uint8_t *b) {
  u128 v = 0;
  for (int i = 15; i >= 0; i--) v = (v << 8) | b[i];
  return v;
}

fp mont(u128 v, const FpCtx &c) { return fp_mul(fp{(uint64_t)v, (uint64_t)(v >> 64)}, c.r2, c); }
bool fp_eq(fp a, fp b) { return a.lo == b.lo && a.hi == b.hi; }

// eq(a, b) = prod_i (a_i b_i + (1 - a_i)(1 - b_i)) over the prime field.
fp fp_eq_at(const fp *a, const fp *b, int n, const FpCtx &c) {
  fp e = c.one;
  for (int i = 0; i < n; i++) {
    const fp ab = fp_mul(a[i], b[i], c);
    const fp na = fp_sub(c.one, a[i], c), nb = fp_sub(c.one, b[i], c);
    e = fp_mul(e, fp_add(ab, fp_mul(na, nb, c), c), c);
  }
  return e;
}

// A prime-field sumcheck round (sumcheck.rs:771-811): the coefficients are
// canonical and below q, p(0) + p(1) equals the claim, they are absorbed as
// one public message, and the claim moves to p(r).
bool fp_round(Transcript &t, const FpCtx &c, u128 q, const uint8_t *coefs, int ncoef, fp &claim,
              fp &r) {
  fp co[4], at_one = fp_zero();
  for (int i = 0; i < ncoef; i++) {
    const u128 v = get_u128(coefs + 16 * i);
    if (v >= q) return false;
    co[i] = mont(v, c);
    at_one = fp_add(at_one, co[i], c);
  }
  if (!fp_eq(fp_add(co[0], at_one, c), claim)) return false;
  t.public_message(coefs, 16 * (size_t)ncoef);
  r = mont(t.challenge_fp(q), c);
  fp v = fp_zero();
  for (int i = ncoef - 1; i >= 0; i--) v = fp_add(fp_mul(v, r, c), co[i], c);
  claim = v;
  return true;
}

// Montgomery eq table over n <= 7 coordinates on the host (coordinate i =
// index bit i).
void fp_eq_small(const fp *pt, int n, const FpCtx &c, fp *out) {
  out[0] = c.one;
  for (int i = 0; i < n; i++) {
    const size_t h = (size_t)1 << i;
    for (size_t k = 0; k < h; k++) {
      const fp one = fp_mul(out[k], pt[i], c);
      out[k + h] = one;
      out[k] = fp_sub(out[k], one, c);
    }
  }
}

// post_gkr's advance (post_gkr/src/lib.rs:290-292).
f128 advance(f128 claim, f128 a0, f128 a2, f128 r) {
  return gadd(a0, gmul(r, gadd(gadd(claim, a2), gmul(r, a2))));
}

// BLAKE3 of one message, default mode.
void blake3_once(const uint8_t *in, size_t len, uint8_t out[32]) {
  Blake3 h;
  h.update(in, len);
  h.finalize(out);
}

}  // namespace

// One failed check: its message, and the reference's verification error.
#define BZ_VERIFY(cond, what)   \
  do {                          \
    if (!(cond)) {              \
      error = (what);           \
      return BZ_ERR_VERIFY;     \
    }                           \
  } while (0)

int ProofSystem::verify(const uint8_t *proof, size_t proof_len, Context *lane) {
  const CircuitSetup &S = *dev_->host;
  Context &ctx = lane ? *lane : Context::get();
  cudaStream_t s = ctx.stream();
  Workspace &W = workspace(ctx);
  Tables &T = tables(s);
  W.staged_serial = 0;  // the verifier reuses the lane's buffers
  const int nr = ceil_log2(S.rows ? S.rows : 1), nc = ceil_log2(S.h_len);
  // ---- proof bytes: root || Spartan section || bitzPCS wire container
  const size_t spartan_len = 16 * (4 * (size_t)nr + 3 + 3 * (size_t)nc);
  if (!proof || proof_len < 32 + spartan_len) {
    error = "proof is shorter than its root and Spartan section";
    return BZ_ERR_MALFORMED;
  }
  const uint8_t *root = proof;
  const uint8_t *outer = proof + 32, *abc = outer + 64 * (size_t)nr, *inner = abc + 48;
  WireView wv;
  int rc = wire_decode(proof + 32 + spartan_len, proof_len - 32 - spartan_len, wv, error);
  if (rc) return rc;
  const char *dom = circuit_name(kind_);
  Transcript t((const uint8_t *)"bitz/circuit-e2e/v2", 19, (const uint8_t *)dom, strlen(dom));
  Narg rd{t, wv.narg, wv.narg_len};
  Hints hs{wv.hints, wv.hints_len};
  const int log_n = pcs_.log_n, m = S.committed_m;
  // ---- receive_commitment (commitment.rs:153-190, ood.rs:56-75)
  t.public_message("bitz/pcs/commit/v1", 18);
  t.public_message(root, 32);
  t.public_message(pcs_enc_.data(), pcs_enc_.size());
  std::vector<f128> ood_pt;
  f128 ood_val = mk(0, 0);
  if (security_ == 100) {
    t.public_message("bitz/pcs/ood/v1", 15);
    for (int i = 0; i < log_n; i++) ood_pt.push_back(t.challenge_f128());
    ood_val = rd.f();
  }
  // ---- bind and the prime (end_to_end.rs:401-455)
  t.public_u64(public_bytes_.size());
  t.public_message(public_bytes_.data(), public_bytes_.size());
  t.public_message(root, 32);
  t.public_u64(7);
  t.public_u64((uint64_t)S.claim_log_cols);
  t.public_f128(generator_);
  t.public_message(pcs_enc_.data(), pcs_enc_.size());
  t.public_message(S.map_digest, 32);
  t.public_message(matrix_digest_, 32);
  t.public_message("bitz/circuit-opening-path/v1", 28);
  const uint8_t path = 1;
  t.public_message(&path, 1);
  const u128 q = t.prime(121);
  const FpCtx fc = make_fp_ctx(q);
  std::vector<uint8_t> params;
  put_u64(params, 7);
  put_u64(params, (uint64_t)S.claim_log_cols);
  put_u128(params, q);
  const uint8_t *gb = reinterpret_cast<const uint8_t *>(&generator_);
  params.insert(params.end(), gb, gb + 16);
  t.public_message(params.data(), params.size());
  // ---- Spartan (piop.rs:117-160): outer cubic rounds, then the inner quadratic
  t.public_message(matrix_digest_, 32);
  std::vector<fp> tau(nr), rx(nr), ry(nc);
  for (int i = 0; i < nr; i++) tau[i] = mont(t.challenge_fp(q), fc);
  fp claim = fp_zero();
  for (int i = 0; i < nr; i++)
    BZ_VERIFY(fp_round(t, fc, q, outer + 64 * i, 4, claim, rx[i]), "Spartan outer round check");
  const u128 az_c = get_u128(abc), bz_c = get_u128(abc + 16), cz_c = get_u128(abc + 32);
  BZ_VERIFY(az_c < q && bz_c < q && cz_c < q, "Spartan claimed evaluations are not canonical");
  const fp az = mont(az_c, fc), bzv = mont(bz_c, fc), cz = mont(cz_c, fc);
  BZ_VERIFY(fp_eq(claim, fp_mul(fp_eq_at(tau.data(), rx.data(), nr, fc),
                                fp_sub(fp_mul(az, bzv, fc), cz, fc), fc)),
            "Spartan outer closing check");
  t.public_message(abc, 48);
  const fp rho = mont(t.challenge_fp(q), fc), rho2 = fp_mul(rho, rho, fc);
  claim = fp_add(fp_add(az, fp_mul(rho, bzv, fc), fc), fp_mul(rho2, cz, fc), fc);
  for (int i = 0; i < nc; i++)
    BZ_VERIFY(fp_round(t, fc, q, inner + 48 * i, 3, claim, ry[i]), "Spartan inner round check");
  const fp fin = claim;
  // D(r_y) on the device
  const size_t R = (size_t)1 << nr, Cn = (size_t)1 << nc;
  W.sp_t.resize(8 * R);
  W.sp_d.resize(4 * Cn);
  W.sp_eqs.resize(4096 * 2 + ((size_t)1 << ((std::max(nr, nc) + 1) / 2 + 1)));
  W.sp_part.resize(3 * kSMs * 8 + 16);
  W.sp_sums.resize(4);
  W.sp_tab.resize(dev_->ntab + 1);
  if (bit_rows_.empty())
    W.bit_rows.resize(1);
  else
    W.bit_rows.upload(bit_rows_.data(), bit_rows_.size(), s);
  SpartanScratch sc;
  for (int i = 0; i < 8; i++) sc.t[i] = W.sp_t.get() + i * R;
  for (int i = 0; i < 4; i++) sc.d[i] = W.sp_d.get() + i * Cn;
  sc.eq_scratch = W.sp_eqs.get();
  sc.partial = W.sp_part.get();
  sc.sums = W.sp_sums.get();
  sc.tab = W.sp_tab.get();
  sc.host = W.host_fp;
  SpartanArgs sa;
  sa.ctx = fc;
  sa.q = q;
  sa.num_row_vars = nr;
  sa.num_col_vars = nc;
  sa.rows = S.rows;
  sa.cols = S.h_len;
  sa.csc_off = dev_->sp_off.get();
  sa.csc_row = dev_->sp_row.get();
  sa.csc_idx = dev_->sp_idx.get();
  sa.col0_nnz = dev_->col0_nnz;
  sa.tab_vals = dev_->tab_vals.get();
  sa.tab_which = dev_->tab_which.get();
  sa.ntab = dev_->ntab;
  sa.bit_rows = W.bit_rows.get();
  sa.n_bit_rows = (int)bit_rows_.size();
  const fp d_ry = spartan_matrix_eval(sa, rx.data(), rho, ry.data(), sc, s);
  // ---- the opening claim (end_to_end.rs:509-528)
  const int sc_cols = S.claim_log_cols;
  const size_t ncol = (size_t)1 << sc_cols;
  std::vector<fp> pt(7 + sc_cols, fp_zero());
  for (int i = 0; i < nc && i < 7 + sc_cols; i++) pt[i] = ry[i];
  std::vector<u128> rows_w(128), cols_w(ncol);
  {
    fp e[128];
    fp_eq_small(pt.data(), 7, fc, e);
    for (int b = 0; b < 128; b++) rows_w[b] = fp_canonical(fp_mul(e[b], d_ry, fc), fc);
  }
  W.cols_fp.resize(ncol + 2);
  W.cols_canon.resize(ncol);
  fp_eq_table(pt.data() + 7, sc_cols, fc, W.cols_fp.get(), sc.eq_scratch, s);
  fp_canonical_device(W.cols_fp.get(), ncol, fc, W.cols_canon.get(), s);
  BZ_CUDA(cudaMemcpyAsync(cols_w.data(), W.cols_canon.get(), ncol * 16, cudaMemcpyDeviceToHost, s));
  BZ_CUDA(stream_wait(s));
  const u128 fin_c = fp_canonical(fin, fc);
  t.public_message("bitz/virtual-statement/v1", 25);
  t.public_message(root, 32);
  {
    std::vector<uint8_t> vp = params;
    put_u64(vp, 7);
    put_u64(vp, (uint64_t)(m - 7));
    t.public_message(vp.data(), vp.size());
  }
  t.public_message(S.map_digest, 32);
  {
    std::vector<uint8_t> ce;
    ce.reserve(16 * (129 + ncol) + 16);
    put_u64(ce, 128);
    for (auto w : rows_w) put_u128(ce, w);
    put_u64(ce, ncol);
    for (auto w : cols_w) put_u128(ce, w);
    put_u128(ce, fin_c);
    t.public_message(ce.data(), ce.size());
  }
  t.public_message(pcs_enc_.data(), pcs_enc_.size());
  // ---- receive_fold (crates/verifier/src/fold.rs:42-77): every fold is at
  // most 128 (q - 1), and sum_j cols_w[j] fold_j = the claim mod q
  std::vector<u128> folds(ncol);
  {
    const u128 bound = (u128)128 * (q - 1);
    fp acc = fp_zero();
    for (size_t j = 0; j < ncol; j++) {
      uint8_t b[16];
      rd.take(b, 16);
      folds[j] = get_u128(b);
      BZ_VERIFY(folds[j] <= bound, "a column fold exceeds 128 (q - 1)");
      acc = fp_add(acc, fp_mul(mont(cols_w[j], fc), mont(folds[j] % q, fc), fc), fc);
    }
    BZ_VERIFY(!rd.short_read, "the proof ends inside the column folds");
    BZ_VERIFY(fp_canonical(acc, fc) == fin_c, "the column folds do not meet the Spartan claim");
  }
  // the images g^fold on the device (the prover's comb)
  W.folds.upload(folds.data(), ncol, s);
  W.images.resize(ncol + 128);
  comb_pow(T.comb.get(), W.folds.get(), (int)ncol, W.images.get() + 128, s);
  W.exps.upload(rows_w.data(), 128, s);
  comb_pow(T.comb.get(), W.exps.get(), 128, W.images.get(), s);
  std::vector<f128> row_images(128);
  BZ_CUDA(cudaMemcpyAsync(row_images.data(), W.images.get(), 128 * 16, cudaMemcpyDeviceToHost, s));
  BZ_VERIFY(rd.grind("bitz/columns/v1", grinding_bits((uint32_t)security_, (uint64_t)sc_cols)),
            "column-fold grinding nonce");
  std::vector<f128> point(sc_cols);
  for (auto &z : point) z = t.challenge_f128();
  // ---- gpgkr_verify (crates/gkr/src/lib.rs:717-772) from e0 = MLE(images)(zeta)
  W.u2.resize(ncol);
  W.eqs.resize(eq_scratch_entries(std::max(sc_cols, std::max(m, log_n))));
  W.acc.resize(512);
  eq_table_device(point.data(), sc_cols, W.u2.get(), W.eqs.get(), s);
  BZ_CUDA(cudaMemsetAsync(W.acc.get(), 0, 16, s));
  dot(W.u2.get(), W.images.get() + 128, ncol, W.acc.get(), Publish{nullptr, nullptr, 0}, s);
  BZ_CUDA(cudaMemcpyAsync(W.host_acc, W.acc.get(), 16, cudaMemcpyDeviceToHost, s));
  BZ_CUDA(stream_wait(s));
  f128 gclaim = mk(W.host_acc[0], W.host_acc[1]);
  const uint32_t gkr_bits = grinding_bits((uint32_t)security_, 3);
  for (int layer = 0; layer < 7; layer++) {
    const int n = (int)point.size();
    std::vector<f128> next(n + 1);
    f128 eq_bound = kOne;
    for (int i = n - 1; i >= 0; i--) {
      const f128 z = point[i];
      const f128 sum_b = rd.f(), sum_inf = rd.f();
      // claim = (1 + z) sum0 + z sum1: the prover sends sum1 when z = 0
      f128 sum0, sum1;
      if (gis_zero(z)) {
        sum0 = gclaim;
        sum1 = sum_b;
      } else {
        sum0 = sum_b;
        sum1 = gmul(gadd(gclaim, gmul(gadd(kOne, z), sum_b)), gf_inv_host(z));
      }
      BZ_VERIFY(rd.grind("gkr/cubic/v1", gkr_bits), "GKR grinding nonce");
      const f128 r = t.challenge_f128();
      next[i] = r;
      const f128 eq_r = gadd(gadd(kOne, r), z);
      // quadratic_at(sum0, sum1, sum_inf, r), then times eq(r, z)
      gclaim = gmul(eq_r, gadd(sum0, gmul(r, gadd(gadd(sum1, sum0), gmul(gadd(r, kOne), sum_inf)))));
      eq_bound = gmul(eq_bound, eq_r);
    }
    const f128 left = rd.f(), right = rd.f();
    BZ_VERIFY(!rd.short_read, "the proof ends inside the GKR layers");
    BZ_VERIFY(geq(gmul(gmul(eq_bound, left), right), gclaim), "GKR layer closing check");
    const f128 tt = t.challenge_f128();
    next[n] = tt;
    gclaim = gadd(left, gmul(tt, gadd(right, left)));
    point = next;
  }
  // ---- gkr_reduce's claim (crates/verifier/src/reduce.rs:27-54) and the
  // transposed query (virtual_map.rs:174-223), on the device as the prover
  const f128 ip_target = gadd(gclaim, kOne);
  std::vector<f128> eqb(128), u1(128);
  eq_table_host(point.data() + sc_cols, 7, eqb.data());
  for (int b = 0; b < 128; b++) u1[b] = gmul(gadd(row_images[b], kOne), eqb[b]);
  W.u1.upload(u1.data(), 128, s);
  eq_table_device(point.data(), sc_cols, W.u2.get(), W.eqs.get(), s);
  const size_t nbits = (size_t)1 << m;
  W.weights.resize(nbits);
  W.w0.resize(2);
  W.mt_dense.resize((size_t)128 << sc_cols);
  mt_transpose(dev_->csc_off.get(), dev_->csc_row.get(), S.f_bits + 1, W.u1.get(), W.u2.get(),
               W.weights.get(), nbits, W.w0.get(), s, W.mt_dense.get(), sc_cols);
  // the weight digest (opening.rs:337-368): the weights' chunk tree on the
  // device, the trailing column weight [1] and the root here
  const size_t nchunks = nbits * 16 / 1024;
  W.b3.resize(16 * nchunks);
  Blake3 dk = Blake3::derive_key("bitz/pcs/bit-inner-product-weights/v1");
  uint32_t left_cv[8];
  f128 w0_h;
  blake3_tree_cv(reinterpret_cast<const uint8_t *>(W.weights.get()), nchunks, dk.key,
                 B3_DERIVE_KEY_MATERIAL, W.b3.get(), left_cv, s, nullptr, W.w0.get(), &w0_h);
  uint8_t digest[32];
  {
    uint8_t one16[64] = {1};
    uint32_t mw[16], right[8], out[8], pm[16];
    b3_load_le(one16, mw, 16);
    b3_compress(dk.key, mw, nchunks, 16, B3_DERIVE_KEY_MATERIAL | B3_CHUNK_START | B3_CHUNK_END,
                right);
    memcpy(pm, left_cv, 32);
    memcpy(pm + 8, right, 32);
    b3_compress(dk.key, pm, 0, 64, B3_DERIVE_KEY_MATERIAL | B3_PARENT | B3_ROOT, out);
    b3_store_le(out, digest, 8);
  }
  const f128 target2 = gadd(ip_target, w0_h);
  t.public_message("bitz/pcs/bit-inner-product/v3", 29);
  t.public_message(root, 32);
  t.public_message(pcs_enc_.data(), pcs_enc_.size());
  t.public_u64(nbits);
  t.public_u64(1);
  t.public_message(digest, 32);
  t.public_f128(target2);
  t.public_message("bitz/pcs/inner-product-sumcheck/v2", 34);
  // ---- post_gkr::verify (post_gkr/src/lib.rs:150-166, sumcheck.rs:112-200)
  std::vector<f128> rho_pt(m);
  f128 pclaim = target2;
  const uint32_t pg_bits = grinding_bits((uint32_t)security_, 2);
  for (int k = 0; k < m; k++) {
    const f128 a0 = rd.f(), a2 = rd.f();
    BZ_VERIFY(rd.grind("bitz/pcs/sumcheck/v1", pg_bits), "inner-product sumcheck grinding nonce");
    const f128 r = t.challenge_f128();
    rho_pt[k] = r;
    pclaim = advance(pclaim, a0, a2, r);
  }
  const f128 v = rd.f();
  BZ_VERIFY(!rd.short_read, "the proof ends inside the inner-product sumcheck");
  {
    // MLE(weights)(rho) on the device: eq(rho, .) against the weights
    W.eq.resize(nbits);
    eq_table_device(rho_pt.data(), m, W.eq.get(), W.eqs.get(), s);
    BZ_CUDA(cudaMemsetAsync(W.acc.get(), 0, 16, s));
    dot(W.eq.get(), W.weights.get(), nbits, W.acc.get(), Publish{nullptr, nullptr, 0}, s);
    BZ_CUDA(cudaMemcpyAsync(W.host_acc, W.acc.get(), 16, cudaMemcpyDeviceToHost, s));
    BZ_CUDA(stream_wait(s));
    const f128 wv = mk(W.host_acc[0], W.host_acc[1]);
    BZ_VERIFY(geq(gmul(wv, v), pclaim), "inner-product sumcheck closing check");
  }
  // ---- the MLE opening with binding (opening.rs:119-135), ring switch
  // (mle.rs:63-123) and OOD batching (ood.rs:77-95)
  t.public_message("bitz/pcs/mle-opening/v1", 23);
  t.public_message(root, 32);
  t.public_message(pcs_enc_.data(), pcs_enc_.size());
  t.public_u64((uint64_t)m);
  for (auto &c : rho_pt) t.public_f128(c);
  t.public_f128(v);
  t.public_message("bitz/pcs/mle-claims/v1", 22);
  std::vector<f128> claims(128);
  for (auto &c : claims) c = rd.f();
  {
    std::vector<f128> pre(128);
    eq_table_host(rho_pt.data(), 7, pre.data());
    wide chk = wzero();
    for (int b = 0; b < 128; b++) wacc(chk, gmul_wide(pre[b], claims[b]));
    BZ_VERIFY(!rd.short_read && geq(greduce(chk), v), "ring-switch claims against the evaluation");
  }
  BZ_VERIFY(rd.grind("bitz/pcs/ring/v1",
                     grinding_bits((uint32_t)security_, 7 + (security_ == 100 ? 1 : 0))),
            "ring-switch grinding nonce");
  t.public_message("bitz/pcs/ring-switch-challenges/v1", 34);
  std::vector<f128> bpt(7), bw(128);
  for (auto &c : bpt) c = t.challenge_f128();
  eq_table_host(bpt.data(), 7, bw.data());
  // transpose.rs:14: the target is sum over v of X^v (sum over the set bits
  // u of claims[v] of bw[u])
  f128 ptarget = mk(0, 0);
  for (int vv = 0; vv < 128; vv++) {
    f128 sv = mk(0, 0);
    for (uint64_t mm = claims[vv].lo; mm; mm &= mm - 1) sv = gadd(sv, bw[__builtin_ctzll(mm)]);
    for (uint64_t mm = claims[vv].hi; mm; mm &= mm - 1) sv = gadd(sv, bw[64 + __builtin_ctzll(mm)]);
    ptarget = gadd(ptarget, gmul_xk(sv, vv));
  }
  const size_t np = (size_t)1 << log_n;
  W.suffix.resize(np);
  eq_table_device(rho_pt.data() + 7, log_n, W.suffix.get(), W.eqs.get(), s);
  W.bw.upload(bw.data(), 128, s);
  W.lb.resize(np);
  W.lb2.resize(np);
  W.lf2.resize(np);
  W.eq.resize(np);
  f128 coef = mk(0, 0);
  if (security_ == 100) {
    t.public_message("bitz/pcs/ood-batching/v1", 24);
    coef = t.challenge_f128();
    ptarget = gadd(ptarget, gmul(coef, ood_val));
    W.eq_ood.resize(np);
    eq_table_device(ood_pt.data(), log_n, W.eq_ood.get(), W.eqs.get(), s);
  }
  packed_basis(W.suffix.get(), np, W.bw.get(), security_ == 100 ? W.eq_ood.get() : nullptr, coef,
               W.lb.get(), s);
  // ---- the Ligerito opening (this library's construction, prover.cpp)
  const uint8_t *lhead = hs.take(4);
  BZ_VERIFY(lhead, "the hint stream ends before the opening");
  const uint32_t llen = (uint32_t)lhead[0] | ((uint32_t)lhead[1] << 8) |
                        ((uint32_t)lhead[2] << 16) | ((uint32_t)lhead[3] << 24);
  BZ_VERIFY((size_t)llen == wv.hints_len - 4, "the opening's length prefix");
  const PcsConfig &cfg = pcs_;
  std::vector<uint32_t> sched;
  for (int i = 0; i < cfg.nlevels; i++) {
    const PcsLevel &L = cfg.levels[i];
    for (int r = 0; r < L.k; r++)
      sched.push_back(security_ == 128 ? (uint32_t)L.fold_grinding
                                       : (uint32_t)(L.fold_grinding - r));
    sched.push_back((uint32_t)L.grinding);
  }
  size_t at = 0;
  auto lig_grind = [&]() {
    const uint32_t bits = sched[at++];
    t.public_message("pcs/flock/pow/v1", 16);
    uint8_t b4[4];
    for (int i = 0; i < 4; i++) b4[i] = (uint8_t)(bits >> (8 * i));
    t.public_message(b4, 4);
    uint8_t seed[16];
    t.squeeze(seed, 16);
    const uint64_t nonce = rd.u64();
    return !rd.short_read && pow_valid(seed, nonce, bits);
  };
  auto sample_vec = [&](size_t n) {
    t.public_message("pcs/flock/sample-vector/v1", 26);
    t.public_u64(n);
    std::vector<f128> out(n);
    for (auto &x : out) x = t.challenge_f128();
    return out;
  };
  t.public_message("flock-ligerito-basis-v0", 23);
  t.public_f128(ptarget);
  f128 lclaim = ptarget;
  uint8_t cur_root[32];
  memcpy(cur_root, root, 32);
  int cur_k = cfg.levels[0].k, cur_rate = cfg.levels[0].log_inv_rate, cur_log_n = log_n;
  std::vector<f128> f_final;
  f128 *b = W.lb.get(), *b2 = W.lb2.get();
  size_t n = np;
  for (int i = 0; i < cfg.nlevels; i++) {
    const PcsLevel &L = cfg.levels[i];
    std::vector<f128> rs;
    for (int r = 0; r < L.k; r++) {
      const f128 a0 = rd.f(), a2 = rd.f();
      BZ_VERIFY(lig_grind(), "Ligerito fold grinding nonce");
      const f128 c = t.challenge_f128();
      rs.push_back(c);
      lclaim = advance(lclaim, a0, a2, c);
      // the basis folds at c (both tables of the fold kernel are the basis)
      quad_fold(b, b, c, b2, W.lf2.get(), n, 0, W.acc.get(), Publish{nullptr, nullptr, 0}, s);
      std::swap(b, b2);
      n /= 2;
    }
    const int l = L.log_msg_cols;
    const bool last = i + 1 == cfg.nlevels;
    uint8_t next_root[32] = {0};
    if (!last) {
      const PcsLevel &N = cfg.levels[i + 1];
      uint8_t rb[36];
      rd.take(rb, 36);
      BZ_VERIFY(!rd.short_read && rb[0] == 32 && !rb[1] && !rb[2] && !rb[3],
                "a Ligerito level's root");
      memcpy(next_root, rb + 4, 32);
      if (N.ood_samples) {
        const std::vector<f128> opt = sample_vec((size_t)l);
        const f128 ov = rd.f();
        const f128 mu = t.challenge_f128();
        eq_table_device(opt.data(), l, W.eq.get(), W.eqs.get(), s);
        axpy(b, mu, W.eq.get(), n, s);  // basis += mu eq(point, .)
        lclaim = gadd(lclaim, gmul(mu, ov));
      }
    } else {
      uint8_t nb[4];
      rd.take(nb, 4);
      const uint32_t fl = (uint32_t)nb[0] | ((uint32_t)nb[1] << 8) | ((uint32_t)nb[2] << 16) |
                          ((uint32_t)nb[3] << 24);
      BZ_VERIFY(!rd.short_read && fl == (1u << l), "the final vector's length");
      f_final.resize(fl);
      for (auto &x : f_final) x = rd.f();
    }
    BZ_VERIFY(lig_grind(), "Ligerito query grinding nonce");
    const std::vector<f128> qs = sample_vec((size_t)L.queries);
    const size_t rows = (size_t)1 << (cur_log_n - cur_k + cur_rate);
    const int width = 1 << cur_k, depth = ceil_log2(rows);
    const uint8_t *qh = hs.take(8);
    BZ_VERIFY(qh, "the hint stream ends before a level's openings");
    uint64_t nq = 0;
    for (int k = 7; k >= 0; k--) nq = (nq << 8) | qh[k];
    BZ_VERIFY(nq == (uint64_t)L.queries, "a level's query count");
    std::vector<f128> eqr((size_t)1 << L.k);
    eq_table_host(rs.data(), L.k, eqr.data());
    std::vector<f128> vals(L.queries);
    std::vector<uint64_t> idx(L.queries);
    for (int qi = 0; qi < L.queries; qi++) {
      idx[qi] = qs[qi].lo & (rows - 1);
      const uint8_t *row = hs.take((size_t)width * 16);
      BZ_VERIFY(row, "the hint stream ends inside an opened row");
      uint8_t node[32];
      blake3_once(row, (size_t)width * 16, node);
      size_t at_node = rows + idx[qi];
      for (int d = 0; d < depth; d++) {
        const uint8_t *sib = hs.take(32);
        BZ_VERIFY(sib, "the hint stream ends inside a Merkle path");
        uint8_t pair[64];
        memcpy(pair, (at_node & 1) ? sib : node, 32);
        memcpy(pair + 32, (at_node & 1) ? node : sib, 32);
        blake3_once(pair, 64, node);
        at_node >>= 1;
      }
      BZ_VERIFY(memcmp(node, cur_root, 32) == 0, "a Merkle path does not reach the root");
      wide acc = wzero();
      for (int c = 0; c < width; c++) {
        f128 e;
        memcpy(&e, row + 16 * c, 16);
        wacc(acc, gmul_wide(e, eqr[c]));
      }
      vals[qi] = greduce(acc);
    }
    const int av = ceil_log2((size_t)L.queries);
    const std::vector<f128> alpha = sample_vec((size_t)av);
    const f128 mu = t.challenge_f128();
    std::vector<f128> beta((size_t)1 << av), sq(L.queries);
    eq_table_host(alpha.data(), av, beta.data());
    for (int qi = 0; qi < L.queries; qi++) {
      sq[qi] = gmul(mu, beta[qi]);
      lclaim = gadd(lclaim, gmul(sq[qi], vals[qi]));
    }
    // the glue on the device: basis += sum_q s_q X(x_q)
    W.qidx.upload(idx.data(), idx.size(), s);
    W.qs.upload(sq.data(), sq.size(), s);
    query_basis(W.qidx.get(), T.wh.get(), W.qs.get(), L.queries, l, b, s);
    if (!last) {
      memcpy(cur_root, next_root, 32);
      cur_log_n = l;
      cur_k = cfg.levels[i + 1].k;
      cur_rate = cfg.levels[i + 1].log_inv_rate;
    }
  }
  BZ_VERIFY(!rd.short_read, "the proof ends inside the opening");
  {
    std::vector<f128> hb(n);
    BZ_CUDA(cudaMemcpyAsync(hb.data(), b, n * 16, cudaMemcpyDeviceToHost, s));
    BZ_CUDA(stream_wait(s));
    BZ_VERIFY(f_final.size() == n, "the final vector's length");
    wide chk = wzero();
    for (size_t j = 0; j < n; j++) wacc(chk, gmul_wide(hb[j], f_final[j]));
    BZ_VERIFY(geq(greduce(chk), lclaim), "the final vector against its basis");
  }
  // both streams spent (crates/verifier/src/verify.rs:69-71, check_eof)
  BZ_VERIFY(rd.pos == rd.len && hs.pos == hs.len, "leftover proof bytes");
  return BZ_OK;
}

}  // namespace bz
