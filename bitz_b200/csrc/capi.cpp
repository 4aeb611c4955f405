// The extern "C" boundary: argument checks, device staging for the host-buffer
// variants, and exception-to-status translation. No exception crosses it.
#include <cuda_runtime.h>
#include <stdlib.h>

#include <mutex>
#include <string>

#include "../../include/bitz_b200.h"
#include "context.hpp"
#include "gkr.hpp"
#include "post_gkr.hpp"
#include "status.hpp"
#include "transcript.hpp"

using namespace bz;

struct bitz_transcript {
  Transcript t;
};

// Prover lanes are streams that each keep a round kernel waiting for their
// host thread; with the CUDA default of 8 hardware work queues, lanes past 8
// share queues, and a waiting kernel at the head of a queue holds back the
// other lanes' launches behind it. When the library is loaded before the
// process creates its CUDA context and the caller has not chosen, ask for 32
// queues (the most the driver gives). A caller's own setting is kept.
__attribute__((constructor)) static void bz_default_work_queues() {
  setenv("CUDA_DEVICE_MAX_CONNECTIONS", "32", 0);
}

static thread_local std::string g_last_error;

static int fail(int code, const std::string &msg) {
  g_last_error = msg;
  return code;
}

namespace bz {
int capi_fail(int code, const std::string &msg) { return fail(code, msg); }
}  // namespace bz

template <class F>
static int guarded(F &&f) {
  try {
    return f();
  } catch (const CudaError &e) {
    return fail(BZ_ERR_CUDA, e.what());
  } catch (const std::exception &e) {
    return fail(BZ_ERR_INTERNAL, e.what());
  } catch (...) {
    return fail(BZ_ERR_INTERNAL, "unknown exception");
  }
}

extern "C" {

const char *bitz_last_error(void) { return g_last_error.c_str(); }

int bitz_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
  return n;
}

int bitz_set_device(int device) {
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return fail(BZ_ERR_CUDA, cudaGetErrorString(e));
  return BZ_OK;
}

bitz_transcript *bitz_transcript_new(const uint8_t *session, size_t slen, const uint8_t *instance,
                                     size_t ilen) {
  try {
    return new bitz_transcript{Transcript(session, slen, instance, ilen)};
  } catch (...) {
    g_last_error = "allocation failed";
    return nullptr;
  }
}

void bitz_transcript_free(bitz_transcript *t) { delete t; }

int bitz_transcript_public(bitz_transcript *t, const void *msg, size_t len) {
  if (!t || (!msg && len)) return fail(BZ_ERR_ARGUMENT, "null argument");
  t->t.public_message(msg, len);
  return BZ_OK;
}

int bitz_transcript_prover(bitz_transcript *t, const void *msg, size_t len) {
  if (!t || (!msg && len)) return fail(BZ_ERR_ARGUMENT, "null argument");
  t->t.prover_message(msg, len);
  return BZ_OK;
}

int bitz_transcript_hint(bitz_transcript *t, const void *msg, size_t len) {
  if (!t || (!msg && len)) return fail(BZ_ERR_ARGUMENT, "null argument");
  t->t.hint(msg, len);
  return BZ_OK;
}

int bitz_transcript_challenge_f128(bitz_transcript *t, uint64_t out[2]) {
  if (!t || !out) return fail(BZ_ERR_ARGUMENT, "null argument");
  f128 c = t->t.challenge_f128();
  out[0] = c.lo;
  out[1] = c.hi;
  return BZ_OK;
}

int bitz_transcript_grind(bitz_transcript *t, const char *label, uint32_t bits) {
  if (!t || !label) return fail(BZ_ERR_ARGUMENT, "null argument");
  if (bits > 32) return fail(BZ_ERR_ARGUMENT, "grinding difficulty exceeds 32 bits");
  t->t.grind(label, bits);
  return BZ_OK;
}

int bitz_transcript_prime(bitz_transcript *t, uint32_t bits, uint8_t out_le[16]) {
  if (!t || !out_le) return fail(BZ_ERR_ARGUMENT, "null argument");
  if (bits < 2 || bits > 126) return fail(BZ_ERR_ARGUMENT, "prime width out of range");
  u128 p = t->t.prime(bits);
  for (int i = 0; i < 16; i++) out_le[i] = (uint8_t)(p >> (8 * i));
  return BZ_OK;
}

size_t bitz_transcript_narg(const bitz_transcript *t, uint8_t *out, size_t cap) {
  if (!t) return 0;
  const auto &v = t->t.narg();
  if (out && cap >= v.size()) memcpy(out, v.data(), v.size());
  return v.size();
}

size_t bitz_transcript_hints(const bitz_transcript *t, uint8_t *out, size_t cap) {
  if (!t) return 0;
  const auto &v = t->t.hints();
  if (out && cap >= v.size()) memcpy(out, v.data(), v.size());
  return v.size();
}

// ------------------------------------------------------------- post-GKR

static int post_gkr_common(const f128 *rows, int log_rows, const f128 *cols, int log_cols,
                           const uint64_t target[2], const f128 *packed, uint32_t security_bits,
                           bitz_transcript *t, uint64_t *point_out, uint64_t value_out[2]) {
  Context &ctx = Context::get();
  PostGkrArgs a;
  a.rows = rows;
  a.log_rows = log_rows;
  a.cols = cols;
  a.log_cols = log_cols;
  a.packed = packed;
  a.target = mk(target[0], target[1]);
  a.grind_bits = grinding_bits(security_bits, 2);
  PostGkrScratch &sc = ctx.post_gkr_scratch((size_t)1 << (log_rows + log_cols - 1));
  f128 point[96], value;
  int rc = post_gkr_prove(a, t->t, sc, ctx.stream(), point, &value);
  if (rc == BZ_ERR_CLAIM) {
    char buf[160];
    snprintf(buf, sizeof buf, "claim does not hold: weighted sum %016llx%016llx",
             (unsigned long long)sc.claim_seen.hi, (unsigned long long)sc.claim_seen.lo);
    return fail(rc, buf);
  }
  if (rc != BZ_OK) return fail(rc, "post-GKR failed");
  for (int i = 0; i < log_rows + log_cols; i++) {
    point_out[2 * i] = point[i].lo;
    point_out[2 * i + 1] = point[i].hi;
  }
  value_out[0] = value.lo;
  value_out[1] = value.hi;
  return BZ_OK;
}

static int check_post_gkr_args(int log_rows, int log_cols, uint32_t security_bits) {
  if (log_rows < 7 || log_cols < 0 || log_rows + log_cols > 40 || log_rows + log_cols < 8)
    return fail(BZ_ERR_ARGUMENT, "unsupported post-GKR shape");
  if (security_bits != 100 && security_bits != 128)
    return fail(BZ_ERR_ARGUMENT, "security_bits must be 100 or 128");
  return BZ_OK;
}

int bitz_post_gkr_prove(const uint64_t *rows, int log_rows, const uint64_t *cols, int log_cols,
                        const uint64_t target[2], const uint64_t *packed, uint32_t security_bits,
                        bitz_transcript *t, uint64_t *point_out, uint64_t value_out[2]) {
  if (!rows || !cols || !target || !packed || !t || !point_out || !value_out)
    return fail(BZ_ERR_ARGUMENT, "null argument");
  if (int rc = check_post_gkr_args(log_rows, log_cols, security_bits)) return rc;
  return guarded([&] {
    Context &ctx = Context::get();
    size_t nr = (size_t)1 << log_rows, nc = (size_t)1 << log_cols;
    size_t np = (nr >> 7) * nc;
    DeviceBuffer<f128> d_rows(nr), d_cols(nc), d_packed(np);
    d_rows.upload((const f128 *)rows, nr, ctx.stream());
    d_cols.upload((const f128 *)cols, nc, ctx.stream());
    d_packed.upload((const f128 *)packed, np, ctx.stream());
    return post_gkr_common(d_rows.get(), log_rows, d_cols.get(), log_cols, target, d_packed.get(),
                           security_bits, t, point_out, value_out);
  });
}

int bitz_post_gkr_prove_dev(const uint64_t *rows_dev, int log_rows, const uint64_t *cols_dev,
                            int log_cols, const uint64_t target[2], const uint64_t *packed_dev,
                            uint32_t security_bits, bitz_transcript *t, uint64_t *point_out,
                            uint64_t value_out[2]) {
  if (!rows_dev || !cols_dev || !target || !packed_dev || !t || !point_out || !value_out)
    return fail(BZ_ERR_ARGUMENT, "null argument");
  if (int rc = check_post_gkr_args(log_rows, log_cols, security_bits)) return rc;
  return guarded([&] {
    return post_gkr_common((const f128 *)rows_dev, log_rows, (const f128 *)cols_dev, log_cols,
                           target, (const f128 *)packed_dev, security_bits, t, point_out,
                           value_out);
  });
}

int bitz_post_gkr_prove_noalloc(const uint64_t *rows_dev, int log_rows, const uint64_t *cols_dev,
                                int log_cols, const uint64_t target[2], const uint64_t *packed_dev,
                                uint32_t security_bits, bitz_transcript *t, void *stream,
                                uint64_t *point_out, uint64_t value_out[2]) {
  if (!rows_dev || !cols_dev || !target || !packed_dev || !t || !point_out || !value_out)
    return fail(BZ_ERR_ARGUMENT, "null argument");
  if (int rc = check_post_gkr_args(log_rows, log_cols, security_bits)) return rc;
  return guarded([&] {
    PostGkrArgs a;
    a.rows = (const f128 *)rows_dev;
    a.log_rows = log_rows;
    a.cols = (const f128 *)cols_dev;
    a.log_cols = log_cols;
    a.packed = (const f128 *)packed_dev;
    a.target = mk(target[0], target[1]);
    a.grind_bits = grinding_bits(security_bits, 2);
    f128 point[64], value;
    std::string err;
    int rc = post_gkr_prove_noalloc(a, t->t, (cudaStream_t)stream, point, &value, err);
    if (rc == BZ_ERR_CLAIM) return fail(rc, "claim does not hold");
    if (rc != BZ_OK) return fail(rc, err.empty() ? "post-GKR failed" : err);
    for (int i = 0; i < log_rows + log_cols; i++) {
      point_out[2 * i] = point[i].lo;
      point_out[2 * i + 1] = point[i].hi;
    }
    value_out[0] = value.lo;
    value_out[1] = value.hi;
    return BZ_OK;
  });
}

// ------------------------------------------------------------------ GKR

static int gkr_common(const f128 *images, const f128 *columns, int log_cols, const uint64_t *zeta,
                      uint32_t security_bits, bitz_transcript *t, uint64_t *point_out,
                      uint64_t claim_out[2]) {
  Context &ctx = Context::get();
  GkrScratch &sc = ctx.gkr_scratch(log_cols);
  sc.live_cols = 0;  // arbitrary columns: all live
  gkr_build(columns, log_cols, images, sc, ctx.stream());
  f128 z[kMaxPointGkr], pt[kMaxPointGkr];
  for (int i = 0; i < log_cols; i++) z[i] = mk(zeta[2 * i], zeta[2 * i + 1]);
  f128 claim = gkr_prove(log_cols, z, grinding_bits(security_bits, 3), t->t, sc, ctx.stream(), pt);
  for (int i = 0; i < log_cols + 7; i++) {
    point_out[2 * i] = pt[i].lo;
    point_out[2 * i + 1] = pt[i].hi;
  }
  claim_out[0] = claim.lo;
  claim_out[1] = claim.hi;
  return BZ_OK;
}

static int check_gkr_args(int log_cols, uint32_t security_bits) {
  if (log_cols < 1 || log_cols > 28) return fail(BZ_ERR_ARGUMENT, "unsupported GKR shape");
  if (security_bits != 100 && security_bits != 128)
    return fail(BZ_ERR_ARGUMENT, "security_bits must be 100 or 128");
  return BZ_OK;
}

int bitz_gkr_prove(const uint64_t *row_images, const uint64_t *columns, int log_cols,
                   const uint64_t *zeta, uint32_t security_bits, bitz_transcript *t,
                   uint64_t *point_out, uint64_t claim_out[2]) {
  if (!row_images || !columns || !zeta || !t || !point_out || !claim_out)
    return fail(BZ_ERR_ARGUMENT, "null argument");
  if (int rc = check_gkr_args(log_cols, security_bits)) return rc;
  return guarded([&] {
    Context &ctx = Context::get();
    size_t nc = (size_t)1 << log_cols;
    DeviceBuffer<f128> d_img(128), d_cols(nc);
    d_img.upload((const f128 *)row_images, 128, ctx.stream());
    d_cols.upload((const f128 *)columns, nc, ctx.stream());
    return gkr_common(d_img.get(), d_cols.get(), log_cols, zeta, security_bits, t, point_out,
                      claim_out);
  });
}

int bitz_gkr_prove_dev(const uint64_t *row_images_dev, const uint64_t *columns_dev, int log_cols,
                       const uint64_t *zeta, uint32_t security_bits, bitz_transcript *t,
                       uint64_t *point_out, uint64_t claim_out[2]) {
  if (!row_images_dev || !columns_dev || !zeta || !t || !point_out || !claim_out)
    return fail(BZ_ERR_ARGUMENT, "null argument");
  if (int rc = check_gkr_args(log_cols, security_bits)) return rc;
  return guarded([&] {
    return gkr_common((const f128 *)row_images_dev, (const f128 *)columns_dev, log_cols, zeta,
                      security_bits, t, point_out, claim_out);
  });
}

int bitz_gkr_outputs(const uint64_t *row_images, const uint64_t *columns, int log_cols,
                     uint64_t *out) {
  if (!row_images || !columns || !out) return fail(BZ_ERR_ARGUMENT, "null argument");
  if (log_cols < 1 || log_cols > 28) return fail(BZ_ERR_ARGUMENT, "unsupported GKR shape");
  return guarded([&] {
    Context &ctx = Context::get();
    size_t nc = (size_t)1 << log_cols;
    DeviceBuffer<f128> d_img(128), d_cols(nc);
    d_img.upload((const f128 *)row_images, 128, ctx.stream());
    d_cols.upload((const f128 *)columns, nc, ctx.stream());
    GkrScratch &sc = ctx.gkr_scratch(log_cols);
    sc.live_cols = 0;
    gkr_build(d_cols.get(), log_cols, d_img.get(), sc, ctx.stream());
    BZ_CUDA(cudaMemcpyAsync(out, sc.layer[7], nc * 16, cudaMemcpyDeviceToHost, ctx.stream()));
    BZ_CUDA(cudaStreamSynchronize(ctx.stream()));
    return BZ_OK;
  });
}

}  // extern "C"
