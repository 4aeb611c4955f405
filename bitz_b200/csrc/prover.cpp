// End-to-end prover orchestration. Fiat-Shamir stays on the host; every bulk
// stage runs on the device, and only round messages, digests, folds and
// Ligerito openings cross back.
#include "prover.hpp"

#include <math.h>
#include <string.h>

#include <chrono>
#include <map>
#include <mutex>

#include "bitz_kernels.hpp"
#include "eq.cuh"
#include "gkr.hpp"
#include "post_gkr.hpp"
#include "status.hpp"
#include "witness.hpp"
#include "prover_internal.hpp"

namespace bz {

void matrix_digest(const CircuitSetup &S, const std::vector<int64_t> &expected_c, uint8_t out[32]);

// ------------------------------------------------------------ PCS ladder

// crates/pcs/src/profiles.rs:26-126, queries and grinding from the closed
// forms its tests check (profiles.rs:188-327).
bool pcs_config(int m, int sec, PcsConfig &cfg) {
  if (m < 20 || m > 35) return false;
  cfg = PcsConfig();
  cfg.m = m;
  cfg.security = sec;
  cfg.log_n = m - 7;
  int remaining = cfg.log_n;
  while (remaining > 5) {
    int folds = cfg.nlevels == 0 ? 4 : std::min(3, remaining - 5);
    remaining -= folds;
    PcsLevel &L = cfg.levels[cfg.nlevels];
    L.k = folds;
    L.log_inv_rate = cfg.nlevels + 1;
    L.log_msg_cols = remaining;
    cfg.nlevels++;
  }
  cfg.final_log_n = remaining;
  for (int i = 0; i < cfg.nlevels; i++) {
    PcsLevel &L = cfg.levels[i];
    double n = ldexp(1.0, L.log_msg_cols + L.log_inv_rate);
    double rho = ldexp(1.0, -L.log_inv_rate);
    if (sec == 128) {
      double delta = 1.0 - rho, gamma = delta / 2.0 - 3.0 / (delta * n);
      int g = 0;
      while ((gamma * n + 3.0 + ((i > 0 && g == 0) ? 1.0 : 0.0)) * ldexp(1.0, -128 - g) >
             ldexp(1.0, -128))
        g++;
      L.fold_grinding = g;
      int q = 1;
      while (pow(1.0 - gamma, q) > ldexp(1.0, -128)) q++;
      L.queries = q;
      L.grinding = 4;
      L.ood_samples = 0;
    } else {
      double eta = 0.02, srho = sqrt(rho), list = 1.0 / (2.0 * eta * srho);
      double gamma = 1.0 - srho - eta;
      double half = fmax(ceil(srho / (2.0 * eta)), 3.0) + 0.5;
      double base =
          (2.0 * pow(half, 5) + 3.0 * half * gamma * rho) / (3.0 * pow(rho, 1.5)) * n + half / srho;
      int g = 0;
      for (;; g++) {
        bool fits = true;
        for (int r = 0; r < L.k; r++) {
          int eff = std::max(g - r, 0);
          double beta = (i > 0 && r == 0 && eff == 0) ? 1.0 : 0.0;
          if (base * ldexp(1.0, L.k - 1 - r) + (2.0 + beta) * list > ldexp(1.0, 28 + eff)) fits = false;
        }
        if (fits) break;
      }
      L.fold_grinding = g;
      double next_list = i + 1 < cfg.nlevels ? 1.0 / (2.0 * eta * sqrt(ldexp(1.0, -(i + 2)))) : 1.0;
      int q = 1;
      for (;; q++) {
        int alpha = 0;
        while ((1 << alpha) < q) alpha++;
        if (pow(srho + eta, q) + (alpha + 1) * next_list * ldexp(1.0, -128) <= ldexp(1.0, -100)) break;
      }
      L.queries = q;
      L.grinding = 0;
      L.ood_samples = i > 0 ? 1 : 0;
    }
  }
  return true;
}

namespace {

double ms_since(std::chrono::steady_clock::time_point t) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t).count();
}

// Phase timer: with BITZ_PHASES set, each phase's host time (after a stream
// sync) is printed to stderr.
struct Phases {
  cudaStream_t s;
  bool on;
  RoundChannel *ch;
  std::chrono::steady_clock::time_point t;
  unsigned long long w0 = 0, n0 = 0;
  Phases(cudaStream_t st, RoundChannel *c)
      : s(st), on(getenv("BITZ_PHASES") != nullptr), ch(c) {
    t = std::chrono::steady_clock::now();
    if (ch) w0 = ch->wait_ns, n0 = ch->waits;
  }
  void mark(const char *name) {
    if (!on) return;
    stream_wait(s);
    double wait_ms = ch ? (ch->wait_ns - w0) * 1e-6 : 0.0;
    unsigned long long waits = ch ? ch->waits - n0 : 0;
    fprintf(stderr, "[phase] %-22s %8.3f ms  (%llu round waits, %.3f ms waiting)\n", name,
            ms_since(t), waits, wait_ms);
    t = std::chrono::steady_clock::now();
    if (ch) w0 = ch->wait_ns, n0 = ch->waits;
  }
};

// Setup cache: one device copy per (circuit, input size).
std::mutex g_setup_mu;
std::map<std::pair<int, size_t>, std::shared_ptr<DeviceSetup>> g_setups;

std::shared_ptr<DeviceSetup> device_setup(int kind, size_t n_inputs, cudaStream_t s) {
  std::lock_guard<std::mutex> lk(g_setup_mu);
  auto key = std::make_pair(kind, n_inputs);
  auto it = g_setups.find(key);
  if (it != g_setups.end()) return it->second;
  auto d = std::make_shared<DeviceSetup>();
  d->host = std::make_shared<CircuitSetup>();
  CircuitSetup &S = *d->host;
  build_circuit_setup(kind, n_inputs, S);
  d->m_off.upload(S.m_off.data(), S.m_off.size(), s);
  d->m_pos.upload(S.m_pos.data(), S.m_pos.size(), s);
  d->csc_off.upload(S.csc_off.data(), S.csc_off.size(), s);
  d->csc_row.upload(S.csc_row.data(), S.csc_row.size(), s);
  for (int k = 0; k < 3; k++) {
    d->abc_off[k].upload(S.abc[k].off.data(), S.abc[k].off.size(), s);
    d->abc_col[k].upload(S.abc[k].col.data(), std::max<size_t>(S.abc[k].col.size(), 1), s);
    d->abc_coef[k].upload(S.abc[k].coef.data(), std::max<size_t>(S.abc[k].coef.size(), 1), s);
  }
  // column-major A, B, C with a table of distinct (matrix, coefficient) pairs
  std::map<std::pair<int, int64_t>, uint16_t> tab;
  std::vector<int64_t> vals;
  std::vector<uint8_t> which;
  std::vector<uint32_t> cnt(S.h_len + 1, 0);
  for (int k = 0; k < 3; k++)
    for (uint32_t c : S.abc[k].col) cnt[c + 1]++;
  for (size_t c = 0; c < S.h_len; c++) cnt[c + 1] += cnt[c];
  size_t nnz = cnt[S.h_len];
  std::vector<uint32_t> row(std::max<size_t>(nnz, 1));
  std::vector<uint16_t> idx(std::max<size_t>(nnz, 1));
  std::vector<uint32_t> cur(cnt.begin(), cnt.end() - 1);
  for (int k = 0; k < 3; k++) {
    const Matrix &M = S.abc[k];
    for (size_t r = 0; r < S.rows; r++)
      for (uint32_t e = M.off[r]; e < M.off[r + 1]; e++) {
        auto key2 = std::make_pair(k, M.coef[e]);
        auto f = tab.find(key2);
        uint16_t id;
        if (f == tab.end()) {
          id = (uint16_t)vals.size();
          tab[key2] = id;
          vals.push_back(M.coef[e]);
          which.push_back((uint8_t)k);
        } else {
          id = f->second;
        }
        uint32_t pos = cur[M.col[e]]++;
        row[pos] = (uint32_t)r;
        idx[pos] = id;
      }
  }
  if (vals.size() > 65535) throw std::runtime_error("too many distinct coefficients");
  d->sp_off.upload(cnt.data(), cnt.size(), s);
  d->sp_row.upload(row.data(), row.size(), s);
  d->sp_idx.upload(idx.data(), idx.size(), s);
  d->tab_vals.upload(vals.data(), vals.size(), s);
  d->tab_which.upload(which.data(), which.size(), s);
  d->ntab = (int)vals.size();
  d->col0_nnz = cnt[1];
  BZ_CUDA(stream_wait(s));
  g_setups[key] = d;
  return d;
}

}  // namespace

Tables &tables(cudaStream_t s) {
  static Tables *t = nullptr;
  static std::mutex mu;
  std::lock_guard<std::mutex> lk(mu);
  if (!t) {
    t = new Tables();
    t->generator = smallest_generator_host();
    std::vector<f128> comb(16 * 256);
    comb_table(t->generator, comb.data());
    t->comb.upload(comb.data(), comb.size(), s);
    t->wh_host.resize(kMaxRsDim * kMaxRsDim);
    subspace_table(kMaxRsDim, t->wh_host.data());
    t->wh.upload(t->wh_host.data(), t->wh_host.size(), s);
    BZ_CUDA(stream_wait(s));
  }
  return *t;
}

// The lane's workspace, created on its first proof.
Workspace &workspace(Context &lane) {
  if (!lane.workspace) lane.workspace = std::make_shared<Workspace>();
  return *lane.workspace;
}

// ----------------------------------------------------------- ProofSystem

static void prepare_statement(int kind, const CircuitSetup &S, const std::vector<uint8_t> &inputs_,
                              const std::vector<uint8_t> &outputs_, std::vector<uint32_t> &states,
                              std::vector<uint32_t> &msgs, std::vector<uint32_t> &fin,
                              std::vector<uint8_t> &bitc);

ProofSystem::ProofSystem(int kind, const uint8_t *inputs, size_t n_inputs, const uint8_t *outputs,
                         int security_bits, Context *lane)
    : kind_(kind), security_(security_bits), inputs_(inputs, inputs + n_inputs),
      outputs_(outputs, outputs + 256) {
  Context &ctx = lane ? *lane : Context::get();
  cudaStream_t s = ctx.stream();
  dev_ = device_setup(kind, n_inputs, s);
  const CircuitSetup &S = *dev_->host;
  if (!pcs_config(S.committed_m, security_bits, pcs_))
    throw std::runtime_error("unsupported PCS shape");
  generator_ = tables(s).generator;
  // the statement-dependent C entries: expected value of every bit constraint
  std::vector<int64_t> ex(n_inputs + 256);
  for (size_t i = 0; i < n_inputs; i++) ex[i] = inputs[i];
  for (int i = 0; i < 256; i++) ex[n_inputs + i] = outputs[i];
  matrix_digest(S, ex, matrix_digest_);
  for (size_t i = 0; i < n_inputs; i++)
    if (inputs[i]) bit_rows_.push_back((uint32_t)i);
  for (int i = 0; i < 256; i++)
    if (outputs[i]) bit_rows_.push_back((uint32_t)(S.rows - 256 + i));
  // circuits.rs:149-160
  put_u64(public_bytes_, n_inputs);
  public_bytes_.insert(public_bytes_.end(), inputs, inputs + n_inputs);
  public_bytes_.insert(public_bytes_.end(), outputs, outputs + 256);
  // commitment.rs:214-221
  const char *v = "bitz/pcs/security/v1";
  pcs_enc_.insert(pcs_enc_.end(), v, v + strlen(v));
  put_u64(pcs_enc_, (uint64_t)1 << S.committed_m);
  for (int i = 0; i < 4; i++) pcs_enc_.push_back((uint8_t)((uint32_t)security_bits >> (8 * i)));
  prepare_statement(kind, S, inputs_, outputs_, states_h_, msgs_h_, fin_h_, bitc_h_);
  static std::atomic<uint64_t> serials{0};
  serial_ = ++serials;
  BZ_CUDA(cudaEventCreate(&ev_start_));
  BZ_CUDA(cudaEventCreate(&ev_stop_));
  BZ_CUDA(stream_wait(s));
}

uint64_t ProofSystem::footprint_bytes(int kind, size_t n_inputs) {
  // compressions and the layout's per-compression sizes (sha256.rs:45,54-60)
  uint64_t c = kind == kCompression ? 1 : kind == kChain ? n_inputs / 512 : n_inputs / 512 + 1;
  uint64_t h = 20456 * c + 2 * (uint64_t)n_inputs + 513, f = 6376 * c + n_inputs;
  int mh = std::max(20, ceil_log2(h)), mf = std::max(20, ceil_log2(f));
  // Spartan column tables and GKR layers (2^mh entries of 16 bytes, six of
  // them with the eq tables), post-GKR tables, and a fixed remainder
  return 96ull * (1ull << mh) + 64ull * (1ull << mf) + (16ull << 20);
}

ProofSystem::~ProofSystem() {
  if (ev_start_) cudaEventDestroy(ev_start_);
  if (ev_stop_) cudaEventDestroy(ev_stop_);
}

void ProofSystem::stage_statement(cudaStream_t s) {
  states_->upload(states_h_.data(), states_h_.size(), s);
  msgs_->upload(msgs_h_.data(), msgs_h_.size(), s);
  offsets_->upload(dev_->host->block_f_offset.data(), dev_->host->block_f_offset.size(), s);
  if (!fin_h_.empty()) fin_->upload(fin_h_.data(), fin_h_.size(), s);  // empty message: no inputs
  bit_c_->upload(bitc_h_.data(), bitc_h_.size(), s);
}

int ProofSystem::witness(cudaStream_t s) {
  const CircuitSetup &S = *dev_->host;
  Workspace &W = workspace(*lane_);
  W.acc.resize(512);
  size_t n_in = inputs_.size();
  size_t fwords = ((size_t)1 << S.committed_m) / 32;
  size_t hwords = ((size_t)1 << (S.claim_log_cols + 7)) / 32;
  f_->resize(fwords);
  h_->resize(hwords);
  BZ_CUDA(cudaMemsetAsync(f_->get(), 0, fwords * 4, s));
  BZ_CUDA(cudaMemsetAsync(h_->get(), 0, hwords * 4, s));
  if (n_in)
    BZ_CUDA(cudaMemcpyAsync(f_->get(), fin_->get(), fin_h_.size() * 4, cudaMemcpyDeviceToDevice, s));
  prod_->resize(3 * S.rows);
  W.flag.resize(1);
  BZ_CUDA(cudaMemsetAsync(W.flag.get(), 0, sizeof(int), s));
  WitnessArgs a;
  a.states = states_->get();
  a.msgs = msgs_->get();
  a.offsets = offsets_->get();
  a.nblocks = (int)S.n_blocks;
  a.f = f_->get();
  a.h_len = S.h_len;
  a.m_off = dev_->m_off.get();
  a.m_pos = dev_->m_pos.get();
  a.h = h_->get();
  a.rows = S.rows;
  a.n_inputs = n_in;
  for (int k = 0; k < 3; k++) {
    a.abc_off[k] = dev_->abc_off[k].get();
    a.abc_col[k] = dev_->abc_col[k].get();
    a.abc_coef[k] = dev_->abc_coef[k].get();
  }
  a.bit_c = bit_c_->get();
  a.prod = prod_->get();
  a.unsat = W.flag.get();
  witness_generate(a, s);
  int *unsat_h = reinterpret_cast<int *>(W.pin_small.get(kPinSmall) + kPinFlag);
  BZ_CUDA(cudaMemcpyAsync(unsat_h, W.flag.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
  BZ_CUDA(stream_wait(s));
  if (*unsat_h) {
    error = "circuit witness does not satisfy the constraints";
    return BZ_ERR_UNSATISFIED;
  }
  return BZ_OK;
}

// The statement's chaining values and message words for every compression
// (the chain is sequential, a few hundred nanoseconds per block on the host);
// the device expands each block's hints in parallel.
static void prepare_statement(int kind, const CircuitSetup &S, const std::vector<uint8_t> &inputs_,
                              const std::vector<uint8_t> &outputs_, std::vector<uint32_t> &states,
                              std::vector<uint32_t> &msgs, std::vector<uint32_t> &fin,
                              std::vector<uint8_t> &bitc) {
  const int kind_ = kind;
  size_t n_in = inputs_.size();
  states.assign(8 * S.n_blocks, 0);
  msgs.assign(16 * S.n_blocks, 0);
  static const uint32_t IV[8] = {0x6a09e667, 0xbb67ae85, 0x3c6ef372, 0xa54ff53a,
                                 0x510e527f, 0x9b05688c, 0x1f83d9ab, 0x5be0cd19};
  uint32_t st[8];
  for (int i = 0; i < 8; i++) st[i] = IV[i];
  if (kind_ == kCompression)
    for (int i = 0; i < 8; i++) {
      uint32_t w = 0;
      for (int j = 0; j < 32; j++) w |= (uint32_t)inputs_[512 + 32 * i + j] << j;
      st[i] = w;
    }
  size_t nmsg = (kind_ == kCompression) ? 1 : n_in / 512;
  for (size_t b = 0; b < S.n_blocks; b++) {
    uint32_t m[16];
    if (b < nmsg) {
      for (int w = 0; w < 16; w++) {
        uint32_t x = 0;
        for (int j = 0; j < 32; j++) {
          size_t bit = b * 512 + 32 * w + (kind_ <= kChain ? j : 31 - j);
          x |= (uint32_t)inputs_[bit] << j;
        }
        m[w] = x;
      }
    } else {  // the padding block of the block-aligned circuits
      memset(m, 0, sizeof m);
      m[0] = 0x80000000u;
      m[14] = (uint32_t)((uint64_t)n_in >> 32);
      m[15] = (uint32_t)n_in;
    }
    for (int i = 0; i < 8; i++) states[8 * b + i] = st[i];
    for (int i = 0; i < 16; i++) msgs[16 * b + i] = m[i];
    sha256_compress_host(st, m);
  }
  fin.assign((n_in + 31) / 32, 0);
  for (size_t i = 0; i < n_in; i++) fin[i / 32] |= (uint32_t)inputs_[i] << (i % 32);
  bitc.assign(n_in + 256, 0);
  for (size_t i = 0; i < n_in; i++) bitc[i] = inputs_[i];
  for (int i = 0; i < 256; i++) bitc[n_in + i] = outputs_[i];
}

int ProofSystem::commit(cudaStream_t s) {
  const CircuitSetup &S = *dev_->host;
  Workspace &W = workspace(*lane_);
  Tables &T = tables(s);
  const PcsLevel &L0 = pcs_.levels[0];
  int log_n = pcs_.log_n;
  size_t rows = (size_t)1 << (log_n - L0.k + L0.log_inv_rate);
  codeword0_->resize(rows << L0.k);
  nodes0_->resize(16 * rows);
  const f128 *fpk = reinterpret_cast<const f128 *>(f_->get());
  RoundChannel *lch = lane_->channel();
  rs_encode(fpk, log_n, L0.k, L0.log_inv_rate, T.wh.get(), codeword0_->get(), lch->err_dev, s);
  f128 *root_h = W.pin_small.get(kPinSmall) + kPinRoot;
  if (rows <= kMerkleBlockMaxRows &&
      merkle_build_posted(codeword0_->get(), rows, L0.k, nodes0_->get(), lch->arm(), s)) {
    // a small tree in one launch that posts its root
    lch->wait(s, reinterpret_cast<uint64_t *>(root_h), 4);
  } else {
    merkle_build(codeword0_->get(), rows, L0.k, nodes0_->get(), s);
    BZ_CUDA(cudaMemcpyAsync(root_h, nodes0_->get() + 8, 32, cudaMemcpyDeviceToHost, s));
    BZ_CUDA(stream_wait(s));
  }
  lch->check_device_error("commit");
  memcpy(root_, root_h, 32);
  const char *dom = circuit_name(kind_);
  ts_.reset(new Transcript((const uint8_t *)"bitz/circuit-e2e/v2", 19, (const uint8_t *)dom,
                           strlen(dom)));
  Transcript &t = *ts_;
  // bind_commitment (commitment.rs:172-176)
  t.public_message("bitz/pcs/commit/v1", 18);
  t.public_message(root_, 32);
  t.public_message(pcs_enc_.data(), pcs_enc_.size());
  ood_point_.clear();
  if (security_ == 100) {
    // ood::prove (ood.rs:44-52): log2(packed_len) coordinates, MLE of the packed witness
    t.public_message("bitz/pcs/ood/v1", 15);
    for (int i = 0; i < log_n; i++) ood_point_.push_back(t.challenge_f128());
    size_t n = (size_t)1 << log_n;
    W.eq_ood.resize(n);
    W.eqs.resize(eq_scratch_entries(log_n));
    eq_table_device(ood_point_.data(), log_n, W.eq_ood.get(), W.eqs.get(), s);
    W.acc.resize(512);
    BZ_CUDA(cudaMemsetAsync(W.acc.get(), 0, 16, s));
    RoundChannel *ch = lane_->channel();
    dot(W.eq_ood.get(), fpk, n, W.acc.get(), ch->arm(), s);
    ch->wait(s, W.host_acc, 2);
    ood_value_ = mk(W.host_acc[0], W.host_acc[1]);
    t.prover_f128(ood_value_);
  }
  (void)S;
  return BZ_OK;
}

// The Ligerito opening (the PCS restatement; see oracle/pcs.c for the
// construction): returns the hint bytes, empty on an internal failure.
std::vector<uint8_t> ProofSystem::ligerito(cudaStream_t s, f128 target) {
  Workspace &W = workspace(*lane_);
  Tables &T = tables(s);
  Transcript &t = *ts_;
  const PcsConfig &cfg = pcs_;
  Phases ph(s, lane_->channel());
  // challenger schedule (ligerito.rs:47-63)
  std::vector<uint32_t> sched;
  for (int i = 0; i < cfg.nlevels; i++) {
    const PcsLevel &L = cfg.levels[i];
    for (int r = 0; r < L.k; r++)
      sched.push_back(cfg.security == 128 ? (uint32_t)L.fold_grinding : (uint32_t)(L.fold_grinding - r));
    sched.push_back((uint32_t)L.grinding);
  }
  size_t at = 0;
  auto grind = [&]() {
    uint32_t bits = sched[at++];
    t.public_message("pcs/flock/pow/v1", 16);
    uint8_t b4[4];
    for (int i = 0; i < 4; i++) b4[i] = (uint8_t)(bits >> (8 * i));
    t.public_message(b4, 4);
    uint8_t seed[16];
    t.squeeze(seed, 16);
    const uint64_t nonce = pow_search(seed, bits);
    t.prover_message(&nonce, 8);
  };
  auto sample_vec = [&](size_t n) {
    t.public_message("pcs/flock/sample-vector/v1", 26);
    t.public_u64(n);
    std::vector<f128> v(n);
    for (auto &x : v) x = t.challenge_f128();
    return v;
  };
  t.public_message("flock-ligerito-basis-v0", 23);
  t.public_f128(target);
  f128 claim = target;
  std::vector<uint8_t> proof;
  size_t n = (size_t)1 << cfg.log_n;
  f128 *f = W.lf.get(), *b = W.lb.get(), *f2 = W.lf2.get(), *b2 = W.lb2.get();
  // the current level's codeword and tree
  const f128 *cw = codeword0_->get();
  const uint32_t *nodes = nodes0_->get();
  int cur_k = cfg.levels[0].k;
  size_t cur_rows = (size_t)1 << (cfg.log_n - cur_k + cfg.levels[0].log_inv_rate);
  DeviceBuffer<f128> *next_cw = W.lig_cw;
  DeviceBuffer<uint32_t> *next_nodes = W.lig_nodes;
  int flip = 0;
  unsigned long long *acc = W.acc.get();
  RoundChannel *ch = lane_->channel();
  for (int i = 0; i < cfg.nlevels; i++) {
    const PcsLevel &L = cfg.levels[i];
    std::vector<f128> rs;
    BZ_CUDA(cudaMemsetAsync(acc, 0, 8 * sizeof(unsigned long long) * (L.k + 1), s));
    // kernels that wait for the host follow the sumchecks' mode
    const bool resident = resident_rounds_enabled();
    const int pg_nb = lane_->pg_mid_blocks();
    if (resident && pg_mid_fits_folds(n, L.k, pg_nb)) {
      // the level's folds in one resident kernel: fold r takes its challenge
      // from the downbox and posts the next message itself
      RoundCtl *ctl = lane_->round_ctl();
      BZ_CUDA(cudaMemsetAsync(ctl, 0, sizeof(RoundCtl) * (L.k + 1), s));
      // no other thread's device allocation while the kernel waits for this one
      ResidentScope gate(true);
      const unsigned long long d0 = ch->down_next + 1;
      quad_sums(b, f, n, acc, ch->arm(), s);
      launch_pg_mid(b, f, n, 0, L.k, 0, 1, b2, f2, acc, ch, ch->next, d0, ctl, pg_nb, s);
      try {
        for (int r = 0; r < L.k; r++) {
          ch->wait(s, W.host_acc, 4);
          f128 a0 = mk(W.host_acc[0], W.host_acc[1]), a2 = mk(W.host_acc[2], W.host_acc[3]);
          t.prover_f128(a0);
          t.prover_f128(a2);
          grind();
          f128 c = t.challenge_f128();
          rs.push_back(c);
          claim = gadd(a0, gmul(c, gadd(gadd(claim, a2), gmul(c, a2))));
          const uint64_t cw[2] = {c.lo, c.hi};
          ch->send(cw, 2);
          if (r + 1 < L.k) ch->arm();
        }
      } catch (...) {  // release the waiting kernel before the lane is reused
        ch->abort();
        stream_wait(s);
        ch->clear_down();
        throw;
      }
      std::swap(f, f2);
      std::swap(b, b2);
      n >>= L.k;
    } else {
      quad_sums(b, f, n, acc, ch->arm(), s);
      for (int r = 0; r < L.k; r++) {
        ch->wait(s, W.host_acc, 4);
        f128 a0 = mk(W.host_acc[0], W.host_acc[1]), a2 = mk(W.host_acc[2], W.host_acc[3]);
        t.prover_f128(a0);
        t.prover_f128(a2);
        grind();
        f128 c = t.challenge_f128();
        rs.push_back(c);
        claim = gadd(a0, gmul(c, gadd(gadd(claim, a2), gmul(c, a2))));
        bool more = r + 1 < L.k;
        quad_fold(b, f, c, b2, f2, n, more, acc + 8 * (r + 1),
                  more ? ch->arm() : Publish{nullptr, nullptr, 0}, s);
        std::swap(f, f2);
        std::swap(b, b2);
        n /= 2;
      }
    }
    int l = L.log_msg_cols;
    bool last = i + 1 == cfg.nlevels;
    int nk = 0;
    size_t nrows = 0;
    if (!last) {
      const PcsLevel &N = cfg.levels[i + 1];
      nk = N.k;
      nrows = (size_t)1 << (l - N.k + N.log_inv_rate);
      next_cw[flip].resize(nrows << N.k);
      next_nodes[flip].resize(16 * nrows);
      rs_encode(f, l, N.k, N.log_inv_rate, T.wh.get(), next_cw[flip].get(), ch->err_dev, s);
      f128 *root_h = W.pin_small.get(kPinSmall) + kPinLevelRoot;
      if (nrows <= kMerkleBlockMaxRows &&
          merkle_build_posted(next_cw[flip].get(), nrows, N.k, next_nodes[flip].get(), ch->arm(),
                              s)) {
        ch->wait(s, reinterpret_cast<uint64_t *>(root_h), 4);
      } else {
        merkle_build(next_cw[flip].get(), nrows, N.k, next_nodes[flip].get(), s);
        BZ_CUDA(cudaMemcpyAsync(root_h, next_nodes[flip].get() + 8, 32, cudaMemcpyDeviceToHost,
                                s));
        BZ_CUDA(stream_wait(s));
      }
      ch->check_device_error("ligerito");
      uint8_t root[36];
      uint32_t len = 32;
      memcpy(root, &len, 4);
      memcpy(root + 4, root_h, 32);
      t.prover_message(root, 36);
      if (N.ood_samples) {
        std::vector<f128> pt = sample_vec((size_t)l);
        W.eqs.resize(eq_scratch_entries(l));
        eq_table_device(pt.data(), l, W.eq.get(), W.eqs.get(), s);
        BZ_CUDA(cudaMemsetAsync(acc, 0, 16, s));
        dot(W.eq.get(), f, n, acc, ch->arm(), s);
        ch->wait(s, W.host_acc, 2);
        f128 v = mk(W.host_acc[0], W.host_acc[1]);
        t.prover_f128(v);
        f128 mu = t.challenge_f128();
        axpy(b, mu, W.eq.get(), n, s);  // basis += mu * eq(point, .)
        claim = gadd(claim, gmul(mu, v));
      }
    } else {
      f128 *hf = W.pin_f.get(n);
      BZ_CUDA(cudaMemcpyAsync(hf, f, n * 16, cudaMemcpyDeviceToHost, s));
      BZ_CUDA(stream_wait(s));
      uint32_t cnt = (uint32_t)n;
      t.prover_message(&cnt, 4);
      t.prover_message(hf, n * 16);  // one f128 message per entry, no framing between
    }
    ph.mark("lig sumcheck+encode");
    // queries into this level's codeword: the rows and Merkle paths are
    // gathered on the device and only they cross to the host
    grind();
    std::vector<f128> qs = sample_vec((size_t)L.queries);
    int width = 1 << cur_k;
    int depth = ceil_log2(cur_rows);
    const size_t stride = (size_t)width + 2 * (size_t)depth;  // 16-byte units per query
    uint64_t *idx = W.pin_idx.get(L.queries);
    for (int q = 0; q < L.queries; q++) idx[q] = qs[q].lo & (cur_rows - 1);
    W.qidx.resize(L.queries);
    BZ_CUDA(cudaMemcpyAsync(W.qidx.get(), idx, (size_t)L.queries * 8, cudaMemcpyHostToDevice, s));
    W.openings.resize(stride * L.queries);
    gather_openings(cw, nodes, cur_rows, width, depth, W.qidx.get(), L.queries, W.openings.get(), s);
    f128 *opened = W.pin_open.get(stride * L.queries);
    BZ_CUDA(cudaMemcpyAsync(opened, W.openings.get(), stride * L.queries * 16,
                            cudaMemcpyDeviceToHost, s));
    BZ_CUDA(stream_wait(s));
    put_u64(proof, (uint64_t)L.queries);
    const uint8_t *ob = reinterpret_cast<const uint8_t *>(opened);
    proof.insert(proof.end(), ob, ob + stride * L.queries * 16);
    std::vector<f128> eqr((size_t)1 << L.k);
    eq_table_host(rs.data(), L.k, eqr.data());
    std::vector<f128> vals(L.queries);
    for (int q = 0; q < L.queries; q++) {
      const f128 *row = opened + q * stride;
      wide v = wzero();
      for (int c = 0; c < width; c++) wacc(v, gmul_wide(row[c], eqr[c]));
      vals[q] = greduce(v);
    }
    int av = ceil_log2((size_t)L.queries);
    std::vector<f128> alpha = sample_vec((size_t)av);
    f128 mu = t.challenge_f128();
    std::vector<f128> beta((size_t)1 << av);
    eq_table_host(alpha.data(), av, beta.data());
    // glue: basis += sum_q s_q X(x_q) with X_j(x) = prod_{t in j} Wh_t(x);
    // the kernel forms Wh_t(x_q) from the uploaded row indices
    f128 *sq = W.pin_qw.get(L.queries);
    for (int q = 0; q < L.queries; q++) {
      sq[q] = gmul(mu, beta[q]);
      claim = gadd(claim, gmul(sq[q], vals[q]));
    }
    W.qs.resize(L.queries);
    BZ_CUDA(cudaMemcpyAsync(W.qs.get(), sq, (size_t)L.queries * 16, cudaMemcpyHostToDevice, s));
    query_basis(W.qidx.get(), T.wh.get(), W.qs.get(), L.queries, l, b, s);
    ph.mark("lig queries+glue");
    if (!last) {
      cw = next_cw[flip].get();
      nodes = next_nodes[flip].get();
      cur_k = nk;
      cur_rows = nrows;
      flip ^= 1;
    }
  }
  // the final vector meets its basis
  f128 *hf = W.pin_f.get(n), *hb = W.pin_b.get(n);
  BZ_CUDA(cudaMemcpyAsync(hf, f, n * 16, cudaMemcpyDeviceToHost, s));
  BZ_CUDA(cudaMemcpyAsync(hb, b, n * 16, cudaMemcpyDeviceToHost, s));
  BZ_CUDA(stream_wait(s));
  f128 chk = mk(0, 0);
  for (size_t j = 0; j < n; j++) chk = gadd(chk, gmul(hb[j], hf[j]));
  if (!geq(chk, claim)) proof.clear();
  return proof;
}

int ProofSystem::prove_after_commit(cudaStream_t s, std::vector<uint8_t> &proof) {
  const CircuitSetup &S = *dev_->host;
  Workspace &W = workspace(*lane_);
  Tables &T = tables(s);
  Context &ctx = *lane_;
  Transcript &t = *ts_;
  Phases ph(s, lane_->channel());
  // bind (end_to_end.rs:442-455)
  t.public_u64(public_bytes_.size());
  t.public_message(public_bytes_.data(), public_bytes_.size());
  t.public_message(root_, 32);
  t.public_u64(7);
  t.public_u64((uint64_t)S.claim_log_cols);
  t.public_f128(generator_);
  t.public_message(pcs_enc_.data(), pcs_enc_.size());
  t.public_message(S.map_digest, 32);
  t.public_message(matrix_digest_, 32);
  t.public_message("bitz/circuit-opening-path/v1", 28);
  uint8_t path = 1;
  t.public_message(&path, 1);
  // sample_and_install_prime + project_contraints (end_to_end.rs:401-435)
  u128 q = t.prime(121);
  FpCtx fc = make_fp_ctx(q);
  std::vector<uint8_t> params;
  put_u64(params, 7);
  put_u64(params, (uint64_t)S.claim_log_cols);
  put_u128(params, q);
  const uint8_t *gb = reinterpret_cast<const uint8_t *>(&generator_);
  params.insert(params.end(), gb, gb + 16);
  t.public_message(params.data(), params.size());
  ph.mark("bind+prime");
  // Spartan
  int nr = ceil_log2(S.rows ? S.rows : 1), nc = ceil_log2(S.h_len);
  size_t R = (size_t)1 << nr, Cn = (size_t)1 << nc;
  W.sp_t.resize(8 * R);
  W.sp_d.resize(4 * Cn);
  W.sp_eqs.resize(4096 * 2 + ((size_t)1 << ((std::max(nr, nc) + 1) / 2 + 1)));
  W.sp_part.resize(3 * kSMs * 8 + 16);
  W.sp_sums.resize(4);
  W.sp_tab.resize(dev_->ntab + 1);
  if (bit_rows_.empty())
    d_bit_rows_->resize(1);
  else
    d_bit_rows_->upload(bit_rows_.data(), bit_rows_.size(), s);
  SpartanScratch sc;
  for (int i = 0; i < 8; i++) sc.t[i] = W.sp_t.get() + i * R;
  for (int i = 0; i < 4; i++) sc.d[i] = W.sp_d.get() + i * Cn;
  sc.eq_scratch = W.sp_eqs.get();
  sc.partial = W.sp_part.get();
  sc.sums = W.sp_sums.get();
  sc.tab = W.sp_tab.get();
  sc.host = W.host_fp;
  sc.channel = ctx.channel();
  sc.ctl = ctx.round_ctl();
  sc.mid_blocks = ctx.sp_mid_blocks();
  SpartanArgs sa;
  sa.ctx = fc;
  sa.q = q;
  sa.num_row_vars = nr;
  sa.num_col_vars = nc;
  sa.rows = S.rows;
  sa.cols = S.h_len;
  sa.prod = prod_->get();
  sa.hbits = h_->get();
  sa.digest = matrix_digest_;
  sa.csc_off = dev_->sp_off.get();
  sa.csc_row = dev_->sp_row.get();
  sa.csc_idx = dev_->sp_idx.get();
  sa.col0_nnz = dev_->col0_nnz;
  sa.tab_vals = dev_->tab_vals.get();
  sa.tab_which = dev_->tab_which.get();
  sa.ntab = dev_->ntab;
  sa.bit_rows = d_bit_rows_->get();
  sa.n_bit_rows = (int)bit_rows_.size();
  SpartanOut so;
  spartan_prove(sa, t, sc, s, so);
  ph.mark("spartan");
  if (!so.ok) {
    error = "Spartan closing check failed";
    return BZ_ERR_INTERNAL;
  }
  // opening_claim (end_to_end.rs:509-528)
  int sc_cols = S.claim_log_cols;
  size_t ncol = (size_t)1 << sc_cols;
  std::vector<fp> pt(7 + sc_cols, fp_zero());
  for (int i = 0; i < nc && i < 7 + sc_cols; i++) pt[i] = so.ry[i];
  std::vector<u128> rows_w(128);
  {
    std::vector<fp> e(128);
    e[0] = fc.one;
    for (int i = 0; i < 7; i++) {
      size_t h = (size_t)1 << i;
      for (size_t k = 0; k < h; k++) {
        fp p = e[k];
        fp one = fp_mul(p, pt[i], fc);
        e[k] = fp_sub(p, one, fc);
        e[k + h] = one;
      }
    }
    for (int b = 0; b < 128; b++) rows_w[b] = fp_canonical(fp_mul(e[b], so.d_at_ry, fc), fc);
  }
  // Device work that needs no further challenge is queued first, so it runs
  // while the host absorbs the claim: the column weights in canonical form,
  // the column folds and row images, and the GKR product layers.
  W.cols_fp.resize(ncol + 2);
  W.cols_canon.resize(ncol);
  fp_eq_table(pt.data() + 7, sc_cols, fc, W.cols_fp.get(), sc.eq_scratch, s);
  fp_canonical_device(W.cols_fp.get(), ncol, fc, W.cols_canon.get(), s);
  u128 *cols_h = W.host_cols.get(ncol);
  BZ_CUDA(cudaMemcpyAsync(cols_h, W.cols_canon.get(), ncol * 16, cudaMemcpyDeviceToHost, s));
  BZ_CUDA(cudaEventRecord(W.ev_cols, s));
  // send_fold (crates/prover/src/fold.rs:38-75) and the GKR build
  W.exps.upload(rows_w.data(), 128, s);
  W.folds.resize(ncol);
  const f128 *hpk = reinterpret_cast<const f128 *>(h_->get());
  fold_columns(hpk, ncol, W.exps.get(), W.folds.get(), s);
  u128 *folds_h = W.host_folds.get(ncol + 128);  // the folds, then the 128 row images
  BZ_CUDA(cudaMemcpyAsync(folds_h, W.folds.get(), ncol * 16, cudaMemcpyDeviceToHost, s));
  W.images.resize(128);
  comb_pow(T.comb.get(), W.exps.get(), 128, W.images.get(), s);
  f128 *row_images_h = reinterpret_cast<f128 *>(folds_h + ncol);
  BZ_CUDA(cudaMemcpyAsync(row_images_h, W.images.get(), 128 * 16, cudaMemcpyDeviceToHost, s));
  BZ_CUDA(cudaEventRecord(W.ev_folds, s));
  GkrScratch &gs = ctx.gkr_scratch(sc_cols);
  gs.live_cols = (S.h_len + 127) / 128;  // packed columns past h's last bit are all zero
  gkr_build(hpk, sc_cols, W.images.get(), gs, s);
  u128 target_p = fp_canonical(so.final_claim, fc);
  // prove_virtual (crates/prover/src/prove.rs:96-152)
  t.public_message("bitz/virtual-statement/v1", 25);
  t.public_message(root_, 32);
  {
    std::vector<uint8_t> vp = params;
    put_u64(vp, 7);
    put_u64(vp, (uint64_t)(S.committed_m - 7));
    t.public_message(vp.data(), vp.size());
  }
  t.public_message(S.map_digest, 32);
  {
    // one public message: 128, the row weights, ncol, the column weights,
    // the target (the sponge has no per-call framing, so it is absorbed in
    // pieces as the column weights arrive)
    std::vector<uint8_t> head;
    head.reserve(16 * 129 + 8);
    put_u64(head, 128);
    for (auto w : rows_w) put_u128(head, w);
    put_u64(head, ncol);
    t.public_message(head.data(), head.size());
    BZ_CUDA(event_wait(W.ev_cols));
    t.public_message(cols_h, ncol * 16);
    std::vector<uint8_t> tail;
    put_u128(tail, target_p);
    t.public_message(tail.data(), tail.size());
  }
  t.public_message(pcs_enc_.data(), pcs_enc_.size());
  ph.mark("claim");
  BZ_CUDA(event_wait(W.ev_folds));
  t.prover_message(folds_h, ncol * 16);
  std::vector<f128> row_images(row_images_h, row_images_h + 128);
  t.grind("bitz/columns/v1", grinding_bits((uint32_t)security_, (uint64_t)sc_cols));
  std::vector<f128> zeta(sc_cols);
  for (auto &z : zeta) z = t.challenge_f128();
  ph.mark("fold");
  // gkr_reduce (crates/prover/src/reduce.rs:17-47); the layers were built above
  std::vector<f128> gpt(sc_cols + 7);
  f128 gclaim = gkr_prove(sc_cols, zeta.data(), grinding_bits((uint32_t)security_, 3), t, gs, s,
                          gpt.data());
  f128 ip_target = gadd(gclaim, mk(1, 0));
  ph.mark("gkr");
  std::vector<f128> eqb(128), u1(128);
  eq_table_host(gpt.data() + sc_cols, 7, eqb.data());
  for (int b = 0; b < 128; b++) u1[b] = gmul(gadd(row_images[b], mk(1, 0)), eqb[b]);
  W.u1.upload(u1.data(), 128, s);
  W.u2.resize(ncol);
  W.eqs.resize(eq_scratch_entries(sc_cols));
  eq_table_device(gpt.data(), sc_cols, W.u2.get(), W.eqs.get(), s);
  // transpose_query (crates/common/src/virtual_map.rs:174-223)
  size_t nbits = (size_t)1 << S.committed_m;
  W.weights.resize(nbits);
  W.w0.resize(2);
  W.mt_dense.resize((size_t)128 << sc_cols);
  mt_transpose(dev_->csc_off.get(), dev_->csc_row.get(), S.f_bits + 1, W.u1.get(), W.u2.get(),
               W.weights.get(), nbits, W.w0.get(), s, W.mt_dense.get(), sc_cols);
  f128 *w0_h = W.pin_small.get(kPinSmall) + kPinW0;
  // the inner-product statement's weight digest (opening.rs:337-368); the
  // weight of column 0 comes back with it
  size_t nchunks = nbits * 16 / 1024;
  W.b3.resize(16 * nchunks);
  Blake3 dk = Blake3::derive_key("bitz/pcs/bit-inner-product-weights/v1");
  uint32_t left[8];
  blake3_tree_cv(reinterpret_cast<const uint8_t *>(W.weights.get()), nchunks, dk.key,
                 B3_DERIVE_KEY_MATERIAL, W.b3.get(), left, s, ctx.channel(), W.w0.get(), w0_h);
  uint8_t digest[32];
  {
    // the column weight [1] is one more 16-byte chunk; the root joins the two
    uint8_t one16[64] = {1};
    uint32_t m[16], right[8], out[8];
    b3_load_le(one16, m, 16);
    b3_compress(dk.key, m, nchunks, 16,
                B3_DERIVE_KEY_MATERIAL | B3_CHUNK_START | B3_CHUNK_END, right);
    uint32_t pm[16];
    memcpy(pm, left, 32);
    memcpy(pm + 8, right, 32);
    b3_compress(dk.key, pm, 0, 64, B3_DERIVE_KEY_MATERIAL | B3_PARENT | B3_ROOT, out);
    b3_store_le(out, digest, 8);
  }
  f128 target2 = gadd(ip_target, *w0_h);
  t.public_message("bitz/pcs/bit-inner-product/v3", 29);
  t.public_message(root_, 32);
  t.public_message(pcs_enc_.data(), pcs_enc_.size());
  t.public_u64(nbits);
  t.public_u64(1);
  t.public_message(digest, 32);
  t.public_f128(target2);
  t.public_message("bitz/pcs/inner-product-sumcheck/v2", 34);
  ph.mark("transpose+digest");
  // post-GKR sumcheck
  W.ones.resize(1);
  f128 *one_h = W.pin_small.get(kPinSmall) + kPinOne;
  *one_h = mk(1, 0);
  BZ_CUDA(cudaMemcpyAsync(W.ones.get(), one_h, 16, cudaMemcpyHostToDevice, s));
  PostGkrArgs pa;
  pa.rows = W.weights.get();
  pa.log_rows = S.committed_m;
  pa.cols = W.ones.get();
  pa.log_cols = 0;
  pa.packed = reinterpret_cast<const f128 *>(f_->get());
  pa.target = target2;
  pa.grind_bits = grinding_bits((uint32_t)security_, 2);
  PostGkrScratch &ps = ctx.post_gkr_scratch(nbits / 2);
  std::vector<f128> rho(S.committed_m);
  f128 v;
  int rc = post_gkr_prove(pa, t, ps, s, rho.data(), &v);
  if (rc) {
    error = "post-GKR claim does not hold";
    return rc;
  }
  ph.mark("post_gkr");
  // prove(Mle) with binding (opening.rs:119-135, 323-335)
  t.public_message("bitz/pcs/mle-opening/v1", 23);
  t.public_message(root_, 32);
  t.public_message(pcs_enc_.data(), pcs_enc_.size());
  t.public_u64((uint64_t)S.committed_m);
  for (auto &c : rho) t.public_f128(c);
  t.public_f128(v);
  // ring switch (mle.rs:63-123)
  int log_n = pcs_.log_n;
  size_t np = (size_t)1 << log_n;
  W.suffix.resize(np);
  W.eqs.resize(eq_scratch_entries(log_n));
  eq_table_device(rho.data() + 7, log_n, W.suffix.get(), W.eqs.get(), s);
  BZ_CUDA(cudaMemsetAsync(W.acc.get(), 0, 256 * 8, s));
  ring_claims(pa.packed, W.suffix.get(), np, W.acc.get(), s);
  f128 *claims_h = W.pin_small.get(kPinSmall) + kPinClaims;
  BZ_CUDA(cudaMemcpyAsync(claims_h, W.acc.get(), 128 * 16, cudaMemcpyDeviceToHost, s));
  BZ_CUDA(stream_wait(s));
  std::vector<f128> claims(claims_h, claims_h + 128);
  {
    std::vector<f128> pre(128);
    eq_table_host(rho.data(), 7, pre.data());
    wide chk = wzero();
    for (int b = 0; b < 128; b++) wacc(chk, gmul_wide(pre[b], claims[b]));
    if (!geq(greduce(chk), v)) {
      error = "ring-switch claims do not match the evaluation";
      return BZ_ERR_INTERNAL;
    }
  }
  t.public_message("bitz/pcs/mle-claims/v1", 22);
  t.prover_message(claims.data(), 128 * 16);
  t.grind("bitz/pcs/ring/v1",
          grinding_bits((uint32_t)security_, 7 + (security_ == 100 ? 1 : 0)));
  t.public_message("bitz/pcs/ring-switch-challenges/v1", 34);
  std::vector<f128> bpt(7);
  for (auto &c : bpt) c = t.challenge_f128();
  std::vector<f128> bw(128);
  eq_table_host(bpt.data(), 7, bw.data());
  // transpose.rs:14: out[u].bit(v) = claims[v].bit(u), and the target is
  // sum over u of out[u] bw[u] = sum over v of X^v (sum over the set bits u
  // of claims[v] of bw[u]): one XOR per set bit and one shift per claim
  f128 ptarget = mk(0, 0);
  for (int vv = 0; vv < 128; vv++) {
    f128 sv = mk(0, 0);
    for (uint64_t m = claims[vv].lo; m; m &= m - 1) sv = gadd(sv, bw[__builtin_ctzll(m)]);
    for (uint64_t m = claims[vv].hi; m; m &= m - 1) sv = gadd(sv, bw[64 + __builtin_ctzll(m)]);
    ptarget = gadd(ptarget, gmul_xk(sv, vv));
  }
  W.bw.upload(bw.data(), 128, s);
  W.lb.resize(np);
  W.lf.resize(np);
  W.lb2.resize(np);
  W.lf2.resize(np);
  W.eq.resize(np);
  f128 coef = mk(0, 0);
  if (security_ == 100) {
    t.public_message("bitz/pcs/ood-batching/v1", 24);
    coef = t.challenge_f128();
    ptarget = gadd(ptarget, gmul(coef, ood_value_));
  }
  packed_basis(W.suffix.get(), np, W.bw.get(), security_ == 100 ? W.eq_ood.get() : nullptr, coef,
               W.lb.get(), s);
  BZ_CUDA(cudaMemcpyAsync(W.lf.get(), f_->get(), np * 16, cudaMemcpyDeviceToDevice, s));
  ph.mark("ring_switch");
  std::vector<uint8_t> lproof = ligerito(s, ptarget);
  ph.mark("ligerito");
  if (lproof.empty()) {
    error = "Ligerito closing check failed";
    return BZ_ERR_INTERNAL;
  }
  uint32_t ll = (uint32_t)lproof.size();
  t.hint(&ll, 4);
  t.hint(lproof.data(), lproof.size());
  // proof bytes: root || Spartan section || wire container (wire_proof.rs:88-104)
  proof.clear();
  proof.insert(proof.end(), root_, root_ + 32);
  for (auto &x : so.outer) put_u128(proof, fp_canonical(x, fc));
  for (int k = 0; k < 3; k++) put_u128(proof, fp_canonical(so.abc[k], fc));
  for (auto &x : so.inner) put_u128(proof, fp_canonical(x, fc));
  const uint8_t magic[8] = {'b', 'i', 't', 'z', 'P', 'C', 'S', 0};
  proof.insert(proof.end(), magic, magic + 8);
  proof.push_back(1);
  proof.push_back(0);
  proof.push_back(32);
  proof.push_back(0);
  for (int i = 0; i < 4; i++) proof.push_back(0);
  put_u64(proof, t.narg().size());
  put_u64(proof, t.hints().size());
  proof.insert(proof.end(), t.narg().begin(), t.narg().end());
  proof.insert(proof.end(), t.hints().begin(), t.hints().end());
  return BZ_OK;
}

void ProofSystem::bind_lane(Context *lane) {
  lane_ = lane ? lane : &Context::get();
  Workspace &W = workspace(*lane_);
  states_ = &W.states, msgs_ = &W.msgs, fin_ = &W.fin, offsets_ = &W.offsets;
  f_ = &W.f, h_ = &W.h, prod_ = &W.prod, bit_c_ = &W.bit_c, d_bit_rows_ = &W.bit_rows;
  codeword0_ = &W.codeword0, nodes0_ = &W.nodes0;
}

int ProofSystem::split_witness(const uint8_t *inputs, size_t n_inputs, Context *lane) {
  if (split_) {
    error = "this system already holds a witness: prove or drop it first";
    return BZ_ERR_ARGUMENT;
  }
  if (n_inputs != inputs_.size()) {  // end_to_end.rs:216-218
    error = "wrong witness input length";
    return BZ_ERR_ARGUMENT;
  }
  for (size_t i = 0; i < n_inputs; i++)
    if (inputs[i] > 1) {
      error = "input bits must be 0 or 1";
      return BZ_ERR_ARGUMENT;
    }
  bind_lane(lane);
  cudaStream_t s = lane_->stream();
  // the witness is computed from these inputs; the bit constraints keep the
  // statement's expected values, so other inputs leave it unsatisfied
  std::vector<uint8_t> in(inputs, inputs + n_inputs);
  std::vector<uint32_t> states, msgs, fin;
  std::vector<uint8_t> bitc_unused;
  prepare_statement(kind_, *dev_->host, in, outputs_, states, msgs, fin, bitc_unused);
  states_->upload(states.data(), states.size(), s);
  msgs_->upload(msgs.data(), msgs.size(), s);
  offsets_->upload(dev_->host->block_f_offset.data(), dev_->host->block_f_offset.size(), s);
  if (!fin.empty()) fin_->upload(fin.data(), fin.size(), s);
  bit_c_->upload(bitc_h_.data(), bitc_h_.size(), s);
  workspace(*lane_).staged_serial = 0;  // not this statement's staging: restage next time
  BZ_CUDA(cudaEventRecord(ev_start_, s));
  int rc = witness(s);
  if (rc) return rc;
  split_ = 1;
  return BZ_OK;
}

int ProofSystem::split_commit() {
  if (split_ != 1) {
    error = split_ ? "the witness is already committed" : "no witness to commit";
    return BZ_ERR_ARGUMENT;
  }
  int rc = commit(lane_->stream());
  if (rc) return rc;
  split_ = 2;
  return BZ_OK;
}

int ProofSystem::split_prove(std::vector<uint8_t> &proof) {
  if (split_ != 2) {
    error = split_ ? "the witness is not committed" : "no committed witness to prove";
    return BZ_ERR_ARGUMENT;
  }
  split_ = 0;
  cudaStream_t s = lane_->stream();
  int rc = prove_after_commit(s, proof);
  BZ_CUDA(cudaEventRecord(ev_stop_, s));
  BZ_CUDA(event_wait(ev_stop_));
  KernelProbe::get().collect();
  return rc;
}

void ProofSystem::split_drop() {
  split_ = 0;
  ts_.reset();
}

int ProofSystem::prove(std::vector<uint8_t> &proof, StageTimes *times, bool restage,
                       Context *lane) {
  if (split_) {
    error = "this system holds a witness of the staged calls: prove or drop it first";
    return BZ_ERR_ARGUMENT;
  }
  bind_lane(lane);
  cudaStream_t s = lane_->stream();
  auto t0 = std::chrono::steady_clock::now();
  Workspace &W = workspace(*lane_);
  BZ_CUDA(cudaEventRecord(ev_start_, s));
  if (restage || W.staged_serial != serial_) {
    stage_statement(s);
    W.staged_serial = serial_;
  }
  int rc = witness(s);
  if (rc) return rc;
  double tw = ms_since(t0);
  auto t1 = std::chrono::steady_clock::now();
  rc = commit(s);
  if (rc) return rc;
  double tc = ms_since(t1);
  auto t2 = std::chrono::steady_clock::now();
  rc = prove_after_commit(s, proof);
  BZ_CUDA(cudaEventRecord(ev_stop_, s));
  BZ_CUDA(event_wait(ev_stop_));
  KernelProbe::get().collect();
  if (times) {
    times->witness_ms = tw;
    times->commit_ms = tc;
    times->prove_ms = ms_since(t2);
    float dm = 0;
    BZ_CUDA(cudaEventElapsedTime(&dm, ev_start_, ev_stop_));
    times->device_ms = dm;
  }
  return rc;
}

void ProofSystem::download_witness(std::vector<uint32_t> &f, std::vector<uint32_t> &h,
                                   std::vector<int64_t> &prod) {
  if (!lane_ || !f_) throw std::runtime_error("no proof has run on this system");
  cudaStream_t s = lane_->stream();
  // this statement's sizes (the lane's buffers may be larger)
  const CircuitSetup &S = *dev_->host;
  f.resize(((size_t)1 << S.committed_m) / 32);
  h.resize(((size_t)1 << (S.claim_log_cols + 7)) / 32);
  prod.resize(3 * S.rows);
  f_->download(f.data(), f.size(), s);
  h_->download(h.data(), h.size(), s);
  prod_->download(prod.data(), prod.size(), s);
  BZ_CUDA(stream_wait(s));
}

}  // namespace bz
