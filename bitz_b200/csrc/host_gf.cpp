// Scalar GF(2^128) helpers on the host: inversion, the additive-FFT subspace
// table, the fixed-base comb and the generator search. Every bulk use of the
// field runs on the device; these are setup-time or per-round scalars.
#include "bitz_kernels.hpp"

namespace bz {

static f128 sqn(f128 a, int k) {
  for (int i = 0; i < k; i++) a = gmul(a, a);
  return a;
}

// Itoh-Tsujii over the chain 1,2,3,6,12,24,48,96,120,126,127
// (crates/field/src/gf128/pow.rs:87-103).
f128 gf_inv_host(f128 a) {
  f128 b1 = a;
  f128 b2 = gmul(sqn(b1, 1), b1);
  f128 b3 = gmul(sqn(b2, 1), b1);
  f128 b6 = gmul(sqn(b3, 3), b3);
  f128 b12 = gmul(sqn(b6, 6), b6);
  f128 b24 = gmul(sqn(b12, 12), b12);
  f128 b48 = gmul(sqn(b24, 24), b24);
  f128 b96 = gmul(sqn(b48, 48), b48);
  f128 b120 = gmul(sqn(b96, 24), b24);
  f128 b126 = gmul(sqn(b120, 6), b6);
  f128 b127 = gmul(sqn(b126, 1), b1);
  return gmul(b127, b127);
}

// W_0(x) = x, W_{t+1}(x) = W_t(x) (W_t(x) + W_t(X^t)); carrying W_t(X^j) for
// every j gives the whole table in d^2 multiplies.
void subspace_table(int d, f128 *wh) {
  f128 w[kMaxRsDim];
  for (int j = 0; j < d; j++) w[j] = j < 64 ? mk(1ull << j, 0) : mk(0, 1ull << (j - 64));
  for (int t = 0; t < d; t++) {
    f128 inv = gf_inv_host(w[t]);
    for (int s = 0; s < kMaxRsDim; s++)
      wh[t * kMaxRsDim + s] = s < d ? (s < t ? mk(0, 0) : gmul(w[s], inv)) : mk(0, 0);
    f128 c = w[t];
    for (int j = t; j < d; j++) w[j] = gmul(w[j], gadd(w[j], c));
  }
}

void comb_table(f128 base, f128 *out) {
  f128 b = base;
  for (int i = 0; i < 16; i++) {
    f128 cur = mk(1, 0);
    for (int d = 0; d < 256; d++) {
      out[i * 256 + d] = cur;
      cur = gmul(cur, b);
    }
    b = sqn(b, 8);
  }
}

static f128 pow_host(f128 a, u128 e) {
  f128 acc = mk(1, 0);
  while (e) {
    if (e & 1) acc = gmul(acc, a);
    a = gmul(a, a);
    e >>= 1;
  }
  return acc;
}

// crates/field/src/gf128/pow.rs:110-127
f128 smallest_generator_host() {
  static const uint64_t f[9] = {3, 5, 17, 257, 641, 65537, 274177, 6700417, 67280421310721ull};
  for (uint64_t n = 2;; n++) {
    f128 a = mk(n, 0);
    bool ok = true;
    for (int i = 0; i < 9 && ok; i++) {
      f128 r = pow_host(a, (~(u128)0) / f[i]);
      if (r.lo == 1 && r.hi == 0) ok = false;
    }
    if (ok) return a;
  }
}

void eq_table_host(const f128 *r, int n, f128 *out) {
  out[0] = mk(1, 0);
  for (int i = 0; i < n; i++) {
    size_t h = (size_t)1 << i;
    for (size_t k = 0; k < h; k++) {
      f128 p = out[k];
      f128 one = gmul(p, r[i]);
      out[k] = gadd(p, one);
      out[k + h] = one;
    }
  }
}

}  // namespace bz
