// TEST INFRASTRUCTURE ONLY -- the parity checker, never the product.
//
// CPU restatement of the reference's RNS-CKKS evaluator path (kenmaro3/ckks-train):
// RnsPoly (crates/ckks-train-core/src/poly.rs), fast/exact base conversion, rescale,
// ModUp/ModDown (crates/ckks-train-core/src/baseconv.rs), the samplers
// (crates/ckks-train-core/src/sampler.rs), CKKS parameters (crates/ckks-train-ckks/src/params.rs),
// keys (keys.rs), hybrid key switching (keyswitch.rs), the Evaluator with its checks,
// scale labels and OpCounter (evaluator.rs, counter.rs), the BSGS products (linalg.rs) and
// bootstrapping with its encoder and setup (oracle_boot.inc).
// The `parallel` feature's data parallelism (crates/ckks-train-ckks/src/par.rs) is
// restated with OpenMP at the same call sites; results are identical for any thread count.
//
// It is exported as a C API (bottom of this file) that the tests, __graft_entry__.smoke()
// and bench.py's CPU-baseline leg load with ctypes. Nothing in the product links it.

#include "oracle_core.hpp"

#include <algorithm>
#include <cmath>
#include <functional>
#include <map>
#include <omp.h>
#include <optional>
#include <set>

namespace orc {

// ---------------------------------------------------------------------------------------
// RnsPoly: crates/ckks-train-core/src/poly.rs:25-330
// ---------------------------------------------------------------------------------------

struct Poly {
  BasisPtr basis;
  std::vector<Limb> limbs;
  bool ntt = false;

  size_t level() const { return limbs.size() - 1; }
  uint64_t n() const { return basis->n; }

  static Poly zero(const BasisPtr& b, size_t level) {  // poly.rs:52-64
    Poly p;
    p.basis = b;
    p.limbs.assign(level + 1, Limb(b->n, 0));
    return p;
  }
  void add_assign(const Poly& o) {  // poly.rs:131-141
    for (size_t i = 0; i < limbs.size(); ++i) {
      const Modulus& m = basis->moduli[i];
      for (uint64_t c = 0; c < n(); ++c) limbs[i][c] = m.add(limbs[i][c], o.limbs[i][c]);
    }
  }
  void sub_assign(const Poly& o) {  // poly.rs:144-154
    for (size_t i = 0; i < limbs.size(); ++i) {
      const Modulus& m = basis->moduli[i];
      for (uint64_t c = 0; c < n(); ++c) limbs[i][c] = m.sub(limbs[i][c], o.limbs[i][c]);
    }
  }
  void neg() {  // poly.rs:157-161
    for (size_t i = 0; i < limbs.size(); ++i) {
      const Modulus& m = basis->moduli[i];
      for (auto& x : limbs[i]) x = m.sub(0, x);
    }
  }
  void mul_assign(const Poly& o) {  // poly.rs:167-182 (Barrett)
    for (size_t i = 0; i < limbs.size(); ++i) {
      const Modulus& m = basis->moduli[i];
      for (uint64_t c = 0; c < n(); ++c) limbs[i][c] = m.mul(limbs[i][c], o.limbs[i][c]);
    }
  }
  void mul_scalar_assign(uint64_t s) {  // poly.rs:185-190 (Shoup)
    for (size_t i = 0; i < limbs.size(); ++i) {
      const Modulus& m = basis->moduli[i];
      Shoup sh = m.shoup(s);
      for (auto& x : limbs[i]) x = m.mul_shoup(x, sh);
    }
  }
  void to_ntt() {  // poly.rs:193-202
    if (ntt) return;
    for (size_t i = 0; i < limbs.size(); ++i) basis->ntt[i].forward(limbs[i].data());
    ntt = true;
  }
  void to_coeff() {  // poly.rs:205-214
    if (!ntt) return;
    for (size_t i = 0; i < limbs.size(); ++i) basis->ntt[i].inverse(limbs[i].data());
    ntt = false;
  }
  void drop_last_limb() {  // poly.rs:221-224
    if (limbs.size() <= 1) throw std::logic_error("cannot drop the last limb at level 0");
    limbs.pop_back();
  }
  // poly.rs:242-296
  Poly automorphism(uint64_t g) const {
    uint64_t nn = n(), two_n = 2 * nn;
    Poly r;
    r.basis = basis;
    r.ntt = ntt;
    r.limbs.resize(limbs.size());
    if (ntt) {
      auto perm = basis->galois_permutation(g);
      for (size_t i = 0; i < limbs.size(); ++i) {
        r.limbs[i].resize(nn);
        for (uint64_t c = 0; c < nn; ++c) r.limbs[i][c] = limbs[i][(*perm)[c]];
      }
    } else {
      g %= two_n;
      for (size_t i = 0; i < limbs.size(); ++i) {
        const Modulus& m = basis->moduli[i];
        r.limbs[i].assign(nn, 0);
        uint64_t e = 0;
        for (uint64_t c = 0; c < nn; ++c) {
          if (e < nn) r.limbs[i][e] = limbs[i][c];
          else r.limbs[i][e - nn] = m.sub(0, limbs[i][c]);
          e += g;
          if (e >= two_n) e -= two_n;
        }
      }
    }
    return r;
  }
  // poly.rs:298-330: centered lift of a level-0 polynomial.
  Poly raise_from_level0(size_t level) const {
    const auto& mods = basis->moduli;
    uint64_t q0 = mods[0].q;
    Limb src = limbs[0];
    if (ntt) basis->ntt[0].inverse(src.data());
    uint64_t half = q0 / 2;
    Poly r;
    r.basis = basis;
    r.ntt = ntt;
    for (size_t i = 0; i <= level; ++i) {
      uint64_t q = mods[i].q;
      if (i == 0) { r.limbs.push_back(limbs[0]); continue; }
      Limb a(n());
      for (uint64_t c = 0; c < n(); ++c) {
        uint64_t x = src[c];
        if (x > half) {
          uint64_t rr = (q0 - x) % q;
          a[c] = rr == 0 ? 0 : q - rr;
        } else {
          a[c] = x % q;
        }
      }
      if (ntt) basis->ntt[i].forward(a.data());
      r.limbs.push_back(std::move(a));
    }
    return r;
  }
};

Poly truncated(const Poly& p, size_t level) {  // keys.rs:141-157
  if (level > p.level()) throw std::logic_error("cannot truncate upwards");
  Poly r = p;
  r.limbs.resize(level + 1);
  return r;
}

// ---------------------------------------------------------------------------------------
// Base conversion: crates/ckks-train-core/src/baseconv.rs:77-235
// ---------------------------------------------------------------------------------------

struct BaseConverter {
  std::vector<Modulus> from, to;
  std::vector<uint64_t> q_hat_inv;                 // (Q/q_j)^{-1} mod q_j
  std::vector<std::vector<uint64_t>> q_hat_mod_p;  // [t][j] = (Q/q_j) mod p_t

  BaseConverter(const std::vector<uint64_t>& f, const std::vector<uint64_t>& t) {  // :96-134
    for (uint64_t q : f) from.emplace_back(q);
    for (uint64_t q : t) to.emplace_back(q);
    auto q_hat_mod = [&](size_t j, const Modulus& m) {
      uint64_t acc = 1 % m.q;
      for (size_t i = 0; i < from.size(); ++i)
        if (i != j) acc = m.mul(acc, from[i].q % m.q);
      return acc;
    };
    for (size_t j = 0; j < from.size(); ++j) q_hat_inv.push_back(from[j].inv_or_throw(q_hat_mod(j, from[j])));
    for (auto& p : to) {
      std::vector<uint64_t> row;
      for (size_t j = 0; j < from.size(); ++j) row.push_back(q_hat_mod(j, p));
      q_hat_mod_p.push_back(row);
    }
  }

  // :183-235. With `exact` and >= 2 sources, e = floor(sum_j f64(y_j) * (1/q_j)) is
  // evaluated with separate round-to-nearest products and sums in source order.
  std::vector<Limb> convert(const std::vector<Limb>& input, bool exact) const {
    size_t n = input[0].size();
    std::vector<Limb> y(from.size(), Limb(n));
    for (size_t j = 0; j < from.size(); ++j) {
      Shoup s = from[j].shoup(q_hat_inv[j]);
      for (size_t c = 0; c < n; ++c) y[j][c] = from[j].mul_shoup(input[j][c], s);
    }
    std::vector<uint64_t> e;
    bool use_e = exact && from.size() > 1;
    if (use_e) {
      std::vector<double> inv(from.size());
      for (size_t j = 0; j < from.size(); ++j) inv[j] = 1.0 / (double)from[j].q;
      e.resize(n);
      for (size_t c = 0; c < n; ++c) {
        volatile double f = -0.0;
        for (size_t j = 0; j < from.size(); ++j) {
          volatile double prod = (double)y[j][c] * inv[j];
          f = f + prod;
        }
        e[c] = (uint64_t)std::floor((double)f);
      }
    }
    std::vector<Limb> out(to.size(), Limb(n, 0));
    for (size_t t = 0; t < to.size(); ++t) {
      const Modulus& p = to[t];
      for (size_t j = 0; j < from.size(); ++j) {
        Shoup s = p.shoup(q_hat_mod_p[t][j]);
        for (size_t c = 0; c < n; ++c) out[t][c] = p.add(out[t][c], p.mul_shoup(y[j][c], s));
      }
      if (use_e) {
        uint64_t qm = 1 % p.q;
        for (auto& m : from) qm = p.mul(qm, m.q % p.q);
        Shoup s = p.shoup(qm);
        for (size_t c = 0; c < n; ++c) out[t][c] = p.sub(out[t][c], p.mul_shoup(e[c], s));
      }
    }
    return out;
  }
};

// baseconv.rs:239-245: (D - 1)/2 mod m for D the product of `factors`.
uint64_t half_mod(const std::vector<Modulus>& factors, const Modulus& m) {
  uint64_t d = 1 % m.q;
  for (auto& f : factors) d = m.mul(d, f.q % m.q);
  return m.mul(m.sub(d, 1 % m.q), (m.q + 1) / 2);
}

// baseconv.rs:258-291
void rescale_by_last(Poly& x) {
  size_t l = x.level();
  if (l < 1) throw std::logic_error("cannot rescale at level 0");
  auto basis = x.basis;
  const Modulus& q_last = basis->moduli[l];
  uint64_t half = q_last.q >> 1;
  Limb last = x.limbs[l];
  if (x.ntt) basis->ntt[l].inverse(last.data());
  for (auto& v : last) v = q_last.add(v, half);
  x.drop_last_limb();
  for (size_t i = 0; i < x.limbs.size(); ++i) {
    const Modulus& m = basis->moduli[i];
    Shoup one = m.shoup(1);
    uint64_t half_i = m.mul_shoup(half, one);
    Limb t(x.n());
    for (size_t c = 0; c < t.size(); ++c) t[c] = m.sub(m.mul_shoup(last[c], one), half_i);
    if (x.ntt) basis->ntt[i].forward(t.data());
    Shoup inv = m.shoup(m.inv_or_throw(q_last.q % m.q));
    for (size_t c = 0; c < t.size(); ++c) x.limbs[i][c] = m.mul_shoup(m.sub(x.limbs[i][c], t[c]), inv);
  }
}

// baseconv.rs:459-511: (q_part, p_part) representing X over Q_l * P divided by P with rounding.
void mod_down(Poly& self, const Poly& special) {
  bool ntt = self.ntt;
  auto basis = self.basis;
  size_t l = self.level();
  auto sp = special.basis;
  std::vector<Modulus> qs(basis->moduli.begin(), basis->moduli.begin() + l + 1);
  std::vector<Modulus> ps(sp->moduli.begin(), sp->moduli.begin() + special.level() + 1);
  std::vector<Limb> src = special.limbs;
  for (size_t t = 0; t < src.size(); ++t) {
    if (ntt) sp->ntt[t].inverse(src[t].data());
    uint64_t h = ps[t].q >> 1;
    for (auto& v : src[t]) v = ps[t].add(v, h);
  }
  std::vector<uint64_t> from, to;
  for (auto& p : ps) from.push_back(p.q);
  for (auto& q : qs) to.push_back(q.q);
  auto converted = BaseConverter(from, to).convert(src, true);
  for (size_t i = 0; i <= l; ++i) {
    const Modulus& m = qs[i];
    uint64_t p_mod = 1 % m.q;
    for (auto& p : ps) p_mod = m.mul(p_mod, p.q % m.q);
    uint64_t p_inv = m.inv_or_throw(p_mod);
    uint64_t half = half_mod(ps, m);
    Limb& t = converted[i];
    for (auto& v : t) v = m.sub(v, half);
    if (ntt) basis->ntt[i].forward(t.data());
    Shoup s = m.shoup(p_inv);
    for (size_t c = 0; c < t.size(); ++c) self.limbs[i][c] = m.mul_shoup(m.sub(self.limbs[i][c], t[c]), s);
  }
}

// ---------------------------------------------------------------------------------------
// CKKS parameters: crates/ckks-train-ckks/src/params.rs:87-157, 181-184, 203-209
// ---------------------------------------------------------------------------------------

struct Params {
  uint32_t log_n = 0;
  std::vector<uint64_t> q, p;
  std::vector<uint32_t> q_bits, p_bits;
  double scale = 0;
  size_t dnum = 0;
  std::optional<size_t> hamming_weight;
  BasisPtr bq, bp;

  uint64_t n() const { return 1ULL << log_n; }
  size_t slots() const { return n() / 2; }
  size_t max_level() const { return q.size() - 1; }
  size_t alpha() const { return q.size() / dnum; }
  double log_pq() const {
    double s = 0;
    for (auto v : q) s += std::log2((double)v);
    for (auto v : p) s += std::log2((double)v);
    return s;
  }
  double scale_at(size_t level) const {  // params.rs:282-289
    if (level > max_level()) throw HeError(INVALID_PARAMS, "level above max_level");
    return level == 0 ? scale : std::exp2((double)q_bits[level]);
  }
};
typedef std::shared_ptr<const Params> ParamsPtr;

// params.rs:87-157: SEAL-style prime generation and hand-out.
ParamsPtr params_from_bits(uint32_t log_n, const std::vector<uint32_t>& q_bits,
                           const std::vector<uint32_t>& p_bits, uint32_t scale_bits, size_t dnum) {
  if (log_n < 1 || log_n > 17) throw HeError(INVALID_PARAMS, "log_n outside [1, 17]");
  if (q_bits.empty() || p_bits.empty()) throw HeError(INVALID_PARAMS, "q_bits and p_bits must be non-empty");
  for (auto b : q_bits) if (b < 2 || b > 60) throw HeError(INVALID_PARAMS, "prime bit size outside 2..=60");
  for (auto b : p_bits) if (b < 2 || b > 60) throw HeError(INVALID_PARAMS, "prime bit size outside 2..=60");
  if (scale_bits < 1 || scale_bits > 60) throw HeError(INVALID_PARAMS, "scale_bits outside 1..=60");
  if (dnum == 0 || q_bits.size() % dnum != 0) throw HeError(INVALID_PARAMS, "dnum must divide the number of q primes");
  uint64_t n = 1ULL << log_n;
  std::vector<uint32_t> all(q_bits);
  all.insert(all.end(), p_bits.begin(), p_bits.end());
  std::vector<uint32_t> distinct(all);
  std::sort(distinct.begin(), distinct.end());
  distinct.erase(std::unique(distinct.begin(), distinct.end()), distinct.end());
  std::map<uint32_t, std::vector<uint64_t>> pools;
  std::map<uint32_t, size_t> next;
  for (auto b : distinct) {
    size_t count = std::count(all.begin(), all.end(), b);
    pools[b] = ntt_primes_skip(b, n, 0, count);
    next[b] = 0;
  }
  std::vector<uint64_t> primes;
  for (auto b : all) {
    auto& pool = pools[b];
    primes.push_back(pool[pool.size() - 1 - next[b]]);
    next[b]++;
  }
  auto P = std::make_shared<Params>();
  P->log_n = log_n;
  P->q.assign(primes.begin(), primes.begin() + q_bits.size());
  P->p.assign(primes.begin() + q_bits.size(), primes.end());
  P->q_bits = q_bits;
  P->p_bits = p_bits;
  P->scale = std::exp2((double)scale_bits);
  P->dnum = dnum;
  P->bq = std::make_shared<RnsBasis>(n, P->q);
  P->bp = std::make_shared<RnsBasis>(n, P->p);
  return P;
}

ParamsPtr params_from_primes(uint32_t log_n, const std::vector<uint64_t>& q, const std::vector<uint64_t>& p,
                             double scale, size_t dnum) {
  if (q.empty() || p.empty()) throw HeError(INVALID_PARAMS, "q and p must be non-empty");
  if (dnum == 0 || q.size() % dnum != 0) throw HeError(INVALID_PARAMS, "dnum must divide the number of q primes");
  auto P = std::make_shared<Params>();
  P->log_n = log_n;
  P->q = q;
  P->p = p;
  for (auto v : q) P->q_bits.push_back(64 - __builtin_clzll(v));
  for (auto v : p) P->p_bits.push_back(64 - __builtin_clzll(v));
  P->scale = scale;
  P->dnum = dnum;
  uint64_t n = 1ULL << log_n;
  std::vector<uint64_t> all(q);
  all.insert(all.end(), p.begin(), p.end());
  RnsBasis check(n, all);  // duplicate / NTT-friendliness checks across Q and P
  P->bq = std::make_shared<RnsBasis>(n, q);
  P->bp = std::make_shared<RnsBasis>(n, p);
  return P;
}

// ---------------------------------------------------------------------------------------
// Samplers: crates/ckks-train-core/src/sampler.rs:31-247
// ---------------------------------------------------------------------------------------

struct Rng {
  ChaCha20 cc;
  explicit Rng(const uint8_t seed[32]) : cc(seed) {}
  uint64_t next_u64() { return cc.next_u64(); }
  uint64_t below(uint64_t bound) {  // :82-91
    uint64_t zone = (UINT64_MAX / bound) * bound;
    for (;;) {
      uint64_t x = next_u64();
      if (x < zone) return x % bound;
    }
  }
  Poly uniform_poly(const BasisPtr& b, size_t level) {  // :98-110
    Poly p;
    p.basis = b;
    for (size_t i = 0; i <= level; ++i) {
      uint64_t q = b->moduli[i].q;
      Limb l(b->n);
      for (auto& v : l) v = below(q);
      p.limbs.push_back(std::move(l));
    }
    return p;
  }
  Poly ternary_poly(const BasisPtr& b, size_t level, std::optional<size_t> hw) {  // :123-150
    uint64_t n = b->n;
    std::vector<int64_t> coeffs(n, 0);
    if (hw) {
      std::vector<size_t> idx(n);
      for (size_t i = 0; i < n; ++i) idx[i] = i;
      for (size_t k = 0; k < *hw; ++k) {
        size_t j = k + (size_t)below(n - k);
        std::swap(idx[k], idx[j]);
        coeffs[idx[k]] = (next_u64() & 1) == 0 ? 1 : -1;
      }
    } else {
      for (auto& c : coeffs) {
        uint64_t r = next_u64() & 3;
        c = r == 0 ? -1 : (r == 1 ? 1 : 0);
      }
    }
    return signed_to_poly(b, level, coeffs);
  }
  Poly gaussian_poly(const BasisPtr& b, size_t level, double sigma) {  // :176-200
    auto cdt = cdt_table(sigma);
    int64_t bound = (int64_t)(cdt.size() / 2);
    size_t last = cdt.size() - 1;
    std::vector<int64_t> coeffs(b->n);
    for (auto& c : coeffs) {
      uint64_t r = next_u64();
      size_t k = std::upper_bound(cdt.begin(), cdt.end(), r) - cdt.begin();  // partition_point(c <= r)
      c = (int64_t)std::min(k, last) - bound;
    }
    return signed_to_poly(b, level, coeffs);
  }
  static std::vector<uint64_t> cdt_table(double sigma) {  // :209-226
    int64_t bound = (int64_t)std::floor(6.0 * sigma);
    double denom = 2.0 * sigma * sigma;
    std::vector<double> w;
    for (int64_t x = -bound; x <= bound; ++x) w.push_back(std::exp(-((double)x) * (double)x / denom));
    double total = -0.0;
    for (double v : w) total += v;
    double acc = 0.0;
    std::vector<uint64_t> cdt;
    for (double v : w) {
      acc += v;
      double f = acc / total * 18446744073709551616.0;
      cdt.push_back(f >= 18446744073709551616.0 ? UINT64_MAX : (uint64_t)f);
    }
    cdt.back() = UINT64_MAX;
    return cdt;
  }
  static Poly signed_to_poly(const BasisPtr& b, size_t level, const std::vector<int64_t>& coeffs) {  // :229-247
    Poly p;
    p.basis = b;
    for (size_t i = 0; i <= level; ++i) {
      uint64_t q = b->moduli[i].q;
      Limb l(b->n);
      for (size_t c = 0; c < coeffs.size(); ++c)
        l[c] = coeffs[c] >= 0 ? (uint64_t)coeffs[c] : q - (uint64_t)(-coeffs[c]);
      p.limbs.push_back(std::move(l));
    }
    return p;
  }
};

// ---------------------------------------------------------------------------------------
// Keys: crates/ckks-train-ckks/src/keys.rs
// ---------------------------------------------------------------------------------------

const double ERROR_STD_DEV = 3.2;  // keys.rs:85
const uint64_t GALOIS_GENERATOR = 3;  // encoder.rs:73

uint64_t galois_elt(uint64_t n, int32_t step) {  // keys.rs:89-103
  uint64_t m = 2 * n;
  int64_t slots = (int64_t)std::max<uint64_t>(n / 2, 1);
  int64_t kk = ((int64_t)step % slots + slots) % slots;
  uint64_t k = (uint64_t)kk, base = GALOIS_GENERATOR % m, acc = 1 % m;
  while (k > 0) {
    if (k & 1) acc = acc * base % m;
    base = base * base % m;
    k >>= 1;
  }
  return acc;
}
uint64_t conjugation_elt(uint64_t n) { return 2 * n - 1; }  // keys.rs:106-108

struct QpPoly {  // keys.rs:112-146
  Poly q, p;
};

struct KskKey {  // keys.rs:229-245
  std::vector<std::pair<QpPoly, QpPoly>> parts;
};

// keys.rs:685-705: centered coefficients of limb 0 copied into every limb of `target`.
Poly lift_small(const Poly& src, const BasisPtr& target) {
  uint64_t q0 = src.basis->moduli[0].q;
  Poly r;
  r.basis = target;
  for (auto& m : target->moduli) {
    uint64_t t = m.q;
    Limb l(src.n());
    for (size_t c = 0; c < l.size(); ++c) {
      uint64_t x = src.limbs[0][c];
      if (x > q0 / 2) {
        uint64_t rr = (q0 - x) % t;
        l[c] = rr == 0 ? 0 : t - rr;
      } else {
        l[c] = x % t;
      }
    }
    r.limbs.push_back(std::move(l));
  }
  return r;
}

QpPoly small_qp(const BasisPtr& bp, Poly q) {  // keys.rs:676-681
  Poly p = lift_small(q, bp);
  q.to_ntt();
  p.to_ntt();
  return QpPoly{q, p};
}

// keys.rs:483-511
std::pair<QpPoly, QpPoly> rlwe_sample_under(Rng& rng, const Params& P, const QpPoly& target, size_t level) {
  Poly aq = rng.uniform_poly(P.bq, level);
  Poly ap = rng.uniform_poly(P.bp, P.bp->len() - 1);
  aq.to_ntt();
  ap.to_ntt();
  QpPoly e = small_qp(P.bp, rng.gaussian_poly(P.bq, level, ERROR_STD_DEV));
  Poly tq = level == target.q.level() ? target.q : truncated(target.q, level);
  auto mk = [](const Poly& a, const Poly& s, const Poly& e) {
    Poly b = a;
    b.mul_assign(s);
    b.neg();
    b.add_assign(e);
    return b;
  };
  Poly bq = mk(aq, tq, e.q), bpp = mk(ap, target.p, e.p);
  return {QpPoly{bq, bpp}, QpPoly{aq, ap}};
}

// keys.rs:520-559
KskKey ksk_under(Rng& rng, const Params& P, const QpPoly& target, const Poly& s_prime, size_t level) {
  size_t n = P.n(), alpha = P.alpha();
  size_t parts_count = level / alpha + 1;
  KskKey key;
  for (size_t j = 0; j < parts_count; ++j) {
    auto ba = rlwe_sample_under(rng, P, target, level);
    Poly gadget;
    gadget.basis = P.bq;
    gadget.ntt = true;
    for (size_t i = 0; i <= level; ++i) {
      const Modulus& m = P.bq->moduli[i];
      if (i >= j * alpha && i < (j + 1) * alpha) {
        uint64_t q = m.q, p_mod = 1 % q;
        for (auto pv : P.p) p_mod = m.mul(p_mod, pv % q);
        Shoup s = m.shoup(p_mod);
        Limb l(n);
        for (size_t c = 0; c < n; ++c) l[c] = m.mul_shoup(s_prime.limbs[i][c], s);
        gadget.limbs.push_back(std::move(l));
      } else {
        gadget.limbs.push_back(Limb(n, 0));
      }
    }
    ba.first.q.add_assign(gadget);
    key.parts.push_back(ba);
  }
  return key;
}

struct KeyGenerator {  // keys.rs:341-467
  ParamsPtr P;
  QpPoly sk;
  Rng rng;
  KeyGenerator(ParamsPtr params, const uint8_t seed[32]) : P(params), rng(seed) {
    uint64_t n = P->n();
    if (P->hamming_weight && (*P->hamming_weight == 0 || *P->hamming_weight > n))
      throw HeError(INVALID_PARAMS, "secret-key Hamming weight must be in 1..=N");
    Poly s = rng.ternary_poly(P->bq, P->max_level(), P->hamming_weight);
    sk = small_qp(P->bp, s);
  }
  std::pair<QpPoly, QpPoly> public_key() { return rlwe_sample_under(rng, *P, sk, P->max_level()); }
  KskKey relin_key() {
    Poly s2 = sk.q;
    s2.mul_assign(sk.q);
    return ksk_under(rng, *P, sk, s2, P->max_level());
  }
  KskKey galois_key(uint64_t elt) {
    uint64_t two_n = 2 * P->n();
    if (elt % 2 == 0 || elt >= two_n) throw HeError(INVALID_PARAMS, "Galois element must be odd and < 2N");
    Poly sp = sk.q.automorphism(elt);
    return ksk_under(rng, *P, sk, sp, P->max_level());
  }
};

// ---------------------------------------------------------------------------------------
// Hybrid key switching: crates/ckks-train-ckks/src/keyswitch.rs:68-319
// ---------------------------------------------------------------------------------------

struct Range { size_t start, end; };

std::vector<Range> digit_ranges(const Params& P, size_t level) {  // :68-74
  std::vector<Range> out;
  size_t alpha = P.alpha();
  for (size_t j = 0; j < P.dnum; ++j) {
    Range r{j * alpha, std::min((j + 1) * alpha, level + 1)};
    if (r.start > level) break;
    out.push_back(r);
  }
  return out;
}

// :140-202: the exact centered lift of one digit to Q_l * P.
QpPoly lift_digit_exact(const Poly& poly, Range digit, const BasisPtr& basis_p) {
  size_t l = poly.level();
  auto basis = poly.basis;
  std::vector<Modulus> digit_moduli(basis->moduli.begin() + digit.start, basis->moduli.begin() + digit.end);
  std::vector<Limb> src;
  for (size_t i = digit.start; i < digit.end; ++i) {
    Limb a = poly.limbs[i];
    basis->ntt[i].inverse(a.data());
    const Modulus& m = basis->moduli[i];
    uint64_t h = m.q >> 1;
    for (auto& v : a) v = m.add(v, h);
    src.push_back(std::move(a));
  }
  std::vector<size_t> others;
  for (size_t i = 0; i <= l; ++i)
    if (i < digit.start || i >= digit.end) others.push_back(i);
  std::vector<std::pair<const Modulus*, const NttTable*>> targets;
  for (size_t i : others) targets.push_back({&basis->moduli[i], &basis->ntt[i]});
  for (size_t t = 0; t < basis_p->len(); ++t) targets.push_back({&basis_p->moduli[t], &basis_p->ntt[t]});
  std::vector<Limb> out;
  if (digit.end - digit.start == 1) {
    const Limb& y = src[0];
    for (auto& tg : targets) {
      const Modulus& m = *tg.first;
      Shoup one = m.shoup(1);
      uint64_t h = half_mod(digit_moduli, m);
      Limb a(y.size());
      for (size_t c = 0; c < a.size(); ++c) a[c] = m.sub(m.mul_shoup(y[c], one), h);
      tg.second->forward(a.data());
      out.push_back(std::move(a));
    }
  } else {
    std::vector<uint64_t> from, to;
    for (auto& m : digit_moduli) from.push_back(m.q);
    for (auto& tg : targets) to.push_back(tg.first->q);
    out = BaseConverter(from, to).convert(src, true);
    for (size_t t = 0; t < targets.size(); ++t) {
      const Modulus& m = *targets[t].first;
      uint64_t h = half_mod(digit_moduli, m);
      for (auto& v : out[t]) v = m.sub(v, h);
      targets[t].second->forward(out[t].data());
    }
  }
  QpPoly r;
  r.q.basis = basis;
  r.q.ntt = true;
  size_t k = 0;
  for (size_t i = 0; i <= l; ++i) {
    if (i >= digit.start && i < digit.end) r.q.limbs.push_back(poly.limbs[i]);
    else r.q.limbs.push_back(out[k++]);
  }
  r.p.basis = basis_p;
  r.p.ntt = true;
  for (; k < out.size(); ++k) r.p.limbs.push_back(out[k]);
  return r;
}

// :82-119 (parallel over digits with the `parallel` feature).
std::vector<QpPoly> decompose(const Params& P, const Poly& poly) {
  if (!poly.ntt) throw std::logic_error("key switching needs NTT form");
  auto ranges = digit_ranges(P, poly.level());
  std::vector<QpPoly> out(ranges.size());
#pragma omp parallel for schedule(dynamic, 1)
  for (size_t j = 0; j < ranges.size(); ++j) out[j] = lift_digit_exact(poly, ranges[j], P.bp);
  return out;
}

// :230-309: u128 inner product per limb, reduced once, then two mod_downs.
std::pair<Poly, Poly> apply_key(const Params& P, const std::vector<QpPoly>& digits, const KskKey& key) {
  size_t l = digits[0].q.level();
  if (digits.size() != digit_ranges(P, l).size()) throw std::logic_error("digit count mismatch");
  if (digits.size() > key.parts.size()) throw std::logic_error("more digits than key parts");
  size_t n = P.n();
  auto inner = [&](const BasisPtr& basis, size_t limbs, bool qpart, Poly& ob, Poly& oa) {
    ob = Poly();
    oa = Poly();
    ob.basis = oa.basis = basis;
    ob.ntt = oa.ntt = true;
    ob.limbs.assign(limbs, Limb());
    oa.limbs.assign(limbs, Limb());
#pragma omp parallel for schedule(dynamic, 1)
    for (size_t i = 0; i < limbs; ++i) {
      const Modulus& m = basis->moduli[i];
      std::vector<u128> acc_b(n, 0), acc_a(n, 0);
      for (size_t j = 0; j < digits.size(); ++j) {
        const Limb& dl = qpart ? digits[j].q.limbs[i] : digits[j].p.limbs[i];
        const Limb& bl = qpart ? key.parts[j].first.q.limbs[i] : key.parts[j].first.p.limbs[i];
        const Limb& al = qpart ? key.parts[j].second.q.limbs[i] : key.parts[j].second.p.limbs[i];
        for (size_t c = 0; c < n; ++c) {
          acc_b[c] += (u128)dl[c] * bl[c];
          acc_a[c] += (u128)dl[c] * al[c];
        }
      }
      Shoup two64 = m.shoup((uint64_t)(((u128)1 << 64) % m.q));
      Shoup one = m.shoup(1);
      Limb rb(n), ra(n);
      for (size_t c = 0; c < n; ++c) {
        rb[c] = m.add(m.mul_shoup((uint64_t)(acc_b[c] >> 64), two64), m.mul_shoup((uint64_t)acc_b[c], one));
        ra[c] = m.add(m.mul_shoup((uint64_t)(acc_a[c] >> 64), two64), m.mul_shoup((uint64_t)acc_a[c], one));
      }
      ob.limbs[i] = std::move(rb);
      oa.limbs[i] = std::move(ra);
    }
  };
  Poly bq, aq, bp, ap;
  inner(P.bq, l + 1, true, bq, aq);
  inner(P.bp, P.bp->len(), false, bp, ap);
  mod_down(bq, bp);
  mod_down(aq, ap);
  return {bq, aq};
}

std::pair<Poly, Poly> key_switch(const Params& P, const Poly& poly, const KskKey& key) {  // :317-319
  return apply_key(P, decompose(P, poly), key);
}

// ---------------------------------------------------------------------------------------
// Evaluator: crates/ckks-train-ckks/src/evaluator.rs, counter.rs, ops.rs (EvalConfig)
// ---------------------------------------------------------------------------------------

struct OpCounter {  // counter.rs:42-58
  uint64_t rotations = 0, relins = 0, ct_ct_tensor = 0, ct_pt_mults = 0, rescales = 0, sse_switches = 0,
           bootstraps = 0;
};

struct EvalConfig {  // ops.rs:111-178
  bool hoist = true, bsgs = true, lazy_relin = true;
};

struct Ciphertext {  // ciphertext.rs:17-60
  std::vector<Poly> c;
  double scale = 0;
  size_t level = 0;
  size_t len() const { return c.size(); }
};

struct Plaintext {
  Poly poly;
  double scale = 0;
  size_t level() const { return poly.level(); }
};

Ciphertext ct_new(std::vector<Poly> c, double scale) {  // ciphertext.rs:36-60
  if (c.size() < 2) throw HeError(INVALID_PARAMS, "a ciphertext needs at least 2 components");
  for (auto& p : c)
    if (!p.ntt) throw HeError(INVALID_PARAMS, "ciphertext components must be in NTT form");
  for (auto& p : c)
    if (p.basis != c[0].basis) throw HeError(INVALID_PARAMS, "ciphertext components over different bases");
  size_t level = c[0].level();
  for (auto& p : c)
    if (p.level() != level) throw HeError(LEVEL_MISMATCH, "level mismatch");
  if (!(std::isfinite(scale) && scale > 0.0))
    throw HeError(INVALID_PARAMS, "ciphertext scale must be positive and finite");
  Ciphertext ct;
  ct.c = std::move(c);
  ct.scale = scale;
  ct.level = level;
  return ct;
}

const double SCALE_TOLERANCE = 1.0 / 1024.0;           // evaluator.rs:96
const uint64_t LABEL_SEARCH_ULPS = 8;                   // evaluator.rs:100
const double MAX_SCALAR_INT = 4611686018427387904.0;   // evaluator.rs:103
const double MIN_PLAIN_SCALE = 1048576.0;               // evaluator.rs:108

void check_level(size_t a, size_t b) {
  if (a != b) throw HeError(LEVEL_MISMATCH, "level mismatch");
}
void check_scale(double a, double b) {  // evaluator.rs:833-839
  if (!(std::fabs(a - b) < SCALE_TOLERANCE * std::min(a, b))) throw HeError(SCALE_MISMATCH, "scale mismatch");
}
void check_plain_scale(double sp) {  // evaluator.rs:111-119
  if (sp < MIN_PLAIN_SCALE) throw HeError(INVALID_PARAMS, "plaintext scale is below 2^20");
}

double exact_product_scale(const Params& P, size_t level, double target) {  // evaluator.rs:739-773
  if (level > P.max_level()) throw HeError(INVALID_PARAMS, "level exceeds max_level");
  if (!(std::isfinite(target) && target > 0.0)) throw HeError(INVALID_PARAMS, "target scale must be positive and finite");
  if (level == 0) throw HeError(NO_LEVELS_LEFT, "no levels left");
  double q = (double)P.q[level];
  double l0 = target * q;
  if (!std::isfinite(l0)) throw HeError(INVALID_PARAMS, "target scale times q overflows");
  uint64_t bits;
  memcpy(&bits, &l0, 8);
  for (uint64_t k = 0; k <= LABEL_SEARCH_ULPS; ++k) {
    for (int s = 0; s < 2; ++s) {
      uint64_t b = s == 0 ? bits + k : bits - k;
      double l;
      memcpy(&l, &b, 8);
      if (l / q == target) return l;
    }
  }
  throw HeError(SCALE_MISMATCH, "scale mismatch");
}

struct Evaluator {
  ParamsPtr P;
  std::shared_ptr<KskKey> relin;
  std::shared_ptr<std::map<uint64_t, std::shared_ptr<KskKey>>> galois;
  EvalConfig config;
  std::mutex mu;
  OpCounter counter;

  template <class F>
  void count(F f) {
    std::lock_guard<std::mutex> lk(mu);
    f(counter);
  }

  void check_basis(const std::vector<Poly>& polys) const {
    for (auto& p : polys)
      if (p.basis != P->bq) throw HeError(INVALID_PARAMS, "operand is not over this evaluator's data basis");
  }
  void check_key_basis(const KskKey& key) const {  // evaluator.rs:680-696
    bool ok = key.parts.size() == P->dnum;
    for (auto& pr : key.parts)
      ok = ok && pr.first.q.basis == P->bq && pr.first.p.basis == P->bp && pr.second.q.basis == P->bq &&
           pr.second.p.basis == P->bp;
    if (!ok) throw HeError(INVALID_PARAMS, "key is not over this evaluator's bases");
  }
  const KskKey& relin_key_checked() const {
    if (!relin) throw HeError(INVALID_PARAMS, "evaluator has no relinearization key");
    check_key_basis(*relin);
    return *relin;
  }
  void check_mul_operands(const Ciphertext& a, const Ciphertext& b) const {  // evaluator.rs:479-496
    check_basis(a.c);
    check_basis(b.c);
    if (a.len() != 2 || b.len() != 2) throw HeError(INVALID_PARAMS, "multiplication needs 2-component ciphertexts");
    check_level(a.level, b.level);
    if (a.level == 0) throw HeError(NO_LEVELS_LEFT, "no levels left");
  }

  Ciphertext add_sub(const Ciphertext& a, const Ciphertext& b, bool sub) const {  // evaluator.rs:699-723
    check_basis(a.c);
    check_basis(b.c);
    check_level(a.level, b.level);
    check_scale(a.scale, b.scale);
    std::vector<Poly> c = a.c;
    for (size_t i = 0; i < b.c.size(); ++i) {
      if (i < c.size()) {
        if (sub) c[i].sub_assign(b.c[i]); else c[i].add_assign(b.c[i]);
      } else {
        Poly q = b.c[i];
        if (sub) q.neg();
        c.push_back(q);
      }
    }
    return ct_new(c, a.scale);
  }
  Ciphertext add(const Ciphertext& a, const Ciphertext& b) const { return add_sub(a, b, false); }
  Ciphertext sub(const Ciphertext& a, const Ciphertext& b) const { return add_sub(a, b, true); }
  Ciphertext negate(const Ciphertext& a) const {
    check_basis(a.c);
    std::vector<Poly> c = a.c;
    for (auto& p : c) p.neg();
    return ct_new(c, a.scale);
  }
  Ciphertext add_plain(const Ciphertext& a, const Plaintext& p) const {
    check_basis(a.c);
    check_basis({p.poly});
    check_level(a.level, p.level());
    check_scale(a.scale, p.scale);
    std::vector<Poly> c = a.c;
    c[0].add_assign(p.poly);
    return ct_new(c, a.scale);
  }
  Ciphertext mul_plain(const Ciphertext& a, const Plaintext& p) {
    check_basis(a.c);
    check_basis({p.poly});
    check_level(a.level, p.level());
    std::vector<Poly> c = a.c;
    for (auto& x : c) x.mul_assign(p.poly);
    Ciphertext r = ct_new(c, a.scale * p.scale);
    count([](OpCounter& k) { k.ct_pt_mults++; });
    return r;
  }
  Ciphertext mul_scalar(const Ciphertext& ct, double value, double target) {  // evaluator.rs:361-376, 777-799
    check_basis(ct.c);
    if (!std::isfinite(value)) throw HeError(INVALID_PARAMS, "scalar must be finite");
    double label = exact_product_scale(*P, ct.level, target);
    check_plain_scale(label / ct.scale);
    double k = std::round(value * (label / ct.scale));
    if (std::fabs(k) >= MAX_SCALAR_INT) throw HeError(INVALID_PARAMS, "scalar integer >= 2^62");
    std::vector<Poly> c = ct.c;
    for (auto& p : c) {
      p.mul_scalar_assign((uint64_t)std::fabs(k));
      if (k < 0.0) p.neg();
    }
    Ciphertext r = ct_new(c, label);
    count([](OpCounter& x) { x.ct_pt_mults++; });
    return r;
  }
  Ciphertext mul_plain_to_scale(const Ciphertext& a, const Plaintext& p, double target) {  // evaluator.rs:393-414
    check_basis(a.c);
    check_basis({p.poly});
    check_level(a.level, p.level());
    double label = exact_product_scale(*P, a.level, target);
    check_plain_scale(label / a.scale);
    if (p.scale != label / a.scale) throw HeError(SCALE_MISMATCH, "scale mismatch");
    std::vector<Poly> c = a.c;
    for (auto& x : c) x.mul_assign(p.poly);
    Ciphertext r = ct_new(c, label);
    count([](OpCounter& x) { x.ct_pt_mults++; });
    return r;
  }
  Ciphertext mul_no_relin(const Ciphertext& a, const Ciphertext& b) {  // evaluator.rs:422-439
    check_mul_operands(a, b);
    auto prod = [](const Poly& p, const Poly& q) {
      Poly r = p;
      r.mul_assign(q);
      return r;
    };
    Poly d0 = prod(a.c[0], b.c[0]);
    Poly d1 = prod(a.c[0], b.c[1]);
    d1.add_assign(prod(a.c[1], b.c[0]));
    Poly d2 = prod(a.c[1], b.c[1]);
    Ciphertext r = ct_new({d0, d1, d2}, a.scale * b.scale);
    count([](OpCounter& x) { x.ct_ct_tensor++; });
    return r;
  }
  Ciphertext relinearize(const Ciphertext& ct) {  // evaluator.rs:441-460
    check_basis(ct.c);
    if (ct.len() != 3) throw HeError(INVALID_PARAMS, "relinearize needs a 3-component ciphertext");
    const KskKey& rk = relin_key_checked();
    std::vector<Poly> c = ct.c;
    Poly c2 = c.back();
    c.pop_back();
    auto kbka = key_switch(*P, c2, rk);
    c[0].add_assign(kbka.first);
    c[1].add_assign(kbka.second);
    Ciphertext r = ct_new(c, ct.scale);
    count([](OpCounter& x) { x.relins++; });
    return r;
  }
  Ciphertext mul(const Ciphertext& a, const Ciphertext& b) {  // evaluator.rs:463-467
    check_mul_operands(a, b);
    relin_key_checked();
    return relinearize(mul_no_relin(a, b));
  }
  Ciphertext rescale(const Ciphertext& ct) {  // evaluator.rs:498-510
    check_basis(ct.c);
    size_t l = ct.level;
    if (l == 0) throw HeError(NO_LEVELS_LEFT, "no levels left");
    std::vector<Poly> c = ct.c;
    for (auto& p : c) rescale_by_last(p);
    Ciphertext r = ct_new(c, ct.scale / (double)P->q[l]);
    count([](OpCounter& x) { x.rescales++; });
    return r;
  }
  Ciphertext mod_switch_to_level(const Ciphertext& ct, size_t level) const {  // evaluator.rs:513-525
    check_basis(ct.c);
    if (level > ct.level) throw HeError(INVALID_PARAMS, "cannot switch a ciphertext up a level");
    std::vector<Poly> c;
    for (auto& p : ct.c) c.push_back(truncated(p, level));
    return ct_new(c, ct.scale);
  }
  Ciphertext relabel(const Ciphertext& ct, double scale) const { return ct_new(ct.c, scale); }  // ops.rs:475-477

  // Rotations: evaluator.rs:534-676
  void check_galois_input(const Ciphertext& ct) const {
    check_basis(ct.c);
    if (ct.len() != 2) throw HeError(INVALID_PARAMS, "rotation needs a 2-component ciphertext");
  }
  std::optional<uint64_t> rotation_elt(int32_t steps) const {
    int64_t slots = (int64_t)P->slots();
    int64_t k = (((int64_t)steps % slots) + slots) % slots;
    if (k == 0) return std::nullopt;
    return galois_elt(P->n(), (int32_t)k);
  }
  const KskKey& galois_key(uint64_t elt) const {
    uint64_t two_n = 2 * P->n();
    if (elt % 2 == 0 || elt >= two_n) throw HeError(INVALID_PARAMS, "Galois element must be odd and < 2N");
    if (!galois) throw HeError(INVALID_PARAMS, "missing galois key");
    auto it = galois->find(elt);
    if (it == galois->end()) throw HeError(INVALID_PARAMS, "missing galois key");
    check_key_basis(*it->second);
    return *it->second;
  }
  void check_rotation_keys(const std::vector<int32_t>& steps) const {
    for (auto s : steps) {
      auto e = rotation_elt(s);
      if (e) galois_key(*e);
    }
  }
  static Ciphertext finish_galois(const Ciphertext& ct, uint64_t elt, const Poly& kb, const Poly& ka) {
    Poly r0 = ct.c[0].automorphism(elt);
    r0.add_assign(kb);
    return ct_new({r0, ka}, ct.scale);
  }
  Ciphertext apply_galois(const Ciphertext& ct, uint64_t elt) {
    const KskKey& gk = galois_key(elt);
    Poly d = ct.c[1].automorphism(elt);
    auto kbka = key_switch(*P, d, gk);
    Ciphertext r = finish_galois(ct, elt, kbka.first, kbka.second);
    count([](OpCounter& x) { x.rotations++; });
    return r;
  }
  Ciphertext rotate(const Ciphertext& ct, int32_t steps) {
    check_galois_input(ct);
    auto e = rotation_elt(steps);
    if (!e) return ct;
    return apply_galois(ct, *e);
  }
  Ciphertext conjugate(const Ciphertext& ct) {
    check_galois_input(ct);
    return apply_galois(ct, conjugation_elt(P->n()));
  }
  std::vector<Ciphertext> hoisted_rotate(const Ciphertext& ct, const std::vector<int32_t>& steps) {  // :572-616
    check_galois_input(ct);
    std::vector<Ciphertext> out(steps.size());
    if (!config.hoist) {
      check_rotation_keys(steps);
#pragma omp parallel for schedule(dynamic, 1)
      for (size_t i = 0; i < steps.size(); ++i) out[i] = rotate(ct, steps[i]);
      return out;
    }
    std::vector<std::pair<uint64_t, const KskKey*>> keys(steps.size(), {0, nullptr});
    bool any = false;
    for (size_t i = 0; i < steps.size(); ++i) {
      auto e = rotation_elt(steps[i]);
      if (e) {
        keys[i] = {*e, &galois_key(*e)};
        any = true;
      }
    }
    std::vector<QpPoly> digits;
    if (any) digits = decompose(*P, ct.c[1]);
    uint64_t nontrivial = 0;
    for (auto& k : keys) nontrivial += k.second != nullptr;
#pragma omp parallel for schedule(dynamic, 1)
    for (size_t i = 0; i < steps.size(); ++i) {
      if (!keys[i].second) {
        out[i] = ct;
        continue;
      }
      uint64_t elt = keys[i].first;
      std::vector<QpPoly> rotated;
      for (auto& d : digits) rotated.push_back(QpPoly{d.q.automorphism(elt), d.p.automorphism(elt)});
      auto kbka = apply_key(*P, rotated, *keys[i].second);
      out[i] = finish_galois(ct, elt, kbka.first, kbka.second);
    }
    count([&](OpCounter& x) { x.rotations += nontrivial; });
    return out;
  }
};

// ---------------------------------------------------------------------------------------
// BSGS: crates/ckks-train-ckks/src/linalg.rs:419-497, 608-680, 801-893
// ---------------------------------------------------------------------------------------

std::pair<size_t, size_t> bsgs_split(size_t d) {  // :419-424
  if (d == 0 || (d & (d - 1))) throw std::logic_error("d must be a power of two");
  uint32_t log_d = __builtin_ctzll(d);
  size_t baby = (size_t)1 << ((log_d + 1) / 2);
  return {baby, d / baby};
}

std::vector<int32_t> bsgs_rotation_steps(size_t d, size_t stride, int64_t offset) {  // :433-497
  auto bg = bsgs_split(d);
  std::vector<int32_t> out;
  for (size_t k2 = 1; k2 < bg.first; ++k2) out.push_back((int32_t)(k2 * stride));
  for (size_t k1 = 0; k1 < bg.second; ++k1) {
    int64_t g = (offset + (int64_t)(bg.first * k1)) * (int64_t)stride;
    if (g != 0) out.push_back((int32_t)g);
  }
  return out;
}

template <class T>
struct Diagonals {
  size_t d = 0, baby = 0, giant = 0, stride = 1;
  int64_t offset = 0;
  std::vector<T> entries;
};

void check_stride(size_t d, size_t stride, size_t slots) {  // :528-536
  if (stride == 0 || slots % (d * stride) != 0)
    throw HeError(INVALID_PARAMS, "d * stride must divide the slot count");
}

template <class T>
void check_entries_lv(const std::vector<T>& e, size_t (*lv)(const T&), double (*sc)(const T&)) {  // :548-560
  if (e.empty()) return;
  for (auto& x : e)
    if (lv(x) != lv(e[0])) throw HeError(LEVEL_MISMATCH, "level mismatch");
  for (auto& x : e)
    if (sc(x) != sc(e[0])) throw HeError(SCALE_MISMATCH, "scale mismatch");
}

inline size_t pt_level(const Plaintext& p) { return p.level(); }
inline double pt_scale(const Plaintext& p) { return p.scale; }
inline size_t ct_level(const Ciphertext& c) { return c.level; }
inline double ct_scale(const Ciphertext& c) { return c.scale; }

// :801-893, one term (matvec_plain / matvec_enc), no skipped entries.
template <class T, class MulF, class FinF>
Ciphertext bsgs_one(Evaluator& ev, const Diagonals<T>& diag, const Ciphertext& x, bool share_giant, MulF mul,
                    FinF finish) {
  size_t baby = diag.baby, giant = diag.giant, stride = diag.stride;
  int64_t offset = diag.offset;
  std::vector<int32_t> steps;
  for (size_t k2 = 0; k2 < baby; ++k2) steps.push_back((int32_t)(k2 * stride));
  std::vector<Ciphertext> xs = ev.hoisted_rotate(x, steps);
  std::vector<std::optional<Ciphertext>> blocks(giant);
  std::vector<std::string> errs(giant);
  std::vector<int> ekind(giant, 0);
#pragma omp parallel for schedule(dynamic, 1)
  for (size_t k1 = 0; k1 < giant; ++k1) {
    try {
      int64_t shift = (offset + (int64_t)(baby * k1)) * (int64_t)stride;
      std::optional<Ciphertext> sum;
      if (!share_giant && shift != 0) {
        for (size_t k2 = 0; k2 < baby; ++k2) {
          Ciphertext t = finish(mul(diag.entries[k1 * baby + k2], xs[k2]));
          t = ev.rotate(t, (int32_t)shift);
          sum = sum ? ev.add(*sum, t) : t;
        }
        blocks[k1] = sum;
        continue;
      }
      for (size_t k2 = 0; k2 < baby; ++k2) {
        Ciphertext t = mul(diag.entries[k1 * baby + k2], xs[k2]);
        sum = sum ? ev.add(*sum, t) : t;
      }
      Ciphertext b = finish(*sum);
      if (shift != 0) b = ev.rotate(b, (int32_t)shift);
      blocks[k1] = b;
    } catch (const HeError& e) {
      errs[k1] = e.what();
      ekind[k1] = e.kind;
    }
  }
  for (size_t k1 = 0; k1 < giant; ++k1)
    if (ekind[k1]) throw HeError((ErrKind)ekind[k1], errs[k1]);
  std::optional<Ciphertext> acc;
  for (auto& b : blocks) {
    if (!b) continue;
    acc = acc ? ev.add(*acc, *b) : *b;
  }
  return *acc;
}

template <class T>
void check_bsgs(Evaluator& ev, const Diagonals<T>& diag, const Ciphertext& x, size_t (*lv)(const T&),
                double (*sc)(const T&)) {  // :680-689
  check_entries_lv(diag.entries, lv, sc);
  for (auto& e : diag.entries)
    if (lv(e) != x.level) throw HeError(LEVEL_MISMATCH, "level mismatch");
  check_stride(diag.d, diag.stride, ev.P->slots());
  ev.check_rotation_keys(bsgs_rotation_steps(diag.d, diag.stride, diag.offset));
}

Ciphertext matvec_plain(Evaluator& ev, const Diagonals<Plaintext>& diag, const Ciphertext& x) {  // :608-622
  ev.check_galois_input(x);
  for (auto& p : diag.entries) ev.check_basis({p.poly});
  check_bsgs<Plaintext>(ev, diag, x, pt_level, pt_scale);
  return bsgs_one(
      ev, diag, x, ev.config.bsgs, [&](const Plaintext& w, const Ciphertext& xr) { return ev.mul_plain(xr, w); },
      [](Ciphertext c) { return c; });
}

Ciphertext matvec_enc(Evaluator& ev, const Diagonals<Ciphertext>& diag, const Ciphertext& x) {  // :642-678
  ev.check_galois_input(x);
  for (auto& c : diag.entries) ev.check_galois_input(c);
  check_bsgs<Ciphertext>(ev, diag, x, ct_level, ct_scale);
  if (x.level == 0) throw HeError(NO_LEVELS_LEFT, "no levels left");
  ev.relin_key_checked();
  if (ev.config.lazy_relin)
    return bsgs_one(
        ev, diag, x, ev.config.bsgs, [&](const Ciphertext& w, const Ciphertext& xr) { return ev.mul_no_relin(w, xr); },
        [&](Ciphertext c) { return ev.relinearize(c); });
  return bsgs_one(
      ev, diag, x, ev.config.bsgs, [&](const Ciphertext& w, const Ciphertext& xr) { return ev.mul(w, xr); },
      [](Ciphertext c) { return c; });
}

#include "oracle_boot.inc"

}  // namespace orc

// =======================================================================================
// C API (ctypes). Buffers are flat little-endian u64 arrays, limb-major: limb i occupies
// [i*N, (i+1)*N). A ciphertext buffer holds its components one after another.
// Functions return 0 on success or an ErrKind; orc_last_error() gives the message.
// =======================================================================================

using namespace orc;

static thread_local std::string g_err;

#define ORC_TRY(...)                               \
  try {                                            \
    __VA_ARGS__;                                   \
    return 0;                                      \
  } catch (const HeError& e) {                     \
    g_err = e.what();                              \
    return (int)e.kind;                            \
  } catch (const std::exception& e) {              \
    g_err = std::string("oracle panic: ") + e.what(); \
    return 100;                                    \
  }

struct OrcParams { ParamsPtr P; };
struct OrcKey { std::shared_ptr<KskKey> k; };
struct OrcKeyGen { std::unique_ptr<KeyGenerator> kg; };
struct OrcEval { std::unique_ptr<Evaluator> ev; };
struct OrcCt { Ciphertext ct; };

static Poly poly_from(const BasisPtr& b, const uint64_t* data, size_t nlimbs, bool ntt) {
  Poly p;
  p.basis = b;
  p.ntt = ntt;
  for (size_t i = 0; i < nlimbs; ++i) p.limbs.emplace_back(data + i * b->n, data + (i + 1) * b->n);
  return p;
}
static void poly_to(const Poly& p, uint64_t* out) {
  for (size_t i = 0; i < p.limbs.size(); ++i) memcpy(out + i * p.n(), p.limbs[i].data(), p.n() * 8);
}

extern "C" {

const char* orc_last_error() { return g_err.c_str(); }
void orc_set_threads(int t) { omp_set_num_threads(t > 0 ? t : 1); }
int orc_get_threads() { return omp_get_max_threads(); }

// --- scalar helpers (pins) ---
int orc_is_prime(uint64_t n) { return is_prime_u64(n) ? 1 : 0; }
int orc_ntt_primes_skip(uint32_t bits, uint64_t n, uint64_t skip, uint64_t count, uint64_t* out) {
  ORC_TRY({
    auto v = ntt_primes_skip(bits, n, skip, count);
    for (size_t i = 0; i < v.size(); ++i) out[i] = v[i];
  })
}
int orc_min_root(uint64_t n, uint64_t q, uint64_t* out) {
  ORC_TRY({ *out = NttTable(n, Modulus(q)).psi; })
}
int orc_barrett(uint64_t q, uint64_t* lo, uint64_t* hi) {
  ORC_TRY({
    Modulus m(q);
    *lo = (uint64_t)m.ratio;
    *hi = (uint64_t)(m.ratio >> 64);
  })
}
uint64_t orc_mulmod(uint64_t q, uint64_t a, uint64_t b) { return Modulus(q).mul(a, b); }
uint64_t orc_mul_shoup(uint64_t q, uint64_t a, uint64_t w) { Modulus m(q); return m.mul_shoup(a, m.shoup(w)); }
uint64_t orc_galois_elt(uint64_t n, int32_t step) { return galois_elt(n, step); }
void orc_galois_perm(uint64_t n, uint64_t g, uint32_t* out) {
  auto v = galois_permutation_ntt(n, g);
  memcpy(out, v.data(), n * 4);
}
void orc_chacha_words(const uint8_t* seed, uint64_t count, uint64_t* out) {
  ChaCha20 c(seed);
  for (uint64_t i = 0; i < count; ++i) out[i] = c.next_u64();
}
void orc_seed_from_u64(uint64_t s, uint8_t* out) { seed_from_u64(s, out); }
void orc_bsgs_split(uint64_t d, uint64_t* baby, uint64_t* giant) {
  auto bg = bsgs_split(d);
  *baby = bg.first;
  *giant = bg.second;
}
int orc_bsgs_steps(uint64_t d, uint64_t stride, int64_t offset, int32_t* out) {
  auto v = bsgs_rotation_steps(d, stride, offset);
  for (size_t i = 0; i < v.size(); ++i) out[i] = v[i];
  return (int)v.size();
}
void orc_cdt_table(double sigma, uint64_t* out, uint64_t* len) {
  auto v = Rng::cdt_table(sigma);
  if (out) memcpy(out, v.data(), v.size() * 8);
  *len = v.size();
}

// --- params ---
int orc_params_from_bits(uint32_t log_n, const uint32_t* qb, uint64_t nq, const uint32_t* pb, uint64_t np,
                         uint32_t scale_bits, uint64_t dnum, OrcParams** out) {
  ORC_TRY({
    *out = new OrcParams{params_from_bits(log_n, std::vector<uint32_t>(qb, qb + nq),
                                          std::vector<uint32_t>(pb, pb + np), scale_bits, dnum)};
  })
}
int orc_params_from_primes(uint32_t log_n, const uint64_t* q, uint64_t nq, const uint64_t* p, uint64_t np,
                           double scale, uint64_t dnum, OrcParams** out) {
  ORC_TRY({
    *out = new OrcParams{params_from_primes(log_n, std::vector<uint64_t>(q, q + nq),
                                            std::vector<uint64_t>(p, p + np), scale, dnum)};
  })
}
void orc_params_free(OrcParams* p) { delete p; }
void orc_params_primes(const OrcParams* p, uint64_t* q, uint64_t* pp) {
  memcpy(q, p->P->q.data(), p->P->q.size() * 8);
  memcpy(pp, p->P->p.data(), p->P->p.size() * 8);
}
double orc_params_log_pq(const OrcParams* p) { return p->P->log_pq(); }
double orc_params_scale_at(const OrcParams* p, uint64_t level) { return p->P->scale_at(level); }
int orc_digit_ranges(const OrcParams* p, uint64_t level, uint64_t* out) {
  auto r = digit_ranges(*p->P, level);
  for (size_t i = 0; i < r.size(); ++i) {
    out[2 * i] = r[i].start;
    out[2 * i + 1] = r[i].end;
  }
  return (int)r.size();
}

// --- polynomial primitives (basis 0 = Q, 1 = P) ---
static BasisPtr pick(const OrcParams* p, int basis) { return basis == 0 ? p->P->bq : p->P->bp; }

int orc_ntt(const OrcParams* p, int basis, uint64_t first_prime, uint64_t nlimbs, uint64_t* data, int inverse) {
  ORC_TRY({
    auto b = pick(p, basis);
    for (uint64_t i = 0; i < nlimbs; ++i) {
      if (inverse) b->ntt[first_prime + i].inverse(data + i * b->n);
      else b->ntt[first_prime + i].forward(data + i * b->n);
    }
  })
}
// op: 0 add, 1 sub, 2 mul (Barrett), 3 neg, 4 mul_scalar (Shoup)
int orc_poly_op(const OrcParams* p, int basis, uint64_t nlimbs, int op, uint64_t* a, const uint64_t* b,
                uint64_t scalar) {
  ORC_TRY({
    auto bs = pick(p, basis);
    Poly x = poly_from(bs, a, nlimbs, true);
    if (op <= 2) {
      Poly y = poly_from(bs, b, nlimbs, true);
      if (op == 0) x.add_assign(y);
      if (op == 1) x.sub_assign(y);
      if (op == 2) x.mul_assign(y);
    } else if (op == 3) {
      x.neg();
    } else {
      x.mul_scalar_assign(scalar);
    }
    poly_to(x, a);
  })
}
int orc_automorphism(const OrcParams* p, int basis, uint64_t nlimbs, const uint64_t* in, uint64_t g, int ntt,
                     uint64_t* out) {
  ORC_TRY({ poly_to(poly_from(pick(p, basis), in, nlimbs, ntt).automorphism(g), out); })
}
// rescale of a level-`level` polynomial (level+1 limbs): writes `level` limbs.
int orc_rescale(const OrcParams* p, const uint64_t* in, uint64_t level, int ntt, uint64_t* out) {
  ORC_TRY({
    Poly x = poly_from(p->P->bq, in, level + 1, ntt);
    rescale_by_last(x);
    poly_to(x, out);
  })
}
// exact centered lift of digit `digit` of a level-`level` NTT-form polynomial.
int orc_mod_up(const OrcParams* p, const uint64_t* in, uint64_t level, uint64_t digit, uint64_t* out_q,
               uint64_t* out_p) {
  ORC_TRY({
    Poly x = poly_from(p->P->bq, in, level + 1, true);
    auto r = digit_ranges(*p->P, level);
    if (digit >= r.size()) throw HeError(INVALID_PARAMS, "digit out of range");
    QpPoly d = lift_digit_exact(x, r[digit], p->P->bp);
    poly_to(d.q, out_q);
    poly_to(d.p, out_p);
  })
}
int orc_mod_down(const OrcParams* p, const uint64_t* q, uint64_t level, const uint64_t* pp, int ntt,
                 uint64_t* out) {
  ORC_TRY({
    Poly x = poly_from(p->P->bq, q, level + 1, ntt);
    Poly y = poly_from(p->P->bp, pp, p->P->p.size(), ntt);
    mod_down(x, y);
    poly_to(x, out);
  })
}
int orc_raise_from_level0(const OrcParams* p, const uint64_t* in, uint64_t level, int ntt, uint64_t* out) {
  ORC_TRY({ poly_to(poly_from(p->P->bq, in, 1, ntt).raise_from_level0(level), out); })
}
// uniform residues from ChaCha20Rng::seed_from_u64(seed), next_u64() % q (the reference
// GPU tests' random_poly, crates/ckks-train-cuda/tests/cases/mod.rs:59-66).
void orc_random_poly(uint64_t seed, const uint64_t* primes, uint64_t nlimbs, uint64_t n, uint64_t* out) {
  uint8_t s[32];
  seed_from_u64(seed, s);
  ChaCha20 c(s);
  for (uint64_t i = 0; i < nlimbs; ++i)
    for (uint64_t k = 0; k < n; ++k) out[i * n + k] = c.next_u64() % primes[i];
}

// --- keys ---
int orc_keygen_new(const OrcParams* p, const uint8_t* seed, OrcKeyGen** out) {
  ORC_TRY({ *out = new OrcKeyGen{std::make_unique<KeyGenerator>(p->P, seed)}; })
}
void orc_keygen_free(OrcKeyGen* k) { delete k; }
// secret key: Q part (L+1 limbs) then P part (k limbs), NTT form.
void orc_keygen_secret(const OrcKeyGen* k, uint64_t* out) {
  poly_to(k->kg->sk.q, out);
  poly_to(k->kg->sk.p, out + k->kg->sk.q.limbs.size() * k->kg->P->n());
}
int orc_keygen_relin(OrcKeyGen* k, OrcKey** out) {
  ORC_TRY({ *out = new OrcKey{std::make_shared<KskKey>(k->kg->relin_key())}; })
}
int orc_keygen_galois(OrcKeyGen* k, uint64_t elt, OrcKey** out) {
  ORC_TRY({ *out = new OrcKey{std::make_shared<KskKey>(k->kg->galois_key(elt))}; })
}
void orc_key_free(OrcKey* k) { delete k; }
uint64_t orc_key_parts(const OrcKey* k) { return k->k->parts.size(); }
uint64_t orc_key_qlimbs(const OrcKey* k) { return k->k->parts[0].first.q.limbs.size(); }
// layout: for each part j: b.q, b.p, a.q, a.p (limb-major) -- the reference's device layout.
void orc_key_export(const OrcKey* k, uint64_t* out) {
  size_t off = 0, n = k->k->parts[0].first.q.n();
  for (auto& pr : k->k->parts) {
    for (const Poly* x : {&pr.first.q, &pr.first.p, &pr.second.q, &pr.second.p}) {
      poly_to(*x, out + off);
      off += x->limbs.size() * n;
    }
  }
}
int orc_key_import(const OrcParams* p, const uint64_t* in, uint64_t parts, uint64_t qlimbs, OrcKey** out) {
  ORC_TRY({
    auto key = std::make_shared<KskKey>();
    size_t n = p->P->n(), k = p->P->p.size(), off = 0;
    for (uint64_t j = 0; j < parts; ++j) {
      QpPoly b, a;
      b.q = poly_from(p->P->bq, in + off, qlimbs, true); off += qlimbs * n;
      b.p = poly_from(p->P->bp, in + off, k, true); off += k * n;
      a.q = poly_from(p->P->bq, in + off, qlimbs, true); off += qlimbs * n;
      a.p = poly_from(p->P->bp, in + off, k, true); off += k * n;
      key->parts.push_back({b, a});
    }
    *out = new OrcKey{key};
  })
}
int orc_key_switch(const OrcParams* p, const OrcKey* key, const uint64_t* in, uint64_t level, uint64_t* out_b,
                   uint64_t* out_a) {
  ORC_TRY({
    Poly x = poly_from(p->P->bq, in, level + 1, true);
    auto r = key_switch(*p->P, x, *key->k);
    poly_to(r.first, out_b);
    poly_to(r.second, out_a);
  })
}

// --- evaluator ---
int orc_eval_new(const OrcParams* p, const OrcKey* relin, const OrcKey* const* gkeys, const uint64_t* elts,
                 uint64_t ngal, int hoist, int bsgs, int lazy, OrcEval** out) {
  ORC_TRY({
    auto ev = std::make_unique<Evaluator>();
    ev->P = p->P;
    if (relin) ev->relin = relin->k;
    if (ngal) {
      ev->galois = std::make_shared<std::map<uint64_t, std::shared_ptr<KskKey>>>();
      for (uint64_t i = 0; i < ngal; ++i) (*ev->galois)[elts[i]] = gkeys[i]->k;
    }
    ev->config = EvalConfig{hoist != 0, bsgs != 0, lazy != 0};
    *out = new OrcEval{std::move(ev)};
  })
}
void orc_eval_free(OrcEval* e) { delete e; }
void orc_eval_counter(OrcEval* e, uint64_t* out7) {
  std::lock_guard<std::mutex> lk(e->ev->mu);
  auto& c = e->ev->counter;
  uint64_t v[7] = {c.rotations, c.relins, c.ct_ct_tensor, c.ct_pt_mults, c.rescales, c.sse_switches, c.bootstraps};
  memcpy(out7, v, sizeof v);
}
void orc_eval_reset_counter(OrcEval* e) {
  std::lock_guard<std::mutex> lk(e->ev->mu);
  e->ev->counter = OpCounter();
}

int orc_ct_new(const OrcEval* e, uint64_t ncomp, uint64_t level, double scale, const uint64_t* data, OrcCt** out) {
  ORC_TRY({
    std::vector<Poly> c;
    size_t per = (level + 1) * e->ev->P->n();
    for (uint64_t i = 0; i < ncomp; ++i) c.push_back(poly_from(e->ev->P->bq, data + i * per, level + 1, true));
    *out = new OrcCt{ct_new(c, scale)};
  })
}
void orc_ct_free(OrcCt* c) { delete c; }
void orc_ct_info(const OrcCt* c, uint64_t* ncomp, uint64_t* level, double* scale) {
  *ncomp = c->ct.len();
  *level = c->ct.level;
  *scale = c->ct.scale;
}
void orc_ct_data(const OrcCt* c, uint64_t* out) {
  size_t per = (c->ct.level + 1) * c->ct.c[0].n();
  for (size_t i = 0; i < c->ct.len(); ++i) poly_to(c->ct.c[i], out + i * per);
}

// Binary/unary ciphertext ops. op codes:
//  0 add, 1 sub, 2 negate, 3 mul_no_relin, 4 relinearize, 5 mul, 6 rescale, 7 conjugate
int orc_ct_op(OrcEval* e, int op, const OrcCt* a, const OrcCt* b, OrcCt** out) {
  ORC_TRY({
    Evaluator& ev = *e->ev;
    Ciphertext r;
    switch (op) {
      case 0: r = ev.add(a->ct, b->ct); break;
      case 1: r = ev.sub(a->ct, b->ct); break;
      case 2: r = ev.negate(a->ct); break;
      case 3: r = ev.mul_no_relin(a->ct, b->ct); break;
      case 4: r = ev.relinearize(a->ct); break;
      case 5: r = ev.mul(a->ct, b->ct); break;
      case 6: r = ev.rescale(a->ct); break;
      case 7: r = ev.conjugate(a->ct); break;
      default: throw HeError(INVALID_PARAMS, "unknown op");
    }
    *out = new OrcCt{std::move(r)};
  })
}
int orc_ct_rotate(OrcEval* e, const OrcCt* a, int32_t steps, OrcCt** out) {
  ORC_TRY({ *out = new OrcCt{e->ev->rotate(a->ct, steps)}; })
}
int orc_ct_hoisted_rotate(OrcEval* e, const OrcCt* a, const int32_t* steps, uint64_t n, OrcCt** outs) {
  ORC_TRY({
    auto v = e->ev->hoisted_rotate(a->ct, std::vector<int32_t>(steps, steps + n));
    for (size_t i = 0; i < v.size(); ++i) outs[i] = new OrcCt{v[i]};
  })
}
int orc_ct_mod_switch(OrcEval* e, const OrcCt* a, uint64_t level, OrcCt** out) {
  ORC_TRY({ *out = new OrcCt{e->ev->mod_switch_to_level(a->ct, level)}; })
}
int orc_ct_relabel(OrcEval* e, const OrcCt* a, double scale, OrcCt** out) {
  ORC_TRY({ *out = new OrcCt{e->ev->relabel(a->ct, scale)}; })
}
int orc_ct_mul_scalar(OrcEval* e, const OrcCt* a, double value, double target, OrcCt** out) {
  ORC_TRY({ *out = new OrcCt{e->ev->mul_scalar(a->ct, value, target)}; })
}
// plaintext ops: 0 add_plain, 1 mul_plain, 2 mul_plain_to_scale(target)
int orc_ct_plain_op(OrcEval* e, int op, const OrcCt* a, const uint64_t* pt, uint64_t pt_level, double pt_scale,
                    double target, OrcCt** out) {
  ORC_TRY({
    Plaintext p{poly_from(e->ev->P->bq, pt, pt_level + 1, true), pt_scale};
    Ciphertext r;
    if (op == 0) r = e->ev->add_plain(a->ct, p);
    else if (op == 1) r = e->ev->mul_plain(a->ct, p);
    else r = e->ev->mul_plain_to_scale(a->ct, p, target);
    *out = new OrcCt{std::move(r)};
  })
}
double orc_exact_product_scale(OrcEval* e, uint64_t level, double target, int* err) {
  try {
    *err = 0;
    return exact_product_scale(*e->ev->P, level, target);
  } catch (const HeError& x) {
    g_err = x.what();
    *err = x.kind;
    return 0;
  }
}
// BSGS: plaintext diagonals (d entries, all at pt_level and pt_scale, flat buffer) or
// ciphertext diagonals (d OrcCt handles).
int orc_matvec_plain(OrcEval* e, uint64_t d, uint64_t stride, const uint64_t* pts, uint64_t pt_level,
                     double pt_scale, const OrcCt* x, OrcCt** out) {
  ORC_TRY({
    if (d == 0 || (d & (d - 1))) throw HeError(INVALID_PARAMS, "d must be a power of two");
    Diagonals<Plaintext> dg;
    dg.d = d;
    auto bg = bsgs_split(d);
    dg.baby = bg.first;
    dg.giant = bg.second;
    dg.stride = stride;
    check_stride(d, stride, e->ev->P->slots());
    size_t per = (pt_level + 1) * e->ev->P->n();
    for (uint64_t i = 0; i < d; ++i)
      dg.entries.push_back(Plaintext{poly_from(e->ev->P->bq, pts + i * per, pt_level + 1, true), pt_scale});
    *out = new OrcCt{matvec_plain(*e->ev, dg, x->ct)};
  })
}
int orc_matvec_enc(OrcEval* e, uint64_t d, uint64_t stride, const OrcCt* const* cts, const OrcCt* x,
                   OrcCt** out) {
  ORC_TRY({
    if (d == 0 || (d & (d - 1))) throw HeError(INVALID_PARAMS, "d must be a power of two");
    Diagonals<Ciphertext> dg;
    dg.d = d;
    auto bg = bsgs_split(d);
    dg.baby = bg.first;
    dg.giant = bg.second;
    dg.stride = stride;
    check_stride(d, stride, e->ev->P->slots());
    for (uint64_t i = 0; i < d; ++i) dg.entries.push_back(cts[i]->ct);
    *out = new OrcCt{matvec_enc(*e->ev, dg, x->ct)};
  })
}

#include "oracle_boot_api.inc"

}  // extern "C"
