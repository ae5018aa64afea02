// TEST INFRASTRUCTURE ONLY -- the parity checker, never the product.
//
// CPU restatement of the ring/RNS layer of the reference (kenmaro3/ckks-train,
// crate ckks-train-core): word-sized modular arithmetic, prime search, the negacyclic
// NTT, the RNS basis with its NTT-form Galois permutation, the ChaCha20 generator and
// the polynomial samplers. Every function cites the reference file:line it follows.
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it.
//
// Build with -ffp-contract=off: the one floating-point step of the path (the overflow
// estimate of exact base conversion) must round every multiply and add separately.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

namespace orc {

typedef unsigned __int128 u128;
typedef std::vector<uint64_t> Limb;

// Error kinds of crates/ckks-train-core/src/error.rs:7-21 (HekitError).
enum ErrKind { OK = 0, INVALID_PARAMS = 1, SCALE_MISMATCH = 2, LEVEL_MISMATCH = 3,
               NO_LEVELS_LEFT = 4, DECODE = 5, DEVICE = 6 };

struct HeError : std::runtime_error {
  ErrKind kind;
  HeError(ErrKind k, const std::string& m) : std::runtime_error(m), kind(k) {}
};

// ---------------------------------------------------------------------------------------
// Modulus / Shoup: crates/ckks-train-core/src/modulus.rs:10-161
// ---------------------------------------------------------------------------------------

// High 128 bits of the 256-bit product x*y (modulus.rs:36-47, written out by columns).
inline u128 mulhi_u128(u128 x, u128 y) {
  u128 x0 = (uint64_t)x, x1 = x >> 64, y0 = (uint64_t)y, y1 = y >> 64;
  u128 p00 = x0 * y0, p01 = x0 * y1, p10 = x1 * y0, p11 = x1 * y1;
  u128 carry = (p00 >> 64) + (uint64_t)p01 + (uint64_t)p10;
  return p11 + (p01 >> 64) + (p10 >> 64) + (carry >> 64);
}

struct Shoup {
  uint64_t w = 0, ws = 0;  // multiplicand and floor(w * 2^64 / q)
};

struct Modulus {
  uint64_t q = 0;
  u128 ratio = 0;  // floor(2^128 / q)

  Modulus() = default;
  // modulus.rs:50-66: 2 <= q < 2^60, ratio = floor(2^128/q).
  explicit Modulus(uint64_t qv) : q(qv) {
    if (qv < 2 || qv >= (1ULL << 60))
      throw HeError(INVALID_PARAMS, "modulus " + std::to_string(qv) + " must satisfy 2 <= q < 2^60");
    u128 all = ~(u128)0;
    ratio = all / qv;
    if (all % qv + 1 == qv) ratio += 1;
  }
  uint64_t value() const { return q; }
  // modulus.rs:79-89
  uint64_t reduce_wide(u128 x) const {
    u128 est = mulhi_u128(x, ratio);
    uint64_t r = (uint64_t)(x - est * q);
    if (r >= q) r -= q;
    return r;
  }
  uint64_t add(uint64_t a, uint64_t b) const { uint64_t s = a + b; return s >= q ? s - q : s; }  // :92-96
  uint64_t sub(uint64_t a, uint64_t b) const { return a >= b ? a - b : a + q - b; }            // :98-102
  uint64_t mul(uint64_t a, uint64_t b) const { return reduce_wide((u128)a * b); }             // :106-109
  uint64_t pow(uint64_t a, uint64_t e) const {                                                 // :111-123
    uint64_t base = a % q, acc = 1 % q;
    while (e > 0) {
      if (e & 1) acc = mul(acc, base);
      base = mul(base, base);
      e >>= 1;
    }
    return acc;
  }
  // :125-139, extended Euclid; returns false when gcd(a, q) != 1.
  bool inv(uint64_t a, uint64_t* out) const {
    __int128 r0 = q, r1 = a % q, t0 = 0, t1 = 1;
    while (r1 != 0) {
      __int128 quo = r0 / r1;
      __int128 r2 = r0 - quo * r1; r0 = r1; r1 = r2;
      __int128 t2 = t0 - quo * t1; t0 = t1; t1 = t2;
    }
    if (r0 != 1) return false;
    __int128 m = (__int128)q;
    __int128 v = t0 % m;
    if (v < 0) v += m;
    *out = (uint64_t)v;
    return true;
  }
  uint64_t inv_or_throw(uint64_t a) const {
    uint64_t r;
    if (!inv(a, &r)) throw std::logic_error("not invertible");
    return r;
  }
  Shoup shoup(uint64_t w) const {  // :142-148
    Shoup s;
    s.w = w % q;
    s.ws = (uint64_t)(((u128)s.w << 64) / q);
    return s;
  }
  uint64_t mul_shoup_lazy(uint64_t a, const Shoup& s) const {  // :152-155
    uint64_t qhat = (uint64_t)(((u128)a * s.ws) >> 64);
    return a * s.w - qhat * q;
  }
  uint64_t mul_shoup(uint64_t a, const Shoup& s) const {  // :158-161
    uint64_t r = mul_shoup_lazy(a, s);
    return r >= q ? r - q : r;
  }
};

// ---------------------------------------------------------------------------------------
// Primes: crates/ckks-train-core/src/primes.rs:5-118
// ---------------------------------------------------------------------------------------

inline uint64_t mulmod_plain(uint64_t a, uint64_t b, uint64_t m) { return (uint64_t)((u128)a * b % m); }
inline uint64_t powmod_plain(uint64_t a, uint64_t e, uint64_t m) {
  uint64_t acc = 1 % m;
  a %= m;
  while (e > 0) {
    if (e & 1) acc = mulmod_plain(acc, a, m);
    a = mulmod_plain(a, a, m);
    e >>= 1;
  }
  return acc;
}

// primes.rs:24-53: deterministic Miller-Rabin with the first twelve prime bases.
inline bool is_prime_u64(uint64_t n) {
  static const uint64_t bases[12] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
  if (n < 2) return false;
  for (uint64_t p : bases) {
    if (n == p) return true;
    if (n % p == 0) return false;
  }
  int s = __builtin_ctzll(n - 1);
  uint64_t d = (n - 1) >> s;
  for (uint64_t a : bases) {
    uint64_t x = powmod_plain(a, d, n);
    if (x == 1 || x == n - 1) continue;
    bool ok = false;
    for (int i = 1; i < s; ++i) {
      x = mulmod_plain(x, x, n);
      if (x == n - 1) { ok = true; break; }
    }
    if (!ok) return false;
  }
  return true;
}

// primes.rs:67-112: primes 2^(bits-1) < q < 2^bits, q = 1 mod 2n, descending, after `skip`.
inline std::vector<uint64_t> ntt_primes_skip(uint32_t bits, uint64_t n, size_t skip, size_t count) {
  if (bits < 2 || bits > 60)
    throw HeError(INVALID_PARAMS, "prime bit size " + std::to_string(bits) + " must be in 2..=60");
  if (n == 0 || (n & (n - 1)) != 0)
    throw HeError(INVALID_PARAMS, "n = " + std::to_string(n) + " must be a power of two");
  u128 step = (u128)n * 2, lo = (u128)1 << (bits - 1), hi = (u128)1 << bits;
  std::vector<uint64_t> out;
  auto not_enough = [&]() {
    return HeError(INVALID_PARAMS, "not enough " + std::to_string(bits) + "-bit primes");
  };
  if (step >= hi) {
    if (count == 0) return out;
    throw not_enough();
  }
  u128 q = (hi - 2) / step * step + 1;
  size_t seen = 0;
  while (out.size() < count) {
    if (q <= lo) throw not_enough();
    if (is_prime_u64((uint64_t)q)) {
      if (seen >= skip) out.push_back((uint64_t)q);
      seen++;
    }
    if (q < step) throw not_enough();
    q -= step;
  }
  return out;
}

// ---------------------------------------------------------------------------------------
// NTT: crates/ckks-train-core/src/ntt.rs:34-232
// ---------------------------------------------------------------------------------------

inline uint64_t bitrev(uint64_t i, uint32_t bits) {
  if (bits == 0) return 0;
  uint64_t r = 0;
  for (uint32_t b = 0; b < bits; ++b) r |= ((i >> b) & 1ULL) << (bits - 1 - b);
  return r;
}

// ntt.rs:66-82: minimal primitive 2n-th root of unity.
inline uint64_t minimal_primitive_root(uint64_t n, const Modulus& m) {
  uint64_t q = m.q, e = (q - 1) / (2 * n), c = 0;
  for (uint64_t g = 2;; ++g) {
    c = m.pow(g, e);
    if (m.pow(c, n) == q - 1) break;
  }
  uint64_t c2 = m.mul(c, c), cur = c, best = c;
  for (uint64_t i = 1; i < n; ++i) {
    cur = m.mul(cur, c2);
    if (cur < best) best = cur;
  }
  return best;
}

struct NttTable {
  uint64_t n = 0;
  Modulus m;
  uint64_t psi = 0;
  std::vector<Shoup> roots, inv_roots;
  Shoup n_inv, w_n_inv;

  NttTable() = default;
  // ntt.rs:89-129
  NttTable(uint64_t nn, const Modulus& mod) : n(nn), m(mod) {
    if (nn < 2 || (nn & (nn - 1)) != 0)
      throw HeError(INVALID_PARAMS, "NTT size " + std::to_string(nn) + " must be a power of two >= 2");
    uint64_t q = m.q;
    if (nn >= q || (q - 1) % (2 * nn) != 0)
      throw HeError(INVALID_PARAMS, "modulus " + std::to_string(q) + " is not 1 mod 2n");
    if (!is_prime_u64(q)) throw HeError(INVALID_PARAMS, "modulus " + std::to_string(q) + " is not prime");
    psi = minimal_primitive_root(nn, m);
    uint64_t psi_inv = m.inv_or_throw(psi), ninv = m.inv_or_throw(nn);
    uint32_t bits = __builtin_ctzll(nn);
    roots.resize(nn);
    inv_roots.resize(nn);
    uint64_t p = 1, pi = 1;
    for (uint64_t i = 0; i < nn; ++i) {  // ntt.rs:54-63 table[bitrev(i)] = base^i
      roots[bitrev(i, bits)] = m.shoup(p);
      inv_roots[bitrev(i, bits)] = m.shoup(pi);
      p = m.mul(p, psi);
      pi = m.mul(pi, psi_inv);
    }
    n_inv = m.shoup(ninv);
    w_n_inv = m.shoup(m.mul(inv_roots[1].w, ninv));
  }

  // ntt.rs:141-179: Harvey CT, natural in, bit-reversed out, lazy in [0, 4q).
  void forward(uint64_t* a) const {
    uint64_t q = m.q, two_q = 2 * q;
    uint64_t t = n, groups = 1;
    while (groups < n / 2) {
      t >>= 1;
      for (uint64_t g = 0; g < groups; ++g) {
        const Shoup& w = roots[groups + g];
        uint64_t* lo = a + 2 * t * g;
        uint64_t* hi = lo + t;
        for (uint64_t k = 0; k < t; ++k) {
          uint64_t x = lo[k];
          uint64_t xr = x >= two_q ? x - two_q : x;
          uint64_t tt = m.mul_shoup_lazy(hi[k], w);
          lo[k] = xr + tt;
          hi[k] = xr + two_q - tt;
        }
      }
      groups <<= 1;
    }
    auto reduce = [&](uint64_t r) {
      r = r >= two_q ? r - two_q : r;
      return r >= q ? r - q : r;
    };
    for (uint64_t g = 0; g < n / 2; ++g) {
      const Shoup& w = roots[n / 2 + g];
      uint64_t x = a[2 * g];
      uint64_t xr = x >= two_q ? x - two_q : x;
      uint64_t tt = m.mul_shoup_lazy(a[2 * g + 1], w);
      a[2 * g] = reduce(xr + tt);
      a[2 * g + 1] = reduce(xr + two_q - tt);
    }
  }

  // ntt.rs:184-232: GS, bit-reversed in, natural out, fused N^-1 in the last stage.
  void inverse(uint64_t* a) const {
    uint64_t q = m.q, two_q = 2 * q;
    uint64_t t = 1, h = n >> 1;
    if (h > 1) {
      for (uint64_t g = 0; g < h; ++g) {
        const Shoup& w = inv_roots[h + g];
        uint64_t x = a[2 * g], y = a[2 * g + 1];
        uint64_t s = x + y;
        a[2 * g] = s >= two_q ? s - two_q : s;
        a[2 * g + 1] = m.mul_shoup_lazy(x + two_q - y, w);
      }
      t = 2;
      h >>= 1;
    }
    while (h > 1) {
      for (uint64_t g = 0; g < h; ++g) {
        const Shoup& w = inv_roots[h + g];
        uint64_t* lo = a + 2 * t * g;
        uint64_t* hi = lo + t;
        for (uint64_t k = 0; k < t; ++k) {
          uint64_t x = lo[k], y = hi[k];
          uint64_t s = x + y, d = x + two_q - y;
          lo[k] = s >= two_q ? s - two_q : s;
          hi[k] = m.mul_shoup_lazy(d, w);
        }
      }
      t <<= 1;
      h >>= 1;
    }
    uint64_t half = n / 2;
    for (uint64_t k = 0; k < half; ++k) {
      uint64_t x = a[k], y = a[k + half];
      uint64_t s = x + y, d = x + two_q - y;
      uint64_t r0 = m.mul_shoup_lazy(s, n_inv), r1 = m.mul_shoup_lazy(d, w_n_inv);
      if (r0 >= q) r0 -= q;
      if (r1 >= q) r1 -= q;
      a[k] = r0;
      a[k + half] = r1;
    }
  }
};

// ---------------------------------------------------------------------------------------
// RNS basis and Galois permutation: crates/ckks-train-core/src/rns.rs:39-175
// ---------------------------------------------------------------------------------------

// rns.rs:162-175 (SEAL's generate_table_ntt).
inline std::vector<uint32_t> galois_permutation_ntt(uint64_t n, uint64_t g) {
  uint32_t log_n = __builtin_ctzll(n);
  uint64_t mask = n - 1;
  std::vector<uint32_t> out(n);
  for (uint64_t i = n; i < 2 * n; ++i) {
    uint64_t reversed = bitrev(i, log_n + 1);
    uint64_t index_raw = ((g * reversed) >> 1) & mask;
    out[i - n] = (uint32_t)bitrev(index_raw, log_n);
  }
  return out;
}

struct RnsBasis {
  uint64_t n = 0;
  std::vector<Modulus> moduli;
  std::vector<NttTable> ntt;
  mutable std::mutex mu;
  mutable std::unordered_map<uint64_t, std::shared_ptr<std::vector<uint32_t>>> galois_cache;

  // rns.rs:65-99
  RnsBasis(uint64_t nn, const std::vector<uint64_t>& qs) : n(nn) {
    if (qs.empty()) throw HeError(INVALID_PARAMS, "RNS basis needs at least one modulus");
    if (nn >= (1ULL << 32)) throw HeError(INVALID_PARAMS, "ring degree must be below 2^32");
    for (size_t i = 0; i < qs.size(); ++i)
      for (size_t j = 0; j < i; ++j)
        if (qs[i] == qs[j]) throw HeError(INVALID_PARAMS, "duplicate modulus in RNS basis");
    for (uint64_t q : qs) {
      Modulus m(q);
      ntt.emplace_back(nn, m);
      moduli.push_back(m);
    }
  }
  size_t len() const { return moduli.size(); }
  // rns.rs:137-152 (cached per element).
  std::shared_ptr<std::vector<uint32_t>> galois_permutation(uint64_t g) const {
    uint64_t two_n = 2 * n;
    g %= two_n;
    std::lock_guard<std::mutex> lk(mu);
    auto it = galois_cache.find(g);
    if (it != galois_cache.end()) return it->second;
    auto p = std::make_shared<std::vector<uint32_t>>(galois_permutation_ntt(n, g));
    galois_cache[g] = p;
    return p;
  }
};
typedef std::shared_ptr<const RnsBasis> BasisPtr;

// ---------------------------------------------------------------------------------------
// ChaCha20 stream of rand_chacha 0.9.0 (ChaCha20Rng): a 32-byte key, 64-bit block counter
// from 0 in state words 12-13, stream id 0 in words 14-15, output words little-endian in
// order, next_u64 = word[2i] | word[2i+1] << 32. Published ChaCha20 (Bernstein 2008).
// Used by crates/ckks-train-core/src/sampler.rs:31-75.
// ---------------------------------------------------------------------------------------

struct ChaCha20 {
  uint32_t key[8];
  uint64_t counter = 0;
  uint32_t buf[16];
  int idx = 16;

  explicit ChaCha20(const uint8_t seed[32]) {
    for (int i = 0; i < 8; ++i)
      key[i] = (uint32_t)seed[4 * i] | ((uint32_t)seed[4 * i + 1] << 8) |
               ((uint32_t)seed[4 * i + 2] << 16) | ((uint32_t)seed[4 * i + 3] << 24);
  }
  static inline uint32_t rotl(uint32_t v, int c) { return (v << c) | (v >> (32 - c)); }
  static inline void qr(uint32_t& a, uint32_t& b, uint32_t& c, uint32_t& d) {
    a += b; d ^= a; d = rotl(d, 16);
    c += d; b ^= c; b = rotl(b, 12);
    a += b; d ^= a; d = rotl(d, 8);
    c += d; b ^= c; b = rotl(b, 7);
  }
  void refill() {
    uint32_t s[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u,
                      key[0], key[1], key[2], key[3], key[4], key[5], key[6], key[7],
                      (uint32_t)counter, (uint32_t)(counter >> 32), 0u, 0u};
    uint32_t x[16];
    memcpy(x, s, sizeof x);
    for (int r = 0; r < 10; ++r) {
      qr(x[0], x[4], x[8], x[12]); qr(x[1], x[5], x[9], x[13]);
      qr(x[2], x[6], x[10], x[14]); qr(x[3], x[7], x[11], x[15]);
      qr(x[0], x[5], x[10], x[15]); qr(x[1], x[6], x[11], x[12]);
      qr(x[2], x[7], x[8], x[13]); qr(x[3], x[4], x[9], x[14]);
    }
    for (int i = 0; i < 16; ++i) buf[i] = x[i] + s[i];
    counter++;
    idx = 0;
  }
  uint32_t next_u32() {
    if (idx >= 16) refill();
    return buf[idx++];
  }
  uint64_t next_u64() {
    uint64_t lo = next_u32();
    uint64_t hi = next_u32();
    return lo | (hi << 32);
  }
};

// rand_core 0.9.5 SeedableRng::seed_from_u64: PCG32 (XSH-RR) output, 4 bytes per step.
inline void seed_from_u64(uint64_t state, uint8_t out[32]) {
  const uint64_t MUL = 6364136223846793005ULL, INC = 11634580027462260723ULL;
  for (int c = 0; c < 8; ++c) {
    state = state * MUL + INC;
    uint32_t xorshifted = (uint32_t)(((state >> 18) ^ state) >> 27);
    uint32_t rot = (uint32_t)(state >> 59);
    uint32_t x = (xorshifted >> rot) | (xorshifted << ((32 - rot) & 31));
    for (int b = 0; b < 4; ++b) out[4 * c + b] = (uint8_t)(x >> (8 * b));
  }
}

}  // namespace orc
