// Host-side number theory for building the device tables: word modular arithmetic,
// Miller-Rabin, SEAL-style NTT-friendly prime hand-out, the minimal primitive 2N-th root
// and bit reversal. Follows crates/ckks-train-core/src/{modulus,primes,ntt}.rs and
// crates/ckks-train-ckks/src/params.rs:87-157.
#pragma once
#include <algorithm>
#include <cstdint>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

namespace ckg {

typedef unsigned __int128 u128;

struct HostMod {
  uint64_t q = 0;
  HostMod() = default;
  explicit HostMod(uint64_t v) : q(v) {}
  uint64_t mul(uint64_t a, uint64_t b) const { return (uint64_t)((u128)a * b % q); }
  uint64_t add(uint64_t a, uint64_t b) const { uint64_t s = a + b; return s >= q ? s - q : s; }
  uint64_t sub(uint64_t a, uint64_t b) const { return a >= b ? a - b : a + q - b; }
  uint64_t pow(uint64_t a, uint64_t e) const {
    uint64_t r = 1 % q;
    a %= q;
    while (e) {
      if (e & 1) r = mul(r, a);
      a = mul(a, a);
      e >>= 1;
    }
    return r;
  }
  // Inverse via Fermat's little theorem (q prime).
  uint64_t inv(uint64_t a) const { return pow(a % q, q - 2); }
  uint64_t shoup(uint64_t w) const { return (uint64_t)(((u128)(w % q) << 64) / q); }
};

inline uint32_t bit_length(uint64_t v) { return v ? 64 - __builtin_clzll(v) : 0; }

inline uint64_t bitrev(uint64_t i, uint32_t bits) {
  uint64_t r = 0;
  for (uint32_t b = 0; b < bits; ++b) r |= ((i >> b) & 1ULL) << (bits - 1 - b);
  return r;
}

inline bool is_prime(uint64_t n) {
  static const uint64_t bases[12] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
  if (n < 2) return false;
  for (uint64_t p : bases) {
    if (n == p) return true;
    if (n % p == 0) return false;
  }
  HostMod m(n);
  uint64_t d = n - 1;
  int s = 0;
  while (!(d & 1)) { d >>= 1; ++s; }
  for (uint64_t a : bases) {
    uint64_t x = m.pow(a, d);
    if (x == 1 || x == n - 1) continue;
    bool comp = true;
    for (int r = 1; r < s; ++r) {
      x = m.mul(x, x);
      if (x == n - 1) { comp = false; break; }
    }
    if (comp) return false;
  }
  return true;
}

// The `count` largest primes 2^(bits-1) < q < 2^bits with q = 1 mod 2n, descending.
inline std::vector<uint64_t> ntt_primes(uint32_t bits, uint64_t n, size_t count) {
  if (bits < 2 || bits > 60) throw std::invalid_argument("prime bit size must be in 2..=60");
  u128 step = (u128)2 * n, lo = (u128)1 << (bits - 1), hi = (u128)1 << bits;
  std::vector<uint64_t> out;
  if (count == 0) return out;
  if (step >= hi) throw std::invalid_argument("not enough NTT-friendly primes");
  u128 q = (hi - 2) / step * step + 1;
  while (out.size() < count) {
    if (q <= lo) throw std::invalid_argument("not enough NTT-friendly primes of " + std::to_string(bits) + " bits");
    if (is_prime((uint64_t)q)) out.push_back((uint64_t)q);
    if (q < step) throw std::invalid_argument("not enough NTT-friendly primes");
    q -= step;
  }
  return out;
}

// SEAL CoeffModulus::Create hand-out (params.rs:122-140): per bit size, the c largest
// primes are handed out from the smallest upwards in order of appearance.
inline void primes_for_bits(uint32_t log_n, const std::vector<uint32_t>& q_bits, const std::vector<uint32_t>& p_bits,
                            std::vector<uint64_t>& q, std::vector<uint64_t>& p) {
  std::vector<uint32_t> all(q_bits);
  all.insert(all.end(), p_bits.begin(), p_bits.end());
  std::map<uint32_t, std::vector<uint64_t>> pools;
  std::map<uint32_t, size_t> next;
  for (uint32_t b : all)
    if (!pools.count(b)) {
      pools[b] = ntt_primes(b, 1ULL << log_n, std::count(all.begin(), all.end(), b));
      next[b] = 0;
    }
  q.clear();
  p.clear();
  for (size_t i = 0; i < all.size(); ++i) {
    auto& pool = pools[all[i]];
    uint64_t v = pool[pool.size() - 1 - next[all[i]]++];
    (i < q_bits.size() ? q : p).push_back(v);
  }
}

// Minimal primitive 2n-th root of unity modulo prime q (ntt.rs:66-82).
inline uint64_t minimal_root(uint64_t n, const HostMod& m) {
  uint64_t q = m.q, e = (q - 1) / (2 * n), c = 0;
  for (uint64_t g = 2;; ++g) {
    c = m.pow(g, e);
    if (m.pow(c, n) == q - 1) break;
  }
  uint64_t c2 = m.mul(c, c), cur = c, best = c;
  for (uint64_t i = 1; i < n; ++i) {
    cur = m.mul(cur, c2);
    best = std::min(best, cur);
  }
  return best;
}

// NTT-form Galois permutation out[i] = in[perm[i]] (crates/ckks-train-core/src/rns.rs:162-175).
inline std::vector<uint32_t> galois_perm(uint64_t n, uint64_t g) {
  uint32_t log_n = __builtin_ctzll(n);
  std::vector<uint32_t> out(n);
  for (uint64_t i = 0; i < n; ++i) {
    uint64_t rev = bitrev(n + i, log_n + 1);
    out[i] = (uint32_t)bitrev(((g * rev) >> 1) & (n - 1), log_n);
  }
  return out;
}

// Galois element of a left rotation by `step` slots: 3^(step mod N/2) mod 2N
// (crates/ckks-train-ckks/src/keys.rs:89-103).
inline uint64_t galois_elt(uint64_t n, int32_t step) {
  uint64_t m = 2 * n;
  int64_t slots = (int64_t)std::max<uint64_t>(n / 2, 1);
  uint64_t k = (uint64_t)((((int64_t)step % slots) + slots) % slots);
  uint64_t base = 3 % m, acc = 1 % m;
  while (k) {
    if (k & 1) acc = (uint64_t)((u128)acc * base % m);
    base = (uint64_t)((u128)base * base % m);
    k >>= 1;
  }
  return acc;
}

}  // namespace ckg
