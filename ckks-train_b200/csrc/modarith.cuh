// Device modular arithmetic for word-sized primes q < 2^60 on the integer pipe.
//
// Every routine returns a value congruent to the exact result; the fully reduced forms
// return the unique residue in [0, q), so results are bit-identical to any other exact
// implementation (the reference reduces with floor(2^128/q) Barrett and Shoup products,
// crates/ckks-train-core/src/modulus.rs:79-161).
#pragma once
#include <cstdint>

#define CKG_DEV __device__ __forceinline__

// Per-prime constants, one record per global prime index (0..L data primes, then the
// special primes). Read through the read-only path.
struct PrimeConst {
  uint64_t q;
  uint64_t two_q;
  uint64_t mu;       // floor(2^(2b) / q), b = bit length of q (Barrett, a*b with a, b < q)
  uint64_t ninv;     // N^-1 mod q and its Shoup companion
  uint64_t ninv_s;
  uint64_t wninv;    // psi^-1 * N^-1 (the fused last inverse stage) and companion
  uint64_t wninv_s;
  uint64_t r64;      // 2^64 mod q and companion (reduction of 128-bit sums)
  uint64_t r64_s;
  uint64_t one_s;    // floor(2^64 / q): Shoup companion of 1 (reduces any u64 to [0, 2q))
  uint32_t b;        // bit length of q
  uint32_t ip_off;   // nonzero: the inner product may take its FP64-assisted form (kernels.cu)
  double qd, qinv;     // q and fl(1/q) for the FP64 butterflies of primes below 2^50
  double ninvd, wninvd;  // ninv and wninv as doubles (exact: < q < 2^50)
};

CKG_DEV uint64_t mul_shoup_lazy(uint64_t a, uint64_t w, uint64_t ws, uint64_t q) {
  uint64_t qh = __umul64hi(a, ws);
  return a * w - qh * q;  // in [0, 2q) for any a < 2^64
}

CKG_DEV uint64_t csub(uint64_t x, uint64_t m) { return x >= m ? x - m : x; }

CKG_DEV uint64_t mul_shoup(uint64_t a, uint64_t w, uint64_t ws, uint64_t q) {
  return csub(mul_shoup_lazy(a, w, ws, q), q);
}

CKG_DEV uint64_t add_mod(uint64_t a, uint64_t b, uint64_t q) { return csub(a + b, q); }
CKG_DEV uint64_t sub_mod(uint64_t a, uint64_t b, uint64_t q) { return a >= b ? a - b : a + q - b; }

// a * b mod q for a, b < q, Barrett with mu = floor(2^(2b)/q): the quotient estimate
// ((x >> (b-1)) * mu) >> (b+1) is at most 2 below the true quotient, so two conditional
// subtractions finish the reduction.
CKG_DEV uint64_t mul_mod(uint64_t a, uint64_t bb, const PrimeConst& p) {
  uint64_t lo = a * bb, hi = __umul64hi(a, bb);
  uint32_t b = p.b;
  uint64_t t = (hi << (65 - b)) | (lo >> (b - 1));  // x >> (b-1) < 2^(b+1)
  uint64_t plo = t * p.mu, phi = __umul64hi(t, p.mu);
  uint64_t est = (phi << (63 - b)) | (plo >> (b + 1));
  uint64_t r = lo - est * p.q;
  r = csub(r, p.q);
  return csub(r, p.q);
}

// Reduces a 128-bit value (hi, lo) modulo q: hi * [2^64]_q + lo via two Shoup products.
CKG_DEV uint64_t reduce128(uint64_t hi, uint64_t lo, const PrimeConst& p) {
  uint64_t a = mul_shoup_lazy(hi, p.r64, p.r64_s, p.q);  // [0, 2q)
  uint64_t c = mul_shoup_lazy(lo, 1, p.one_s, p.q);      // [0, 2q)
  uint64_t s = csub(a, p.q) + csub(c, p.q);
  return csub(s, p.q);
}

// 128-bit accumulate: (hi, lo) += a * b.
CKG_DEV void mac128(uint64_t& hi, uint64_t& lo, uint64_t a, uint64_t b) {
  uint64_t plo = a * b, phi = __umul64hi(a, b);
  asm("add.cc.u64 %0, %0, %2;\n\taddc.u64 %1, %1, %3;" : "+l"(lo), "+l"(hi) : "l"(plo), "l"(phi));
}
