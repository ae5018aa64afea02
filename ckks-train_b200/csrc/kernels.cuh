// Launch descriptors shared by the device kernels and the host engine.
//
// Kernels take their work lists by value (`__grid_constant__` parameter structs), so a
// launch needs no separate descriptor upload and a captured CUDA graph keeps its own copy.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "modarith.cuh"

namespace ckg {

// One limb of a batched limb-wise kernel: N words at src (read) and dst (written; may
// equal src), reduced modulo the prime with global index `prime`.
struct LimbRef {
  const uint64_t* src;
  uint64_t* dst;
  uint32_t prime;
  uint32_t aux;  // kernel-specific (e.g. the second operand's limb offset)
};

constexpr int kMaxLimbs = 256;  // per launch; larger lists are split by the host
struct LimbBatch {
  int count;
  int pad;
  LimbRef r[kMaxLimbs];
};

// Element-wise binary op over limbs: out = a (op) b, b given per limb.
struct BinRef {
  const uint64_t* a;
  const uint64_t* b;
  uint64_t* out;
  uint32_t prime;
  uint32_t pad;
};
constexpr int kMaxBin = 192;
struct BinBatch {
  int count;
  int op;  // 0 add, 1 sub, 2 mul
  BinRef r[kMaxBin];
};

// Base conversion job: source limbs (coefficient form) -> target limbs (coefficient form)
// out_t = (sum_j y_j * (S/s_j mod t) - e * (S mod t) - h_t) mod t,
// y_j = [(x_j + h_j) * (S/s_j)^-1]_{s_j}, e = floor(sum_j f64(y_j) * f64(1/s_j)) when n_src > 1.
// `table` points at a device record laid out by ConvLayout below.
constexpr int kMaxSrc = 16;
constexpr int kMaxDst = 64;
struct ConvJob {
  const uint64_t* src;   // n_src limbs, limb j at src + j * src_stride
  uint64_t* dst;         // n_dst limbs, limb t at dst + t * dst_stride
  const uint64_t* table;
  uint64_t src_stride;
  uint64_t dst_stride;
  int n_dst;             // targets of this job
  int pad;
};
constexpr int kMaxConv = 32;
struct ConvBatch {
  int count;
  int n_src;
  int n_dst;
  int pad;
  ConvJob j[kMaxConv];
};

// Table record (u64 words):
//   header, 1 word: the number of leading dst records in the FP64-assisted form
//   src block, 5 words per source j: prime, qhat_inv, qhat_inv_shoup, half_j, bits(1.0/s_j)
//   dst block, (8 + 2 n_src) words per target t, in one of two forms:
//   - exact: prime, (t - [S]_t), (t - [h]_t), t, [2^64]_t, its Shoup companion, floor(2^64/t),
//     out, then w_tj = [S/s_j]_t split into 30-bit halves (low half in bits 0..29, high half in
//     bits 32..61), then n_src unused words;
//   - FP64-assisted: prime, (t - [S]_t), (t - [h]_t), t, bits(1/t), bits((t - [S]_t)/t),
//     bits((t - [h]_t)/t), out | two_stage << 32, then w_tj whole, then bits(w_tj / t);
//   `out` is the target's limb position in the job's output (records may be reordered).
struct ConvLayout {
  static constexpr int kHeadWords = 1;
  static constexpr int kSrcWords = 5;
  static __host__ __device__ int dst_words(int n_src) { return 8 + 2 * n_src; }
  static __host__ __device__ int size(int n_src, int n_dst) {
    return kHeadWords + kSrcWords * n_src + dst_words(n_src) * n_dst;
  }
  // The tensor-core block follows the records at the next 16-byte boundary (tables start on
  // one), for n_src <= kTcMaxSrc and n_dst <= kTcMaxDst:
  //   word 0: K | N << 32 (K = 32 or 64 operand bytes per coefficient, N = MMA width, a
  //   multiple of 16 >= 8 n_dst), word 1: 0; then 6 words per target in output order: t,
  //   bits(1/t), t - [S]_t, t - [h]_t, bits(f64(t - [S]_t)), bits(f64(t - [h]_t)); then the
  //   B operand: N rows (target o, byte b at row 8 o + b) of K bytes, row (o, b) holding at
  //   byte 8 j + a the byte b of [2^(8a) w_oj]_t, stored as 8-row x 16-byte core matrices (row
  //   group stride 8 K bytes, K-chunk stride 128).
  static constexpr int kTcMaxSrc = 8;
  static constexpr int kTcMaxDst = 32;
  static __host__ __device__ int tc_offset(int n_src, int n_dst) { return (size(n_src, n_dst) + 1) & ~1; }
};
// FP64-assisted records serve at most this many sources (kernel register arrays).
constexpr int kMaxSrcF64 = 8;

// Key-switch inner product of one level-l polynomial (module docs of keyswitch.cu).
constexpr int kMaxDigits = 16;
struct IpJob {
  int level;                          // l
  int ndig;                           // digits at level l
  int key_q;                          // data limbs per key part (the key's max level + 1)
  int pad;
  const uint64_t* in;                 // the switched polynomial (NTT form, l+1 limbs)
  const uint64_t* conv[kMaxDigits];   // digit j's converted limbs (targets, NTT form)
  const uint64_t* key;                // key base: part j, b/a, (L+1+k) limbs
  uint64_t* out_b;                    // l+1+k limbs
  uint64_t* out_a;
  const uint32_t* perm;               // optional NTT-form Galois permutation (hoisting)
};
constexpr int kMaxIp = 16;
struct IpBatch {
  int count;
  int alpha;   // primes per digit
  int L;       // max level of the parameters (special prime t has global index L+1+t)
  int k;       // special primes
  IpJob j[kMaxIp];
};

// Finish of ModDown / rescale: out_i = (x_i - t_i) * c_i (+ add_i) mod q_i.
struct FinRef {
  const uint64_t* x;
  const uint64_t* t;
  const uint64_t* add;       // may be null
  const uint32_t* add_perm;  // optional: the addend is read as add[add_perm[c]]
  uint64_t* out;
  uint64_t c;            // the constant and its Shoup companion
  uint64_t c_s;
  uint32_t prime;
  uint32_t pad;
};
constexpr int kMaxFin = 96;
struct FinBatch {
  int count;
  int pad;
  FinRef r[kMaxFin];
};

// Ciphertext tensor product per limb: d0 = a0 b0, d1 = a0 b1 + a1 b0, d2 = a1 b1.
struct TensorRef {
  const uint64_t* a0;
  const uint64_t* a1;
  const uint64_t* b0;
  const uint64_t* b1;
  uint64_t* d0;
  uint64_t* d1;
  uint64_t* d2;
  uint32_t prime;
  uint32_t pad;
};
constexpr int kMaxTensor = 96;
struct TensorBatch {
  int count;
  int pad;
  TensorRef r[kMaxTensor];
};

// Fused plaintext multiply-accumulate over the limbs of 2-component ciphertexts:
// out_c[i] = sum_t x_c[t][i] * w[t][i] (c = 0, 1), limb i at offset i * N of every base
// pointer, prime index i.
constexpr int kMaxMacTerms = 48;
struct MacBatch {
  int count, limbs;
  uint64_t* out0;
  uint64_t* out1;
  const uint64_t* x0[kMaxMacTerms];
  const uint64_t* x1[kMaxMacTerms];
  const uint64_t* w[kMaxMacTerms];
};

// Fused ciphertext-ciphertext multiply-accumulate (the inner sums of BSGS with encrypted
// diagonals): out0 = sum_t a0_t b0_t, out1 = sum_t (a0_t b1_t + a1_t b0_t), out2 = sum_t a1_t b1_t,
// limb i at offset i * N of every base pointer, prime index i.
constexpr int kMaxMacTensorTerms = 32;
struct MacTensorBatch {
  int count, limbs;
  uint64_t* out0;
  uint64_t* out1;
  uint64_t* out2;
  const uint64_t* a0[kMaxMacTensorTerms];
  const uint64_t* a1[kMaxMacTensorTerms];
  const uint64_t* b0[kMaxMacTensorTerms];
  const uint64_t* b1[kMaxMacTensorTerms];
};

// Multiplication of limbs by a per-prime constant (Shoup pair per global prime index).
constexpr int kMaxPrimes = 64;
struct ScalarTable {
  uint64_t w[kMaxPrimes];
  uint64_t ws[kMaxPrimes];
};

// Work lists resident in device memory (the batched path): the same kernels read
// items through a pointer instead of a by-value array.
struct LimbPtrs {
  int count;
  int pad;
  const LimbRef* r;
};
struct ConvPtrs {
  int count;
  int n_src;
  int n_dst;
  int pad;
  const ConvJob* j;
};
struct IpPtrs {
  int count;
  int alpha;
  int L;
  int k;
  const IpJob* j;
};
struct FinPtrs {
  int count;
  int pad;
  const FinRef* r;
};
struct BinPtrs {
  int count;
  int op;
  const BinRef* r;
};
struct TensorPtrs {
  int count;
  int pad;
  const TensorRef* r;
};
// Gather through a per-limb permutation (NTT-form automorphism of many ciphertexts).
struct GatherRef {
  const uint64_t* src;
  uint64_t* dst;
  const uint32_t* perm;
};
struct GatherPtrs {
  int count;
  int pad;
  const GatherRef* r;
};

// One segment of a packed download: `rows` rows of `row_words` words at `pitch` words apart in
// the source, written contiguously at dst (rows * row_words < 2^32).
struct PackSeg {
  const uint64_t* src;
  uint64_t* dst;
  uint64_t pitch;
  uint32_t rows;
  uint32_t row_words;
};

}  // namespace ckg
