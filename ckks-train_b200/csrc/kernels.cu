// sm_100a kernels of the RNS-CKKS evaluator path: batched negacyclic NTT / INTT, base
// conversion (ModUp / ModDown / rescale), the key-switch inner product, the ModDown and
// rescale finish, element-wise ops and the NTT-form automorphism.
//
// Arithmetic is 64-bit integer on the IMAD pipe, except the NTT butterflies of primes below
// 2^50, which run exactly on the FP64 pipe (see kF64Bound), and the overflow estimate of
// exact base conversion, done with __dmul_rn / __dadd_rn so that no multiply-add is
// contracted (crates/ckks-train-core/src/baseconv.rs:198-206).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <stdexcept>
#include <vector>
#include <type_traits>

#include "kernels.cuh"
#include "launch.hpp"
#include "bounds_refs.hpp"

namespace ckg {

// ------------------------------------------------------------------------------------
// NTT. Forward: Harvey Cooley-Tukey, natural order in, bit-reversed order out, values
// lazily in [0, 4q) between stages (crates/ckks-train-core/src/ntt.rs:141-179); inverse:
// Gentleman-Sande with N^-1 fused into the last stage (ntt.rs:184-232). Twiddles are the
// full-N tables roots[bitrev(i)] = psi^i as (w, floor(w 2^64 / q)) pairs.
//
// N = 2^logN >= 2^12 runs in two passes over a 2^(logN-8) x 256 matrix view of each limb
// (element x = 256 * row + col). The first logN - 8 forward stages pair elements of one
// column (stride >= 256), the last 8 pair elements of one row. Each pass loads a tile,
// runs its stages in registers as two radix-2^E phases with one shared-memory exchange,
// and writes the tile back (in place or to another buffer).
// ------------------------------------------------------------------------------------

namespace {

constexpr int kRowLog = 8;
constexpr int kRow = 1 << kRowLog;  // 256
constexpr int kCols = 16;           // columns per CTA in the column pass
constexpr int kRowsPerCta = 16;     // rows per CTA in the row pass
constexpr int kRowPad = kRow + kRow / 16;  // padded row stride in shared memory

// High 64 bits of a * b from three of the four 32x32 partial products: the dropped low
// product and carries make it at most 2 below the exact value.
CKG_DEV uint64_t mulhi_approx(uint64_t a, uint64_t b) {
  const uint32_t a0 = (uint32_t)a, a1 = (uint32_t)(a >> 32), b0 = (uint32_t)b, b1 = (uint32_t)(b >> 32);
  const uint64_t mid = (uint64_t)__umulhi(a0, b1) + __umulhi(a1, b0);
  return (uint64_t)a1 * b1 + mid;
}

// Harvey butterfly. Exact form (any prime < 2^60): values in [0, 4q) between stages. LAZY
// form (primes below 2^57): the Shoup quotient comes from mulhi_approx, so t = w*y mod q
// lies in [0, 4q), and x is never brought back down: values grow by at most 4q per stage
// from [0, q), so all 16 stages of N = 2^16 stay below 65q < 2^64 and one reduction at the
// end suffices.
template <bool LAZY>
CKG_DEV void ct_bf(uint64_t& x, uint64_t& y, const ulonglong2 w, uint64_t q, uint64_t two_q) {
  if (LAZY) {
    const uint64_t t = y * w.x - mulhi_approx(y, w.y) * q;
    const uint64_t xr = x;
    x = xr + t;
    y = xr + 2 * two_q - t;
  } else {
    const uint64_t xr = csub(x, two_q);
    const uint64_t t = mul_shoup_lazy(y, w.x, w.y, q);
    x = xr + t;
    y = xr + two_q - t;
  }
}

// Primes below this bound take the lazy forward path.
constexpr uint64_t kLazyBound = 1ULL << 57;

CKG_DEV void gs_bf(uint64_t& x, uint64_t& y, const ulonglong2 w, uint64_t q, uint64_t two_q) {
  uint64_t s = x + y;
  uint64_t d = x + two_q - y;
  x = csub(s, two_q);
  y = mul_shoup_lazy(d, w.x, w.y, q);
}

CKG_DEV ulonglong2 ldtw(const ulonglong2* t, uint32_t i) { return __ldg(t + i); }

CKG_DEV int pad_idx(int k) { return k + (k >> 4); }

// FP64 butterflies for primes below 2^50, on the FP64 pipe instead of IMAD. Values are exact
// integers held in doubles, signed and lazy (bounds at mulmod_f64 and ct_bf_f64 / gs_bf_f64).
// w*y mod q: hi = fl(w y) and lo = fma(w, y, -hi) hold the exact product; k = rint(hi / q) by the
// native rounding instruction; fma(-k, q, hi) + lo = w y - k q is then an integer below 2^53 in
// magnitude and every step is exact. Inputs and outputs of a transform are canonical u64; between
// its two passes the limb holds the raw doubles.
constexpr uint64_t kF64Bound = 1ULL << 50;
constexpr double kTwo52 = 4503599627370496.0;

CKG_DEV double f64_of(uint64_t x) {  // exact for x < 2^52
  return __dsub_rn(__longlong_as_double((long long)(x | 0x4330000000000000ULL)), kTwo52);
}
CKG_DEV uint64_t u64_of(double v) {  // v an integer in [0, 2^52)
  return (uint64_t)__double_as_longlong(__dadd_rn(v, kTwo52)) & 0xFFFFFFFFFFFFFULL;
}
CKG_DEV double bits_dbl(uint64_t v) { return __longlong_as_double((long long)v); }
CKG_DEV uint64_t dbl_bits(double v) { return (uint64_t)__double_as_longlong(v); }
CKG_DEV double rint_f64(double v) { return rint(v); }  // round to nearest integer (|v| < 2^51 here)

// w y mod q, signed and exact, for |y| < 8q, 0 <= w < q < 2^50: |w y / q| < 2^53 and the
// rounded quotient is within 0.5 + 3 |y| 2^-53 of it, so the result lies in (-3.5q, 3.5q),
// and |hi - k q| + |lo| < 2^53 keeps every step exact.
CKG_DEV double mulmod_f64(double y, double w, double q, double qinv) {
  const double hi = __dmul_rn(y, w);
  const double lo = __fma_rn(y, w, -hi);
  const double k = rint_f64(__dmul_rn(hi, qinv));
  return __dadd_rn(__fma_rn(-k, q, hi), lo);
}
// x - q rint(x / q): |x| < 8q -> |result| <= q/2 + 1.
CKG_DEV double red_f64(double x, double q, double qinv) { return __fma_rn(-rint_f64(__dmul_rn(x, qinv)), q, x); }
CKG_DEV uint64_t canon_u64(double x, double q, double qinv) {
  const double r = red_f64(x, q, qinv);
  return u64_of(r < 0.0 ? __dadd_rn(r, q) : r);
}
// Cooley-Tukey. With RED the additive input is first reduced to [-q/2, q/2]; the passes set
// RED on every other stage. With |t| <= (0.5 + 0.375 |y|/q) q (q < 2^50), a RED stage after
// inputs below b q gives outputs below (1 + 0.375 b) q and a plain stage after inputs below
// a q gives (1.375 a + 0.5) q: the pair settles at a = 2.45, b = 3.87, so every value stays
// below 3.9q, inside the 8q that mulmod_f64 and red_f64 accept.
template <bool RED>
CKG_DEV void ct_bf_f64(double& x, double& y, double w, double q, double qinv) {
  const double t = mulmod_f64(y, w, q, qinv);
  const double xr = RED ? red_f64(x, q, qinv) : x;
  x = __dadd_rn(xr, t);
  y = __dsub_rn(xr, t);
}
// Gentleman-Sande: the sum is reduced, the difference multiplied. From inputs below c q the
// outputs stay below q/2 + 1 and (0.5 + 0.75 c) q, which settles at c = 2: values below 2q,
// differences below 4q.
CKG_DEV void gs_bf_f64(double& x, double& y, double w, double q, double qinv) {
  const double s = __dadd_rn(x, y), d = __dsub_rn(x, y);
  x = red_f64(s, q, qinv);
  y = mulmod_f64(d, w, q, qinv);
}

// The centred lift of x in [0, ql) to prime q: x when x <= (ql - 1) / 2, else x - ql, reduced
// mod q (one_s = floor(2^64 / q)). It equals the one-source exact base conversion of the rescale
// (x + h mod ql, lifted, minus h with h = (ql - 1) / 2; crates/ckks-train-core/src/baseconv.rs:258-291).
CKG_DEV uint64_t centred_lift(uint64_t x, uint64_t ql, uint64_t q, uint64_t one_s) {
  const bool neg = x > (ql >> 1);
  const uint64_t m = neg ? ql - x : x;
  const uint64_t r = csub(mul_shoup_lazy(m, 1, one_s, q), q);
  return neg && r ? q - r : r;
}

// Forward column pass: stages 0..LOGS-1 on 2^LOGS-point columns (stride 256).
// Column block `cb` (columns cb * 16 ..); with `tile` the input columns are read from that
// shared-memory copy ([row][16] words, the same buffer as `sm`) instead of ref.src: every thread
// writes its exchange words where it read its inputs, so no barrier is needed between the two.
template <int LOGS, bool LAZY>
CKG_DEV void fwd_cols_body(const LimbRef& ref, uint64_t q, const ulonglong2* roots, uint64_t* sm, uint64_t lift_q,
                           uint64_t one_s, int cb, const uint64_t* tile) {
  constexpr int E1 = (LOGS + 1) / 2, E2 = LOGS / 2, TPS = 1 << E2, V = 1 << (E1 - E2);
  const uint64_t two_q = 2 * q;
  const int c = threadIdx.x % kCols, ts = threadIdx.x / kCols;
  const int col = cb * kCols + c;
  uint64_t x[1 << E1];
#pragma unroll
  for (int j = 0; j < (1 << E1); ++j)
    x[j] = tile ? tile[(ts + TPS * j) * kCols + c] : ref.src[col + (size_t)kRow * (ts + TPS * j)];
  if (lift_q) {
#pragma unroll
    for (int j = 0; j < (1 << E1); ++j) x[j] = centred_lift(x[j], lift_q, q, one_s);
  }
#pragma unroll
  for (int r = 0; r < E1; ++r) {
    const int half = 1 << (E1 - 1 - r);
#pragma unroll
    for (int j = 0; j < (1 << E1); ++j)
      if (!(j & half)) ct_bf<LAZY>(x[j], x[j + half], ldtw(roots, (1u << r) + (j >> (E1 - r))), q, two_q);
  }
#pragma unroll
  for (int j = 0; j < (1 << E1); ++j) sm[(ts + TPS * j) * kCols + c] = x[j];
  __syncthreads();
#pragma unroll
  for (int v = 0; v < V; ++v) {
    const int t2 = ts + TPS * v;
    uint64_t y[1 << E2];
#pragma unroll
    for (int j = 0; j < (1 << E2); ++j) y[j] = sm[((t2 << E2) + j) * kCols + c];
#pragma unroll
    for (int r = E1; r < LOGS; ++r) {
      const int half = 1 << (LOGS - 1 - r);
#pragma unroll
      for (int j = 0; j < (1 << E2); ++j)
        if (!(j & half)) {
          const int k = (t2 << E2) + j;
          ct_bf<LAZY>(y[j], y[j + half], ldtw(roots, (1u << r) + (k >> (LOGS - r))), q, two_q);
        }
    }
#pragma unroll
    for (int j = 0; j < (1 << E2); ++j) ref.dst[col + (size_t)kRow * ((t2 << E2) + j)] = y[j];
  }
}

// The same pass with FP64 butterflies; writes the raw doubles for the row pass.
template <int LOGS>
CKG_DEV void fwd_cols_body_f64(const LimbRef& ref, const PrimeConst* P, const double* roots, uint64_t* sm,
                               uint64_t lift_q, int cb, const uint64_t* tile) {
  constexpr int E1 = (LOGS + 1) / 2, E2 = LOGS / 2, TPS = 1 << E2, V = 1 << (E1 - E2);
  const double q = __ldg(&P->qd), qinv = __ldg(&P->qinv);
  const int c = threadIdx.x % kCols, ts = threadIdx.x / kCols;
  const int col = cb * kCols + c;
  double x[1 << E1];
  auto in = [&](int j) { return tile ? tile[(ts + TPS * j) * kCols + c] : ref.src[col + (size_t)kRow * (ts + TPS * j)]; };
  if (lift_q) {
    const uint64_t qi = __ldg(&P->q), one_s = __ldg(&P->one_s);
#pragma unroll
    for (int j = 0; j < (1 << E1); ++j) x[j] = f64_of(centred_lift(in(j), lift_q, qi, one_s));
  } else {
#pragma unroll
    for (int j = 0; j < (1 << E1); ++j) x[j] = f64_of(in(j));
  }
#pragma unroll
  for (int r = 0; r < E1; ++r) {
    const int half = 1 << (E1 - 1 - r);
#pragma unroll
    for (int j = 0; j < (1 << E1); ++j)
      if (!(j & half)) {
        if (r % 2 == 0) ct_bf_f64<true>(x[j], x[j + half], __ldg(roots + (1u << r) + (j >> (E1 - r))), q, qinv);
        else ct_bf_f64<false>(x[j], x[j + half], __ldg(roots + (1u << r) + (j >> (E1 - r))), q, qinv);
      }
  }
#pragma unroll
  for (int j = 0; j < (1 << E1); ++j) sm[(ts + TPS * j) * kCols + c] = dbl_bits(x[j]);
  __syncthreads();
#pragma unroll
  for (int v = 0; v < V; ++v) {
    const int t2 = ts + TPS * v;
    double y[1 << E2];
#pragma unroll
    for (int j = 0; j < (1 << E2); ++j) y[j] = bits_dbl(sm[((t2 << E2) + j) * kCols + c]);
#pragma unroll
    for (int r = E1; r < LOGS; ++r) {
      const int half = 1 << (LOGS - 1 - r);
#pragma unroll
      for (int j = 0; j < (1 << E2); ++j)
        if (!(j & half)) {
          const int k = (t2 << E2) + j;
          if (r % 2 == 0) ct_bf_f64<true>(y[j], y[j + half], __ldg(roots + (1u << r) + (k >> (LOGS - r))), q, qinv);
          else ct_bf_f64<false>(y[j], y[j + half], __ldg(roots + (1u << r) + (k >> (LOGS - r))), q, qinv);
        }
    }
#pragma unroll
    for (int j = 0; j < (1 << E2); ++j) ref.dst[col + (size_t)kRow * ((t2 << E2) + j)] = dbl_bits(y[j]);
  }
}

template <int LOGS, class B>
__global__ void __launch_bounds__(kCols * (1 << (LOGS / 2)), LOGS <= 8 ? 4 : 1)
    k_ntt_fwd_cols(const __grid_constant__ B b, const PrimeConst* __restrict__ pc,
                   const ulonglong2* __restrict__ tw, const double* __restrict__ twd, int log_n, int in_place) {
  extern __shared__ uint64_t sm[];  // [2^LOGS][kCols]
  LimbRef ref = b.r[blockIdx.y];
  // aux = p + 1: src is a limb of prime p in coefficient form, read through its centred lift
  // (the rescale's one-source conversion fused into the load; never in place).
  const uint64_t lift_q = ref.aux ? __ldg(&pc[ref.aux - 1].q) : 0;
  if (in_place && !ref.aux) ref.src = ref.dst;
  const uint64_t q = __ldg(&pc[ref.prime].q);
  if (q < kF64Bound) {
    fwd_cols_body_f64<LOGS>(ref, pc + ref.prime, twd + ((size_t)ref.prime << log_n), sm, lift_q, blockIdx.x, nullptr);
    return;
  }
  const ulonglong2* roots = tw + ((size_t)ref.prime << log_n);
  const uint64_t one_s = __ldg(&pc[ref.prime].one_s);
  if (q < kLazyBound) fwd_cols_body<LOGS, true>(ref, q, roots, sm, lift_q, one_s, blockIdx.x, nullptr);
  else fwd_cols_body<LOGS, false>(ref, q, roots, sm, lift_q, one_s, blockIdx.x, nullptr);
}

// Forward row pass: stages s0..s0+7 (s0 = logN - 8) on 256-point rows, final reduction.
// `store(i, col, v)` receives the reduced value of row (CTA row i, column col).
template <bool LAZY, class Store>
CKG_DEV void fwd_rows_body(const uint64_t* base, const PrimeConst* P, const ulonglong2* roots, int log_n,
                           uint64_t* sm, Store store) {
  const uint64_t q = __ldg(&P->q), two_q = 2 * q;
  const int s0 = log_n - kRowLog;
  const int t = threadIdx.x % 16, rr = threadIdx.x / 16;
  const uint32_t row = blockIdx.x * kRowsPerCta + rr;
  const uint64_t* src = base + (size_t)row * kRow;
  uint64_t x[16];
#pragma unroll
  for (int j = 0; j < 16; ++j) x[j] = src[t + 16 * j];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int half = 1 << (3 - r);
#pragma unroll
    for (int j = 0; j < 16; ++j)
      if (!(j & half))
        ct_bf<LAZY>(x[j], x[j + half], ldtw(roots, (1u << (s0 + r)) + (row << r) + (j >> (4 - r))), q, two_q);
  }
  uint64_t* srow = sm + rr * kRowPad;
#pragma unroll
  for (int j = 0; j < 16; ++j) srow[pad_idx(t + 16 * j)] = x[j];
  __syncwarp();
  // A row's 16 threads form half a warp, so the exchange only needs a warp barrier.
#pragma unroll
  for (int j = 0; j < 16; ++j) x[j] = srow[pad_idx(16 * t + j)];
#pragma unroll
  for (int r = 4; r < 8; ++r) {
    const int half = 1 << (7 - r);
#pragma unroll
    for (int j = 0; j < 16; ++j)
      if (!(j & half)) {
        const int k = 16 * t + j;
        ct_bf<LAZY>(x[j], x[j + half], ldtw(roots, (1u << (s0 + r)) + (row << r) + (k >> (8 - r))), q, two_q);
      }
  }
  if (LAZY) {
    const uint64_t one_s = __ldg(&P->one_s);
#pragma unroll
    for (int j = 0; j < 16; ++j) srow[pad_idx(16 * t + j)] = csub(mul_shoup_lazy(x[j], 1, one_s, q), q);
  } else {
#pragma unroll
    for (int j = 0; j < 16; ++j) srow[pad_idx(16 * t + j)] = csub(csub(x[j], two_q), q);
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < kRowsPerCta; ++i) store(i, threadIdx.x, sm[i * kRowPad + pad_idx(threadIdx.x)]);
}

// The row pass with FP64 butterflies over the raw doubles of the FP64 column pass.
template <class Store>
CKG_DEV void fwd_rows_body_f64(const uint64_t* base, const PrimeConst* P, const double* roots, int log_n,
                               uint64_t* sm, Store store) {
  const double q = __ldg(&P->qd), qinv = __ldg(&P->qinv);
  const int s0 = log_n - kRowLog;
  const int t = threadIdx.x % 16, rr = threadIdx.x / 16;
  const uint32_t row = blockIdx.x * kRowsPerCta + rr;
  const uint64_t* src = base + (size_t)row * kRow;
  double x[16];
#pragma unroll
  for (int j = 0; j < 16; ++j) x[j] = bits_dbl(src[t + 16 * j]);
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int half = 1 << (3 - r);
#pragma unroll
    for (int j = 0; j < 16; ++j)
      if (!(j & half))
        if (r % 2 == 0) ct_bf_f64<true>(x[j], x[j + half], __ldg(roots + (1u << (s0 + r)) + (row << r) + (j >> (4 - r))), q, qinv);
        else ct_bf_f64<false>(x[j], x[j + half], __ldg(roots + (1u << (s0 + r)) + (row << r) + (j >> (4 - r))), q, qinv);
  }
  uint64_t* srow = sm + rr * kRowPad;
#pragma unroll
  for (int j = 0; j < 16; ++j) srow[pad_idx(t + 16 * j)] = dbl_bits(x[j]);
  __syncwarp();
#pragma unroll
  for (int j = 0; j < 16; ++j) x[j] = bits_dbl(srow[pad_idx(16 * t + j)]);
#pragma unroll
  for (int r = 4; r < 8; ++r) {
    const int half = 1 << (7 - r);
#pragma unroll
    for (int j = 0; j < 16; ++j)
      if (!(j & half)) {
        const int k = 16 * t + j;
        if (r % 2 == 0) ct_bf_f64<true>(x[j], x[j + half], __ldg(roots + (1u << (s0 + r)) + (row << r) + (k >> (8 - r))), q, qinv);
        else ct_bf_f64<false>(x[j], x[j + half], __ldg(roots + (1u << (s0 + r)) + (row << r) + (k >> (8 - r))), q, qinv);
      }
  }
#pragma unroll
  for (int j = 0; j < 16; ++j) srow[pad_idx(16 * t + j)] = canon_u64(x[j], q, qinv);
  __syncthreads();
#pragma unroll
  for (int i = 0; i < kRowsPerCta; ++i) store(i, threadIdx.x, sm[i * kRowPad + pad_idx(threadIdx.x)]);
}

template <class B>
__global__ void __launch_bounds__(256, 4)
    k_ntt_fwd_rows(const __grid_constant__ B b, const PrimeConst* __restrict__ pc,
                   const ulonglong2* __restrict__ tw, const double* __restrict__ twd, int log_n, int in_place) {
  __shared__ uint64_t sm[kRowsPerCta * kRowPad];
  const LimbRef ref = b.r[blockIdx.y];
  const uint64_t* src = in_place ? ref.dst : ref.src;
  const PrimeConst* P = pc + ref.prime;
  uint64_t* dst = ref.dst + (size_t)blockIdx.x * kRowsPerCta * kRow;
  auto store = [&](int i, int col, uint64_t v) { dst[i * kRow + col] = v; };
  const uint64_t q = __ldg(&P->q);
  if (q < kF64Bound) {
    fwd_rows_body_f64(src, P, twd + ((size_t)ref.prime << log_n), log_n, sm, store);
    return;
  }
  const ulonglong2* roots = tw + ((size_t)ref.prime << log_n);
  if (q < kLazyBound) fwd_rows_body<true>(src, P, roots, log_n, sm, store);
  else fwd_rows_body<false>(src, P, roots, log_n, sm, store);
}

// The row pass of the forward NTT of t (its column pass already run in place) fused with
// the ModDown / rescale finish: out = (x - NTT(t)) * c (+ add[perm]), so NTT(t) is never
// written back (crates/ckks-train-core/src/baseconv.rs:286-289, 505-510).
template <class B>
__global__ void __launch_bounds__(256, 4)
    k_ntt_fwd_rows_finish(const __grid_constant__ B fb, const PrimeConst* __restrict__ pc,
                          const ulonglong2* __restrict__ tw, const double* __restrict__ twd, int log_n) {
  __shared__ uint64_t sm[kRowsPerCta * kRowPad];
  const FinRef& r = fb.r[blockIdx.y];
  const PrimeConst* P = pc + r.prime;
  const uint64_t q = __ldg(&P->q);
  const ulonglong2* roots = tw + ((size_t)r.prime << log_n);
  const size_t base = (size_t)blockIdx.x * kRowsPerCta * kRow;
  auto keep = [](int, int, uint64_t) {};  // the transformed rows stay in shared memory
  if (q < kF64Bound) fwd_rows_body_f64(r.t, P, twd + ((size_t)r.prime << log_n), log_n, sm, keep);
  else if (q < kLazyBound) fwd_rows_body<true>(r.t, P, roots, log_n, sm, keep);
  else fwd_rows_body<false>(r.t, P, roots, log_n, sm, keep);
  // Finish, 8 rows at a time so their loads (x, the permutation, the gathered addend) are in
  // flight together; x, add and perm are only read here and `out` is a separate buffer.
  const uint64_t* __restrict__ xs = r.x;
  const uint64_t* __restrict__ adds = r.add;
  const uint32_t* __restrict__ pm = r.add_perm;
  uint64_t* __restrict__ outp = r.out;
  const uint64_t c = r.c, c_s = r.c_s;
  const int col = threadIdx.x;
#pragma unroll
  for (int h = 0; h < kRowsPerCta; h += 8) {
    uint64_t xv[8], av[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) xv[i] = __ldg(xs + base + (h + i) * kRow + col);
    if (adds) {
      if (pm) {
        uint32_t pv[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) pv[i] = __ldg(pm + base + (h + i) * kRow + col);
#pragma unroll
        for (int i = 0; i < 8; ++i) av[i] = __ldg(adds + pv[i]);
      } else {
#pragma unroll
        for (int i = 0; i < 8; ++i) av[i] = __ldg(adds + base + (h + i) * kRow + col);
      }
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const uint64_t v = sm[(h + i) * kRowPad + pad_idx(col)];
      uint64_t o = mul_shoup(sub_mod(xv[i], v, q), c, c_s, q);
      if (adds) o = add_mod(o, av[i], q);
      outp[base + (h + i) * kRow + col] = o;
    }
  }
}

// 8-byte asynchronous global -> shared copy (cp.async, no register staging) and the wait for
// all of this thread's copies.
CKG_DEV void cp_async8(void* smem, const void* gmem) {
  const uint32_t sa = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(sa), "l"(gmem) : "memory");
}
CKG_DEV void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

// Inverse row pass with FP64 butterflies: canonical input, raw doubles out.
CKG_DEV void inv_rows_body_f64(const LimbRef& ref, const PrimeConst* P, const double* roots, int log_n,
                               uint64_t* sm) {
  const double q = __ldg(&P->qd), qinv = __ldg(&P->qinv);
  const int t = threadIdx.x % 16, rr = threadIdx.x / 16;
  const uint32_t row = blockIdx.x * kRowsPerCta + rr;
  uint64_t* srow = sm + rr * kRowPad;
  double x[16];
#pragma unroll
  for (int j = 0; j < 16; ++j) x[j] = f64_of(srow[pad_idx(16 * t + j)]);
  // The row's words are in registers: its shared-memory slot now takes the twiddles of stages
  // 0-3, 128 >> u words for stage u at [256 - (256 >> u), ...), loaded in one batch of 15 per
  // thread instead of one dependent round of global loads per stage; tw_idx spreads each stage's
  // stride-(8 >> u) reads over the banks.
  // The copies are asynchronous (cp.async), so they hold no registers while in flight.
  auto tw_idx = [](int w) { return w + (w >> 3); };  // < 272 for w < 240
  __syncwarp();
#pragma unroll
  for (int i = 0; i < 15; ++i) {
    const int u = i < 8 ? 0 : i < 12 ? 1 : i < 14 ? 2 : 3;
    const int w = t + 16 * i, m = w - (256 - (256 >> u));
    cp_async8(srow + tw_idx(w), roots + (1u << (log_n - 1 - u)) + (row << (7 - u)) + m);
  }
  cp_async_wait_all();
  __syncwarp();
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    const int d = 1 << u;
#pragma unroll
    for (int j = 0; j < 16; ++j)
      if (!(j & d)) {
        const uint32_t k = 16 * t + j;
        const double w = bits_dbl(srow[tw_idx((256 - (256 >> u)) + (k >> (u + 1)))]);
        gs_bf_f64(x[j], x[j + d], w, q, qinv);
      }
  }
  __syncwarp();  // every thread of the row has read its twiddles
#pragma unroll
  for (int j = 0; j < 16; ++j) srow[pad_idx(16 * t + j)] = dbl_bits(x[j]);
  __syncwarp();
#pragma unroll
  for (int j = 0; j < 16; ++j) x[j] = bits_dbl(srow[pad_idx(t + 16 * j)]);
#pragma unroll
  for (int u = 4; u < 8; ++u) {
    const int d = 1 << (u - 4);
#pragma unroll
    for (int j = 0; j < 16; ++j)
      if (!(j & d)) {
        const uint32_t k = t + 16 * j;
        const uint32_t h = 1u << (log_n - 1 - u);
        gs_bf_f64(x[j], x[j + d], __ldg(roots + h + (row << (7 - u)) + (k >> (u + 1))), q, qinv);
      }
  }
  uint64_t* dst = ref.dst + (size_t)row * kRow;
#pragma unroll
  for (int j = 0; j < 16; ++j) dst[t + 16 * j] = dbl_bits(x[j]);
}

// Inverse row pass: GS stages u = 0..7 (pair distance 2^u) within 256-point rows.
template <class B>
__global__ void __launch_bounds__(256, 4)
    k_ntt_inv_rows(const __grid_constant__ B b, const PrimeConst* __restrict__ pc,
                   const ulonglong2* __restrict__ tw, const double* __restrict__ twd, int log_n, int in_place) {
  __shared__ uint64_t sm[kRowsPerCta * kRowPad];
  LimbRef ref = b.r[blockIdx.y];
  if (in_place) ref.src = ref.dst;
  const uint64_t q = __ldg(&pc[ref.prime].q), two_q = 2 * q;
  const ulonglong2* roots = tw + ((size_t)ref.prime << log_n);
  const uint64_t* src = ref.src + (size_t)blockIdx.x * kRowsPerCta * kRow;
#pragma unroll
  for (int i = 0; i < kRowsPerCta; ++i) sm[i * kRowPad + pad_idx(threadIdx.x)] = src[i * kRow + threadIdx.x];
  __syncthreads();
  if (q < kF64Bound) {
    inv_rows_body_f64(ref, pc + ref.prime, twd + ((size_t)ref.prime << log_n), log_n, sm);
    return;
  }
  const int t = threadIdx.x % 16, rr = threadIdx.x / 16;
  const uint32_t row = blockIdx.x * kRowsPerCta + rr;
  uint64_t* srow = sm + rr * kRowPad;
  uint64_t x[16];
#pragma unroll
  for (int j = 0; j < 16; ++j) x[j] = srow[pad_idx(16 * t + j)];
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    const int d = 1 << u;
#pragma unroll
    for (int j = 0; j < 16; ++j)
      if (!(j & d)) {
        const uint32_t k = 16 * t + j;
        const uint32_t h = 1u << (log_n - 1 - u);
        gs_bf(x[j], x[j + d], ldtw(roots, h + (row << (7 - u)) + (k >> (u + 1))), q, two_q);
      }
  }
#pragma unroll
  for (int j = 0; j < 16; ++j) srow[pad_idx(16 * t + j)] = x[j];
  __syncwarp();
#pragma unroll
  for (int j = 0; j < 16; ++j) x[j] = srow[pad_idx(t + 16 * j)];
#pragma unroll
  for (int u = 4; u < 8; ++u) {
    const int d = 1 << (u - 4);
#pragma unroll
    for (int j = 0; j < 16; ++j)
      if (!(j & d)) {
        const uint32_t k = t + 16 * j;
        const uint32_t h = 1u << (log_n - 1 - u);
        gs_bf(x[j], x[j + d], ldtw(roots, h + (row << (7 - u)) + (k >> (u + 1))), q, two_q);
      }
  }
  uint64_t* dst = ref.dst + (size_t)row * kRow;
#pragma unroll
  for (int j = 0; j < 16; ++j) dst[t + 16 * j] = x[j];
}

// Inverse column pass: GS stages u = 8..logN-1 on 2^LOGS-point columns, N^-1 fused into
// the last stage, output in [0, q).
// Inverse column pass with FP64 butterflies over the raw doubles of the row pass; N^-1 in
// the last stage, canonical output.
template <int LOGS>
CKG_DEV void inv_cols_body_f64(const LimbRef& ref, const PrimeConst* P, const double* roots, uint64_t* sm, int cb,
                               const uint64_t* tile) {
  constexpr int F1 = (LOGS + 1) / 2, F2 = LOGS / 2, TPS = 1 << F2, V = 1 << (F1 - F2);
  const double q = __ldg(&P->qd), qinv = __ldg(&P->qinv);
  const int c = threadIdx.x % kCols, ts = threadIdx.x / kCols;
  const int col = cb * kCols + c;
  double x[1 << F1];
#pragma unroll
  for (int j = 0; j < (1 << F1); ++j)
    x[j] = bits_dbl(tile ? tile[((ts << F1) + j) * kCols + c] : ref.src[col + (size_t)kRow * ((ts << F1) + j)]);
#pragma unroll
  for (int v = 0; v < F1; ++v) {
    const int d = 1 << v;
#pragma unroll
    for (int j = 0; j < (1 << F1); ++j)
      if (!(j & d)) {
        const uint32_t k = (ts << F1) + j;
        gs_bf_f64(x[j], x[j + d], __ldg(roots + (1u << (LOGS - 1 - v)) + (k >> (v + 1))), q, qinv);
      }
  }
#pragma unroll
  for (int j = 0; j < (1 << F1); ++j) sm[((ts << F1) + j) * kCols + c] = dbl_bits(x[j]);
  __syncthreads();
  const double ninv = __ldg(&P->ninvd), wninv = __ldg(&P->wninvd);
#pragma unroll
  for (int vv = 0; vv < V; ++vv) {
    const int t2 = ts + TPS * vv;
    double y[1 << F2];
#pragma unroll
    for (int j = 0; j < (1 << F2); ++j) y[j] = bits_dbl(sm[(t2 + (j << F1)) * kCols + c]);
#pragma unroll
    for (int v = F1; v < LOGS - 1; ++v) {
      const int d = 1 << (v - F1);
#pragma unroll
      for (int j = 0; j < (1 << F2); ++j)
        if (!(j & d)) {
          const uint32_t k = t2 + (j << F1);
          gs_bf_f64(y[j], y[j + d], __ldg(roots + (1u << (LOGS - 1 - v)) + (k >> (v + 1))), q, qinv);
        }
    }
    uint64_t out[1 << F2];
    {  // last stage: pairs (k, k + 2^(LOGS-1)), times N^-1
      const int d = 1 << (F2 - 1);
#pragma unroll
      for (int j = 0; j < (1 << F2); ++j)
        if (!(j & d)) {
          out[j] = canon_u64(mulmod_f64(__dadd_rn(y[j], y[j + d]), ninv, q, qinv), q, qinv);
          out[j + d] = canon_u64(mulmod_f64(__dsub_rn(y[j], y[j + d]), wninv, q, qinv), q, qinv);
        }
    }
#pragma unroll
    for (int j = 0; j < (1 << F2); ++j) ref.dst[col + (size_t)kRow * (t2 + (j << F1))] = out[j];
  }
}

// The inverse column pass with integer butterflies (primes from 2^50 on).
template <int LOGS>
CKG_DEV void inv_cols_body(const LimbRef& ref, const PrimeConst* P, const ulonglong2* roots, uint64_t* sm, int cb,
                           const uint64_t* tile) {
  constexpr int F1 = (LOGS + 1) / 2, F2 = LOGS / 2, TPS = 1 << F2, V = 1 << (F1 - F2);
  const uint64_t q = __ldg(&P->q), two_q = 2 * q;
  const int c = threadIdx.x % kCols, ts = threadIdx.x / kCols;
  const int col = cb * kCols + c;
  uint64_t x[1 << F1];
#pragma unroll
  for (int j = 0; j < (1 << F1); ++j)
    x[j] = tile ? tile[((ts << F1) + j) * kCols + c] : ref.src[col + (size_t)kRow * ((ts << F1) + j)];
  // local stage v: pair distance 2^v, twiddle index 2^(LOGS-1-v) + (k >> (v+1))
#pragma unroll
  for (int v = 0; v < F1; ++v) {
    const int d = 1 << v;
#pragma unroll
    for (int j = 0; j < (1 << F1); ++j)
      if (!(j & d)) {
        const uint32_t k = (ts << F1) + j;
        gs_bf(x[j], x[j + d], ldtw(roots, (1u << (LOGS - 1 - v)) + (k >> (v + 1))), q, two_q);
      }
  }
#pragma unroll
  for (int j = 0; j < (1 << F1); ++j) sm[((ts << F1) + j) * kCols + c] = x[j];
  __syncthreads();
  const uint64_t ninv = __ldg(&P->ninv), ninv_s = __ldg(&P->ninv_s);
  const uint64_t wninv = __ldg(&P->wninv), wninv_s = __ldg(&P->wninv_s);
#pragma unroll
  for (int vv = 0; vv < V; ++vv) {
    const int t2 = ts + TPS * vv;
    uint64_t y[1 << F2];
#pragma unroll
    for (int j = 0; j < (1 << F2); ++j) y[j] = sm[(t2 + (j << F1)) * kCols + c];
#pragma unroll
    for (int v = F1; v < LOGS - 1; ++v) {
      const int d = 1 << (v - F1);
#pragma unroll
      for (int j = 0; j < (1 << F2); ++j)
        if (!(j & d)) {
          const uint32_t k = t2 + (j << F1);
          gs_bf(y[j], y[j + d], ldtw(roots, (1u << (LOGS - 1 - v)) + (k >> (v + 1))), q, two_q);
        }
    }
    {  // last stage: pairs (k, k + 2^(LOGS-1)), times N^-1
      const int d = 1 << (F2 - 1);
#pragma unroll
      for (int j = 0; j < (1 << F2); ++j)
        if (!(j & d)) {
          uint64_t s = y[j] + y[j + d], df = y[j] + two_q - y[j + d];
          y[j] = csub(mul_shoup_lazy(s, ninv, ninv_s, q), q);
          y[j + d] = csub(mul_shoup_lazy(df, wninv, wninv_s, q), q);
        }
    }
#pragma unroll
    for (int j = 0; j < (1 << F2); ++j) ref.dst[col + (size_t)kRow * (t2 + (j << F1))] = y[j];
  }
}

template <int LOGS, class B>
__global__ void __launch_bounds__(kCols * (1 << (LOGS / 2)), LOGS <= 8 ? 4 : 1)
    k_ntt_inv_cols(const __grid_constant__ B b, const PrimeConst* __restrict__ pc,
                   const ulonglong2* __restrict__ tw, const double* __restrict__ twd, int log_n, int in_place) {
  extern __shared__ uint64_t sm[];  // [2^LOGS][kCols]
  LimbRef ref = b.r[blockIdx.y];
  if (in_place) ref.src = ref.dst;
  const PrimeConst* P = pc + ref.prime;
  if (__ldg(&P->q) < kF64Bound) inv_cols_body_f64<LOGS>(ref, P, twd + ((size_t)ref.prime << log_n), sm, blockIdx.x, nullptr);
  else inv_cols_body<LOGS>(ref, P, tw + ((size_t)ref.prime << log_n), sm, blockIdx.x, nullptr);
}

// ------------------------------------------------------------------------------------
// Persistent column passes with TMA staging. Each CTA walks the list's (limb, column block)
// tiles with a stride of the grid. A tile (2^LOGS rows of 16 words, 128 bytes apart from row to
// row by 2 KB) is one box of a 3-D tensor map over the list's region (256 columns x 2^LOGS rows x
// limbs, a limb being N words): a single cp.async.bulk.tensor copy brings it into shared memory,
// completing on the stage's mbarrier, two stages deep, so the next tile is in flight while one is
// transformed and a stage is refilled as soon as its tile is done. The stage buffer is also the
// pass's exchange buffer. Waits are bounded (about a second of clock): on timeout the kernel
// records a fault (g_ntt_fault = 1), drains its copies (bounded) and returns; a limb outside the
// map's region is not copied and records fault 3 (the host checks every list first).
// ------------------------------------------------------------------------------------

__device__ int g_ntt_fault;

CKG_DEV uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
CKG_DEV void mbar_init1(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
}
CKG_DEV bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  const long long t0 = clock64();
  for (;;) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (ok) return true;
    if (clock64() - t0 > (2LL << 30)) {
      atomicExch(&g_ntt_fault, 1);
      return false;
    }
  }
}
CKG_DEV void mbar_expect(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// Box (x, y, z) of a 3-D tensor map into shared memory (no multicast).
CKG_DEV void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

template <int LOGS, bool INV, class B>
__global__ void __launch_bounds__(kCols * (1 << (LOGS / 2)), LOGS <= 8 ? 3 : 1)
    k_ntt_cols_tma(const __grid_constant__ B b, const __grid_constant__ CUtensorMap map, const uint64_t* base,
                   uint64_t region_limbs, const PrimeConst* __restrict__ pc, const ulonglong2* __restrict__ tw,
                   const double* __restrict__ twd, int log_n, int in_place, int items) {
  constexpr int TILE = (1 << LOGS) * kCols;  // words per stage
  constexpr int NBLK = kRow / kCols;         // column blocks per limb
  extern __shared__ __align__(128) uint64_t smt[];
  uint64_t* bars = smt + 2 * TILE;
  __shared__ int stage_ok[2];
  auto source = [&](const LimbRef& r) -> const uint64_t* {
    return (INV ? in_place : (in_place && !r.aux)) ? r.dst : r.src;
  };
  auto issue = [&](int item, int s) {  // by one thread
    const uint64_t off = (uint64_t)(source(b.r[item / NBLK]) - base);
    const uint64_t z = off >> log_n;
    const bool ok = (off & ((1ull << log_n) - 1)) == 0 && z < region_limbs;
    stage_ok[s] = ok;
    if (!ok) atomicExch(&g_ntt_fault, 3);
    mbar_expect(&bars[s], ok ? TILE * 8 : 0);
    if (ok) tma_load_3d(smt + s * TILE, &map, (item % NBLK) * kCols, 0, (int)z, &bars[s]);
  };
  if (threadIdx.x == 0) {
    mbar_init1(&bars[0]);
    mbar_init1(&bars[1]);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  const int G = gridDim.x;
  int issued = 0;  // tiles issued by this CTA (thread 0's count)
  if (threadIdx.x == 0) {
    if ((int)blockIdx.x < items) issue(blockIdx.x, 0), ++issued;
    if ((int)blockIdx.x + G < items) issue(blockIdx.x + G, 1), ++issued;
  }
  int k = 0;
  for (int item = blockIdx.x; item < items; item += G, ++k) {
    const int s = k & 1;
    const bool ok = mbar_wait_bounded(&bars[s], (k >> 1) & 1);
    if (__syncthreads_or(!ok)) break;
    uint64_t* tile = smt + s * TILE;
    if (stage_ok[s]) {
      LimbRef ref = b.r[item / NBLK];
      ref.src = source(ref);
      const int cb = item % NBLK;
      const PrimeConst* P = pc + ref.prime;
      const uint64_t q = __ldg(&P->q);
      if (!INV) {
        const uint64_t lift_q = ref.aux ? __ldg(&pc[ref.aux - 1].q) : 0;
        if (q < kF64Bound) {
          fwd_cols_body_f64<LOGS>(ref, P, twd + ((size_t)ref.prime << log_n), tile, lift_q, cb, tile);
        } else {
          const ulonglong2* roots = tw + ((size_t)ref.prime << log_n);
          const uint64_t one_s = __ldg(&P->one_s);
          if (q < kLazyBound) fwd_cols_body<LOGS, true>(ref, q, roots, tile, lift_q, one_s, cb, tile);
          else fwd_cols_body<LOGS, false>(ref, q, roots, tile, lift_q, one_s, cb, tile);
        }
      } else {
        if (q < kF64Bound) inv_cols_body_f64<LOGS>(ref, P, twd + ((size_t)ref.prime << log_n), tile, cb, tile);
        else inv_cols_body<LOGS>(ref, P, tw + ((size_t)ref.prime << log_n), tile, cb, tile);
      }
    }
    // every thread is done with the stage; its exchange writes (generic proxy) are ordered
    // before the copy (async proxy) that refills it
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0 && item + 2 * G < items) issue(item + 2 * G, s), ++issued;
  }
  // After a timeout, copies issued for tiles not yet waited on may still be in flight: wait
  // for them (bounded) before the shared memory is released.
  if (threadIdx.x == 0)
    for (int kk = k; kk < issued; ++kk) mbar_wait_bounded(&bars[kk & 1], (kk >> 1) & 1);
}

// Small transforms (logN <= 11): one CTA per limb, the limb in shared memory, radix-2.
template <class B>
__global__ void k_ntt_small(const __grid_constant__ B b, const PrimeConst* __restrict__ pc,
                            const ulonglong2* __restrict__ twf, const ulonglong2* __restrict__ twi, int log_n,
                            int inverse) {
  extern __shared__ uint64_t sm[];
  const LimbRef ref = b.r[blockIdx.y];
  const PrimeConst* P = pc + ref.prime;
  const uint64_t q = __ldg(&P->q), two_q = 2 * q;
  const int n = 1 << log_n, half_n = n >> 1;
  for (int i = threadIdx.x; i < n; i += blockDim.x) sm[i] = ref.src[i];
  __syncthreads();
  if (!inverse) {
    const ulonglong2* roots = twf + ((size_t)ref.prime << log_n);
    for (int s = 0; s < log_n; ++s) {
      const int t = half_n >> s;
      for (int bf = threadIdx.x; bf < half_n; bf += blockDim.x) {
        const int g = bf / t, k = bf % t;
        const int i0 = 2 * t * g + k;
        ct_bf<false>(sm[i0], sm[i0 + t], ldtw(roots, (1u << s) + g), q, two_q);
      }
      __syncthreads();
    }
    for (int i = threadIdx.x; i < n; i += blockDim.x) ref.dst[i] = csub(csub(sm[i], two_q), q);
  } else {
    const ulonglong2* roots = twi + ((size_t)ref.prime << log_n);
    for (int u = 0; u < log_n - 1; ++u) {
      const int t = 1 << u;
      for (int bf = threadIdx.x; bf < half_n; bf += blockDim.x) {
        const int g = bf / t, k = bf % t;
        const int i0 = 2 * t * g + k;
        gs_bf(sm[i0], sm[i0 + t], ldtw(roots, (half_n >> u) + g), q, two_q);
      }
      __syncthreads();
    }
    const uint64_t ninv = __ldg(&P->ninv), ninv_s = __ldg(&P->ninv_s);
    const uint64_t wninv = __ldg(&P->wninv), wninv_s = __ldg(&P->wninv_s);
    for (int k = threadIdx.x; k < half_n; k += blockDim.x) {
      uint64_t x = sm[k], y = sm[k + half_n];
      ref.dst[k] = csub(mul_shoup_lazy(x + y, ninv, ninv_s, q), q);
      ref.dst[k + half_n] = csub(mul_shoup_lazy(x + two_q - y, wninv, wninv_s, q), q);
    }
  }
}

// ------------------------------------------------------------------------------------
// Base conversion (ModUp digit lift, ModDown P -> Q, rescale last-prime lift).
// Each thread converts two coefficients (c and c + 256). The source words are read once;
// y_j stays in registers split into 30-bit halves, so every product of a target's sum
// sum_j y_j w_tj is one 32x32->64 multiply-add into one of four 64-bit accumulators
// (A = lo*lo, B1 = lo*hi, B2 = hi*lo, C = hi*hi, each < 16 * 2^60), assembled into 128
// bits and reduced once. The target records (weights pre-split, reduction constants)
// are staged in shared memory. Exact conversion (n_src > 1) subtracts e * S with the f64
// estimate e = floor(sum_j f64(y_j) * f64(1/s_j)), each product and sum rounded to nearest
// in source order starting from the first product (crates/ckks-train-core/src/baseconv.rs:198-206).
// ------------------------------------------------------------------------------------

CKG_DEV void add128(uint64_t& hi, uint64_t& lo, uint64_t bhi, uint64_t blo) {
  asm("add.cc.u64 %0, %0, %2;\n\taddc.u64 %1, %1, %3;" : "+l"(lo), "+l"(hi) : "l"(blo), "l"(bhi));
}

// (hi, lo) mod q with the reduction constants of a target record.
CKG_DEV uint64_t reduce128_rec(uint64_t hi, uint64_t lo, const uint64_t* rec) {
  const uint64_t q = rec[3];
  const uint64_t a = csub(mul_shoup_lazy(hi, rec[4], rec[5], q), q);
  const uint64_t b = csub(mul_shoup_lazy(lo, 1, rec[6], q), q);
  return csub(a + b, q);
}

constexpr uint64_t kMask30 = (1ULL << 30) - 1;

// f64(v) rounded to nearest (ties to even), on the FP64 pipe: both 32-bit halves are exact
// doubles (2^52 + x - 2^52), and one FMA rounds hi 2^32 + lo once. Equal to __ull2double_rn.
CKG_DEV double u64_to_f64_rn(uint64_t v) {
  const double hi = __dsub_rn(__hiloint2double(0x43300000, (int)(uint32_t)(v >> 32)), 4503599627370496.0);
  const double lo = __dsub_rn(__hiloint2double(0x43300000, (int)(uint32_t)v), 4503599627370496.0);
  return __fma_rn(hi, 4294967296.0, lo);
}

// One pass over the sources, then every target record of the job's table. Each thread converts
// kBconvU coefficients (c, c + 256, ...). y_j = [(x_j + h_j) qhat_j^-1]_{s_j} stays in registers; the
// overflow estimate is e = floor(sum_j f64(y_j) f64(1/s_j)) (0 for one source). NS is the source
// count (1..8), or 0 for more sources, which have exact records only.
//
// FP64-assisted records (the first `head` of the table; the host admits a target only when the
// bound below holds): V = sum_j y_j w_tj + e (t - [S]_t) + (t - [h]_t) is summed mod 2^64 with
// 64-bit multiply-adds, its quotient by t is estimated by an FP64 FMA chain over f64(y_j) and
// f64(w_tj / t), and r = V - k t (k = rint of the estimate) is exact as a signed 64-bit value
// since |V / t - k| t <= 2^62. A second rounded quotient of f64(r) brings r into (-t, t)
// (records flagged two_stage), and one conditional add into [0, t).
//
// Exact records: y_j split into 30-bit halves, so every product is a 32x32->64 multiply-add
// into one of four 64-bit accumulators (A = lo*lo, B1 = lo*hi, B2 = hi*lo, C = hi*hi, each
// < 16 * 2^60), assembled into 128 bits and reduced once.
constexpr int kBconvU = 1;  // coefficients per thread (registers: one y_j per source each)

template <int NS, class B>
__global__ void __launch_bounds__(256)
    k_bconv(const __grid_constant__ B cb, const PrimeConst* __restrict__ pc, int n) {
  constexpr int K = NS > 0 ? NS : kMaxSrc;
  __shared__ uint64_t sd[kMaxDst * (8 + 2 * kMaxSrc)];
  const ConvJob& job = cb.j[blockIdx.y];
  const uint64_t* tab = job.table;
  const int head = (int)__ldg(tab);
  const int n_src = NS > 0 ? NS : cb.n_src;
  const int dw = ConvLayout::dst_words(n_src);
  const uint64_t* src_tab = tab + ConvLayout::kHeadWords;
  {
    const uint64_t* dtab = src_tab + ConvLayout::kSrcWords * n_src;
    for (int i = threadIdx.x; i < dw * job.n_dst; i += blockDim.x) sd[i] = __ldg(dtab + i);
  }
  constexpr int U = kBconvU;
  const int c0 = blockIdx.x * (256 * U) + threadIdx.x;
  bool ok[U];
#pragma unroll
  for (int u = 0; u < U; ++u) ok[u] = c0 + 256 * u < n;
  uint64_t y[U][K];
  uint64_t e[U];
  {
    double f[U];
#pragma unroll
    for (int j = 0; j < K; ++j) {
      if (j < n_src) {
        const uint64_t* s = src_tab + ConvLayout::kSrcWords * j;
        const uint32_t p = (uint32_t)__ldg(s);
        const uint64_t q = __ldg(&pc[p].q), h = __ldg(s + 3), w = __ldg(s + 1), ws = __ldg(s + 2);
        const double inv = __longlong_as_double((long long)__ldg(s + 4));
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const uint64_t x = ok[u] ? job.src[j * job.src_stride + c0 + 256 * u] : 0;
          const uint64_t yj = mul_shoup(add_mod(x, h, q), w, ws, q);
          y[u][j] = yj;
          const double prod = __dmul_rn(u64_to_f64_rn(yj), inv);
          f[u] = j == 0 ? prod : __dadd_rn(f[u], prod);
        }
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) e[u] = n_src > 1 ? (uint64_t)floor(f[u]) : 0;
  }
  __syncthreads();
  for (int t = 0; t < (NS > 0 ? head : 0); ++t) {
    const uint64_t* d = sd + dw * t;
    uint64_t S[U];
    double Af[U];
#pragma unroll
    for (int u = 0; u < U; ++u) S[u] = 0, Af[u] = 0.0;
#pragma unroll
    for (int j = 0; j < K; ++j) {
      const uint64_t w = d[8 + j];
      const double wq = __longlong_as_double((long long)d[8 + n_src + j]);
#pragma unroll
      for (int u = 0; u < U; ++u) {
        S[u] += y[u][j] * w;
        Af[u] = __fma_rn(u64_to_f64_rn(y[u][j]), wq, Af[u]);
      }
    }
    const uint64_t negS = d[1], negH = d[2], q = d[3];
    const double qinv = __longlong_as_double((long long)d[4]);
    const double nS = __longlong_as_double((long long)d[5]), nH = __longlong_as_double((long long)d[6]);
    const uint64_t meta = d[7];
    const size_t out = (size_t)(uint32_t)meta * job.dst_stride;
    const bool two_stage = (meta >> 32) != 0;
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const uint64_t V = S[u] + e[u] * negS + negH;
      const double A = __dadd_rn(__fma_rn((double)e[u], nS, Af[u]), nH);
      const uint64_t k = (uint64_t)__double2ll_rn(A);
      int64_t r = (int64_t)(V - k * q);
      if (two_stage) {
        // |r| <= 2^62: the rounded quotient of f64(r) is within 1 of r / t's nearest integer
        const double rq = __dmul_rn(__ll2double_rn(r), qinv);
        r -= __double2ll_rn(rq) * (int64_t)q;
      }
      if (r < 0) r += (int64_t)q;
      if (ok[u]) job.dst[out + c0 + 256 * u] = (uint64_t)r;
    }
  }
  for (int t = head; t < job.n_dst; ++t) {
    const uint64_t* d = sd + dw * t;
    uint64_t A[U], B1[U], B2[U], Cc[U];
#pragma unroll
    for (int u = 0; u < U; ++u) A[u] = B1[u] = B2[u] = Cc[u] = 0;
#pragma unroll
    for (int j = 0; j < K; ++j) {
      if (j < n_src) {
        const uint64_t w = d[8 + j];
        const uint32_t wl = (uint32_t)w, wh = (uint32_t)(w >> 32);
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const uint32_t yl = (uint32_t)(y[u][j] & kMask30), yh = (uint32_t)(y[u][j] >> 30);
          A[u] += (uint64_t)yl * wl;
          B1[u] += (uint64_t)yl * wh;
          B2[u] += (uint64_t)yh * wl;
          Cc[u] += (uint64_t)yh * wh;
        }
      }
    }
    const uint64_t negS = d[1], negH = d[2];
    const size_t out = (size_t)(uint32_t)d[7] * job.dst_stride;
#pragma unroll
    for (int u = 0; u < U; ++u) {
      uint64_t lo = A[u], hi = 0;
      add128(hi, lo, B1[u] >> 34, B1[u] << 30);
      add128(hi, lo, B2[u] >> 34, B2[u] << 30);
      add128(hi, lo, Cc[u] >> 4, Cc[u] << 60);
      add128(hi, lo, 0, e[u] * negS);  // e < 16, so e * (t - [S]_t) < 2^64
      add128(hi, lo, 0, negH);
      if (ok[u]) job.dst[out + c0 + 256 * u] = reduce128_rec(hi, lo, d);
    }
  }
}

// f64(v) for v < 2^52, exact: the bits of 2^52 + v minus 2^52.
CKG_DEV double f64_small(uint64_t v) {
  return __dsub_rn(__longlong_as_double((long long)(v | 0x4330000000000000ULL)), 4503599627370496.0);
}
// rint(x) as an integer for 0 <= x < 2^52: 2^52 + x rounds to an integer in [2^52, 2^53).
CKG_DEV uint64_t rint_small(double x) {
  return (uint64_t)__double_as_longlong(__dadd_rn(x, 4503599627370496.0)) - 0x4330000000000000ULL;
}
// The FP64-assisted inner-product result: S = V mod 2^64, A ~ V / q within delta < off, base =
// off q: x = S - rint(A) q + base is V + (off - k) q in [0, (off + delta) q) < 2^53.
CKG_DEV uint64_t ip_finish_f64(uint64_t S, double A, uint64_t q, double q_d, double qinv, uint64_t base) {
  const uint64_t x = S - rint_small(A) * q + base;
  const int64_t r = (int64_t)(x - rint_small(__dmul_rn(u64_to_f64_rn(x), qinv)) * q);
  return (uint64_t)(r < 0 ? r + (int64_t)q : r);
}

// ------------------------------------------------------------------------------------
// Key-switch inner product (crates/ckks-train-ckks/src/keyswitch.rs:230-309): for every
// limb i of Q_l * P, out_b = sum_j d_j * b_j and out_a = sum_j d_j * a_j, accumulated
// exactly and reduced once. Digit j's limb i is the input polynomial's limb when prime i
// belongs to digit j, else the converted limb; with a Galois permutation every digit word is
// read at perm[c] (hoisted rotation). Each thread computes two adjacent coefficients (c, c + 1)
// with 16-byte loads and stores, so the job, limb and digit addressing is shared by both; a job
// whose buffers are not all 16-byte aligned (the input may be a caller's pointer) reads and
// writes the pair as two words.
// ------------------------------------------------------------------------------------

CKG_DEV bool aligned16(const void* p) { return ((uintptr_t)p & 15) == 0; }
CKG_DEV ulonglong2 ld_pair(const uint64_t* p, bool vec) {
  return vec ? __ldg(reinterpret_cast<const ulonglong2*>(p)) : make_ulonglong2(__ldg(p), __ldg(p + 1));
}
CKG_DEV ulonglong2 ldcs_pair(const uint64_t* p, bool vec) {
  return vec ? __ldcs(reinterpret_cast<const ulonglong2*>(p)) : make_ulonglong2(__ldcs(p), __ldcs(p + 1));
}
CKG_DEV void st_pair(uint64_t* p, uint64_t x, uint64_t y, bool vec) {
  if (vec) {
    *reinterpret_cast<ulonglong2*>(p) = make_ulonglong2(x, y);
  } else {
    p[0] = x;
    p[1] = y;
  }
}

template <class B>
__global__ void __launch_bounds__(256, std::is_same<B, IpPtrs>::value ? 4 : 1)
    k_inner_product(const __grid_constant__ B ib, const PrimeConst* __restrict__ pc, int log_n) {
  const int n = 1 << log_n;
  // By-value lists: grid (coefficient-pair blocks, limbs, jobs). Device-resident lists (the
  // batched path, jobs sorted by key): grid (jobs, coefficient-pair blocks, limbs), so the jobs
  // that share a key read the same key block back to back and it is served from L2.
  constexpr bool kJobFast = std::is_same<B, IpPtrs>::value;
  const IpJob& job = ib.j[kJobFast ? blockIdx.x : blockIdx.z];
  const int i = kJobFast ? blockIdx.z : blockIdx.y;  // limb of Q_l * P: 0..l data, l+1..l+k special
  const int c = 2 * ((kJobFast ? blockIdx.y : blockIdx.x) * blockDim.x + threadIdx.x);
  const int l = job.level;
  if (c >= n || i > l + ib.k) return;
  const bool is_q = i <= l;
  const uint32_t prime = is_q ? i : (ib.L + 1) + (i - l - 1);
  const int key_limb = is_q ? i : job.key_q + (i - l - 1);
  const size_t key_limbs = (size_t)(job.key_q + ib.k);
  const bool gather = job.perm != nullptr;
  uint32_t s0 = (uint32_t)c, s1 = (uint32_t)c + 1;
  if (gather) {
    s0 = __ldg(job.perm + c);
    s1 = __ldg(job.perm + c + 1);
  }
  const bool vin = !gather && aligned16(job.in);
  const bool vkey = aligned16(job.key);
  const bool vout = aligned16(job.out_b) && aligned16(job.out_a);
  // By-value lists (one op's jobs) load the words of up to 4 digits before their products so
  // the loads overlap; the batched grid, whose many resident jobs already keep loads in
  // flight, keeps one digit per step (measured faster there).
  constexpr int kChunk = kJobFast ? 1 : 4;
  auto load = [&](int j0, ulonglong2* dv, ulonglong2* kbv, ulonglong2* kav) {
#pragma unroll
    for (int u = 0; u < kChunk; ++u) {
      const int j = j0 + u;
      if (j < job.ndig) {
        const int start = j * ib.alpha;
        const int end = min(start + ib.alpha, l + 1);
        const uint64_t* base;
        bool vec;
        if (is_q && i >= start && i < end) {
          base = job.in + ((size_t)i << log_n);
          vec = vin;
        } else {
          const int t = i < start ? i : i - (end - start);
          base = job.conv[j] + ((size_t)t << log_n);
          vec = !gather && aligned16(job.conv[j]);
        }
        dv[u] = gather ? make_ulonglong2(__ldg(base + s0), __ldg(base + s1)) : ld_pair(base + c, vec);
        kbv[u] = ldcs_pair(job.key + ((size_t)(2 * j) * key_limbs + key_limb) * n + c, vkey);
        kav[u] = ldcs_pair(job.key + ((size_t)(2 * j + 1) * key_limbs + key_limb) * n + c, vkey);
      }
    }
  };
  const PrimeConst& P = pc[prime];
  const size_t o = ((size_t)i << log_n) + c;
  if (P.ip_off) {
    // FP64-assisted (data primes below 2^50 whose digit sums allow it, PrimeConst::ip_off):
    // S = sum_j d_j k_j mod 2^64 on the integer pipe; A = sum_j d_j fl(k_j / q) by FMA, within
    // delta < ip_off of the quotient, so x = S - rint(A) q + ip_off q lies in [0, 2^53); a
    // second rounded quotient of x (exact in f64) brings it into (-q, q), one add into [0, q).
    const double q_d = P.qd, qinv = P.qinv;
    uint64_t Sb0 = 0, Sa0 = 0, Sb1 = 0, Sa1 = 0;
    double Ab0 = 0.0, Aa0 = 0.0, Ab1 = 0.0, Aa1 = 0.0;
    for (int j0 = 0; j0 < job.ndig; j0 += kChunk) {
      ulonglong2 dv[kChunk], kbv[kChunk], kav[kChunk];
      load(j0, dv, kbv, kav);
#pragma unroll
      for (int u = 0; u < kChunk; ++u) {
        if (j0 + u >= job.ndig) break;
        const ulonglong2 d = dv[u], kb = kbv[u], ka = kav[u];
        Sb0 += d.x * kb.x;
        Sa0 += d.x * ka.x;
        Sb1 += d.y * kb.y;
        Sa1 += d.y * ka.y;
        const double dd0 = f64_small(d.x), dd1 = f64_small(d.y);
        Ab0 = __fma_rn(dd0, __dmul_rn(f64_small(kb.x), qinv), Ab0);
        Aa0 = __fma_rn(dd0, __dmul_rn(f64_small(ka.x), qinv), Aa0);
        Ab1 = __fma_rn(dd1, __dmul_rn(f64_small(kb.y), qinv), Ab1);
        Aa1 = __fma_rn(dd1, __dmul_rn(f64_small(ka.y), qinv), Aa1);
      }
    }
    const uint64_t q = P.q, base = (uint64_t)P.ip_off * q;
    st_pair(job.out_b + o, ip_finish_f64(Sb0, Ab0, q, q_d, qinv, base), ip_finish_f64(Sb1, Ab1, q, q_d, qinv, base),
            vout);
    st_pair(job.out_a + o, ip_finish_f64(Sa0, Aa0, q, q_d, qinv, base), ip_finish_f64(Sa1, Aa1, q, q_d, qinv, base),
            vout);
    return;
  }
  // 30-bit halves: four 64-bit accumulators per output, each < 16 * 2^60 (at most 16 digits).
  uint64_t acc[2][2][4] = {};  // [coefficient][b, a][lo*lo, lo*hi, hi*lo, hi*hi]
  for (int j0 = 0; j0 < job.ndig; j0 += kChunk) {
    ulonglong2 dv[kChunk], kbv[kChunk], kav[kChunk];
    load(j0, dv, kbv, kav);
#pragma unroll
    for (int u = 0; u < kChunk; ++u) {
      if (j0 + u >= job.ndig) break;
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const uint64_t d = e ? dv[u].y : dv[u].x, kb = e ? kbv[u].y : kbv[u].x, ka = e ? kav[u].y : kav[u].x;
        const uint32_t dl = (uint32_t)(d & kMask30), dh = (uint32_t)(d >> 30);
        const uint32_t bl = (uint32_t)(kb & kMask30), bh = (uint32_t)(kb >> 30);
        const uint32_t al = (uint32_t)(ka & kMask30), ah = (uint32_t)(ka >> 30);
        acc[e][0][0] += (uint64_t)dl * bl;
        acc[e][0][1] += (uint64_t)dl * bh;
        acc[e][0][2] += (uint64_t)dh * bl;
        acc[e][0][3] += (uint64_t)dh * bh;
        acc[e][1][0] += (uint64_t)dl * al;
        acc[e][1][1] += (uint64_t)dl * ah;
        acc[e][1][2] += (uint64_t)dh * al;
        acc[e][1][3] += (uint64_t)dh * ah;
      }
    }
  }
  uint64_t r[2][2];
#pragma unroll
  for (int e = 0; e < 2; ++e)
#pragma unroll
    for (int ba = 0; ba < 2; ++ba) {
      const uint64_t* a = acc[e][ba];
      uint64_t lo = a[0], hi = 0;
      add128(hi, lo, a[1] >> 34, a[1] << 30);
      add128(hi, lo, a[2] >> 34, a[2] << 30);
      add128(hi, lo, a[3] >> 4, a[3] << 60);
      r[e][ba] = reduce128(hi, lo, P);
    }
  st_pair(job.out_b + o, r[0][0], r[1][0], vout);
  st_pair(job.out_a + o, r[0][1], r[1][1], vout);
}

// ------------------------------------------------------------------------------------
// ModDown / rescale finish (baseconv.rs:286-289, 505-510): out = (x - t) * c (+ add).
// ------------------------------------------------------------------------------------

template <class B>
__global__ void __launch_bounds__(256)
    k_finish(const __grid_constant__ B fb, const PrimeConst* __restrict__ pc, int n) {
  const FinRef& r = fb.r[blockIdx.y];
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  const uint64_t q = __ldg(&pc[r.prime].q);
  uint64_t v = mul_shoup(sub_mod(r.x[c], r.t[c], q), r.c, r.c_s, q);
  if (r.add) v = add_mod(v, r.add[r.add_perm ? __ldg(r.add_perm + c) : c], q);
  r.out[c] = v;
}

// ------------------------------------------------------------------------------------
// Element-wise ops (crates/ckks-train-core/src/poly.rs:131-190) and the NTT-form
// automorphism gather (poly.rs:255-262).
// ------------------------------------------------------------------------------------

template <class B>
__global__ void __launch_bounds__(256)
    k_binary(const __grid_constant__ B bb, const PrimeConst* __restrict__ pc, int n) {
  const BinRef& r = bb.r[blockIdx.y];
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  const PrimeConst& P = pc[r.prime];
  const uint64_t a = r.a[c], b = r.b[c];
  uint64_t v;
  if (bb.op == 0) v = add_mod(a, b, P.q);
  else if (bb.op == 1) v = sub_mod(a, b, P.q);
  else v = mul_mod(a, b, P);
  r.out[c] = v;
}

// op 0: negate; op 1: multiply by the per-limb Shoup constant (aux selects it from
// `consts`, 2 words per entry); op 2: copy; op 3: gather through `perm`.
__global__ void __launch_bounds__(256)
    k_unary(const __grid_constant__ LimbBatch b, const PrimeConst* __restrict__ pc, int n, int op,
            const uint64_t* __restrict__ consts, const uint32_t* __restrict__ perm) {
  const LimbRef& r = b.r[blockIdx.y];
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  const uint64_t q = __ldg(&pc[r.prime].q);
  uint64_t v;
  if (op == 0) {
    v = sub_mod(0, r.src[c], q);
  } else if (op == 1) {
    v = mul_shoup(r.src[c], __ldg(consts + 2 * r.aux), __ldg(consts + 2 * r.aux + 1), q);
  } else if (op == 2) {
    v = r.src[c];
  } else {
    v = r.src[__ldg(perm + c)];
  }
  r.dst[c] = v;
}

// Packed download: each blockIdx.y copies one segment (rows at a source pitch) into its
// contiguous destination, 16 bytes per access when every address and length is even.
__global__ void __launch_bounds__(256) k_pack(const PackSeg* __restrict__ segs) {
  const PackSeg sg = segs[blockIdx.y];
  const uint32_t total = sg.rows * sg.row_words;
  const uint32_t step = gridDim.x * blockDim.x;
  const bool vec = ((((uintptr_t)sg.src | (uintptr_t)sg.dst) & 15) == 0) && !(sg.pitch & 1) && !(sg.row_words & 1);
  if (vec) {
    for (uint32_t w = 2 * (blockIdx.x * blockDim.x + threadIdx.x); w < total; w += 2 * step) {
      const uint32_t r = w / sg.row_words, c = w - r * sg.row_words;
      const ulonglong2 v = __ldcs(reinterpret_cast<const ulonglong2*>(sg.src + r * sg.pitch + c));
      __stcs(reinterpret_cast<ulonglong2*>(sg.dst + w), v);
    }
  } else {
    for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < total; w += step) {
      const uint32_t r = w / sg.row_words, c = w - r * sg.row_words;
      sg.dst[w] = __ldcs(sg.src + r * sg.pitch + c);
    }
  }
}

template <class B>
__global__ void __launch_bounds__(256) k_gather(const __grid_constant__ B gb, int n) {
  const GatherRef& r = gb.r[blockIdx.y];
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  r.dst[c] = r.src[__ldg(r.perm + c)];
}

template <class B>
__global__ void __launch_bounds__(256)
    k_tensor(const __grid_constant__ B tb, const PrimeConst* __restrict__ pc, int n) {
  const TensorRef& r = tb.r[blockIdx.y];
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  const PrimeConst& P = pc[r.prime];
  const uint64_t a0 = r.a0[c], a1 = r.a1[c], b0 = r.b0[c], b1 = r.b1[c];
  r.d0[c] = mul_mod(a0, b0, P);
  r.d1[c] = add_mod(mul_mod(a0, b1, P), mul_mod(a1, b0, P), P.q);
  r.d2[c] = mul_mod(a1, b1, P);
}

// mode 0: dst = src * w (Shoup pair per prime); mode 1: dst = src + w (w < q).
__global__ void __launch_bounds__(256)
    k_scalar(const __grid_constant__ LimbBatch b, const __grid_constant__ ScalarTable st,
             const PrimeConst* __restrict__ pc, int n, int mode) {
  const LimbRef& r = b.r[blockIdx.y];
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  const uint64_t q = __ldg(&pc[r.prime].q);
  r.dst[c] = mode == 0 ? mul_shoup(r.src[c], st.w[r.prime], st.ws[r.prime], q) : add_mod(r.src[c], st.w[r.prime], q);
}

// One pass over every term's limb: 128-bit accumulation of up to kMaxMacTerms products
// (each < 2^120), one reduction per output word.
__global__ void __launch_bounds__(256)
    k_mac_plain(const __grid_constant__ MacBatch b, const PrimeConst* __restrict__ pc, int n) {
  const int i = blockIdx.y;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  const size_t off = (size_t)i * n + c;
  uint64_t h0 = 0, l0 = 0, h1 = 0, l1 = 0;
  for (int t = 0; t < b.count; ++t) {
    const uint64_t w = __ldg(b.w[t] + off);
    mac128(h0, l0, __ldg(b.x0[t] + off), w);
    mac128(h1, l1, __ldg(b.x1[t] + off), w);
  }
  const PrimeConst P = pc[i];
  b.out0[off] = reduce128(h0, l0, P);
  b.out1[off] = reduce128(h1, l1, P);
}

// The same over ciphertext pairs: the three tensor components summed over the terms in 128 bits
// (each product < 2^120, at most 2 * kMaxMacTensorTerms of them per sum), one reduction each,
// equal to the reduced products added one by one.
__global__ void __launch_bounds__(256)
    k_mac_tensor(const __grid_constant__ MacTensorBatch b, const PrimeConst* __restrict__ pc, int n) {
  const int i = blockIdx.y;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  const size_t off = (size_t)i * n + c;
  uint64_t h0 = 0, l0 = 0, h1 = 0, l1 = 0, h2 = 0, l2 = 0;
  for (int t = 0; t < b.count; ++t) {
    const uint64_t x0 = __ldg(b.a0[t] + off), x1 = __ldg(b.a1[t] + off);
    const uint64_t y0 = __ldg(b.b0[t] + off), y1 = __ldg(b.b1[t] + off);
    mac128(h0, l0, x0, y0);
    mac128(h1, l1, x0, y1);
    mac128(h1, l1, x1, y0);
    mac128(h2, l2, x1, y1);
  }
  const PrimeConst P = pc[i];
  b.out0[off] = reduce128(h0, l0, P);
  b.out1[off] = reduce128(h1, l1, P);
  b.out2[off] = reduce128(h2, l2, P);
}

// Centered lift of a level-0 coefficient-form limb (src of every ref) into prime r.prime:
// residues above (q_0 - 1) / 2 are read as negative (poly.rs:298-345).
__global__ void __launch_bounds__(256)
    k_lift_level0(const __grid_constant__ LimbBatch b, const PrimeConst* __restrict__ pc, int n) {
  const LimbRef& r = b.r[blockIdx.y];
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  const uint64_t q0 = __ldg(&pc[0].q), q = __ldg(&pc[r.prime].q);
  const uint64_t x = r.src[c];
  uint64_t v;
  if (x > q0 / 2) {
    const uint64_t m = (q0 - x) % q;
    v = m ? q - m : 0;
  } else {
    v = x % q;
  }
  r.dst[c] = v;
}

template <class T>
void set_smem(T* fn, int bytes) {
  cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link against libcuda).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return (PFN_cuTensorMapEncodeTiled_v12000) nullptr;
    return (PFN_cuTensorMapEncodeTiled_v12000)p;
  }();
  return fn;
}

// The tensor map of a region of `limbs` limbs (N words each) from `base`: 256 columns x N/256
// rows x limbs, boxes of 16 columns x all rows x one limb.
bool limb_tensor_map(CUtensorMap* map, const uint64_t* base, uint64_t limbs, int log_n) {
  auto enc = tensor_map_encoder();
  if (!enc || log_n < 12 || log_n > 16 || ((uintptr_t)base & 15)) return false;
  const cuuint32_t rows = 1u << (log_n - kRowLog);
  cuuint64_t dims[3] = {(cuuint64_t)kRow, rows, limbs};
  cuuint64_t strides[2] = {(cuuint64_t)kRow * 8, ((cuuint64_t)1 << log_n) * 8};
  cuuint32_t box[3] = {(cuuint32_t)kCols, rows, 1};
  cuuint32_t es[3] = {1, 1, 1};
  return enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT64, 3, (void*)base, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
         CUDA_SUCCESS;
}

// The region the column pass reads of a by-value list: from its lowest source, when every source
// lies a whole number of limbs above it.
template <class B>
bool list_region(const B& b, int count, int in_place, bool inverse, int log_n, LimbRegion* out) {
  if constexpr (std::is_same<B, LimbBatch>::value) {
    auto src = [&](const LimbRef& r) { return (inverse ? in_place : (in_place && !r.aux)) ? r.dst : r.src; };
    const uint64_t* lo = src(b.r[0]);
    for (int i = 1; i < count; ++i) lo = std::min(lo, (const uint64_t*)src(b.r[i]));
    uint64_t hi = 0;
    for (int i = 0; i < count; ++i) {
      const uint64_t off = (uint64_t)(src(b.r[i]) - lo);
      if (off & ((1ull << log_n) - 1)) return false;
      hi = std::max(hi, (off >> log_n) + 1);
    }
    *out = LimbRegion{lo, hi};
    return true;
  }
  return false;
}

template <int LOGS, bool INV, class B>
bool launch_cols_tma(const B& b, int count, const DevTables& d, int in_place, cudaStream_t st, LimbRegion reg) {
  CUtensorMap map;
  if (!limb_tensor_map(&map, reg.base, reg.limbs, d.log_n)) return false;
  const int smem = 2 * (1 << LOGS) * kCols * 8 + 16;
  const int threads = kCols * (1 << (LOGS / 2));
  auto fn = k_ntt_cols_tma<LOGS, INV, B>;
  set_smem(fn, smem);
  static const int per_sm = [&] {
    int v = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, fn, threads, smem);
    return v > 0 ? v : 1;
  }();
  const int items = count * (kRow / kCols);
  const int grid = std::min(items, std::max(1, d.sms) * per_sm);
  fn<<<grid, threads, smem, st>>>(b, map, reg.base, reg.limbs, d.prime, INV ? d.tw_inv : d.tw_fwd,
                                  INV ? d.twd_inv : d.twd_fwd, d.log_n, in_place, items);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return true;
}

template <int LOGS, class B>
void launch_cols(bool inverse, const B& b, int count, const DevTables& d, int in_place, cudaStream_t st,
                 const LimbRegion* region) {
  if (d.ntt_tma && LOGS <= 8) {
    LimbRegion reg{};
    if (region ? (reg = *region, true) : list_region(b, count, in_place, inverse, d.log_n, &reg)) {
      if (inverse ? launch_cols_tma<LOGS, true>(b, count, d, in_place, st, reg)
                  : launch_cols_tma<LOGS, false>(b, count, d, in_place, st, reg))
        return;
    }
  }
  const int smem = (1 << LOGS) * kCols * 8;
  const int threads = kCols * (1 << (LOGS / 2));
  dim3 grid(kRow / kCols, count);
  if (!inverse) {
    if (smem > 48 * 1024) set_smem(k_ntt_fwd_cols<LOGS, B>, smem);
    k_ntt_fwd_cols<LOGS, B><<<grid, threads, smem, st>>>(b, d.prime, d.tw_fwd, d.twd_fwd, d.log_n, in_place);
  } else {
    if (smem > 48 * 1024) set_smem(k_ntt_inv_cols<LOGS, B>, smem);
    k_ntt_inv_cols<LOGS, B><<<grid, threads, smem, st>>>(b, d.prime, d.tw_inv, d.twd_inv, d.log_n, in_place);
  }
  g_launches.fetch_add(1, std::memory_order_relaxed);
}

template <class B>
void launch_cols_any(bool inverse, const B& b, int count, const DevTables& d, int in_place, cudaStream_t st,
                     const LimbRegion* region = nullptr) {
  switch (d.log_n - kRowLog) {
    case 4: launch_cols<4>(inverse, b, count, d, in_place, st, region); break;
    case 5: launch_cols<5>(inverse, b, count, d, in_place, st, region); break;
    case 6: launch_cols<6>(inverse, b, count, d, in_place, st, region); break;
    case 7: launch_cols<7>(inverse, b, count, d, in_place, st, region); break;
    case 8: launch_cols<8>(inverse, b, count, d, in_place, st, region); break;
    case 9: launch_cols<9>(inverse, b, count, d, in_place, st, region); break;
    default: break;
  }
}

// Both passes of a batched transform: src -> dst, then dst in place.
template <class B>
void ntt_passes(const DevTables& d, const B& b, int count, bool inverse, cudaStream_t st,
                const LimbRegion* region = nullptr) {
  if (count == 0) return;
  if (d.log_n <= 11) {
    const int n = 1 << d.log_n;
    const int threads = n / 2 < 512 ? (n / 2 < 32 ? 32 : n / 2) : 512;
    k_ntt_small<B><<<dim3(1, count), threads, n * 8, st>>>(b, d.prime, d.tw_fwd, d.tw_inv, d.log_n, inverse);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    return;
  }
  const dim3 rgrid((1 << d.log_n) / (kRow * kRowsPerCta), count);
  if (!inverse) {
    launch_cols_any(false, b, count, d, 0, st, region);
    k_ntt_fwd_rows<B><<<rgrid, 256, 0, st>>>(b, d.prime, d.tw_fwd, d.twd_fwd, d.log_n, 1);
  } else {
    k_ntt_inv_rows<B><<<rgrid, 256, 0, st>>>(b, d.prime, d.tw_inv, d.twd_inv, d.log_n, 0);
    launch_cols_any(true, b, count, d, 1, st, region);
  }
  g_launches.fetch_add(1, std::memory_order_relaxed);
}

template <class B>
void bconv_launch(const DevTables& d, const B& cb, int count, int n_src, cudaStream_t st) {
  const int n = 1 << d.log_n;
  dim3 grid((n + 256 * kBconvU - 1) / (256 * kBconvU), count);
  switch (n_src) {
    case 1: k_bconv<1, B><<<grid, 256, 0, st>>>(cb, d.prime, n); break;
    case 2: k_bconv<2, B><<<grid, 256, 0, st>>>(cb, d.prime, n); break;
    case 3: k_bconv<3, B><<<grid, 256, 0, st>>>(cb, d.prime, n); break;
    case 4: k_bconv<4, B><<<grid, 256, 0, st>>>(cb, d.prime, n); break;
    case 5: k_bconv<5, B><<<grid, 256, 0, st>>>(cb, d.prime, n); break;
    case 6: k_bconv<6, B><<<grid, 256, 0, st>>>(cb, d.prime, n); break;
    case 7: k_bconv<7, B><<<grid, 256, 0, st>>>(cb, d.prime, n); break;
    case 8: k_bconv<8, B><<<grid, 256, 0, st>>>(cb, d.prime, n); break;
    default: k_bconv<0, B><<<grid, 256, 0, st>>>(cb, d.prime, n); break;
  }
  g_launches.fetch_add(1, std::memory_order_relaxed);
}

}  // namespace

// ------------------------------------------------------------------------------------
// Host launchers (declared in launch.hpp). By-value lists longer than one launch's
// capacity are split; device-resident lists run in one launch. Every launch goes to
// stream `st` and is counted in g_launches.
// ------------------------------------------------------------------------------------

std::atomic<uint64_t> g_launches{0};

void launch_ntt(const DevTables& d, const LimbRef* refs, int count, bool inverse, cudaStream_t st) {
  bounds::refs(refs, count, (size_t)1 << d.log_n, "NTT limb");
  LimbBatch b;
  for (int off = 0; off < count; off += kMaxLimbs) {
    b.count = count - off < kMaxLimbs ? count - off : kMaxLimbs;
    for (int i = 0; i < b.count; ++i) b.r[i] = refs[off + i];
    ntt_passes(d, b, b.count, inverse, st);
  }
}

// Device lists go in waves of d.ntt_wave limbs: a wave's column pass and row pass run back to
// back, so the intermediate limbs can stay in L2 between them.
void launch_ntt_ptr(const DevTables& d, const LimbRef* dev_refs, int count, bool inverse, cudaStream_t st,
                    const LimbRegion* region) {
  const int wave = d.ntt_wave > 0 ? d.ntt_wave : count;
  for (int off = 0; off < count; off += wave) {
    const int c = std::min(wave, count - off);
    ntt_passes(d, LimbPtrs{c, 0, dev_refs + off}, c, inverse, st, region);
  }
}

void launch_bconv(const DevTables& d, const ConvJob* jobs, int count, int n_src, int n_dst, cudaStream_t st) {
  if (bounds::enabled()) {
    std::vector<ConvJob> chk(jobs, jobs + count);
    for (ConvJob& j : chk) j.n_dst = n_dst;
    bounds::refs(chk.data(), chk.size(), n_src, (size_t)1 << d.log_n, "base conversion");
  }
  ConvBatch cb;
  cb.n_src = n_src;
  cb.n_dst = n_dst;
  for (int off = 0; off < count; off += kMaxConv) {
    cb.count = count - off < kMaxConv ? count - off : kMaxConv;
    for (int i = 0; i < cb.count; ++i) {
      cb.j[i] = jobs[off + i];
      cb.j[i].n_dst = n_dst;
    }
    if (!launch_bconv_tc(d, cb, cb.count, n_src, n_dst, st)) bconv_launch(d, cb, cb.count, n_src, st);
  }
}

void launch_bconv_ptr(const DevTables& d, const ConvJob* dev_jobs, int count, int n_src, cudaStream_t st,
                      int max_dst) {
  if (!count) return;
  if (max_dst > 0 && launch_bconv_tc_ptr(d, dev_jobs, count, n_src, max_dst, st)) return;
  bconv_launch(d, ConvPtrs{count, n_src, 0, 0, dev_jobs}, count, n_src, st);
}

void launch_inner_product(const DevTables& d, int alpha, int L, int k, const IpJob* jobs, int count, cudaStream_t st) {
  bounds::refs(jobs, count, alpha, k, (size_t)1 << d.log_n, "inner product");
  IpBatch ib;
  ib.alpha = alpha;
  ib.L = L;
  ib.k = k;
  const int n = 1 << d.log_n;
  for (int off = 0; off < count; off += kMaxIp) {
    ib.count = count - off < kMaxIp ? count - off : kMaxIp;
    int max_limbs = 0;
    for (int i = 0; i < ib.count; ++i) {
      ib.j[i] = jobs[off + i];
      max_limbs = std::max(max_limbs, jobs[off + i].level + 1 + k);
    }
    k_inner_product<IpBatch><<<dim3((n / 2 + 255) / 256, max_limbs, ib.count), 256, 0, st>>>(ib, d.prime, d.log_n);
    g_launches.fetch_add(1, std::memory_order_relaxed);
  }
}

void launch_inner_product_ptr(const DevTables& d, int alpha, int L, int k, const IpJob* dev_jobs, int count,
                              int max_limbs, cudaStream_t st) {
  if (!count) return;
  const int n = 1 << d.log_n;
  k_inner_product<IpPtrs><<<dim3(count, (n / 2 + 255) / 256, max_limbs), 256, 0, st>>>(IpPtrs{count, alpha, L, k, dev_jobs},
                                                                                  d.prime, d.log_n);
  g_launches.fetch_add(1, std::memory_order_relaxed);
}

void launch_ntt_finish(const DevTables& d, const FinRef* refs, int count, cudaStream_t st, const LimbRef* cols) {
  bounds::refs(refs, count, (size_t)1 << d.log_n, "NTT + finish");
  if (cols) bounds::refs(cols, count, (size_t)1 << d.log_n, "NTT + finish column pass");
  if (cols && d.log_n <= 11) throw std::logic_error("launch_ntt_finish: explicit column passes need N >= 2^12");
  if (d.log_n <= 11) {  // small transforms: separate NTT and finish
    std::vector<LimbRef> lr(count);
    for (int i = 0; i < count; ++i) lr[i] = LimbRef{refs[i].t, const_cast<uint64_t*>(refs[i].t), refs[i].prime, 0};
    launch_ntt(d, lr.data(), count, false, st);
    launch_finish(d, refs, count, st);
    return;
  }
  LimbBatch b;
  FinBatch fb;
  const dim3 rgrid((1 << d.log_n) / (kRow * kRowsPerCta), 1);
  for (int off = 0; off < count; off += kMaxFin) {
    const int cnt = count - off < kMaxFin ? count - off : kMaxFin;
    b.count = cnt;
    fb.count = cnt;
    for (int i = 0; i < cnt; ++i) {
      fb.r[i] = refs[off + i];
      b.r[i] = cols ? cols[off + i] : LimbRef{refs[off + i].t, const_cast<uint64_t*>(refs[off + i].t), refs[off + i].prime, 0};
    }
    launch_cols_any(false, b, cnt, d, 1, st);
    k_ntt_fwd_rows_finish<FinBatch><<<dim3(rgrid.x, cnt), 256, 0, st>>>(fb, d.prime, d.tw_fwd, d.twd_fwd, d.log_n);
    g_launches.fetch_add(1, std::memory_order_relaxed);
  }
}

void launch_ntt_finish_ptr(const DevTables& d, const LimbRef* dev_cols, const FinRef* dev_fin, int count,
                           cudaStream_t st, const LimbRegion* region) {
  if (!count) return;
  if (d.log_n <= 11) {
    launch_ntt_ptr(d, dev_cols, count, false, st);
    launch_finish_ptr(d, dev_fin, count, st);
    return;
  }
  const int wave = d.ntt_wave > 0 ? d.ntt_wave : count;
  for (int off = 0; off < count; off += wave) {
    const int c = std::min(wave, count - off);
    launch_cols_any(false, LimbPtrs{c, 0, dev_cols + off}, c, d, 1, st, region);
    k_ntt_fwd_rows_finish<FinPtrs><<<dim3((1 << d.log_n) / (kRow * kRowsPerCta), c), 256, 0, st>>>(
        FinPtrs{c, 0, dev_fin + off}, d.prime, d.tw_fwd, d.twd_fwd, d.log_n);
    g_launches.fetch_add(1, std::memory_order_relaxed);
  }
}

void launch_finish(const DevTables& d, const FinRef* refs, int count, cudaStream_t st) {
  bounds::refs(refs, count, (size_t)1 << d.log_n, "finish");
  FinBatch fb;
  const int n = 1 << d.log_n;
  for (int off = 0; off < count; off += kMaxFin) {
    fb.count = count - off < kMaxFin ? count - off : kMaxFin;
    for (int i = 0; i < fb.count; ++i) fb.r[i] = refs[off + i];
    k_finish<FinBatch><<<dim3((n + 255) / 256, fb.count), 256, 0, st>>>(fb, d.prime, n);
    g_launches.fetch_add(1, std::memory_order_relaxed);
  }
}

void launch_finish_ptr(const DevTables& d, const FinRef* dev_refs, int count, cudaStream_t st) {
  if (!count) return;
  const int n = 1 << d.log_n;
  k_finish<FinPtrs><<<dim3((n + 255) / 256, count), 256, 0, st>>>(FinPtrs{count, 0, dev_refs}, d.prime, n);
  g_launches.fetch_add(1, std::memory_order_relaxed);
}

void launch_binary(const DevTables& d, const BinRef* refs, int count, int op, cudaStream_t st) {
  bounds::refs(refs, count, (size_t)1 << d.log_n, "element-wise op");
  BinBatch bb;
  bb.op = op;
  const int n = 1 << d.log_n;
  for (int off = 0; off < count; off += kMaxBin) {
    bb.count = count - off < kMaxBin ? count - off : kMaxBin;
    for (int i = 0; i < bb.count; ++i) bb.r[i] = refs[off + i];
    k_binary<BinBatch><<<dim3((n + 255) / 256, bb.count), 256, 0, st>>>(bb, d.prime, n);
    g_launches.fetch_add(1, std::memory_order_relaxed);
  }
}

void launch_binary_ptr(const DevTables& d, const BinRef* dev_refs, int count, int op, cudaStream_t st) {
  if (!count) return;
  const int n = 1 << d.log_n;
  k_binary<BinPtrs><<<dim3((n + 255) / 256, count), 256, 0, st>>>(BinPtrs{count, op, dev_refs}, d.prime, n);
  g_launches.fetch_add(1, std::memory_order_relaxed);
}

void launch_unary(const DevTables& d, const LimbRef* refs, int count, int op, const uint64_t* consts,
                  const uint32_t* perm, cudaStream_t st) {
  bounds::refs(refs, count, (size_t)1 << d.log_n, "unary op");
  bounds::perm(perm, (size_t)1 << d.log_n, "unary op permutation");
  LimbBatch b;
  const int n = 1 << d.log_n;
  for (int off = 0; off < count; off += kMaxLimbs) {
    b.count = count - off < kMaxLimbs ? count - off : kMaxLimbs;
    for (int i = 0; i < b.count; ++i) b.r[i] = refs[off + i];
    k_unary<<<dim3((n + 255) / 256, b.count), 256, 0, st>>>(b, d.prime, n, op, consts, perm);
    g_launches.fetch_add(1, std::memory_order_relaxed);
  }
}

void launch_pack(const PackSeg* dev_segs, int count, cudaStream_t st) {
  for (int i = 0; i < count; i += 65535) {
    const int m = std::min(65535, count - i);
    k_pack<<<dim3(64, m), 256, 0, st>>>(dev_segs + i);
    g_launches.fetch_add(1, std::memory_order_relaxed);
  }
}

void launch_gather_ptr(const DevTables& d, const GatherRef* dev_refs, int count, cudaStream_t st) {
  if (!count) return;
  const int n = 1 << d.log_n;
  k_gather<GatherPtrs><<<dim3((n + 255) / 256, count), 256, 0, st>>>(GatherPtrs{count, 0, dev_refs}, n);
  g_launches.fetch_add(1, std::memory_order_relaxed);
}

void launch_tensor(const DevTables& d, const TensorRef* refs, int count, cudaStream_t st) {
  bounds::refs(refs, count, (size_t)1 << d.log_n, "tensor product");
  TensorBatch tb;
  const int n = 1 << d.log_n;
  for (int off = 0; off < count; off += kMaxTensor) {
    tb.count = count - off < kMaxTensor ? count - off : kMaxTensor;
    for (int i = 0; i < tb.count; ++i) tb.r[i] = refs[off + i];
    k_tensor<TensorBatch><<<dim3((n + 255) / 256, tb.count), 256, 0, st>>>(tb, d.prime, n);
    g_launches.fetch_add(1, std::memory_order_relaxed);
  }
}

void launch_tensor_ptr(const DevTables& d, const TensorRef* dev_refs, int count, cudaStream_t st) {
  if (!count) return;
  const int n = 1 << d.log_n;
  k_tensor<TensorPtrs><<<dim3((n + 255) / 256, count), 256, 0, st>>>(TensorPtrs{count, 0, dev_refs}, d.prime, n);
  g_launches.fetch_add(1, std::memory_order_relaxed);
}

void launch_scalar(const DevTables& d, const LimbRef* refs, int count, const ScalarTable& table, cudaStream_t st,
                   int mode) {
  bounds::refs(refs, count, (size_t)1 << d.log_n, "scalar op");
  LimbBatch b;
  const int n = 1 << d.log_n;
  for (int off = 0; off < count; off += kMaxLimbs) {
    b.count = count - off < kMaxLimbs ? count - off : kMaxLimbs;
    for (int i = 0; i < b.count; ++i) b.r[i] = refs[off + i];
    k_scalar<<<dim3((n + 255) / 256, b.count), 256, 0, st>>>(b, table, d.prime, n, mode);
    g_launches.fetch_add(1, std::memory_order_relaxed);
  }
}

void launch_mac_plain(const DevTables& d, const MacBatch& b, cudaStream_t st) {
  const int n = 1 << d.log_n;
  if (bounds::enabled()) {
    const size_t w = (size_t)b.limbs * n;
    bounds::limb(b.out0, w, "plaintext MAC");
    bounds::limb(b.out1, w, "plaintext MAC");
    for (int t = 0; t < b.count; ++t) {
      bounds::limb(b.x0[t], w, "plaintext MAC");
      bounds::limb(b.x1[t], w, "plaintext MAC");
      bounds::limb(b.w[t], w, "plaintext MAC");
    }
  }
  k_mac_plain<<<dim3((n + 255) / 256, b.limbs), 256, 0, st>>>(b, d.prime, n);
  g_launches.fetch_add(1, std::memory_order_relaxed);
}

void launch_mac_tensor(const DevTables& d, const MacTensorBatch& b, cudaStream_t st) {
  const int n = 1 << d.log_n;
  if (bounds::enabled()) {
    const size_t w = (size_t)b.limbs * n;
    for (const void* o : {(const void*)b.out0, (const void*)b.out1, (const void*)b.out2}) bounds::limb(o, w, "tensor MAC");
    for (int t = 0; t < b.count; ++t)
      for (const void* x : {(const void*)b.a0[t], (const void*)b.a1[t], (const void*)b.b0[t], (const void*)b.b1[t]})
        bounds::limb(x, w, "tensor MAC");
  }
  k_mac_tensor<<<dim3((n + 255) / 256, b.limbs), 256, 0, st>>>(b, d.prime, n);
  g_launches.fetch_add(1, std::memory_order_relaxed);
}

void launch_lift_level0(const DevTables& d, const LimbRef* refs, int count, cudaStream_t st) {
  bounds::refs(refs, count, (size_t)1 << d.log_n, "level-0 lift");
  LimbBatch b;
  const int n = 1 << d.log_n;
  for (int off = 0; off < count; off += kMaxLimbs) {
    b.count = count - off < kMaxLimbs ? count - off : kMaxLimbs;
    for (int i = 0; i < b.count; ++i) b.r[i] = refs[off + i];
    k_lift_level0<<<dim3((n + 255) / 256, b.count), 256, 0, st>>>(b, d.prime, n);
    g_launches.fetch_add(1, std::memory_order_relaxed);
  }
}

}  // namespace ckg
