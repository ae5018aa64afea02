// Exact fast base conversion on the tensor cores (tcgen05.mma, kind::i8).
//
// Base conversion computes, per coefficient and target prime t,
//   out_t = (sum_j y_j w_tj + e (t - [S]_t) + (t - [h]_t)) mod t,   y_j < s_j < 2^60,
// with y_j = [(x_j + h_j) qhat_j^-1]_{s_j}, w_tj = [S / s_j]_t and the overflow count
// e = floor(sum_j f64(y_j) f64(1/s_j)) (crates/ckks-train-core/src/baseconv.rs:167-235). Write
// y_j = sum_a y_j[a] 2^(8a) in bytes; then sum_j y_j w_tj is congruent mod t to
// sum_b 2^(8b) C_b with C_b = sum_(j,a) y_j[a] W[t, b][j, a], W[t, b][j, a] = byte b of
// [2^(8a) w_tj]_t. C is an exact u8 x u8 -> s32 matrix product (every C_b < 64 * 255^2 < 2^22):
// the A operand is the y_j words themselves (their little-endian bytes are the y_j[a]), one row
// of K = 8 n_src bytes per coefficient; the B operand is the table's byte-split weights, one row
// per (target, byte). The epilogue reduces V = sum_b 2^(8b) C_b + e (t - [S]_t) + (t - [h]_t)
// (< 2^79) with an FP64 quotient (reduce_target): V mod 2^64 in integers, V / t estimated in
// FP64; for t >= 2^30 the rounded quotient is within 0.72 of V / t, so V - q t, computed mod
// 2^64, lies in (-t, t) and one conditional add or subtract gives the canonical residue. Results equal the integer kernels'
// (k_bconv) bit for bit; the overflow estimate is the same __dmul_rn / __dadd_rn chain.
//
// One CTA is one warpgroup: thread i owns coefficient i of each 128-coefficient tile, which is
// row i of the MMA (M = 128) and TMEM lane i of the accumulator. Per tile: every thread computes
// its y_j and e and stores the A row in shared memory; one thread issues the MMAs (K = 32 bytes
// each) and commits them to an mbarrier; the threads load the next tile's sources while the
// tensor core runs, then read their accumulator row (8 columns per target) with tcgen05.ld and
// reduce. The B operand (<= 16 KB) is brought into shared memory once per CTA by a bulk copy
// (cp.async.bulk) completing on an mbarrier. Every wait is bounded (about a second of clock):
// on timeout the kernel records a device fault (g_device_fault), frees its TMEM and returns.
#include <cuda_runtime.h>

#include <algorithm>

#include "kernels.cuh"
#include "launch.hpp"

namespace ckg {

__device__ int g_device_fault;

namespace {

constexpr int kTcRows = 128;  // coefficients per tile: MMA M, threads per warpgroup, TMEM lanes
constexpr int kTcAutoMinSrc = 6;

CKG_DEV uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor (sm_100): start address, leading-dimension byte offset (the
// distance of the two 16-byte K chunks an MMA of K = 32 bytes reads), stride-dimension byte
// offset (the distance of adjacent 8-row groups), version 1, no swizzle.
CKG_DEV uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// Instruction descriptor of kind::i8: s32 accumulator (bits 4-5 = 2), A and B unsigned 8-bit
// (formats 0), both K-major, N >> 3 at bit 17, M >> 4 at bit 24.
CKG_DEV uint32_t idesc_u8(uint32_t m, uint32_t n) { return (2u << 4) | ((n >> 3) << 17) | ((m >> 4) << 24); }

CKG_DEV void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(bar)), "r"(count) : "memory");
}
CKG_DEV bool mbar_try_wait(uint64_t* bar, uint32_t phase) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(saddr(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}
// Waits for `phase` to complete, for at most about a second; records a device fault on timeout.
CKG_DEV bool mbar_wait(uint64_t* bar, uint32_t phase) {
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, phase)) {
    if (clock64() - t0 > (2LL << 30)) {
      atomicExch(&g_device_fault, 1);
      return false;
    }
  }
  return true;
}
// Bulk copy global -> shared (no multicast), completing `bytes` on the mbarrier.
CKG_DEV void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(bar)), "r"(bytes) : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   saddr(dst)),
               "l"(src), "r"(bytes), "r"(saddr(bar))
               : "memory");
}
CKG_DEV void tmem_alloc(uint32_t* slot, uint32_t ncols) {  // by one whole warp
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(slot)), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
CKG_DEV void tmem_dealloc(uint32_t taddr, uint32_t ncols) {  // by one whole warp
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
CKG_DEV void tc_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
CKG_DEV void tc_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
CKG_DEV void async_proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
CKG_DEV void mma_u8(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\ttcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(
          d),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}
CKG_DEV void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(saddr(bar))
               : "memory");
}
// f64(v) rounded to nearest, on the FP64 pipe (as kernels.cu u64_to_f64_rn).
CKG_DEV double u64_f64_rn(uint64_t v) {
  const double hi = __dsub_rn(__hiloint2double(0x43300000, (int)(uint32_t)(v >> 32)), 4503599627370496.0);
  const double lo = __dsub_rn(__hiloint2double(0x43300000, (int)(uint32_t)v), 4503599627370496.0);
  return __fma_rn(hi, 4294967296.0, lo);
}

// 32 consecutive accumulator columns (4 targets) of this thread's lane.
CKG_DEV void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
        "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]),
        "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
        "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(v[0]), "+r"(v[1]), "+r"(v[2]), "+r"(v[3]), "+r"(v[4]), "+r"(v[5]), "+r"(v[6]), "+r"(v[7]),
                 "+r"(v[8]), "+r"(v[9]), "+r"(v[10]), "+r"(v[11]), "+r"(v[12]), "+r"(v[13]), "+r"(v[14]),
                 "+r"(v[15]), "+r"(v[16]), "+r"(v[17]), "+r"(v[18]), "+r"(v[19]), "+r"(v[20]), "+r"(v[21]),
                 "+r"(v[22]), "+r"(v[23]), "+r"(v[24]), "+r"(v[25]), "+r"(v[26]), "+r"(v[27]), "+r"(v[28]),
                 "+r"(v[29]), "+r"(v[30]), "+r"(v[31])
               :
               : "memory");
}

// f64(v) for v < 2^52, exact: the bits of 2^52 + v minus 2^52.
CKG_DEV double f64_exact(uint64_t v) {
  return __dsub_rn(__longlong_as_double((long long)(v | 0x4330000000000000ULL)), 4503599627370496.0);
}

// Target record in shared memory (kTcRec words): t, bits(1/t), t - [S]_t, t - [h]_t, and the last
// two as doubles.
constexpr int kTcRec = 6;

// V = sum_b 2^(8b) c[b] + e (t - [S]_t) + (t - [h]_t) mod t from the 8 partial sums of one target
// (c[b] < 2^22). V = vl + 2^32 vh with vl, vh < 2^47 exact; V mod 2^64 in integers; an FP64
// estimate A of V in three rounded steps (|A - V| < 2^26.6 for V < 2^79), the quotient
// k = rint(A fl(1/t)) is within 0.72 of V / t for t >= 2^30 (0.5 rounding, 0.1 from A, 0.125 from
// fl(1/t) and the product), so r = V - k t computed mod 2^64 lies in (-t, t).
CKG_DEV uint64_t reduce_target(const uint32_t* c, uint64_t e, double ed, const uint64_t* T) {
  const uint64_t t = T[0];
  const uint64_t vl = (uint64_t)c[0] + ((uint64_t)c[1] << 8) + ((uint64_t)c[2] << 16) + ((uint64_t)c[3] << 24);
  const uint64_t vh = (uint64_t)c[4] + ((uint64_t)c[5] << 8) + ((uint64_t)c[6] << 16) + ((uint64_t)c[7] << 24);
  const uint64_t lo = vl + (vh << 32) + e * T[2] + T[3];
  double a = __fma_rn(f64_exact(vh), 4294967296.0, f64_exact(vl));
  a = __fma_rn(ed, __longlong_as_double((long long)T[4]), a);
  a = __dadd_rn(a, __longlong_as_double((long long)T[5]));
  const int64_t k = __double2ll_rn(__dmul_rn(a, __longlong_as_double((long long)T[1])));
  int64_t r = (int64_t)(lo - (uint64_t)k * t);
  r += r < 0 ? (int64_t)t : 0;
  r -= r >= (int64_t)t ? (int64_t)t : 0;
  return (uint64_t)r;
}

constexpr int kTcThreads = 2 * kTcRows;  // two warpgroups share each tile

// Shared memory of one CTA: A (128 rows x KB bytes), B (<= 256 rows x KB), the sources' f64
// products and the overflow counts of a tile, target and source records, two mbarriers, the
// TMEM address slot and the fault flag.
template <int KB>
struct TcSmem {
  uint8_t a[kTcRows * KB];
  uint8_t b[256 * KB];
  double prod[ConvLayout::kTcMaxSrc][kTcRows];
  uint64_t e[kTcRows];
  uint64_t trec[kTcRec * ConvLayout::kTcMaxDst];
  uint64_t srec[ConvLayout::kSrcWords * ConvLayout::kTcMaxSrc];
  uint64_t bar[2];
  uint32_t tslot;
  int fault;
};

// Per tile: thread (g, r) of warpgroup g computes y_j and f64(y_j) / s_j of coefficient r for
// its half of the sources and stores them (A row r, products); one thread issues the MMAs as
// soon as A is complete while warpgroup 0 sums the products in source order into e; both
// warpgroups prefetch their half of the next tile's sources, wait for the MMA, and reduce half
// of the targets each, four at a time (one 32-column TMEM load).
template <int NS, class B>
__global__ void __launch_bounds__(kTcThreads)
    k_bconv_tc(const __grid_constant__ B cb, const PrimeConst* __restrict__ pc, int n, int tiles_per_cta,
               uint32_t ncols) {
  constexpr int KB = NS <= 4 ? 32 : 64;  // operand bytes per coefficient (y words, zero-padded)
  constexpr int NW = KB / 8;
  constexpr int H = (NS + 1) / 2;        // sources of warpgroup 0; warpgroup 1 takes the rest
  extern __shared__ __align__(128) unsigned char smem_raw[];
  TcSmem<KB>& S = *reinterpret_cast<TcSmem<KB>*>(smem_raw);
  const ConvJob& job = cb.j[blockIdx.y];
  const int nd = job.n_dst;
  const uint64_t* tab = job.table;
  const uint64_t* tc = tab + ConvLayout::tc_offset(NS, nd);
  const uint64_t head = __ldg(tc);
  const uint32_t N = (uint32_t)(head >> 32);
  // a table without a valid block for this width (the host never launches one) does nothing
  const bool bad = (uint32_t)head != (uint32_t)KB || N < 8 * (uint32_t)nd || N > 256 || (N & 15) || N > ncols ||
                   ncols < 32 * (uint32_t)((nd + 3) / 4);
  const int tid = threadIdx.x, warp = tid >> 5, g = tid >> 7, r = tid & (kTcRows - 1);
  if (tid == 0) {
    mbar_init(&S.bar[0], 1);
    mbar_init(&S.bar[1], 1);
    S.fault = bad;
    if (bad) atomicExch(&g_device_fault, 2);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) tmem_alloc(&S.tslot, ncols);
  for (int i = tid; i < kTcRec * nd; i += kTcThreads) S.trec[i] = __ldg(tc + 2 + i);
  for (int i = tid; i < ConvLayout::kSrcWords * NS; i += kTcThreads) S.srec[i] = __ldg(tab + ConvLayout::kHeadWords + i);
  tc_before_sync();
  __syncthreads();
  tc_after_sync();
  const uint32_t tmem = S.tslot;
  if (tid == 0 && !bad) bulk_g2s(S.b, tc + 2 + kTcRec * nd, N * KB, &S.bar[0]);
  const int tile0 = blockIdx.x * tiles_per_cta;
  const int tile_end = bad ? tile0 : min(tile0 + tiles_per_cta, n / kTcRows);
  const int j0 = g == 0 ? 0 : H, j1 = g == 0 ? H : NS;  // this thread's sources
  const uint64_t* src = job.src;
  const size_t sstride = job.src_stride;
  uint64_t x[H];
  auto load = [&](int tile) {
    const size_t c = (size_t)tile * kTcRows + r;
#pragma unroll
    for (int u = 0; u < H; ++u)
      if (j0 + u < j1) x[u] = __ldg(src + (j0 + u) * sstride + c);
  };
  if (tile0 < tile_end) load(tile0);
  const uint32_t lane_base = (uint32_t)((warp & 3) * 32) << 16;
  const uint32_t idesc = idesc_u8(kTcRows, N);
  const uint32_t a_base = saddr(S.a), b_base = saddr(S.b);
  uint64_t* arow = reinterpret_cast<uint64_t*>(S.a + (r >> 3) * (8 * KB) + (r & 7) * 16);
  const int groups = (nd + 3) / 4, gsplit = (groups + 1) / 2;
  const int ga = g == 0 ? 0 : gsplit, gb = g == 0 ? gsplit : groups;  // this warpgroup's target groups
  uint32_t phase = 0;
  for (int tile = tile0; tile < tile_end; ++tile) {
    // y_j (word j of A row r: byte a of word j is y_j[a]) and f64(y_j) / s_j of this half
    double pr[H];
#pragma unroll
    for (int u = 0; u < H; ++u) {
      const int j = j0 + u;
      if (j < j1) {
        const uint64_t* s = S.srec + ConvLayout::kSrcWords * j;
        const uint64_t q = __ldg(&pc[(uint32_t)s[0]].q);
        const uint64_t yj = mul_shoup(add_mod(x[u], s[3], q), s[1], s[2], q);
        arow[(j >> 1) * 16 + (j & 1)] = yj;
        pr[u] = __dmul_rn(u64_f64_rn(yj), __longlong_as_double((long long)s[4]));
        if (g == 1) S.prod[j][r] = pr[u];
      }
    }
    if (g == 1 && NS == 2 * H - 1)  // odd source count: warpgroup 1 zeroes the padding word
      arow[(NS >> 1) * 16 + (NS & 1)] = 0;
#pragma unroll
    for (int j = (NS + 1) & ~1; j < NW; ++j)
      if (g == 0) arow[(j >> 1) * 16 + (j & 1)] = 0;
    async_proxy_fence();
    tc_before_sync();
    __syncthreads();
    if (S.fault) break;
    if (tid == 0) {
      if (tile == tile0 && !mbar_wait(&S.bar[0], 0)) {
        S.fault = 1;
      } else {
        tc_after_sync();
#pragma unroll
        for (int kk = 0; kk < KB / 32; ++kk)
          mma_u8(tmem, sdesc(a_base + kk * 256, 128, 8 * KB), sdesc(b_base + kk * 256, 128, 8 * KB), idesc, kk);
        mma_commit(&S.bar[1]);
      }
    }
    // the overflow count e = floor(sum_j f64(y_j) f64(1/s_j)), summed in source order from the
    // first product (crates/ckks-train-core/src/baseconv.rs:198-206)
    if (g == 0) {
      double f = pr[0];
#pragma unroll
      for (int j = 1; j < NS; ++j) f = __dadd_rn(f, j < H ? pr[j < H ? j : 0] : S.prod[j][r]);
      S.e[r] = NS > 1 ? (uint64_t)floor(f) : 0;
    }
    if (tile + 1 < tile_end) load(tile + 1);  // in flight while the tensor core runs
    // warp 0 polls the MMA's completion; the others wait at the barrier without issuing
    if (warp == 0 && !mbar_wait(&S.bar[1], phase)) S.fault = 1;
    phase ^= 1;
    tc_before_sync();
    __syncthreads();  // e is visible; the MMA has completed for every thread
    tc_after_sync();
    if (!S.fault) {
      const uint64_t e = S.e[r];
      const double ed = (double)e;
      const size_t dstride = job.dst_stride;
      uint64_t* dst = job.dst + (size_t)tile * kTcRows + r + (size_t)(4 * ga) * dstride;
      for (int gi = ga; gi < gb; ++gi) {
        uint32_t v[32];
        tmem_ld32(tmem + lane_base + 32 * gi, v);
        uint64_t out[4];
#pragma unroll
        for (int u = 0; u < 4; ++u)
          out[u] = reduce_target(v + 8 * u, e, ed, S.trec + kTcRec * min(4 * gi + u, nd - 1));
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          if (4 * gi + u < nd) *dst = out[u];
          dst += dstride;
        }
      }
    }
    tc_before_sync();
    __syncthreads();  // A, the products and the accumulator are free for the next tile
  }
  if (tile0 >= tile_end && !bad) {
    // the B copy was issued: wait for it (bounded) before the CTA's shared memory goes away
    if (tid == 0) mbar_wait(&S.bar[0], 0);
  }
  tc_before_sync();
  __syncthreads();
  tc_after_sync();
  if (warp == 0) tmem_dealloc(tmem, ncols);
}

template <int NS, class B>
void tc_launch(const DevTables& d, const B& cb, int count, int max_dst, cudaStream_t st) {
  constexpr int KB = NS <= 4 ? 32 : 64;
  const int n = 1 << d.log_n;
  const int tiles = n / kTcRows;
  uint32_t ncols = 32;
  while (ncols < (uint32_t)(8 * max_dst)) ncols <<= 1;  // the MMA width N <= ncols
  // CTAs per SM are capped by shared memory so that their TMEM never exceeds the SM's 512 columns.
  const int per_sm = std::min(8, 512 / (int)ncols);
  int smem = (int)sizeof(TcSmem<KB>);
  if (per_sm < 8) smem = std::max(smem, 233472 / (per_sm + 1));
  // enough CTAs for every SM, several tiles each
  const long total = (long)tiles * count;
  const int tpc = (int)std::max(1L, std::min(16L, total / (148L * per_sm * 2)));
  auto fn = k_bconv_tc<NS, B>;
  cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  fn<<<dim3((tiles + tpc - 1) / tpc, count), kTcThreads, smem, st>>>(cb, d.prime, n, tpc, ncols);
  g_launches.fetch_add(1, std::memory_order_relaxed);
}

template <class B>
bool tc_dispatch(const DevTables& d, const B& cb, int count, int n_src, int max_dst, cudaStream_t st) {
  // auto mode (1) takes the tensor cores from kTcAutoMinSrc sources on, where they measured
  // faster than the integer kernels (fewer sources: cheap integer sums, small grids); mode 2 at
  // any source count
  const int min_src = d.bconv_tc == 2 ? 1 : kTcAutoMinSrc;
  if (!d.bconv_tc || d.log_n < 7 || n_src < min_src || n_src > ConvLayout::kTcMaxSrc || max_dst < 1 ||
      max_dst > ConvLayout::kTcMaxDst)
    return false;
  switch (n_src) {
    case 1: tc_launch<1>(d, cb, count, max_dst, st); break;
    case 2: tc_launch<2>(d, cb, count, max_dst, st); break;
    case 3: tc_launch<3>(d, cb, count, max_dst, st); break;
    case 4: tc_launch<4>(d, cb, count, max_dst, st); break;
    case 5: tc_launch<5>(d, cb, count, max_dst, st); break;
    case 6: tc_launch<6>(d, cb, count, max_dst, st); break;
    case 7: tc_launch<7>(d, cb, count, max_dst, st); break;
    default: tc_launch<8>(d, cb, count, max_dst, st); break;
  }
  return true;
}

}  // namespace

bool launch_bconv_tc(const DevTables& d, const ConvBatch& cb, int count, int n_src, int max_dst, cudaStream_t st) {
  return tc_dispatch(d, cb, count, n_src, max_dst, st);
}

bool launch_bconv_tc_ptr(const DevTables& d, const ConvJob* dev_jobs, int count, int n_src, int max_dst,
                         cudaStream_t st) {
  return tc_dispatch(d, ConvPtrs{count, n_src, max_dst, 0, dev_jobs}, count, n_src, max_dst, st);
}

int device_fault_take() {
  int v = 0;
  if (cudaMemcpyFromSymbol(&v, g_device_fault, sizeof v) != cudaSuccess) return -1;
  if (v) {
    const int zero = 0;
    cudaMemcpyToSymbol(g_device_fault, &zero, sizeof zero);
  }
  return v;
}

}  // namespace ckg
