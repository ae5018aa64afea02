// Host-side launchers of the device kernels (kernels.cu).
#pragma once
#include <cuda_runtime.h>

#include <atomic>

#include "kernels.cuh"

namespace ckg {

// Kernel launches issued by this library since it was loaded.
extern std::atomic<uint64_t> g_launches;

// Device tables of one context: per-prime constants and the twiddle tables.
struct DevTables {
  const PrimeConst* prime;   // [n_primes]
  const ulonglong2* tw_fwd;  // [n_primes][N] (w, w') with roots[bitrev(i)] = psi^i
  const ulonglong2* tw_inv;  // [n_primes][N] inverse roots
  const double* twd_fwd;     // [n_primes][N] the same roots as doubles (FP64 butterflies)
  const double* twd_inv;
  int log_n;
  int ntt_wave;  // limbs per column + row launch pair of device-list transforms (0: all at once)
  int bconv_tc;  // tensor-core conversions (<= 8 sources, <= 32 targets): 0 off, 1 from 6 sources, 2 all
  int ntt_tma;   // nonzero: NTT column passes run persistent with TMA-staged tiles (tensor maps)
  int sms;       // streaming multiprocessors of the device
};

// A device region holding whole limbs (N words each) from `base`: the TMA-staged column passes
// read the limbs of a list through one tensor map over it.
struct LimbRegion {
  const uint64_t* base;
  uint64_t limbs;
};

void launch_ntt(const DevTables& d, const LimbRef* refs, int count, bool inverse, cudaStream_t st);
void launch_bconv(const DevTables& d, const ConvJob* jobs, int count, int n_src, int n_dst, cudaStream_t st);
void launch_inner_product(const DevTables& d, int alpha, int L, int k, const IpJob* jobs, int count, cudaStream_t st);
void launch_finish(const DevTables& d, const FinRef* refs, int count, cudaStream_t st);
// Forward NTT of each FinRef's t (in place for the column pass) fused with its finish:
// out = (x - NTT(t)) * c (+ add). `dev_cols` holds the matching in-place LimbRefs of t.
// `cols`, when given, are the column passes' own refs (one per FinRef, N >= 2^12), e.g. a
// centred-lift load (LimbRef::aux); by default each column pass runs in place on the FinRef's t.
void launch_ntt_finish(const DevTables& d, const FinRef* refs, int count, cudaStream_t st,
                       const LimbRef* cols = nullptr);
void launch_ntt_finish_ptr(const DevTables& d, const LimbRef* dev_cols, const FinRef* dev_fin, int count,
                           cudaStream_t st, const LimbRegion* region = nullptr);
void launch_binary(const DevTables& d, const BinRef* refs, int count, int op, cudaStream_t st);
void launch_unary(const DevTables& d, const LimbRef* refs, int count, int op, const uint64_t* consts,
                  const uint32_t* perm, cudaStream_t st);

void launch_tensor(const DevTables& d, const TensorRef* refs, int count, cudaStream_t st);

// The same kernels over work lists resident in device memory (one launch each).
// `region`: every limb the column passes read lies in it (enables the TMA-staged passes).
void launch_ntt_ptr(const DevTables& d, const LimbRef* dev_refs, int count, bool inverse, cudaStream_t st,
                    const LimbRegion* region = nullptr);
// max_dst: the largest job's target count (0: unknown, the integer kernel runs).
void launch_bconv_ptr(const DevTables& d, const ConvJob* dev_jobs, int count, int n_src, cudaStream_t st,
                      int max_dst = 0);
// The tensor-core conversion (bconv_tc.cu); false when it does not apply (d.bconv_tc off, more
// than 8 sources or 32 targets, N < 2^7), in which case nothing was launched.
bool launch_bconv_tc(const DevTables& d, const ConvBatch& cb, int count, int n_src, int max_dst, cudaStream_t st);
bool launch_bconv_tc_ptr(const DevTables& d, const ConvJob* dev_jobs, int count, int n_src, int max_dst,
                         cudaStream_t st);
// Reads and clears the current device's fault word: nonzero when a kernel's bounded wait ran out
// (1) or it was handed a table without its tensor-core block (2); -1 when it cannot be read.
int device_fault_take();
void launch_inner_product_ptr(const DevTables& d, int alpha, int L, int k, const IpJob* dev_jobs, int count,
                              int max_limbs, cudaStream_t st);
void launch_finish_ptr(const DevTables& d, const FinRef* dev_refs, int count, cudaStream_t st);
void launch_binary_ptr(const DevTables& d, const BinRef* dev_refs, int count, int op, cudaStream_t st);
void launch_tensor_ptr(const DevTables& d, const TensorRef* dev_refs, int count, cudaStream_t st);
void launch_gather_ptr(const DevTables& d, const GatherRef* dev_refs, int count, cudaStream_t st);
// Copies `count` segments (a device array) into their contiguous destinations.
void launch_pack(const PackSeg* dev_segs, int count, cudaStream_t st);
// mode 0: multiply by the per-prime Shoup constant; mode 1: add the per-prime constant.
void launch_scalar(const DevTables& d, const LimbRef* refs, int count, const ScalarTable& table, cudaStream_t st,
                   int mode = 0);
void launch_mac_plain(const DevTables& d, const MacBatch& b, cudaStream_t st);
void launch_mac_tensor(const DevTables& d, const MacTensorBatch& b, cudaStream_t st);
// Centered lift of the coefficient-form level-0 limb `src` into the prime of each ref.
void launch_lift_level0(const DevTables& d, const LimbRef* refs, int count, cudaStream_t st);

}  // namespace ckg
