/*
 * ckg.h -- C ABI of the B200-native RNS-CKKS evaluator path (libckg.so, sm_100a).
 *
 * A drop-in for the device backend behind the `HeOps` evaluator interface of
 * kenmaro3/ckks-train (crates/ckks-train-ckks/src/ops.rs:198-356), i.e. for what
 * `CudaEvaluator` (crates/ckks-train-cuda/src/evaluator.rs:123, 522) and its launch
 * sequences (crates/ckks-train-cuda/src/ks.rs:270-470, basis.rs:455-514) do today.
 *
 * Conventions
 *  - Every function returns CKG_OK (0) or one of the CKG_* status codes, mirroring
 *    HekitError (crates/ckks-train-core/src/error.rs:7-21) plus OOM and TIMEOUT;
 *    ckg_last_error() returns the calling thread's message for the last failure.
 *    Nothing aborts or panics across this boundary.
 *  - Polynomials are limb-major u64 arrays: limb i (residues modulo prime i) occupies
 *    words [i*N, (i+1)*N). A ciphertext is its components one after another.
 *  - Prime indices are global: 0..L are the data primes q_0..q_L, L+1..L+k the special
 *    primes p_0..p_{k-1} (CkksParams::q() and ::p(), crates/ckks-train-ckks/src/params.rs).
 *  - "Device" pointers are CUDA device addresses on the context's device; "host"
 *    pointers are ordinary (pageable or pinned) memory. All work is queued on the
 *    context's stream; ckg_ctx_sync() waits for it. Downloads synchronise.
 *  - Results are bit-identical to the reference's CPU path (crates/ckks-train-core,
 *    crates/ckks-train-ckks) on the same inputs.
 */
#ifndef CKG_H
#define CKG_H

#include <stdint.h>

#if defined(__GNUC__)
#define CKG_API __attribute__((visibility("default")))
#else
#define CKG_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ckg_ctx ckg_ctx;   /* parameters + device tables + stream (CudaDevice, device.rs:290-384) */
typedef struct ckg_key ckg_key;   /* device-resident key-switching key (DeviceKsk, keyswitch.rs:53-216) */
typedef struct ckg_eval ckg_eval; /* evaluator: keys, EvalConfig, OpCounter (CudaEvaluator) */
typedef struct ckg_ct ckg_ct;     /* ciphertext handle; clones share the device buffer (ciphertext.rs) */
typedef struct ckg_pt ckg_pt;     /* plaintext handle (NTT form) */

enum {
  CKG_OK = 0,
  CKG_INVALID_PARAMS = 1,   /* HekitError::InvalidParams */
  CKG_SCALE_MISMATCH = 2,   /* HekitError::ScaleMismatch */
  CKG_LEVEL_MISMATCH = 3,   /* HekitError::LevelMismatch */
  CKG_NO_LEVELS_LEFT = 4,   /* HekitError::NoLevelsLeft */
  CKG_DECODE = 5,           /* HekitError::Decode */
  CKG_DEVICE = 6,           /* HekitError::Device */
  CKG_OOM = 7,              /* HekitError::Device (out of device memory) */
  CKG_TIMEOUT = 8,          /* HekitError::Device (a bounded wait gave up) */
  CKG_CANCELLED = 9         /* serving loop only: request cancelled before admission (no counterpart) */
};

/* EvalConfig flags (crates/ckks-train-ckks/src/ops.rs:111-178). */
enum { CKG_HOIST = 1, CKG_BSGS = 2, CKG_LAZY_RELIN = 4, CKG_OPTIMIZED = 7 };

CKG_API const char* ckg_last_error(void);
CKG_API uint32_t ckg_abi_version(void);
/* Number of kernel launches this library has issued since it was loaded. */
CKG_API uint64_t ckg_launch_count(void);

/* ---- parameters and context -------------------------------------------------------- */

/* SEAL-style prime hand-out of CkksParams::new (crates/ckks-train-ckks/src/params.rs:87-157):
 * fills q_out[nq] and p_out[np]. */
CKG_API int ckg_primes_for_bits(uint32_t log_n, const uint32_t* q_bits, uint32_t nq, const uint32_t* p_bits, uint32_t np,
                        uint64_t* q_out, uint64_t* p_out);

/* CudaDevice::new (crates/ckks-train-cuda/src/device.rs:290-384): uploads the NTT and
 * base-conversion tables for the primes q[0..nq), p[0..np) of ring degree 2^log_n with
 * `dnum` key-switching digits. `stream` is a cudaStream_t to use, or NULL for an own one. */
CKG_API int ckg_ctx_create(uint32_t log_n, const uint64_t* q, uint32_t nq, const uint64_t* p, uint32_t np, uint32_t dnum,
                   int device, void* stream, ckg_ctx** out);
CKG_API void ckg_ctx_destroy(ckg_ctx* ctx);
CKG_API int ckg_ctx_sync(ckg_ctx* ctx);
CKG_API void* ckg_ctx_stream(ckg_ctx* ctx);

/* ---- device-buffer primitives (device pointers) ------------------------------------ */

/* NttTable::forward / ::inverse on every limb (crates/ckks-train-core/src/ntt.rs:141-232);
 * limb i of src/dst uses global prime primes[i]. src may equal dst. */
CKG_API int ckg_ntt(ckg_ctx* ctx, const uint64_t* src, uint64_t* dst, const uint32_t* primes, uint32_t nlimbs, int inverse);

/* RnsPoly add/sub/mul_assign (poly.rs:131-182): op 0 add, 1 sub, 2 pointwise product. */
CKG_API int ckg_poly_binary(ckg_ctx* ctx, int op, const uint64_t* a, const uint64_t* b, uint64_t* out, uint32_t first_prime,
                    uint32_t nlimbs);
/* RnsPoly::neg and ::mul_scalar_assign (poly.rs:157-190). */
CKG_API int ckg_poly_negate(ckg_ctx* ctx, const uint64_t* a, uint64_t* out, uint32_t first_prime, uint32_t nlimbs);
CKG_API int ckg_poly_mul_scalar(ckg_ctx* ctx, const uint64_t* a, uint64_t scalar, uint64_t* out, uint32_t first_prime,
                        uint32_t nlimbs);
/* RnsPoly::automorphism in NTT form (poly.rs:242-262, rns.rs:137-175). out must not alias in. */
CKG_API int ckg_automorphism(ckg_ctx* ctx, const uint64_t* in, uint64_t* out, uint32_t nlimbs, uint64_t galois_elt);
/* RnsPoly::rescale_by_last in NTT form (crates/ckks-train-core/src/baseconv.rs:258-291):
 * in has level+1 limbs, out receives level limbs. */
CKG_API int ckg_rescale(ckg_ctx* ctx, const uint64_t* in, uint32_t level, uint64_t* out);
/* The exact centered lift of digit `digit` of a level-`level` NTT-form polynomial to
 * Q_level * P (keyswitch.rs:140-202): out_q gets level+1 limbs, out_p the k special limbs. */
CKG_API int ckg_mod_up(ckg_ctx* ctx, const uint64_t* in, uint32_t level, uint32_t digit, uint64_t* out_q, uint64_t* out_p);
/* RnsPoly::mod_down (baseconv.rs:459-511), NTT form: (q_part, p_part) over Q_level * P
 * divided by P with rounding -> out (level+1 limbs). */
CKG_API int ckg_mod_down(ckg_ctx* ctx, const uint64_t* q_part, uint32_t level, const uint64_t* p_part, uint64_t* out);

/* Key upload (DeviceKsk, crates/ckks-train-cuda/src/keyswitch.rs:110-216). host_key holds
 * `parts` parts, each b_j then a_j, each q_limbs data limbs then the k special limbs (NTT
 * form); galois_elt is 0 for a relinearization key. One device allocation per key. */
CKG_API int ckg_key_upload(ckg_ctx* ctx, const uint64_t* host_key, uint32_t parts, uint32_t q_limbs, uint64_t galois_elt,
                   ckg_key** out);
/* The same from a device buffer in that layout (copied). */
CKG_API int ckg_key_upload_device(ckg_ctx* ctx, const uint64_t* dev_key, uint32_t parts, uint32_t q_limbs,
                                  uint64_t galois_elt, ckg_key** out);
CKG_API void ckg_key_free(ckg_key* key);
CKG_API uint64_t ckg_key_bytes(const ckg_key* key);

/* keyswitch::key_switch (crates/ckks-train-ckks/src/keyswitch.rs:317-319): in is NTT form
 * at `level`; out_b, out_a receive level+1 limbs each. */
CKG_API int ckg_key_switch(ckg_ctx* ctx, const ckg_key* key, const uint64_t* in, uint32_t level, uint64_t* out_b,
                   uint64_t* out_a);

/* ckg_key_switch without any device allocation. It has no counterpart in the reference.
 * It is for callers that cannot allocate device memory while serving a request, for
 * example a serving process that reserved its whole HBM budget up front and must not fail
 * or stall on an allocation mid-request, or an embedding runtime that owns every device
 * allocation. The caller still passes the input and both outputs.
 *  - The working space is one fixed array of 128 MiB in device memory, held by every GPU
 *    that loads this library until the process exits. A level whose key switch needs more
 *    (e.g. N = 2^16 with 32 data + 4 special primes at its top level) is rejected with
 *    CKG_INVALID_PARAMS and a message stating both sizes; N = 2^16 with 24 + 8 primes and
 *    3 digits fits at every level.
 *  - Every call made outside stream capture looks up that array's device address on the
 *    context's device (so a device reset and a new context are followed); a call made
 *    while the stream captures reuses the last address found, so make the first call on a
 *    device before any stream capture.
 *  - Every call shares the array and leaves it holding its own intermediates; nothing in
 *    it needs to start at zero (each call writes every word it reads). Calls that overlap
 *    on the GPU, for instance from two contexts with different streams on one device,
 *    race on it: order them on one stream. */
CKG_API int ckg_key_switch_noalloc(ckg_ctx* ctx, const ckg_key* key, const uint64_t* in, uint32_t level,
                                   uint64_t* out_b, uint64_t* out_a);

/* ---- evaluator (HeOps, crates/ckks-train-ckks/src/ops.rs:198-356) ------------------- */

/* Evaluator::with_config (evaluator.rs:193-206): relin may be NULL; galois[0..ngal) are
 * Galois keys (their elements set at upload); flags = CKG_* EvalConfig bits. */
CKG_API int ckg_eval_create(ckg_ctx* ctx, const ckg_key* relin, const ckg_key* const* galois, uint32_t ngal, uint32_t flags,
                    ckg_eval** out);
CKG_API void ckg_eval_destroy(ckg_eval* ev);
/* HeOps::fork: same keys and flags, counter at zero. */
CKG_API int ckg_eval_fork(const ckg_eval* ev, ckg_eval** out);
CKG_API uint32_t ckg_eval_config(const ckg_eval* ev);
/* OpCounter (crates/ckks-train-ckks/src/counter.rs:42-58) as 7 words: rotations, relins,
 * ct_ct_tensor, ct_pt_mults, rescales, sse_switches, bootstraps. */
CKG_API void ckg_eval_counter(const ckg_eval* ev, uint64_t out[7]);
CKG_API void ckg_eval_reset_counter(ckg_eval* ev);
CKG_API void ckg_eval_add_counts(ckg_eval* ev, const uint64_t counts[7]);
CKG_API int ckg_eval_has_relin_key(const ckg_eval* ev);
CKG_API int ckg_eval_has_galois_key(const ckg_eval* ev, int32_t step);

/* upload_ct / download_ct (ops.rs:241-257): host buffer of ncomp * (level+1) * N words. */
CKG_API int ckg_ct_upload(ckg_eval* ev, const uint64_t* host, uint32_t ncomp, uint32_t level, double scale, ckg_ct** out);
/* The same from a device buffer (copied). */
CKG_API int ckg_ct_upload_device(ckg_eval* ev, const uint64_t* dev, uint32_t ncomp, uint32_t level, double scale,
                         ckg_ct** out);
CKG_API int ckg_ct_download(const ckg_ct* ct, uint64_t* host);
/* The same without waiting: queued on the context's stream (host should be pinned);
 * the data is in place after ckg_ctx_sync(). */
CKG_API int ckg_ct_download_async(const ckg_ct* ct, uint64_t* host);
/* Copy of the ciphertext into a device buffer (ncomp * (level+1) * N words), queued. */
CKG_API int ckg_ct_download_device(const ckg_ct* ct, uint64_t* dev);
CKG_API void ckg_ct_info(const ckg_ct* ct, uint32_t* ncomp, uint32_t* level, double* scale);
/* Clone shares the device buffer: no allocation, cannot fail (ops.rs:17-20). */
CKG_API ckg_ct* ckg_ct_clone(const ckg_ct* ct);
CKG_API void ckg_ct_free(ckg_ct* ct);
CKG_API int ckg_eval_owns(const ckg_eval* ev, const ckg_ct* ct);

CKG_API int ckg_pt_upload(ckg_eval* ev, const uint64_t* host, uint32_t level, double scale, ckg_pt** out);
CKG_API int ckg_pt_upload_device(ckg_eval* ev, const uint64_t* dev, uint32_t level, double scale, ckg_pt** out);
CKG_API void ckg_pt_info(const ckg_pt* pt, uint32_t* level, double* scale);

/* Overlapped host transfers (no reference counterpart). The same uploads and downloads on two
 * transfer streams of the context, so the uploads of the next batch, the compute of this one
 * and the downloads of the last one run at once, both PCIe directions included. Host memory
 * should be pinned (else the copies are staged and do not overlap) and must stay untouched
 * until its copy completes. Work queued on the context after an upload waits for that upload;
 * a download copies the ciphertext as queued work leaves it, and the ciphertext's memory is
 * not reused before the copy ends, even if its handle is freed at once.
 * ckg_ctx_join_transfers makes the context's stream wait for every transfer queued so far
 * (record a completion event after it); ckg_ctx_sync also waits for them on the host. */
CKG_API int ckg_ct_upload_overlap(ckg_eval* ev, const uint64_t* host, uint32_t ncomp, uint32_t level, double scale,
                                  ckg_ct** out);
CKG_API int ckg_pt_upload_overlap(ckg_eval* ev, const uint64_t* host, uint32_t level, double scale, ckg_pt** out);
CKG_API int ckg_ct_download_overlap(const ckg_ct* ct, uint64_t* host);
CKG_API int ckg_ctx_join_transfers(ckg_ctx* ctx);
/* Host-side accounting since the context was created, up to 9 words in this order: upload calls,
 * bytes uploaded, host ns in the upload pool's allocations, host ns queueing the upload copies,
 * bytes the upload pool holds now, download calls, host ns queueing downloads, device
 * allocations retried after handing cached pool memory back, and transfer blocks reused while
 * still in use (the new transfer waits on the device for the block's last use). */
CKG_API int ckg_ctx_transfer_stats(ckg_ctx* ctx, uint64_t* out, uint32_t n);
/* Hands the device memory the context keeps cached back to the driver: completed transfer
 * blocks and the unused blocks of its pools and of the device's default pool (nothing in use
 * is touched). A device allocation that runs out of memory does this for every context of the
 * process before it fails. */
CKG_API int ckg_ctx_trim(ckg_ctx* ctx);
/* Pinned host memory for the overlapped transfers, allocated by the library's own CUDA runtime
 * (portable: pinned for every context). Free it only when no queued copy still uses it. */
CKG_API int ckg_host_alloc(uint64_t bytes, void** out);
CKG_API void ckg_host_free(void* p);
/* Lists of the same in one call each: the uploads share one device allocation and one
 * stream dependency (every entry is checked before anything is queued; on an error no handle
 * is made); the downloads share one stream dependency and must come from one context. */
CKG_API int ckg_ct_upload_overlap_list(ckg_eval* ev, uint32_t count, const uint64_t* const* hosts,
                                       const uint32_t* ncomp, const uint32_t* levels, const double* scales,
                                       ckg_ct** out);
CKG_API int ckg_pt_upload_overlap_list(ckg_eval* ev, uint32_t count, const uint64_t* const* hosts,
                                       const uint32_t* levels, const double* scales, ckg_pt** out);
CKG_API int ckg_ct_download_overlap_list(uint32_t count, const ckg_ct* const* cts, uint64_t* const* hosts);
CKG_API ckg_pt* ckg_pt_clone(const ckg_pt* pt);
CKG_API void ckg_pt_free(ckg_pt* pt);

/* Ciphertext arithmetic; each has the checks, errors, scale labels and counts of the
 * Evaluator method of the same name (crates/ckks-train-ckks/src/evaluator.rs). */
CKG_API int ckg_add(ckg_eval* ev, const ckg_ct* a, const ckg_ct* b, ckg_ct** out);                  /* :232 */
CKG_API int ckg_sub(ckg_eval* ev, const ckg_ct* a, const ckg_ct* b, ckg_ct** out);                  /* :237 */
CKG_API int ckg_negate(ckg_eval* ev, const ckg_ct* a, ckg_ct** out);                                /* :242 */
CKG_API int ckg_add_plain(ckg_eval* ev, const ckg_ct* a, const ckg_pt* p, ckg_ct** out);            /* :251 */
CKG_API int ckg_mul_plain(ckg_eval* ev, const ckg_ct* a, const ckg_pt* p, ckg_ct** out);            /* :262 */
CKG_API int ckg_mul_scalar(ckg_eval* ev, const ckg_ct* a, double value, double target_scale, ckg_ct** out); /* :361 */
CKG_API int ckg_mul_plain_to_scale(ckg_eval* ev, const ckg_ct* a, const ckg_pt* p, double target_scale,
                           ckg_ct** out);                                                   /* :393 */
CKG_API int ckg_mul_no_relin(ckg_eval* ev, const ckg_ct* a, const ckg_ct* b, ckg_ct** out);         /* :422 */
CKG_API int ckg_relinearize(ckg_eval* ev, const ckg_ct* a, ckg_ct** out);                           /* :441 */
CKG_API int ckg_mul(ckg_eval* ev, const ckg_ct* a, const ckg_ct* b, ckg_ct** out);                  /* :463 */
CKG_API int ckg_rescale_ct(ckg_eval* ev, const ckg_ct* a, ckg_ct** out);                            /* :498 */
CKG_API int ckg_mod_switch_to_level(ckg_eval* ev, const ckg_ct* a, uint32_t level, ckg_ct** out);   /* :513 */
CKG_API int ckg_relabel(ckg_eval* ev, const ckg_ct* a, double scale, ckg_ct** out);                 /* ops.rs:302 */
CKG_API int ckg_rotate(ckg_eval* ev, const ckg_ct* a, int32_t steps, ckg_ct** out);                 /* :534 */
CKG_API int ckg_conjugate(ckg_eval* ev, const ckg_ct* a, ckg_ct** out);                             /* :547 */
/* outs[0..nsteps) receive the rotations in step order (evaluator.rs:572-616). */
CKG_API int ckg_hoisted_rotate(ckg_eval* ev, const ckg_ct* a, const int32_t* steps, uint32_t nsteps, ckg_ct** outs);
CKG_API int ckg_exact_product_scale(const ckg_eval* ev, uint32_t level, double target_scale, double* out); /* :739 */
/* W x for pre-rotated BSGS diagonals (crates/ckks-train-ckks/src/linalg.rs:608-680): d
 * entries in entries[k1*baby + k2] order, `stride` lanes. */
CKG_API int ckg_matvec_plain(ckg_eval* ev, uint32_t d, uint32_t stride, const ckg_pt* const* entries, const ckg_ct* x,
                     ckg_ct** out);
CKG_API int ckg_matvec_enc(ckg_eval* ev, uint32_t d, uint32_t stride, const ckg_ct* const* entries, const ckg_ct* x,
                   ckg_ct** out);
/* CudaEvaluator::matvec_enc_batch (crates/ckks-train-cuda/src/evaluator.rs:437-520): njobs
 * products W_i x_i, job i with d[i] entries at entries[o_i .. o_i + d[i]) (o_i = d[0] + ... +
 * d[i-1]), stride[i] and input xs[i]; outs[i] receives W_i x_i. Every job is checked as
 * ckg_matvec_enc, in order, before any work (the first failure is returned, nothing counted);
 * results and counts equal those of the jobs run one by one. With the optimized EvalConfig the
 * jobs run stage by stage together (all hoisted baby rotations, all inner sums, all
 * relinearizations, all giant rotations: one key-switch launch sequence per stage and level)
 * where the reference spreads whole jobs over streams. */
CKG_API int ckg_matvec_enc_batch(ckg_eval* ev, uint32_t njobs, const uint32_t* d, const uint32_t* stride,
                                 const ckg_ct* const* entries, const ckg_ct* const* xs, ckg_ct** outs);
/* The same for plaintext diagonals (ckg_matvec_plain per job; no counterpart in the reference,
 * which batches only encrypted diagonals). */
CKG_API int ckg_matvec_plain_batch(ckg_eval* ev, uint32_t njobs, const uint32_t* d, const uint32_t* stride,
                                   const ckg_pt* const* entries, const ckg_ct* const* xs, ckg_ct** outs);

/* ---- batched execution at uneven levels ----------------------------------------------
 * A batch holds many ops on ciphertexts of any levels and runs them as one sequence of
 * launches (one per stage for a chunk of ops), optionally captured once into a CUDA graph
 * and replayed. Each op has the checks, errors and result of the evaluator op it stands
 * for (HMult+relinearize+rescale = Evaluator::mul then ::rescale, evaluator.rs:463-510;
 * rotate = evaluator.rs:534-540; mul_plain then rescale = evaluator.rs:262-271, 498-510),
 * checked when the op is added; the outputs are returned at once and hold their values
 * after run / launch_graph completes on the context's stream. Every run adds the ops'
 * counts to the evaluator's OpCounter. Mat-vec products batch through ckg_matvec_enc_batch /
 * ckg_matvec_plain_batch. */
typedef struct ckg_batch ckg_batch;
CKG_API int ckg_batch_create(ckg_eval* ev, ckg_batch** out);
CKG_API void ckg_batch_destroy(ckg_batch* b);
CKG_API int ckg_batch_mul_relin_rescale(ckg_batch* b, const ckg_ct* x, const ckg_ct* y, ckg_ct** out);
CKG_API int ckg_batch_rotate(ckg_batch* b, const ckg_ct* x, int32_t steps, ckg_ct** out);
CKG_API int ckg_batch_mul_plain_rescale(ckg_batch* b, const ckg_ct* x, const ckg_pt* p, ckg_ct** out);
CKG_API int ckg_batch_run(ckg_batch* b);
CKG_API int ckg_batch_capture_graph(ckg_batch* b);
CKG_API int ckg_batch_launch_graph(ckg_batch* b);
CKG_API uint64_t ckg_batch_key_switches(const ckg_batch* b);

/* ---- tuning (no reference counterpart) ---------------------------------------------------
 * Two launch-shape knobs, both bit-neutral (every choice computes the same words):
 * - the NTT limb wave of a context: device-list transforms run as column + row launch pairs
 *   over waves of this many limbs, so the intermediate can stay in L2 (0: one pair for all);
 * - the chunk size of a batch: key-switching ops per launch sequence (default 128).
 * ckg_batch_autotune times every pair of the grid {0, 32, 64, 128, 256} x {64, 128, 256} on
 * the batch's own ops (`reps` graph replays each after a warm-up, no OpCounter change), keeps
 * the fastest (the default shape 0 x 128 when it is within 1% of it): the wave on the context,
 * the chunk size on the batch (rebuilt at its next
 * run or capture). `trials` receives 3 words per trial (wave, chunk size, microseconds per
 * replay), at most `max_trials` of them; `n_trials` the count. */
CKG_API int ckg_ctx_set_ntt_wave(ckg_ctx* ctx, int32_t limbs);
CKG_API int32_t ckg_ctx_ntt_wave(ckg_ctx* ctx);
/* Base conversion engine of a context (bit-neutral; no reference counterpart: the reference's
 * basis_convert runs on CUDA cores). Conversions of <= 8 sources and <= 32 targets can run as
 * exact u8 x u8 -> s32 products on the tensor cores (tcgen05) with an FP64-quotient reduction.
 * Mode 1 (the default when N >= 2^7 and every prime has at least 30 bits) uses them from 6
 * sources on, where they measured faster than the integer kernels; 2 for every source count;
 * 0 never. Setting 1 or 2 on a context that does not qualify fails with CKG_INVALID_PARAMS. */
CKG_API int ckg_ctx_set_bconv_tc(ckg_ctx* ctx, int32_t on);
CKG_API int32_t ckg_ctx_bconv_tc(ckg_ctx* ctx);
/* NTT column-pass staging of a context (bit-neutral; no reference counterpart). 1: persistent
 * column passes whose tiles reach shared memory as one box of a 3-D tensor map per tile
 * (cp.async.bulk.tensor), two stages deep; lists whose limbs do not all lie whole limbs apart
 * in one region take the per-tile kernels. 0 (the default, measured faster at N = 2^16): per-tile
 * kernels that load their tile with ordinary loads. */
CKG_API int ckg_ctx_set_ntt_tma(ckg_ctx* ctx, int32_t on);
CKG_API int32_t ckg_ctx_ntt_tma(ckg_ctx* ctx);
/* Reads and clears the device fault word of the context's device: 0 when no kernel recorded a
 * fault, 1 when a kernel's bounded wait ran out (it freed its tensor memory and returned without
 * its results), 2 when a conversion table lacked its tensor-core block; ckg_ctx_sync also checks
 * it and fails with CKG_DEVICE. */
CKG_API int ckg_device_fault(ckg_ctx* ctx, int32_t* code);
CKG_API int ckg_batch_set_chunk_items(ckg_batch* b, int32_t items);
CKG_API int32_t ckg_batch_chunk_items(const ckg_batch* b);
CKG_API int ckg_batch_autotune(ckg_batch* b, int32_t reps, int32_t* trials, int32_t max_trials, int32_t* n_trials);

/* ---- SEAL 4.1 wire format (crates/ckks-train-ckks/src/seal_compat.rs) ------------------
 * Ciphertexts and plaintexts serialized as Microsoft SEAL 4.1 writes them with
 * compr_mode_type::none (layout at seal_compat.rs:11-33): requests that arrive as bytes are
 * parsed on the host and uploaded, results are written back byte-identical to SEAL's own
 * save. Interop needs SEAL's parameters (ring degree and primes in SEAL's order, SEAL's last
 * prime as the single special prime). Reading treats the bytes as untrusted, as
 * seal_compat.rs:313-455 does: every length is checked against the bytes present, the
 * parms_id must name a data level of the parameters (not the key level), ciphertexts must be
 * in NTT form with 2..16 components and correction factor 1, scales positive and finite,
 * every residue reduced, nothing trailing; compressed and seeded objects are rejected. All
 * failures are CKG_INVALID_PARAMS with a message.
 * Functions marked host need no GPU; they take the data primes q[0..nq) and the special
 * primes p[0..np) of the parameters. */
/* host: SEAL's parms_id of the moduli m[0..count) at ring degree 2^log_n (seal_compat.rs:86-109). */
CKG_API int ckg_seal_parms_id(uint32_t log_n, const uint64_t* m, uint32_t count, uint64_t out[4]);
/* host: serialized length of a ciphertext (ncomp > 0) or a plaintext (ncomp = 0) at `level`. */
CKG_API uint64_t ckg_seal_bytes(uint32_t log_n, uint32_t ncomp, uint32_t level);
/* host: serialize NTT-form words (component-major, limb, coefficient) at `level`; `cap` bytes
 * in `out`, `*len` receives the length (also when `cap` is too small). ncomp = 0: a plaintext. */
CKG_API int ckg_seal_encode(uint32_t log_n, const uint64_t* q, uint32_t nq, const uint64_t* words, uint32_t ncomp,
                            uint32_t level, double scale, uint8_t* out, uint64_t cap, uint64_t* len);
/* host: parse a ciphertext (plaintext = 0) or plaintext (plaintext = 1); `cap` words in
 * `words`, `*nwords` receives the word count (also when `cap` is too small). */
CKG_API int ckg_seal_decode(uint32_t log_n, const uint64_t* q, uint32_t nq, const uint64_t* p, uint32_t np,
                            const uint8_t* bytes, uint64_t len, int plaintext, uint64_t* words, uint64_t cap,
                            uint64_t* nwords, uint32_t* ncomp, uint32_t* level, double* scale);
/* The same through the device: parse and upload (load_ciphertext / load_plaintext), and
 * download and serialize (save_ciphertext). */
CKG_API int ckg_ct_from_seal(ckg_eval* ev, const uint8_t* bytes, uint64_t len, ckg_ct** out);
CKG_API int ckg_pt_from_seal(ckg_eval* ev, const uint8_t* bytes, uint64_t len, ckg_pt** out);
CKG_API int ckg_ct_to_seal(const ckg_ct* ct, uint8_t* out, uint64_t cap, uint64_t* len);

/* ---- bootstrapping ---------------------------------------------------------------------
 * The device side of the reference's bootstrap (crates/ckks-train-ckks/src/bootstrap/): the
 * BootstrapArithmetic ops (poly.rs:453-486), ModRaise with sparse-secret encapsulation
 * (modraise.rs:53-73; to_sparse: 1 part at level 0, to_dense: dnum parts at max_level,
 * both uploaded with ckg_key_upload and Galois element 0), CoeffToSlot / SlotToCoeff over
 * encoded stages (linear.rs:776-859), the level-optimal Chebyshev evaluation
 * (poly.rs:655-714), EvalMod (evalmod.rs:147-189) and the assembled bootstrap
 * (bootstrapper.rs:385-473). Checks, errors, scale labels and OpCounter increments are the
 * CPU code's. Boot parameter arrays `bp` hold 7 words: log_slots, ctos_levels,
 * evalmod_levels, stoc_levels, k_intervals, cheb_degree, double_angle (params.rs:35-66).
 * A stage (ckg_lt) is one LinearTransform (linear.rs:482-497): direction 0 = CoeffToSlot,
 * 1 = SlotToCoeff; `entries` holds d plaintext handles in BSGS order (entry k1*baby + k2 is
 * diagonal offset + baby*k1 + k2 at `stride`, pre-rotated), NULL for an all-zero diagonal;
 * `second` is NULL or d more entries (the conjugate's diagonals in CoeffToSlot's last
 * stage, im's in SlotToCoeff's first). Handles copy what they keep. */
CKG_API int ckg_boot_mul_const(ckg_eval* ev, const ckg_ct* a, double value, double scale, ckg_ct** out); /* :380 */
CKG_API int ckg_boot_add_const(ckg_eval* ev, const ckg_ct* a, double value, ckg_ct** out);               /* :404 */
CKG_API int ckg_boot_zero(ckg_eval* ev, uint32_t level, double scale, ckg_ct** out);                    /* :436 */
CKG_API int ckg_boot_relabel(ckg_eval* ev, const ckg_ct* a, double scale, ckg_ct** out);                /* :481 */
CKG_API int ckg_mul_by_x_half(ckg_eval* ev, const ckg_ct* a, ckg_ct** out);          /* linear.rs:921-936 */
CKG_API int ckg_mod_raise(ckg_eval* ev, const ckg_ct* a, const ckg_key* to_sparse, const ckg_key* to_dense,
                          ckg_ct** out);
typedef struct ckg_lt ckg_lt;
CKG_API int ckg_lt_create(int direction, uint32_t level, double scale, uint32_t d, uint32_t stride, int64_t offset,
                          const ckg_pt* const* entries, const ckg_pt* const* second, ckg_lt** out);
CKG_API void ckg_lt_free(ckg_lt* lt);
CKG_API int ckg_coeff_to_slot(ckg_eval* ev, const ckg_ct* a, const ckg_lt* const* stages, uint32_t n, ckg_ct** re,
                              ckg_ct** im);
CKG_API int ckg_slot_to_coeff(ckg_eval* ev, const ckg_ct* re, const ckg_ct* im, const ckg_lt* const* stages,
                              uint32_t n, ckg_ct** out);
CKG_API int ckg_eval_chebyshev(ckg_eval* ev, const ckg_ct* a, const double* coeffs, uint32_t n, double lo, double hi,
                               double target_scale, ckg_ct** out);
CKG_API int ckg_eval_mod(ckg_eval* ev, const ckg_ct* a, const uint32_t* bp, const double* coeffs, uint32_t n,
                         ckg_ct** out);
typedef struct ckg_boot ckg_boot;
/* scales: {evalmod_scale, stoc_input_scale, delta} (bootstrapper.rs:207-230); galois: the
 * stages' rotation keys and the conjugation key; to_sparse / to_dense both NULL: ModRaise
 * under the main key. */
CKG_API int ckg_boot_create(ckg_ctx* ctx, const uint32_t* bp, const ckg_lt* const* ctos, uint32_t nctos,
                            const ckg_lt* const* stoc, uint32_t nstoc, const ckg_key* const* galois, uint32_t ngal,
                            const ckg_key* to_sparse, const ckg_key* to_dense, const double* coeffs, uint32_t ncoeffs,
                            const double* scales, ckg_boot** out);
CKG_API void ckg_boot_destroy(ckg_boot* b);
CKG_API int ckg_bootstrap(ckg_boot* b, ckg_eval* ev, const ckg_ct* a, ckg_ct** out);
CKG_API uint32_t ckg_boot_output_level(const ckg_boot* b);

/* ---- bootstrap setup (what the reference's Bootstrapper::new prepares on the host,
 * bootstrapper.rs:250-290): the encoder (encoder.rs:215-283), the special-DFT stages adapted
 * and encoded at their exact diagonal scales (linear.rs:401-677, linalg.rs:334-369), their
 * rotation steps (linear.rs:432-450) and the EvalMod series (evalmod.rs:58-96). The f64 steps
 * follow the reference's operation order, so encodings carry the reference's integers.
 * Functions marked host need no GPU. Keys are not generated here (they are the owner's). */
/* values: `count` complex numbers as (re, im) pairs; NTT-form device plaintext at `level`. */
CKG_API int ckg_encode_complex(ckg_eval* ev, const double* values, uint32_t count, double scale, uint32_t level,
                               ckg_pt** out);
/* host: the same encoding over the data primes q[0..nq), coefficient form, (level+1) x 2^log_n. */
CKG_API int ckg_encode_complex_host(uint32_t log_n, const uint64_t* q, uint32_t nq, const double* values,
                                    uint32_t count, double scale, uint32_t level, uint64_t* out);
/* host: rotation steps of both transforms (n set to the count; out may be NULL). */
CKG_API int ckg_boot_rotation_steps(const uint32_t* bp, int32_t* out, uint32_t cap, uint32_t* n);
/* host: the cheb_degree + 1 EvalMod coefficients. */
CKG_API int ckg_evalmod_coeffs(const uint32_t* bp, double* out, uint32_t cap);
/* host: layout of stage `stage` of a direction: info = {d, stride, offset, has_second,
 * stages}; kept[i] / kept[d + i]: entry i of the main / second diagonals is stored. */
CKG_API int ckg_boot_plan(const uint32_t* bp, int direction, uint32_t stage, int64_t* info, uint8_t* kept);
/* (evalmod_scale, stoc_input_scale) for inputs at scale delta (bootstrapper.rs:207-230). */
CKG_API int ckg_boot_stage_scales(ckg_ctx* ctx, const uint32_t* bp, double delta, double* out2);
/* All stages of a direction, encoded on this evaluator's context (out holds `cap` handles). */
CKG_API int ckg_boot_encode_stages(ckg_eval* ev, const uint32_t* bp, int direction, double delta, ckg_lt** out,
                                   uint32_t cap);
/* A bootstrapper whose stages and EvalMod series are encoded here (ckg_boot_create with
 * ckg_boot_encode_stages, ckg_evalmod_coeffs and ckg_boot_stage_scales). */
CKG_API int ckg_boot_create_encoded(ckg_eval* ev, const uint32_t* bp, double delta, const ckg_key* const* galois,
                                    uint32_t ngal, const ckg_key* to_sparse, const ckg_key* to_dense, ckg_boot** out);

/* ---- serving loop ----------------------------------------------------------------------
 * No counterpart in the reference, which runs one HeOps call at a time. A server admits
 * requests from many key owners as they arrive and runs them with continuous batching:
 * while one batch computes, the next is admitted, its missing keys are copied up on a
 * second stream and it is queued behind (at most `max_inflight` batches on the device).
 * Every key is registered once into pinned host memory; device copies are cached LRU and
 * evicted (spilled back to the host copy) to keep the cached keys plus the working space of
 * the queued batches within `hbm_budget_bytes`. A request that cannot fit even alone fails
 * with CKG_OOM. Request kinds and the HeOps call each one stands for, with that call's
 * checks and errors (crates/ckks-train-ckks/src/ops.rs:20-108):
 *   mul        Evaluator::mul then ::rescale (evaluator.rs:463-510), relinearization key;
 *   rotate     Evaluator::rotate (evaluator.rs:534-540), the step's Galois key;
 *   mul_plain  Evaluator::mul_plain then ::rescale (evaluator.rs:262-271, 498-510);
 *   matvec     matvec_plain with hoisted BSGS (linalg.rs:608-622), the step keys;
 *   bootstrap  Bootstrapper::bootstrap (bootstrapper.rs:385-473), one per flight, in its own
 *              completion segment.
 * Each result is bit-identical to the op run on its own. ckg_server_result waits for one
 * request (timeout_ms < 0: no limit; CKG_TIMEOUT leaves it pending), returns its status
 * (the op's error text via ckg_last_error), its output and times_us = {submitted, admitted,
 * completed} in microseconds since the server was created, then forgets it. Inputs and
 * outputs are ordinary ciphertext handles of the context; the context must outlive the
 * server. ckg_server_destroy cancels waiting requests and waits for queued batches.
 * Stats (ckg_server_stats, up to 17 words in this order): submitted, completed, failed,
 * cancelled, batches, multi_owner_batches, max_batch_requests, key_hits, key_misses,
 * key_evictions, key_upload_bytes, key_bytes, peak_key_bytes, peak_device_bytes,
 * budget_waits, pending, hbm_budget. */
typedef struct ckg_server ckg_server;
enum { CKG_REQ_MUL = 0, CKG_REQ_ROTATE = 1, CKG_REQ_MUL_PLAIN = 2, CKG_REQ_MATVEC = 3, CKG_REQ_BOOTSTRAP = 4 };
/* ckg_server_create flags beside the CKG_HOIST / CKG_BSGS / CKG_LAZY_RELIN bits: compute lanes.
 * CKG_SERVE_BOOT_LANE runs bootstrap flights on a stream of their own and all other flights on
 * another; CKG_SERVE_BOOT_LANES_2 gives bootstraps two streams (two bootstraps at once). Each
 * lane has its own memory pool; the other flights' lane takes up to max_inflight flights, a
 * bootstrap lane one. The bootstrap lanes run at the
 * device's highest stream priority unless CKG_SERVE_LANES_EQUAL_PRIORITY is set. Lanes start
 * after the client's work queued on the context's stream when the flight is built, and every
 * output is handed back to the context's stream when its request completes. */
enum { CKG_SERVE_BOOT_LANE = 256, CKG_SERVE_BOOT_LANES_2 = 512, CKG_SERVE_LANES_EQUAL_PRIORITY = 1024 };
CKG_API int ckg_server_create(ckg_ctx* ctx, uint64_t hbm_budget_bytes, uint32_t max_batch_ks, uint32_t max_inflight,
                              uint32_t flags, ckg_server** out);
CKG_API void ckg_server_destroy(ckg_server* s);
CKG_API int ckg_server_add_owner(ckg_server* s, uint32_t* owner);
/* key: the layout of ckg_key_upload; galois_elt 0 registers the relinearization key. */
CKG_API int ckg_server_add_key(ckg_server* s, uint32_t owner, const uint64_t* key, int device_src, uint32_t parts,
                               uint32_t q_limbs, uint64_t galois_elt);
/* The owner's SSE keys for its bootstrap requests (to_sparse: 1 part, 1 data limb; to_dense:
 * dnum parts, L+1 data limbs; the layout of ckg_key_upload). */
CKG_API int ckg_server_add_sse_keys(ckg_server* s, uint32_t owner, const uint64_t* to_sparse, const uint64_t* to_dense,
                                    int device_src);
/* Encodes the bootstrap stages and EvalMod series once (bp: 7 words, as ckg_boot_create) so
 * bootstrap requests (bootstrapper.rs:385-473, the owner's relinearization, rotation,
 * conjugation and SSE keys) can be served; inputs at level 0 and scale delta. */
CKG_API int ckg_server_enable_bootstrap(ckg_server* s, const uint32_t* bp, double delta);
CKG_API int ckg_server_submit_bootstrap(ckg_server* s, uint32_t owner, const ckg_ct* a, uint64_t* id);
CKG_API int ckg_server_submit_mul(ckg_server* s, uint32_t owner, const ckg_ct* a, const ckg_ct* b, uint64_t* id);
CKG_API int ckg_server_submit_rotate(ckg_server* s, uint32_t owner, const ckg_ct* a, int32_t steps, uint64_t* id);
CKG_API int ckg_server_submit_mul_plain(ckg_server* s, uint32_t owner, const ckg_ct* a, const ckg_pt* p, uint64_t* id);
CKG_API int ckg_server_submit_matvec(ckg_server* s, uint32_t owner, uint32_t d, uint32_t stride,
                                     const ckg_pt* const* diag, const ckg_ct* x, uint64_t* id);
CKG_API int ckg_server_result(ckg_server* s, uint64_t id, int64_t timeout_ms, ckg_ct** out, double* times_us);
CKG_API int ckg_server_cancel(ckg_server* s, uint64_t id, int* cancelled);
CKG_API int ckg_server_drain(ckg_server* s, int64_t timeout_ms);
CKG_API int ckg_server_stats(const ckg_server* s, uint64_t* out, uint32_t n);
CKG_API int ckg_server_owner_counter(const ckg_server* s, uint32_t owner, uint64_t* out7);
/* Test hook: the next `count` key uploads fail as an allocation failure would. */
CKG_API int ckg_server_inject_upload_failures(ckg_server* s, uint32_t count);

/* Opt-in bounds checking (CKG_CHECK_BOUNDS=1 in the environment): before each launch, and before
 * a batch uploads its work lists, every buffer a kernel will touch is checked on the host against
 * the device allocations the library made: a range that starts in a live allocation must end in
 * it, and one that starts in recently freed memory is a use after free. A violation fails the call
 * with CKG_DEVICE and a message naming the buffer; nothing is queued. Buffers the library did not
 * allocate pass unchecked. Test hook over the registry: op 0 turns checking on (bytes != 0) or off,
 * 1 records an allocation [p, p + bytes), 2 records the free of the allocation at p, 3 checks
 * [p, p + bytes). */
CKG_API int ckg_debug_bounds(int op, uint64_t p, uint64_t bytes);

#ifdef __cplusplus
}
#endif

#endif /* CKG_H */
