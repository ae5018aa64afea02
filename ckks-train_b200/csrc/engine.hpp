// Device context and the polynomial-level algorithms of the evaluator path built from the
// kernels: NTT/INTT, rescale, ModUp (exact centered digit lift), ModDown, hybrid key
// switching (single, batched and hoisted).
//
// Layout in HBM: a polynomial at level l is l+1 limbs of N words, limb-major and
// contiguous; a ciphertext is its components one after another. An element of Q_l * P
// ("extended" polynomial) is l+1 data limbs followed by the k special limbs. A key is
// dnum parts, each b then a, each (key_q + k) limbs (data primes 0..key_q-1, then P).
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "host_math.hpp"
#include "kernels.cuh"
#include "launch.hpp"

namespace ckg {

// Status codes of the C ABI (include/ckg.h).
enum Status {
  ST_OK = 0,
  ST_INVALID_PARAMS = 1,
  ST_SCALE_MISMATCH = 2,
  ST_LEVEL_MISMATCH = 3,
  ST_NO_LEVELS_LEFT = 4,
  ST_DECODE = 5,
  ST_DEVICE = 6,
  ST_OOM = 7,
  ST_TIMEOUT = 8,
};

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] void throw_cuda(cudaError_t e, const char* what);
#define CKG_CUDA(x)                              \
  do {                                           \
    cudaError_t e_ = (x);                        \
    if (e_ != cudaSuccess) ::ckg::throw_cuda(e_, #x); \
  } while (0)

// The context's stream, shared by the context and every allocation made on it, so the
// stream outlives the last stream-ordered free whatever order handles are released in.
struct StreamRes {
  cudaStream_t s = nullptr;
  int device = 0;
  bool own = false;
  ~StreamRes();
};
typedef std::shared_ptr<StreamRes> StreamPtr;

// Device blocks of the overlapped transfers, kept for reuse: a block comes back with an event
// that completes when its last reader is done, and is handed out again only after that event
// (so the next step's uploads never depend on how a memory pool tracks cross-stream frees).
struct XferCache {
  struct Block {
    uint64_t* p;
    size_t words;
    cudaEvent_t done;
  };
  static constexpr size_t kMaxBlocks = 16;
  static constexpr int kReuseDepth = 2;  // fitting blocks in use before one is reused in use
  std::mutex mu;
  std::vector<Block> blocks;  // oldest first
  size_t max_bytes = 0;       // kept at most (a third of the device's memory)
  int device = 0;
  cudaMemPool_t pool = nullptr;  // where new blocks come from and trimmed ones go back
  StreamPtr stream;               // the upload stream (allocations and trims)
  // A block of words..5/4 words: a completed one, else (when kReuseDepth fitting blocks are in
  // use) the oldest of them with `on` made to wait for its last use; null otherwise.
  uint64_t* take(size_t words, cudaStream_t on);
  std::atomic<uint64_t> waited{0};  // blocks handed out still in use
  void give(uint64_t* p, size_t words, cudaEvent_t done);  // takes ownership of `done`
  void trim();  // completed blocks back to the pool
  ~XferCache();
};
typedef std::shared_ptr<XferCache> XferCachePtr;

// A stream-ordered device allocation of `words` u64.
struct DevBuf {
  uint64_t* p = nullptr;
  size_t words = 0;
  StreamPtr sres;
  // Copies still reading the buffer on other streams (overlapped downloads): the free on
  // `sres` waits for them.
  std::vector<cudaEvent_t> waits;
  int device = 0;
  bool pooled = true;
  XferCachePtr cache;  // set: the block returns to this cache instead of being freed
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf();
};
typedef std::shared_ptr<DevBuf> DevBufPtr;

struct Context;

// A compute lane: a second stream beside a context's own, with its own memory pool, which
// reuses a freed block only once its free has completed (so the lane never waits on work
// queued on another stream). While a thread holds a LaneScope for a context, every launch,
// allocation and free it makes through that context goes to the lane.
struct Lane {
  StreamPtr sres;
  cudaMemPool_t pool = nullptr;
  Lane(int device, int priority = 0);  // stream priority (lower number: scheduled first)
  ~Lane();
  Lane(const Lane&) = delete;
  Lane& operator=(const Lane&) = delete;
};
struct LaneBinding {
  const Context* ctx = nullptr;
  const Lane* lane = nullptr;
};
extern thread_local LaneBinding tl_lane;
class LaneScope {
 public:
  LaneScope(const Context& c, const Lane& l) : prev_(tl_lane) { tl_lane = LaneBinding{&c, &l}; }
  ~LaneScope() { tl_lane = prev_; }
  LaneScope(const LaneScope&) = delete;
  LaneScope& operator=(const LaneScope&) = delete;

 private:
  LaneBinding prev_;
};

// A context's stream as its users see it: the context's own, or the calling thread's lane.
class CtxStream {
 public:
  explicit CtxStream(const Context* c) : c_(c) {}
  operator cudaStream_t() const;

 private:
  const Context* c_;
};

// A key-switching key resident in HBM (one allocation).
struct DevKey {
  Context* ctx = nullptr;
  DevBufPtr buf;
  uint32_t parts = 0;   // digits the key serves
  uint32_t q_limbs = 0; // data limbs per part (max level + 1 of the key)
  uint64_t elt = 0;     // Galois element (0 for a relinearization key)
};

struct Context {
  int device = 0;
  StreamPtr sres;
  CtxStream stream{this};
  StreamPtr cur_sres() const {  // the stream frees of buffers allocated now are ordered on
    return tl_lane.ctx == this && tl_lane.lane ? tl_lane.lane->sres : sres;
  }
  uint32_t log_n = 0;
  uint64_t n = 0;
  uint32_t nq = 0, k = 0, dnum = 0, alpha = 0, L = 0;
  std::vector<uint64_t> primes;  // q_0..q_L, p_0..p_{k-1}
  std::vector<HostMod> mods;
  DevTables dt{};
  PrimeConst* d_prime = nullptr;
  ulonglong2* d_tw_fwd = nullptr;
  ulonglong2* d_tw_inv = nullptr;
  double* d_twd_fwd = nullptr;
  double* d_twd_inv = nullptr;
  uint64_t* d_conv = nullptr;  // all conversion tables
  uint64_t* d_consts = nullptr;  // finish constants (Shoup pairs)
  std::vector<size_t> modup_off;    // [l * dnum + j] word offset into d_conv
  std::vector<size_t> moddown_off;  // [l]
  std::vector<size_t> rescale_off;  // [l], l >= 1
  std::vector<std::pair<uint64_t, uint64_t>> pinv;                 // P^-1 mod q_i
  std::vector<std::vector<std::pair<uint64_t, uint64_t>>> qlinv;  // [l][i] q_l^-1 mod q_i
  std::mutex mu;
  std::map<uint64_t, uint32_t*> perms;  // NTT-form Galois permutations on the device

  Context(uint32_t log_n, const std::vector<uint64_t>& q, const std::vector<uint64_t>& p, uint32_t dnum, int device,
          cudaStream_t st);
  ~Context();

  uint32_t digits_at(uint32_t l) const { return (l + alpha) / alpha < dnum ? (l + alpha) / alpha : dnum; }
  uint32_t digit_start(uint32_t j) const { return j * alpha; }
  uint32_t digit_end(uint32_t j, uint32_t l) const { return std::min((j + 1) * alpha, l + 1); }
  uint32_t p_prime(uint32_t t) const { return L + 1 + t; }  // global index of special prime t
  const uint32_t* perm(uint64_t elt);                       // cached device permutation
  const uint64_t* x_half();  // NTT form of the monomial X^(N/2) over q_0..q_L (cached)
  uint64_t* d_xhalf = nullptr;
  DevBufPtr alloc(size_t words);                            // stream-ordered, on `stream`
  void activate() const;                                    // makes `device` current

  // Overlapped host transfers: an upload stream and a download stream beside `stream`
  // (created on first use). Buffers they fill are allocated on the upload stream and freed on
  // `stream`, which waits for the copy before its first use.
  // Upload buffers come from their own pool, which reuses a freed block only once its free
  // has completed (no stream wait inserted): the next uploads never wait for queued compute.
  StreamPtr xfer_in, xfer_out;
  cudaMemPool_t xpool = nullptr;
  XferCachePtr xcache;
  uint64_t* xfer_block(size_t words, cudaStream_t on);  // from the cache, else a new block of the upload pool
  void transfer_streams();
  DevBufPtr upload_overlapped(const uint64_t* host, size_t words);
  // Several host buffers into one allocation (one copy each, one stream dependency):
  // part i starts at offsets[i] words (256-byte aligned).
  struct HostPart {
    const uint64_t* host;
    size_t words;
  };
  DevBufPtr upload_overlapped_list(const std::vector<HostPart>& parts, std::vector<size_t>& offsets);
  void download_overlapped(const DevBufPtr& buf, const uint64_t* dev, size_t row_words, size_t pitch_words,
                           size_t rows, uint64_t* host);
  struct DevPart {
    const DevBufPtr* buf;
    const uint64_t* dev;
    size_t row_words, pitch_words, rows;
    uint64_t* host;
  };
  void download_overlapped_list(const std::vector<DevPart>& parts);
  void join_transfers();  // `stream` waits for every transfer queued so far
  void sync_transfers();  // the host waits for them

  // Host-built records (batch work lists) copied to the device on `stream` through a pinned
  // staging ring, so the call returns at once: a copy from pageable memory can make the host
  // wait for the work already queued on the stream. A slot is reused once its copy completed.
  // Not allowed while the stream is being captured (the graph would read a reused slot).
  void upload_staged(void* dst, const void* src, size_t bytes);

  // Hands the device memory this context keeps cached back to the driver: completed transfer
  // blocks, the unused blocks of the upload pool, of its lanes' pools and of the device's
  // default pool. trim_all() does it for every live context of the process (an allocation that
  // runs out of memory calls it before it fails).
  void trim();
  static void trim_all();

  // Two lanes for work one caller splits over concurrent host threads (the bootstrap's two
  // independent EvalMods), created on first use and kept for the context's life.
  Lane& aux_lane(int i);
  std::mutex aux_mu;
  std::unique_ptr<Lane> aux_lanes[2];

  // Host-side accounting of the overlapped transfers and allocation retries (ckg_ctx_transfer_stats).
  std::atomic<uint64_t> st_upload_calls{0}, st_upload_bytes{0}, st_upload_alloc_ns{0}, st_upload_copy_ns{0},
      st_download_calls{0}, st_download_ns{0}, st_alloc_retries{0};
  std::mutex stage_mu;
  unsigned char* stage = nullptr;
  size_t stage_cap = 0, stage_head = 0;
  struct StageUse {
    size_t off, len;
    cudaEvent_t done;
  };
  std::deque<StageUse> stage_used;
};

// ---- polynomial-level algorithms (all asynchronous on ctx.stream) -------------------

// In-place (or out-of-place) NTT of `count` contiguous limbs with primes first..first+count-1.
void ntt_poly(Context& c, const uint64_t* src, uint64_t* dst, uint32_t first_prime, uint32_t count, bool inverse);
void ntt_limbs(Context& c, const std::vector<LimbRef>& refs, bool inverse);

// Rescale by the last prime of each level-l input (NTT form): out gets l limbs.
void rescale_many(Context& c, const std::vector<const uint64_t*>& in, uint32_t l, const std::vector<uint64_t*>& out);

// ModDown of extended polynomials (NTT form): out_i = (x_i - conv(round(X/P))_i) * P^-1 (+ add).
struct ModDownJob {
  const uint64_t* qpart;  // l+1 limbs
  const uint64_t* ppart;  // k limbs
  uint64_t* out;          // l+1 limbs
  const uint64_t* add;    // optional addend (l+1 limbs)
  const uint32_t* add_perm;
};
void mod_down_many(Context& c, const std::vector<ModDownJob>& jobs, uint32_t l);

// Exact centered lift of every digit of each level-l input (NTT form): conv[j] receives
// the T_j = l+1-alpha_j+k converted limbs (data primes outside the digit, then P), NTT form.
// `conv_out[i]` is a buffer of conv_words(l) words per input; digit j starts at conv_offset(j).
size_t conv_limbs(const Context& c, uint32_t l);
size_t conv_offset_limbs(const Context& c, uint32_t l, uint32_t j);
void mod_up_many(Context& c, const std::vector<const uint64_t*>& in, uint32_t l, const std::vector<uint64_t*>& conv_out);

// Key switching (keyswitch.rs:230-319) of d (NTT form, level l) with `key`:
// out_b = ModDown(sum_j d_j b_j) (+ add_b), out_a likewise. With `perm` the digits of `in`
// are read through the Galois permutation (hoisting); `conv` may carry precomputed digits.
struct KsJob {
  const uint64_t* in;
  const DevKey* key;
  uint64_t* out_b;
  uint64_t* out_a;
  const uint64_t* add_b = nullptr;
  const uint64_t* add_a = nullptr;
  const uint32_t* add_b_perm = nullptr;
  const uint32_t* perm = nullptr;     // digit permutation (hoisted rotation)
  const uint64_t* conv = nullptr;     // precomputed ModUp of `in` (hoisting); null = compute
};
void key_switch_many(Context& c, const std::vector<KsJob>& jobs, uint32_t l);

// Scratch words a key switch of one level-l polynomial needs (for the caller-provided
// scratch variant).
size_t key_switch_scratch_words(const Context& c, uint32_t l);
void key_switch_with_scratch(Context& c, const KsJob& job, uint32_t l, uint64_t* scratch);

}  // namespace ckg
