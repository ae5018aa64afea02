// Serving loop: continuous batching of evaluator requests from many key owners on one device.
//
// Client threads submit requests at any time: HMult+relinearize+rescale, rotation,
// plaintext-multiply+rescale and plaintext BSGS mat-vec, each on behalf of a key owner whose
// evaluation keys were registered once. Every key lives in pinned host memory; a device copy
// is kept in an LRU cache whose bytes, together with the working space of the batches on the
// device, stay within an HBM budget. A worker thread admits waiting requests in arrival
// order into the next batch as soon as a batch slot (at most `max_inflight` batches queued on
// the device) and the budget allow, evicting the least recently used keys that the batch
// does not need, uploads the missing keys on a copy stream (so they cross PCIe while the
// previous batch computes), and queues the batch: all its key-switching ops, from every
// owner, go through one Batch launch sequence; mat-vecs run through the owner's evaluator
// (hoisted baby steps) right behind it on the same stream. A completion thread watches each
// batch's event, stamps the requests' completion times and releases the batch's keys and
// working space, which lets the worker admit more. Each result is bit-identical to the same
// op run alone: batching only changes which launch computes a ciphertext, never how.
//
// The reference has no serving loop; each request type maps onto its HeOps call
// (crates/ckks-train-ckks/src/ops.rs:20-108) with that call's checks and errors.
#pragma once
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <list>
#include <map>
#include <thread>
#include <unordered_map>

#include "batch.hpp"
#include "boot.hpp"

namespace ckg {

enum ReqKind : uint32_t { REQ_MUL = 0, REQ_ROTATE = 1, REQ_MUL_PLAIN = 2, REQ_MATVEC = 3, REQ_BOOTSTRAP = 4 };
constexpr int ST_CANCELLED = 9;  // request cancelled before it was admitted

struct ServerConfig {
  size_t hbm_budget = 0;         // bytes: device key copies + working space of queued batches
  uint32_t max_batch_ks = 128;   // key switches admitted into one batch
  uint32_t max_inflight = 2;     // batches queued on the device at once (per lane)
  EvalConfig eval;
  // Compute lanes (boot_lanes >= 1): bootstrap flights on `boot_lanes` streams of their own, every
  // other flight on one more, all beside the context's stream (which then carries only the
  // client's own work); the bootstrap lanes at the device's highest stream priority unless
  // boot_priority is off. 0: every flight on the context's stream.
  uint32_t boot_lanes = 0;
  bool boot_priority = true;
};

struct ServerStats {
  uint64_t submitted = 0, completed = 0, failed = 0, cancelled = 0, batches = 0, multi_owner_batches = 0;
  uint64_t max_batch_requests = 0, key_hits = 0, key_misses = 0, key_evictions = 0, key_upload_bytes = 0;
  uint64_t key_bytes = 0, peak_key_bytes = 0, peak_device_bytes = 0, budget_waits = 0, pending = 0;
};

class Server {
 public:
  Server(Context* ctx, const ServerConfig& cfg);
  ~Server();  // cancels waiting requests, waits for the batches on the device

  uint32_t add_owner();
  // Registers a key of `owner` (Galois element `elt`, 0 for the relinearization key) by
  // copying it into pinned host memory; the layout is the one ckg_key_upload takes.
  void add_key(uint32_t owner, const uint64_t* src, bool device_src, uint32_t parts, uint32_t q_limbs, uint64_t elt);
  // The owner's sparse-secret-encapsulation keys (to_sparse: 1 part at level 0; to_dense:
  // dnum parts at the top level), needed by its bootstrap requests.
  void add_sse_keys(uint32_t owner, const uint64_t* to_sparse, const uint64_t* to_dense, bool device_src);
  // Encodes the bootstrap stages and EvalMod series once (shared by every owner: they do not
  // depend on keys) so that bootstrap requests can be served; inputs must be at level 0 and
  // scale `delta`. Each bootstrap runs in its own completion segment.
  void enable_bootstrap(const BootParams& bp, double delta);

  uint64_t submit_mul(uint32_t owner, const Ct& a, const Ct& b);
  uint64_t submit_rotate(uint32_t owner, const Ct& a, int32_t steps);
  uint64_t submit_mul_plain(uint32_t owner, const Ct& a, const Pt& p);
  uint64_t submit_matvec(uint32_t owner, uint32_t d, uint32_t stride, const std::vector<Pt>& diag, const Ct& x);
  uint64_t submit_bootstrap(uint32_t owner, const Ct& a);

  // Waits up to timeout_ms (negative: no limit) for request `id`. On completion returns its
  // status (ST_OK with *out set, or the op's error with *err), fills times (microseconds
  // since the server started: submitted, admitted, completed) and forgets the request;
  // returns ST_TIMEOUT and keeps it if it is still running.
  int result(uint64_t id, int64_t timeout_ms, Ct* out, double times[3], std::string* err);
  bool cancel(uint64_t id);
  bool drain(int64_t timeout_ms);  // waits until no request is waiting or running
  ServerStats stats() const;
  OpCounter owner_counter(uint32_t owner) const;
  void inject_upload_failures(uint32_t n);  // the next n key uploads fail as if out of memory

 private:
  typedef std::chrono::steady_clock Clock;
  struct HostKey {
    uint64_t* host = nullptr;  // pinned
    size_t words = 0;
    uint32_t parts = 0, q_limbs = 0;
    uint64_t elt = 0;
    int role = 0;  // 0 relinearization, 1 Galois, 2 SSE to_sparse, 3 SSE to_dense
    KeyPtr dev;  // the cache's reference to the device copy
    // Completes when the copy that made `dev` has landed: a flight on another lane than the
    // one whose upload made it waits for this before its first read.
    std::shared_ptr<CUevent_st> ready;
    std::list<HostKey*>::iterator lru;
    ~HostKey();
  };
  struct Owner {
    std::unique_ptr<HostKey> relin, to_sparse, to_dense;
    std::map<uint64_t, std::unique_ptr<HostKey>> galois;
    OpCounter counter;
  };
  struct Req {
    uint64_t id = 0;
    uint32_t owner = 0;
    ReqKind kind = REQ_MUL;
    Ct a, b, out;
    Pt p;
    std::vector<Pt> diag;
    int32_t steps = 0;
    uint32_t d = 0, stride = 0;
    uint64_t ks = 0;          // key switches
    size_t work_bytes = 0;    // device working space while it runs
    std::vector<HostKey*> keys;
    int status = -1;          // -1 while waiting or running
    std::string err;
    Clock::time_point t_submit, t_admit, t_done;
  };
  typedef std::shared_ptr<Req> ReqPtr;
  struct Flight;  // one batch on the device

  uint64_t enqueue(ReqPtr r);
  void keys_of(Req& r);
  void worker();
  void completer();
  KeyPtr upload(HostKey* hk);
  std::unique_ptr<HostKey> host_key(const uint64_t* src, bool device_src, uint32_t parts, uint32_t q_limbs,
                                    uint64_t elt);
  void finish(Req& r, int status, const std::string& err);

  Context* ctx_;
  ServerConfig cfg_;
  StreamPtr copy_;
  Clock::time_point t0_;
  std::shared_ptr<std::atomic<int64_t>> key_bytes_;  // live device key copies, cached or held by a batch
  mutable std::mutex mu_;
  std::condition_variable cv_work_, cv_done_, cv_flight_;
  std::vector<std::unique_ptr<Owner>> owners_;
  std::unordered_map<uint64_t, ReqPtr> reqs_;
  std::deque<ReqPtr> pending_;
  std::deque<Flight*> flights_;
  std::vector<std::unique_ptr<Lane>> lanes_;  // with boot_lanes: [0] the batch lane, then the bootstrap lanes
  std::vector<uint32_t> inflight_lane_;       // flights queued per lane (one entry without lanes)
  std::list<HostKey*> lru_;  // front = most recently used
  size_t inflight_work_ = 0;
  uint64_t next_id_ = 1;
  uint32_t fail_uploads_ = 0;
  uint64_t done_gen_ = 0;     // batches completed
  bool building_ = false;     // the worker holds admitted requests outside the lock
  bool stop_ = false, worker_exited_ = false;
  ServerStats st_;
  bool boot_ = false;  // bootstrap template (enable_bootstrap)
  BootParams boot_bp_;
  double boot_delta_ = 0, boot_em_ = 0, boot_si_ = 0;
  std::vector<LtPtr> boot_ctos_, boot_stoc_;
  std::vector<double> boot_coeffs_;
  std::vector<uint64_t> boot_elts_;
  std::thread worker_, completer_;
};

}  // namespace ckg
