// Serving loop (serve.hpp): admission by HBM budget, LRU key residency with spill to pinned
// host memory, continuous batching over the Batch executor, per-request timestamps.
#include <algorithm>
#include <optional>
#include <set>
#include <unordered_set>

#include "bootsetup.hpp"
#include "serve.hpp"
#include "bounds.hpp"

namespace ckg {

namespace {

double us_since(std::chrono::steady_clock::time_point t0, std::chrono::steady_clock::time_point t) {
  return std::chrono::duration<double, std::micro>(t - t0).count();
}

}  // namespace

// A flight is what one worker iteration queued on the device: the batch of key-switching
// ops, then each mat-vec and each bootstrap, every one closed by its own event (a segment), so
// a request completes when its own work does. With two lanes a flight runs on one lane's
// stream; its outputs are handed to the context's stream once it completes.
struct Server::Flight {
  struct Segment {
    cudaEvent_t done = nullptr;
    std::vector<ReqPtr> reqs;
  };
  int lane = 0;
  cudaStream_t stream = nullptr;  // where its work runs
  bool rehome = false;            // outputs were allocated on a lane
  size_t next_seg = 0;            // segments completed so far
  std::vector<Segment> segs;
  std::map<uint32_t, std::unique_ptr<Evaluator>> evs;  // per owner, holding the flight's keys
  std::unique_ptr<Batch> batch;                        // refers to evs: released first
  std::vector<std::unique_ptr<Bootstrapper>> boots;
  std::vector<ReqPtr> reqs;
  size_t work = 0;
  ~Flight() {
    batch.reset();
    boots.clear();
    evs.clear();
    for (auto& s : segs)
      if (s.done) cudaEventDestroy(s.done);
  }
  void close_segment(cudaStream_t st, std::vector<ReqPtr> rs) {
    Segment s;
    s.reqs = std::move(rs);
    if (cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming) != cudaSuccess) s.done = nullptr;
    if (s.done) cudaEventRecord(s.done, st);
    segs.push_back(std::move(s));
  }
};

Server::HostKey::~HostKey() {
  dev.reset();
  if (host) cudaFreeHost(host);
}

Server::Server(Context* ctx, const ServerConfig& cfg) : ctx_(ctx), cfg_(cfg) {
  if (!cfg_.hbm_budget) throw Error(ST_INVALID_PARAMS, "the HBM budget must be positive");
  if (!cfg_.max_batch_ks) throw Error(ST_INVALID_PARAMS, "max_batch_ks must be positive");
  if (!cfg_.max_inflight) throw Error(ST_INVALID_PARAMS, "max_inflight must be positive");
  ctx_->activate();
  copy_ = std::make_shared<StreamRes>();
  copy_->device = ctx_->device;
  copy_->own = true;
  CKG_CUDA(cudaStreamCreateWithFlags(&copy_->s, cudaStreamNonBlocking));
  if (cfg_.boot_lanes > 4) throw Error(ST_INVALID_PARAMS, "at most 4 bootstrap lanes");
  if (cfg_.boot_lanes) {
    // Bootstraps are long chains of small launches that bound the tail: their lanes may get the
    // device's highest stream priority, so the batches fill the SMs they leave idle.
    int least = 0, greatest = 0;
    CKG_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    lanes_.push_back(std::make_unique<Lane>(ctx_->device, least));
    for (uint32_t i = 0; i < cfg_.boot_lanes; ++i)
      lanes_.push_back(std::make_unique<Lane>(ctx_->device, cfg_.boot_priority ? greatest : least));
  }
  inflight_lane_.assign(std::max<size_t>(1, lanes_.size()), 0);
  t0_ = Clock::now();
  key_bytes_ = std::make_shared<std::atomic<int64_t>>(0);
  worker_ = std::thread([this] { worker(); });
  completer_ = std::thread([this] { completer(); });
}

Server::~Server() {
  {
    std::lock_guard<std::mutex> lk(mu_);
    stop_ = true;
    for (auto& r : pending_) finish(*r, ST_CANCELLED, "server shut down before the request was admitted");
    pending_.clear();
  }
  cv_work_.notify_all();
  cv_done_.notify_all();
  worker_.join();
  {
    std::lock_guard<std::mutex> lk(mu_);
    worker_exited_ = true;
  }
  cv_flight_.notify_all();
  completer_.join();
  reqs_.clear();
  try {
    ctx_->activate();
  } catch (...) {
  }
  boot_ctos_.clear();
  boot_stoc_.clear();
  for (auto& o : owners_) {  // device copies are freed on the copy stream before it goes
    for (auto* hk : {o->relin.get(), o->to_sparse.get(), o->to_dense.get()})
      if (hk) hk->dev.reset();
    for (auto& g : o->galois) g.second->dev.reset();
  }
  owners_.clear();
}

uint32_t Server::add_owner() {
  std::lock_guard<std::mutex> lk(mu_);
  owners_.push_back(std::make_unique<Owner>());
  return (uint32_t)owners_.size() - 1;
}

void Server::add_key(uint32_t owner, const uint64_t* src, bool device_src, uint32_t parts, uint32_t q_limbs,
                     uint64_t elt) {
  const Context& c = *ctx_;
  if (!src) throw Error(ST_INVALID_PARAMS, "null key data");
  if (!parts || parts > c.dnum) throw Error(ST_INVALID_PARAMS, "key parts must be in 1..=dnum");
  if (!q_limbs || q_limbs > c.L + 1) throw Error(ST_INVALID_PARAMS, "key data limbs must be in 1..=L+1");
  if (elt && (elt % 2 == 0 || elt >= 2 * c.n)) throw Error(ST_INVALID_PARAMS, "Galois element must be odd and < 2N");
  {
    std::lock_guard<std::mutex> lk(mu_);
    if (owner >= owners_.size()) throw Error(ST_INVALID_PARAMS, "unknown key owner");
    Owner& o = *owners_[owner];
    if (elt ? o.galois.count(elt) != 0 : (bool)o.relin)
      throw Error(ST_INVALID_PARAMS, "the owner already has this key");
  }
  auto hk = host_key(src, device_src, parts, q_limbs, elt);
  hk->role = elt ? 1 : 0;
  std::lock_guard<std::mutex> lk(mu_);
  Owner& o = *owners_[owner];
  if (elt ? o.galois.count(elt) != 0 : (bool)o.relin) throw Error(ST_INVALID_PARAMS, "the owner already has this key");
  if (elt)
    o.galois[elt] = std::move(hk);
  else
    o.relin = std::move(hk);
}

std::unique_ptr<Server::HostKey> Server::host_key(const uint64_t* src, bool device_src, uint32_t parts,
                                                 uint32_t q_limbs, uint64_t elt) {
  auto hk = std::make_unique<HostKey>();
  hk->words = (size_t)parts * 2 * (q_limbs + ctx_->k) * ctx_->n;
  hk->parts = parts;
  hk->q_limbs = q_limbs;
  hk->elt = elt;
  ctx_->activate();
  CKG_CUDA(cudaHostAlloc((void**)&hk->host, hk->words * 8, cudaHostAllocPortable));
  if (device_src) {
    CKG_CUDA(cudaMemcpyAsync(hk->host, src, hk->words * 8, cudaMemcpyDeviceToHost, copy_->s));
    CKG_CUDA(cudaStreamSynchronize(copy_->s));
  } else {
    std::copy(src, src + hk->words, hk->host);
  }
  return hk;
}

void Server::add_sse_keys(uint32_t owner, const uint64_t* to_sparse, const uint64_t* to_dense, bool device_src) {
  if (!to_sparse || !to_dense) throw Error(ST_INVALID_PARAMS, "null key data");
  {
    std::lock_guard<std::mutex> lk(mu_);
    if (owner >= owners_.size()) throw Error(ST_INVALID_PARAMS, "unknown key owner");
    if (owners_[owner]->to_sparse) throw Error(ST_INVALID_PARAMS, "the owner already has SSE keys");
  }
  auto ts = host_key(to_sparse, device_src, 1, 1, 0);  // modraise.rs:109-129 shapes
  auto td = host_key(to_dense, device_src, ctx_->dnum, ctx_->L + 1, 0);
  ts->role = 2;
  td->role = 3;
  std::lock_guard<std::mutex> lk(mu_);
  Owner& o = *owners_[owner];
  if (o.to_sparse) throw Error(ST_INVALID_PARAMS, "the owner already has SSE keys");
  o.to_sparse = std::move(ts);
  o.to_dense = std::move(td);
}

void Server::enable_bootstrap(const BootParams& bp, double delta) {
  Evaluator enc(ctx_, nullptr, {}, cfg_.eval);  // keyless: only encodes
  auto ctos = encode_boot_stages(enc, bp, DIR_COEFF_TO_SLOT, delta);
  auto stoc = encode_boot_stages(enc, bp, DIR_SLOT_TO_COEFF, delta);
  auto coeffs = evalmod_coeffs(bp);
  auto sc = boot_stage_scales(*ctx_, bp, delta);
  std::vector<uint64_t> elts;
  for (int32_t s : boot_rotation_steps(bp)) elts.push_back(galois_elt(ctx_->n, s));
  elts.push_back(2 * ctx_->n - 1);
  CKG_CUDA(cudaStreamSynchronize(ctx_->stream));
  std::lock_guard<std::mutex> lk(mu_);
  if (boot_) throw Error(ST_INVALID_PARAMS, "bootstrap requests are already enabled");
  boot_bp_ = bp;
  boot_delta_ = delta;
  boot_ctos_ = std::move(ctos);
  boot_stoc_ = std::move(stoc);
  boot_coeffs_ = std::move(coeffs);
  boot_em_ = sc.first;
  boot_si_ = sc.second;
  boot_elts_ = std::move(elts);
  boot_ = true;
}

// ---- submission ----------------------------------------------------------------------

uint64_t Server::enqueue(ReqPtr r) {
  if (!r->a || r->a->ctx != ctx_) throw Error(ST_INVALID_PARAMS, "operand is not over this server's context");
  std::lock_guard<std::mutex> lk(mu_);
  if (stop_) throw Error(ST_INVALID_PARAMS, "server is shutting down");
  if (r->owner >= owners_.size()) throw Error(ST_INVALID_PARAMS, "unknown key owner");
  r->id = next_id_++;
  r->t_submit = Clock::now();
  reqs_[r->id] = r;
  pending_.push_back(r);
  st_.submitted++;
  cv_work_.notify_one();
  return r->id;
}

uint64_t Server::submit_mul(uint32_t owner, const Ct& a, const Ct& b) {
  auto r = std::make_shared<Req>();
  r->owner = owner;
  r->kind = REQ_MUL;
  r->a = a;
  r->b = b;
  r->ks = 1;
  if (a) {
    const uint32_t l = a->level;
    r->work_bytes = (Batch::scratch_words(*ctx_, Batch::MUL, l, a->ncomp) + 2 * (size_t)std::max(l, 1u) * ctx_->n) * 8;
  }
  return enqueue(r);
}

uint64_t Server::submit_rotate(uint32_t owner, const Ct& a, int32_t steps) {
  auto r = std::make_shared<Req>();
  r->owner = owner;
  r->kind = REQ_ROTATE;
  r->a = a;
  r->steps = steps;
  const int64_t slots = (int64_t)ctx_->n / 2;
  r->ks = (((int64_t)steps % slots) + slots) % slots != 0;
  if (a) r->work_bytes = (Batch::scratch_words(*ctx_, Batch::ROT, a->level, a->ncomp) + 2 * (size_t)(a->level + 1) * ctx_->n) * 8;
  return enqueue(r);
}

uint64_t Server::submit_mul_plain(uint32_t owner, const Ct& a, const Pt& p) {
  auto r = std::make_shared<Req>();
  r->owner = owner;
  r->kind = REQ_MUL_PLAIN;
  r->a = a;
  r->p = p;
  if (a)
    r->work_bytes =
        (Batch::scratch_words(*ctx_, Batch::PMUL, a->level, a->ncomp) + (size_t)a->ncomp * (a->level + 1) * ctx_->n) * 8;
  return enqueue(r);
}

uint64_t Server::submit_matvec(uint32_t owner, uint32_t d, uint32_t stride, const std::vector<Pt>& diag, const Ct& x) {
  auto r = std::make_shared<Req>();
  r->owner = owner;
  r->kind = REQ_MATVEC;
  r->a = x;
  r->d = d;
  r->stride = stride;
  r->diag = diag;
  if (d && (d & (d - 1)) == 0) {
    const int64_t slots = (int64_t)ctx_->n / 2;
    for (int32_t s : rotation_steps(d, stride)) r->ks += (((int64_t)s % slots) + slots) % slots != 0;
    if (x) {
      // hoisted baby-step ciphertexts, the giant-step temporaries and the key-switch
      // scratch (the hoisted path groups its key switches into at most 2 GiB)
      const size_t ct_words = 2 * (size_t)(x->level + 1) * ctx_->n;
      const size_t baby = bsgs_split(d).first;
      const size_t ks = std::min<size_t>(((size_t)2 << 30) / 8,
                                         std::max<size_t>(baby, 1) * key_switch_scratch_words(*ctx_, x->level));
      r->work_bytes = ((baby + 6) * ct_words + conv_limbs(*ctx_, x->level) * ctx_->n + ks) * 8;
    }
  }
  return enqueue(r);
}

uint64_t Server::submit_bootstrap(uint32_t owner, const Ct& a) {
  auto r = std::make_shared<Req>();
  r->owner = owner;
  r->kind = REQ_BOOTSTRAP;
  r->a = a;
  {
    std::lock_guard<std::mutex> lk(mu_);
    if (!boot_) throw Error(ST_INVALID_PARAMS, "bootstrap requests are not enabled on this server");
  }
  // ciphertexts at the top level and the hoisted key-switch scratch of the widest stage
  const size_t ct_words = 2 * (size_t)(ctx_->L + 1) * ctx_->n;
  r->work_bytes = (32 * ct_words + 8 * key_switch_scratch_words(*ctx_, ctx_->L)) * 8;
  return enqueue(r);
}

// ---- results -------------------------------------------------------------------------

void Server::finish(Req& r, int status, const std::string& err) {
  if (r.status != -1) return;
  r.status = status;
  r.err = err;
  r.t_done = Clock::now();
  if (status == ST_OK)
    st_.completed++;
  else if (status == ST_CANCELLED)
    st_.cancelled++;
  else
    st_.failed++;
}

int Server::result(uint64_t id, int64_t timeout_ms, Ct* out, double times[3], std::string* err) {
  std::unique_lock<std::mutex> lk(mu_);
  auto it = reqs_.find(id);
  if (it == reqs_.end()) throw Error(ST_INVALID_PARAMS, "unknown request id (results are returned once)");
  ReqPtr r = it->second;
  auto ready = [&] { return r->status != -1; };
  if (timeout_ms < 0)
    cv_done_.wait(lk, ready);
  else if (!cv_done_.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready))
    return ST_TIMEOUT;
  if (times) {
    times[0] = us_since(t0_, r->t_submit);
    times[1] = r->t_admit == Clock::time_point() ? times[0] : us_since(t0_, r->t_admit);
    times[2] = us_since(t0_, r->t_done);
  }
  if (out) *out = r->status == ST_OK ? r->out : Ct();
  if (err) *err = r->err;
  reqs_.erase(it);
  return r->status;
}

bool Server::cancel(uint64_t id) {
  std::lock_guard<std::mutex> lk(mu_);
  for (auto it = pending_.begin(); it != pending_.end(); ++it)
    if ((*it)->id == id) {
      finish(**it, ST_CANCELLED, "request cancelled before it was admitted");
      pending_.erase(it);
      cv_done_.notify_all();
      return true;
    }
  return false;
}

bool Server::drain(int64_t timeout_ms) {
  std::unique_lock<std::mutex> lk(mu_);
  auto idle = [&] { return pending_.empty() && flights_.empty() && !building_; };
  if (timeout_ms < 0) {
    cv_done_.wait(lk, idle);
    return true;
  }
  return cv_done_.wait_for(lk, std::chrono::milliseconds(timeout_ms), idle);
}

ServerStats Server::stats() const {
  std::lock_guard<std::mutex> lk(mu_);
  ServerStats s = st_;
  s.key_bytes = (uint64_t)std::max<int64_t>(0, *key_bytes_);
  s.pending = pending_.size();
  return s;
}

OpCounter Server::owner_counter(uint32_t owner) const {
  std::lock_guard<std::mutex> lk(mu_);
  if (owner >= owners_.size()) throw Error(ST_INVALID_PARAMS, "unknown key owner");
  return owners_[owner]->counter;
}

void Server::inject_upload_failures(uint32_t n) {
  std::lock_guard<std::mutex> lk(mu_);
  fail_uploads_ = n;
}

// ---- the worker: admission, residency, batching ---------------------------------------

void Server::keys_of(Req& r) {
  r.keys.clear();
  Owner& o = *owners_[r.owner];
  auto galois = [&](int32_t steps) {
    const int64_t slots = (int64_t)ctx_->n / 2;
    const int64_t k = (((int64_t)steps % slots) + slots) % slots;
    if (!k) return;
    auto it = o.galois.find(galois_elt(ctx_->n, (int32_t)k));
    if (it != o.galois.end() && std::find(r.keys.begin(), r.keys.end(), it->second.get()) == r.keys.end())
      r.keys.push_back(it->second.get());
  };
  if ((r.kind == REQ_MUL || r.kind == REQ_BOOTSTRAP) && o.relin) r.keys.push_back(o.relin.get());
  if (r.kind == REQ_ROTATE) galois(r.steps);
  if (r.kind == REQ_MATVEC && r.d && (r.d & (r.d - 1)) == 0)
    for (int32_t s : rotation_steps(r.d, r.stride)) galois(s);
  if (r.kind == REQ_BOOTSTRAP) {
    for (uint64_t e : boot_elts_) {
      auto it = o.galois.find(e);
      if (it != o.galois.end()) r.keys.push_back(it->second.get());
    }
    if (o.to_sparse && o.to_dense) {
      r.keys.push_back(o.to_sparse.get());
      r.keys.push_back(o.to_dense.get());
    }
  }
}

KeyPtr Server::upload(HostKey* hk) {
  {
    std::lock_guard<std::mutex> lk(mu_);
    if (fail_uploads_) {
      fail_uploads_--;
      throw Error(ST_OOM, "out of device memory (injected key-upload failure)");
    }
  }
  const int64_t bytes = (int64_t)hk->words * 8;
  auto buf = std::make_shared<DevBuf>();
  buf->sres = copy_;
  buf->device = ctx_->device;
  buf->words = hk->words;
  CKG_CUDA(cudaMallocAsync((void**)&buf->p, hk->words * 8, copy_->s));
  bounds::track(buf->p, hk->words * 8);
  CKG_CUDA(cudaMemcpyAsync(buf->p, hk->host, hk->words * 8, cudaMemcpyHostToDevice, copy_->s));
  auto counter = key_bytes_;
  *counter += bytes;
  KeyPtr k(new DevKey(), [counter, bytes](DevKey* p) {
    delete p;
    *counter -= bytes;
  });
  k->ctx = ctx_;
  k->buf = buf;
  k->parts = hk->parts;
  k->q_limbs = hk->q_limbs;
  k->elt = hk->elt;
  return k;
}

void Server::worker() {
  try {
    ctx_->activate();
  } catch (...) {
  }
  std::unique_lock<std::mutex> lk(mu_);
  // The lane of the earliest waiting request whose lane has room (-1: none). Without lanes every
  // request is on lane 0 in arrival order; with them bootstraps go to a free bootstrap lane (1..,
  // one bootstrap in flight per lane, so the lanes add concurrency without holding more working
  // space and keys), the others to lane 0, and either kind may pass a waiting request of the other.
  const bool laned = !lanes_.empty();
  auto boot_class = [&](const Req& r) { return laned && r.kind == REQ_BOOTSTRAP; };
  auto boot_lane_free = [&]() -> int {
    int best = -1;
    for (int l = 1; l < (int)lanes_.size(); ++l)
      if (inflight_lane_[l] < 1 && (best < 0 || inflight_lane_[l] < inflight_lane_[best])) best = l;
    return best;
  };
  auto pick = [&]() -> int {
    for (const ReqPtr& r : pending_) {
      if (boot_class(*r)) {
        const int l = boot_lane_free();
        if (l >= 0) return l;
      } else if (inflight_lane_[0] < cfg_.max_inflight) {
        return 0;
      }
      if (!laned) break;
    }
    return -1;
  };
  while (true) {
    cv_work_.wait(lk, [&] { return stop_ || pick() >= 0; });
    if (stop_) break;
    const int lane = pick();
    // ---- admission (under the lock): arrival order, key-switch cap, HBM budget
    std::vector<ReqPtr> batch;
    std::vector<HostKey*> need;
    std::unordered_set<HostKey*> need_set;
    size_t new_bytes = 0, work = 0;
    uint64_t ks = 0;
    bool wait_memory = false;
    for (auto pit = pending_.begin(); pit != pending_.end();) {
      ReqPtr r = *pit;
      if (boot_class(*r) != (lane >= 1)) {  // the other lanes' request keeps its place
        ++pit;
        continue;
      }
      keys_of(*r);
      if (!batch.empty() && ks + r->ks > cfg_.max_batch_ks) break;
      if (r->kind == REQ_BOOTSTRAP && std::any_of(batch.begin(), batch.end(), [](const ReqPtr& x) {
            return x->kind == REQ_BOOTSTRAP;
          }))
        break;  // one bootstrap per flight
      size_t extra = 0;
      for (HostKey* hk : r->keys)
        if (!hk->dev && !need_set.count(hk)) extra += hk->words * 8;
      auto used = [&] { return (size_t)std::max<int64_t>(0, *key_bytes_) + inflight_work_ + work + new_bytes; };
      // make room: drop the least recently used device copies nobody else holds
      for (auto it = lru_.end(); used() + extra + r->work_bytes > cfg_.hbm_budget && it != lru_.begin();) {
        --it;
        HostKey* hk = *it;
        if (need_set.count(hk) || std::find(r->keys.begin(), r->keys.end(), hk) != r->keys.end()) continue;
        if (hk->dev.use_count() != 1) continue;  // a batch on the device still reads it
        it = lru_.erase(it);
        hk->dev.reset();  // stream-ordered free on the copy stream
        hk->ready.reset();
        st_.key_evictions++;
      }
      if (used() + extra + r->work_bytes > cfg_.hbm_budget) {
        if (batch.empty() && flights_.empty()) {
          // nothing on the device holds memory and every other key copy is gone: the
          // request can never fit
          pit = pending_.erase(pit);
          finish(*r, ST_OOM,
                 "request needs " + std::to_string(extra + r->work_bytes) +
                     " bytes of device memory beyond its resident keys; the serving budget is " +
                     std::to_string(cfg_.hbm_budget));
          cv_done_.notify_all();
          continue;
        }
        if (batch.empty()) wait_memory = true;
        break;
      }
      pit = pending_.erase(pit);
      for (HostKey* hk : r->keys)
        if (need_set.insert(hk).second) {
          need.push_back(hk);
          if (!hk->dev) new_bytes += hk->words * 8;
        }
      work += r->work_bytes;
      ks += r->ks;
      r->t_admit = Clock::now();
      batch.push_back(r);
    }
    if (batch.empty()) {
      if (wait_memory) {
        st_.budget_waits++;
        const uint64_t g = done_gen_;
        cv_work_.wait(lk, [&] { return stop_ || done_gen_ != g; });
      }
      continue;
    }
    std::vector<HostKey*> to_upload;
    std::vector<std::shared_ptr<CUevent_st>> hit_ready;  // copies of resident keys, maybe in flight
    for (HostKey* hk : need) {
      if (hk->dev) {
        st_.key_hits++;
        lru_.splice(lru_.begin(), lru_, hk->lru);
        if (hk->ready && std::find(hit_ready.begin(), hit_ready.end(), hk->ready) == hit_ready.end())
          hit_ready.push_back(hk->ready);
      } else {
        st_.key_misses++;
        to_upload.push_back(hk);
      }
    }
    building_ = true;
    inflight_work_ += work;
    lk.unlock();

    // ---- keys, batch and launches (outside the lock)
    auto f = std::make_unique<Flight>();
    f->reqs = batch;
    f->work = work;
    f->lane = lane;
    Lane* ln = laned ? lanes_[lane].get() : nullptr;
    std::optional<LaneScope> scope;  // this thread's launches through ctx_ go to the lane
    if (ln) scope.emplace(*ctx_, *ln);
    f->stream = ctx_->stream;
    f->rehome = ln != nullptr;
    std::map<HostKey*, std::pair<int, std::string>> failed;
    std::map<HostKey*, KeyPtr> fresh;
    std::shared_ptr<CUevent_st> copied_ev;
    try {
      ctx_->activate();
      if (ln) {  // the lane runs after the client's work queued on the context's stream so far
        cudaEvent_t ready;
        CKG_CUDA(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
        cudaEventRecord(ready, ctx_->sres->s);
        cudaStreamWaitEvent(ln->sres->s, ready, 0);
        cudaEventDestroy(ready);
      }
      // resident keys whose copy another flight issued (possibly on another lane)
      for (auto& e : hit_ready) CKG_CUDA(cudaStreamWaitEvent(ctx_->stream, e.get(), 0));
      for (HostKey* hk : to_upload) {
        try {
          fresh[hk] = upload(hk);
        } catch (const Error& e) {
          failed[hk] = {e.code, e.what()};
        }
      }
      if (!fresh.empty()) {  // the compute stream waits for the key copies
        cudaEvent_t copied;
        CKG_CUDA(cudaEventCreateWithFlags(&copied, cudaEventDisableTiming));
        copied_ev.reset(copied, [](cudaEvent_t e) { cudaEventDestroy(e); });
        CKG_CUDA(cudaEventRecord(copied, copy_->s));
        CKG_CUDA(cudaStreamWaitEvent(ctx_->stream, copied, 0));
      }
    } catch (const std::exception& e) {
      for (HostKey* hk : to_upload)
        if (!fresh.count(hk)) failed[hk] = {ST_DEVICE, e.what()};
    }
    std::vector<std::pair<ReqPtr, std::pair<int, std::string>>> errs;
    {
      std::lock_guard<std::mutex> g(mu_);
      for (auto& kv : fresh) {
        kv.first->dev = kv.second;
        kv.first->ready = copied_ev;
        lru_.push_front(kv.first);
        kv.first->lru = lru_.begin();
        st_.key_upload_bytes += kv.first->words * 8;
      }
      st_.peak_key_bytes = std::max<uint64_t>(st_.peak_key_bytes, (uint64_t)std::max<int64_t>(0, *key_bytes_));
      st_.peak_device_bytes = std::max<uint64_t>(
          st_.peak_device_bytes, (uint64_t)std::max<int64_t>(0, *key_bytes_) + inflight_work_);
      // per-owner evaluators over this batch's keys
      std::map<uint32_t, std::pair<KeyPtr, std::vector<KeyPtr>>> keys;
      for (auto& r : batch) {
        auto& slot = keys[r->owner];
        for (HostKey* hk : r->keys) {
          if (!hk->dev) continue;
          if (hk->role == 0)
            slot.first = hk->dev;
          else if (hk->role == 1 && std::find(slot.second.begin(), slot.second.end(), hk->dev) == slot.second.end())
            slot.second.push_back(hk->dev);
        }
      }
      for (auto& kv : keys)
        f->evs[kv.first] = std::make_unique<Evaluator>(ctx_, kv.second.first, kv.second.second, cfg_.eval);
    }
    std::set<uint32_t> owners_in_batch;
    std::unordered_set<const Req*> placed;  // requests whose work closed a segment
    auto failed_req = [&](const ReqPtr& r) {
      return std::any_of(errs.begin(), errs.end(), [&](auto& x) { return x.first == r; });
    };
    try {
      f->batch = std::make_unique<Batch>(f->evs.begin()->second.get());
      std::vector<ReqPtr> in_batch;
      for (auto& r : batch) {
        auto bad = std::find_if(r->keys.begin(), r->keys.end(), [&](HostKey* hk) { return failed.count(hk) != 0; });
        if (bad != r->keys.end()) {
          errs.push_back({r, failed[*bad]});
          continue;
        }
        if (r->kind == REQ_MATVEC || r->kind == REQ_BOOTSTRAP) continue;
        Evaluator* ev = f->evs[r->owner].get();
        try {
          if (r->kind == REQ_MUL)
            r->out = f->batch->mul_relin_rescale(r->a, r->b, ev);
          else if (r->kind == REQ_ROTATE)
            r->out = f->batch->rotate(r->a, r->steps, ev);
          else
            r->out = f->batch->mul_plain_rescale(r->a, r->p, ev);
          owners_in_batch.insert(r->owner);
          in_batch.push_back(r);
        } catch (const Error& e) {
          errs.push_back({r, {e.code, e.what()}});
        }
      }
      if (f->batch->size()) f->batch->run();
      if (!in_batch.empty()) {
        for (auto& r : in_batch) placed.insert(r.get());
        f->close_segment(ctx_->stream, in_batch);
      }
      // Mat-vecs: each checked on its own (a failing request fails alone), then one batched call
      // per owner (all hoisted baby rotations, inner sums and giant rotations of the owner's
      // requests as one launch sequence per stage) and one completion segment for them.
      std::map<uint32_t, std::vector<ReqPtr>> matvecs;
      for (auto& r : batch) {
        if (r->kind != REQ_MATVEC || failed_req(r)) continue;
        try {
          f->evs[r->owner]->check_matvec_plain(r->d, r->stride, r->diag, r->a);
          matvecs[r->owner].push_back(r);
        } catch (const Error& e) {
          errs.push_back({r, {e.code, e.what()}});
        }
      }
      for (auto& kv : matvecs) {
        std::vector<MatvecJob<Pt>> jobs;
        for (auto& r : kv.second) jobs.push_back(MatvecJob<Pt>{r->d, r->stride, r->diag, r->a});
        try {
          std::vector<Ct> outs = f->evs[kv.first]->matvec_plain_batch(jobs);
          for (size_t i = 0; i < outs.size(); ++i) {
            kv.second[i]->out = outs[i];
            placed.insert(kv.second[i].get());
          }
          owners_in_batch.insert(kv.first);
          f->close_segment(ctx_->stream, kv.second);
        } catch (const Error& e) {
          for (auto& r : kv.second) errs.push_back({r, {e.code, e.what()}});
        }
      }
      for (auto& r : batch) {
        if (r->kind != REQ_BOOTSTRAP || failed_req(r)) continue;
        try {
          std::vector<KeyPtr> gk;
          KeyPtr ts, td;
          for (HostKey* hk : r->keys) {
            if (!hk->dev) continue;
            if (hk->role == 1) gk.push_back(hk->dev);
            if (hk->role == 2) ts = hk->dev;
            if (hk->role == 3) td = hk->dev;
          }
          auto bs = std::make_unique<Bootstrapper>(ctx_, boot_bp_, boot_ctos_, boot_stoc_, gk, ts, td, boot_coeffs_,
                                                   boot_em_, boot_si_, boot_delta_);
          r->out = bs->bootstrap(*f->evs[r->owner], r->a);
          f->boots.push_back(std::move(bs));
          owners_in_batch.insert(r->owner);
          placed.insert(r.get());
          f->close_segment(ctx_->stream, {r});
        } catch (const Error& e) {
          errs.push_back({r, {e.code, e.what()}});
        }
      }
    } catch (const std::exception& e) {
      const int code = dynamic_cast<const Error*>(&e) ? dynamic_cast<const Error*>(&e)->code : ST_DEVICE;
      for (auto& r : batch)
        if (!placed.count(r.get()) && !failed_req(r)) errs.push_back({r, {code, e.what()}});
    }

    lk.lock();
    for (auto& e : errs) finish(*e.first, e.second.first, e.second.second);
    if (!errs.empty()) cv_done_.notify_all();
    st_.batches++;
    if (owners_in_batch.size() > 1) st_.multi_owner_batches++;
    st_.max_batch_requests = std::max<uint64_t>(st_.max_batch_requests, batch.size());
    inflight_lane_[lane]++;
    flights_.push_back(f.release());
    building_ = false;
    cv_flight_.notify_all();
  }
}

void Server::completer() {
  try {
    ctx_->activate();
  } catch (...) {
  }
  // Flights complete in any order (two lanes): each pass polls every queued flight's next
  // segments, completes what is done and releases finished flights.
  while (true) {
    std::vector<Flight*> snap;
    {
      std::unique_lock<std::mutex> lk(mu_);
      cv_flight_.wait(lk, [&] { return !flights_.empty() || worker_exited_; });
      if (flights_.empty()) break;
      snap.assign(flights_.begin(), flights_.end());
    }
    bool progress = false;
    for (Flight* f : snap) {
      while (f->next_seg < f->segs.size()) {  // each segment completes its own requests
        auto& seg = f->segs[f->next_seg];
        cudaError_t e = cudaSuccess;
        if (seg.done) {
          e = cudaEventQuery(seg.done);
          if (e == cudaErrorNotReady) break;
        } else {
          // No completion event could be created: wait for the flight's whole stream, so the
          // flight's working space and keys are released only after its kernels have run.
          cudaStreamSynchronize(f->stream);
          e = cudaErrorUnknown;
        }
        {
          std::lock_guard<std::mutex> lk(mu_);
          const auto t = Clock::now();
          for (auto& r : seg.reqs) {
            if (r->status != -1) continue;
            if (e == cudaSuccess) {
              // a lane's output is freed on the context's stream from now on, after the
              // client's later work on it
              if (f->rehome && r->out) r->out->buf->sres = ctx_->sres;
              finish(*r, ST_OK, "");
              r->t_done = t;
            } else {
              finish(*r, ST_DEVICE, std::string("device error in a served batch: ") + cudaGetErrorString(e));
            }
          }
        }
        cv_done_.notify_all();
        f->next_seg++;
        progress = true;
      }
      if (f->next_seg < f->segs.size()) continue;
      {
        std::lock_guard<std::mutex> lk(mu_);
        for (auto& kv : f->evs) {
          OpCounter c = kv.second->counter();
          OpCounter& o = owners_[kv.first]->counter;
          o.rotations += c.rotations;
          o.relins += c.relins;
          o.ct_ct_tensor += c.ct_ct_tensor;
          o.ct_pt_mults += c.ct_pt_mults;
          o.rescales += c.rescales;
          o.sse_switches += c.sse_switches;
          o.bootstraps += c.bootstraps;
        }
      }
      cv_done_.notify_all();
      // release the flight's keys and working space, then let the worker admit more
      const size_t work = f->work;
      const int lane = f->lane;
      delete f;
      {
        std::lock_guard<std::mutex> lk(mu_);
        flights_.erase(std::find(flights_.begin(), flights_.end(), f));
        inflight_work_ -= work;
        inflight_lane_[lane]--;
        done_gen_++;
      }
      progress = true;
      cv_work_.notify_all();
      cv_done_.notify_all();
    }
    if (!progress) std::this_thread::sleep_for(std::chrono::microseconds(20));
  }
}

}  // namespace ckg
