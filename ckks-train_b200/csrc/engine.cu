// Device context set-up (prime constants, twiddle and conversion tables) and the
// polynomial-level algorithms of the evaluator path. See engine.hpp for the layouts.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>

#include "engine.hpp"
#include "bounds.hpp"

namespace ckg {

[[noreturn]] void throw_cuda(cudaError_t e, const char* what) {
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    throw Error(ST_OOM, std::string("out of device memory: ") + what);
  }
  throw Error(ST_DEVICE, std::string(cudaGetErrorName(e)) + " (" + cudaGetErrorString(e) + ") at " + what);
}

StreamRes::~StreamRes() {
  if (!own || !s) return;
  cudaSetDevice(device);
  cudaStreamSynchronize(s);
  cudaStreamDestroy(s);
}

DevBuf::~DevBuf() {
  if (!p) return;
  bounds::untrack(p);
  int cur = 0;
  cudaGetDevice(&cur);
  if (cur != device) cudaSetDevice(device);
  for (cudaEvent_t e : waits) {
    cudaStreamWaitEvent(sres->s, e, 0);
    cudaEventDestroy(e);
  }
  cudaEvent_t done = nullptr;
  if (cache && cudaEventCreateWithFlags(&done, cudaEventDisableTiming) == cudaSuccess &&
      cudaEventRecord(done, sres->s) == cudaSuccess) {
    cache->give(p, words, done);
  } else {
    if (done) cudaEventDestroy(done);
    if (pooled) cudaFreeAsync(p, sres->s);
    else cudaFree(p);
  }
  if (cur != device) cudaSetDevice(cur);
}

uint64_t* XferCache::take(size_t words, cudaStream_t on) {
  std::lock_guard<std::mutex> lk(mu);
  auto fits = [&](const Block& b) { return b.words >= words && b.words <= words + words / 4; };
  // the smallest fitting block whose last use has completed
  int best = -1;
  for (int i = 0; i < (int)blocks.size(); ++i) {
    const Block& b = blocks[i];
    if (!fits(b) || (best >= 0 && b.words >= blocks[best].words)) continue;
    if (cudaEventQuery(b.done) != cudaSuccess) continue;
    best = i;
  }
  if (best < 0) {
    // Else, once kReuseDepth fitting blocks are in use (enough for the transfers of one step to
    // overlap the compute and copies of the steps before it), the oldest of them, which `on`
    // waits for (stream-ordered reuse): a further block would cost a fresh mapping of device
    // memory on the host's critical path, the wait only the rest of work the device is running.
    int in_use = 0;
    for (const Block& b : blocks) in_use += fits(b);
    if (in_use < kReuseDepth) return nullptr;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(on, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone) {
      cudaGetLastError();
      return nullptr;
    }
    for (int i = 0; i < (int)blocks.size() && best < 0; ++i)
      if (fits(blocks[i]) && cudaStreamWaitEvent(on, blocks[i].done, 0) == cudaSuccess) best = i;
    cudaGetLastError();
    if (best < 0) return nullptr;
    waited++;
  }
  uint64_t* p = blocks[best].p;
  cudaEventDestroy(blocks[best].done);
  blocks.erase(blocks.begin() + best);
  return p;
}

void XferCache::give(uint64_t* p, size_t words, cudaEvent_t done) {
  std::lock_guard<std::mutex> lk(mu);
  blocks.push_back({p, words, done});
  // at most kMaxBlocks and max_bytes kept: the oldest completed ones beyond that go back to the pool
  auto bytes = [&] {
    size_t b = 0;
    for (const Block& x : blocks) b += x.words * 8;
    return b;
  };
  for (size_t i = 0; (blocks.size() > kMaxBlocks || bytes() > max_bytes) && i < blocks.size();) {
    if (cudaEventQuery(blocks[i].done) == cudaSuccess) {
      cudaEventDestroy(blocks[i].done);
      cudaFreeAsync(blocks[i].p, stream->s);
      blocks.erase(blocks.begin() + i);
    } else {
      ++i;
    }
  }
}

void XferCache::trim() {
  std::lock_guard<std::mutex> lk(mu);
  for (size_t i = 0; i < blocks.size();) {
    if (cudaEventQuery(blocks[i].done) == cudaSuccess) {
      cudaEventDestroy(blocks[i].done);
      cudaFreeAsync(blocks[i].p, stream->s);
      blocks[i] = blocks.back();
      blocks.pop_back();
    } else {
      ++i;
    }
  }
  // The frees above are stream-ordered: let them land (unless the stream is being captured)
  // so that the trim below hands the blocks back to the device.
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(stream->s, &cap) == cudaSuccess && cap == cudaStreamCaptureStatusNone)
    cudaStreamSynchronize(stream->s);
  if (pool) cudaMemPoolTrimTo(pool, 0);
}

XferCache::~XferCache() {
  int cur = 0;
  cudaGetDevice(&cur);
  if (cur != device) cudaSetDevice(device);
  for (Block& b : blocks) {
    cudaEventSynchronize(b.done);
    cudaEventDestroy(b.done);
    cudaFreeAsync(b.p, stream->s);
  }
  if (stream) cudaStreamSynchronize(stream->s);
  if (cur != device) cudaSetDevice(cur);
}

void Context::activate() const { CKG_CUDA(cudaSetDevice(device)); }

thread_local LaneBinding tl_lane;

namespace {
// Two registries under two locks that are never held together: a context's trim takes its
// auxiliary-lane lock under g_ctx_mu, and creating an auxiliary lane registers it under
// g_lane_mu while that lock is held.
std::mutex g_ctx_mu;
std::vector<Context*> g_ctxs;  // every live context (Context::trim_all)
std::mutex g_lane_mu;
std::vector<const Lane*> g_lanes;  // every live lane (their pools are trimmed too)
}  // namespace

CtxStream::operator cudaStream_t() const {
  return tl_lane.ctx == c_ && tl_lane.lane ? tl_lane.lane->sres->s : c_->sres->s;
}

Lane::Lane(int device, int priority) {
  sres = std::make_shared<StreamRes>();
  sres->device = device;
  CKG_CUDA(cudaStreamCreateWithPriority(&sres->s, cudaStreamNonBlocking, priority));
  sres->own = true;
  cudaMemPoolProps props{};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = device;
  CKG_CUDA(cudaMemPoolCreate(&pool, &props));
  uint64_t thr = UINT64_MAX;
  int no = 0;
  CKG_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
  CKG_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolReuseAllowInternalDependencies, &no));
  std::lock_guard<std::mutex> lk(g_lane_mu);
  g_lanes.push_back(this);
}

Lane::~Lane() {
  {
    std::lock_guard<std::mutex> lk(g_lane_mu);
    g_lanes.erase(std::remove(g_lanes.begin(), g_lanes.end(), this), g_lanes.end());
  }
  if (sres && sres->s) cudaStreamSynchronize(sres->s);
  if (pool) cudaMemPoolDestroy(pool);  // released once its last block is freed
}

void Context::transfer_streams() {
  for (StreamPtr* sp : {&xfer_in, &xfer_out}) {
    if (*sp) continue;
    auto r = std::make_shared<StreamRes>();
    r->device = device;
    CKG_CUDA(cudaStreamCreateWithFlags(&r->s, cudaStreamNonBlocking));
    r->own = true;
    *sp = r;
  }
  if (!xpool) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    CKG_CUDA(cudaMemPoolCreate(&xpool, &props));
    uint64_t thr = UINT64_MAX;
    int no = 0;
    CKG_CUDA(cudaMemPoolSetAttribute(xpool, cudaMemPoolAttrReleaseThreshold, &thr));
    CKG_CUDA(cudaMemPoolSetAttribute(xpool, cudaMemPoolReuseAllowInternalDependencies, &no));
  }
  if (!xcache) {
    xcache = std::make_shared<XferCache>();
    xcache->device = device;
    xcache->pool = xpool;
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
      cudaGetLastError();
      total_b = (size_t)96 << 30;
    }
    xcache->max_bytes = total_b / 3;
    xcache->stream = xfer_in;
  }
}

uint64_t* Context::xfer_block(size_t words, cudaStream_t on) {
  transfer_streams();
  if (uint64_t* p = xcache->take(words, on)) {  // free, or `on` waits for its last use
    bounds::track(p, words * 8);
    return p;
  }
  uint64_t* p = nullptr;
  cudaError_t e = cudaMallocFromPoolAsync((void**)&p, words * 8, xpool, on);
  if (e == cudaErrorMemoryAllocation) {  // cached blocks still in flight elsewhere: return the rest
    cudaGetLastError();
    st_alloc_retries++;
    trim_all();
    e = cudaMallocFromPoolAsync((void**)&p, words * 8, xpool, on);
  }
  if (e != cudaSuccess) throw_cuda(e, "transfer block allocation");
  bounds::track(p, words * 8);
  return p;
}

namespace {
// `to` waits for the work queued on `from` so far.
void stream_after(cudaStream_t to, cudaStream_t from) {
  cudaEvent_t e;
  CKG_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  cudaError_t err = cudaEventRecord(e, from);
  if (err == cudaSuccess) err = cudaStreamWaitEvent(to, e, 0);
  cudaEventDestroy(e);
  if (err != cudaSuccess) throw_cuda(err, "cudaStreamWaitEvent");
}
}  // namespace

DevBufPtr Context::upload_overlapped(const uint64_t* host, size_t words) {
  activate();
  transfer_streams();
  auto b = std::make_shared<DevBuf>();
  b->sres = cur_sres();  // freed in compute order, after every use there
  b->device = device;
  b->words = words;
  if (!words) return b;
  b->p = xfer_block(words, xfer_in->s);
  b->cache = xcache;
  CKG_CUDA(cudaMemcpyAsync(b->p, host, words * 8, cudaMemcpyHostToDevice, xfer_in->s));
  stream_after(stream, xfer_in->s);
  return b;
}

DevBufPtr Context::upload_overlapped_list(const std::vector<HostPart>& parts, std::vector<size_t>& offsets) {
  activate();
  transfer_streams();
  auto b = std::make_shared<DevBuf>();
  b->sres = cur_sres();
  b->device = device;
  offsets.assign(parts.size(), 0);
  size_t total = 0;
  for (size_t i = 0; i < parts.size(); ++i) {
    offsets[i] = total;
    total += (parts[i].words + 31) & ~(size_t)31;
  }
  b->words = total;
  if (!total) return b;
  const auto t0 = std::chrono::steady_clock::now();
  b->p = xfer_block(total, xfer_in->s);
  b->cache = xcache;
  const auto t1 = std::chrono::steady_clock::now();
  // one copy per run of parts that are adjacent both in host memory and in the block
  for (size_t i = 0; i < parts.size();) {
    size_t j = i + 1, words = parts[i].words;
    while (j < parts.size() && parts[j].host == parts[i].host + words && offsets[j] == offsets[i] + words) {
      words += parts[j].words;
      ++j;
    }
    if (words)
      CKG_CUDA(cudaMemcpyAsync(b->p + offsets[i], parts[i].host, words * 8, cudaMemcpyHostToDevice, xfer_in->s));
    i = j;
  }
  stream_after(stream, xfer_in->s);
  const auto t2 = std::chrono::steady_clock::now();
  st_upload_calls++;
  st_upload_bytes += total * 8;
  st_upload_alloc_ns += std::chrono::duration_cast<std::chrono::nanoseconds>(t1 - t0).count();
  st_upload_copy_ns += std::chrono::duration_cast<std::chrono::nanoseconds>(t2 - t1).count();
  return b;
}

void Context::download_overlapped(const DevBufPtr& buf, const uint64_t* dev, size_t row_words, size_t pitch_words,
                                  size_t rows, uint64_t* host) {
  activate();
  transfer_streams();
  stream_after(xfer_out->s, stream);  // the data is final once the compute stream gets here
  if (pitch_words == row_words)
    CKG_CUDA(cudaMemcpyAsync(host, dev, rows * row_words * 8, cudaMemcpyDeviceToHost, xfer_out->s));
  else
    CKG_CUDA(cudaMemcpy2DAsync(host, row_words * 8, dev, pitch_words * 8, row_words * 8, rows,
                               cudaMemcpyDeviceToHost, xfer_out->s));
  // the buffer's free waits for this copy; finished earlier copies are dropped from the list
  auto& w = buf->waits;
  for (size_t i = 0; i < w.size();) {
    if (cudaEventQuery(w[i]) == cudaSuccess) {
      cudaEventDestroy(w[i]);
      w[i] = w.back();
      w.pop_back();
    } else {
      ++i;
    }
  }
  cudaEvent_t e;
  CKG_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  CKG_CUDA(cudaEventRecord(e, xfer_out->s));
  w.push_back(e);
}

void Context::download_overlapped_list(const std::vector<DevPart>& parts) {
  activate();
  transfer_streams();
  if (parts.empty()) return;
  const auto t0 = std::chrono::steady_clock::now();
  const cudaStream_t st = stream;
  // One kernel packs every part into one staging block on the compute stream; the download
  // stream then copies each run of adjacent host destinations with one transfer (the copies
  // read only the staging block, so the parts' buffers are free once the pack has run).
  std::vector<PackSeg> segs(parts.size());
  size_t total = 0;
  for (size_t i = 0; i < parts.size(); ++i) {
    const DevPart& d = parts[i];
    const size_t w = d.rows * d.row_words;
    if (w >= ((size_t)1 << 32) || d.row_words >= ((size_t)1 << 32))
      throw Error(ST_INVALID_PARAMS, "a download part above 2^32 words");
    segs[i] = PackSeg{d.dev, nullptr, d.pitch_words, (uint32_t)d.rows, (uint32_t)d.row_words};
    total += w;
  }
  if (!total) return;
  uint64_t* stage = xfer_block(total, st);
  size_t off = 0;
  for (PackSeg& sg : segs) {
    sg.dst = stage + off;
    off += (size_t)sg.rows * sg.row_words;
  }
  DevBufPtr desc = alloc((segs.size() * sizeof(PackSeg) + 7) / 8);
  upload_staged(desc->p, segs.data(), segs.size() * sizeof(PackSeg));
  launch_pack(reinterpret_cast<const PackSeg*>(desc->p), (int)segs.size(), st);
  CKG_CUDA(cudaGetLastError());
  // a part whose buffer is freed on another stream: that free waits for the pack
  std::vector<DevBuf*> seen;
  for (const DevPart& d : parts) {
    DevBuf* b = d.buf->get();
    if (b->sres->s == st || std::find(seen.begin(), seen.end(), b) != seen.end()) continue;
    seen.push_back(b);
    cudaEvent_t e;
    CKG_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    CKG_CUDA(cudaEventRecord(e, st));
    b->waits.push_back(e);
  }
  stream_after(xfer_out->s, st);
  off = 0;
  for (size_t i = 0; i < parts.size();) {
    size_t j = i + 1, bytes = (size_t)segs[i].rows * segs[i].row_words * 8;
    while (j < parts.size() &&
           (const unsigned char*)parts[j].host == (const unsigned char*)parts[i].host + bytes) {
      bytes += (size_t)segs[j].rows * segs[j].row_words * 8;
      ++j;
    }
    CKG_CUDA(cudaMemcpyAsync(parts[i].host, stage + off, bytes, cudaMemcpyDeviceToHost, xfer_out->s));
    off += bytes / 8;
    i = j;
  }
  cudaEvent_t copied;
  CKG_CUDA(cudaEventCreateWithFlags(&copied, cudaEventDisableTiming));
  CKG_CUDA(cudaEventRecord(copied, xfer_out->s));
  bounds::untrack(stage);
  xcache->give(stage, total, copied);  // reused once the copies are done
  st_download_calls++;
  st_download_ns += std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now() - t0).count();
}

void Context::upload_staged(void* dst, const void* src, size_t bytes) {
  if (!bytes) return;
  activate();
  cudaStream_t st = stream;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  CKG_CUDA(cudaStreamIsCapturing(st, &cap));
  if (cap != cudaStreamCaptureStatusNone)
    throw Error(ST_INVALID_PARAMS, "a batch is built before stream capture (use the batch's own graph capture)");
  std::lock_guard<std::mutex> lk(stage_mu);
  const size_t need = (bytes + 255) & ~(size_t)255;
  if (need > stage_cap) {  // grow: every copy out of the old ring completes first
    for (auto& u : stage_used) {
      cudaEventSynchronize(u.done);
      cudaEventDestroy(u.done);
    }
    stage_used.clear();
    if (stage) cudaFreeHost(stage);
    stage = nullptr;
    stage_cap = std::max(need * 4, (size_t)32 << 20);
    CKG_CUDA(cudaMallocHost((void**)&stage, stage_cap));
    stage_head = 0;
  }
  if (stage_head + need > stage_cap) stage_head = 0;
  for (auto it = stage_used.begin(); it != stage_used.end();) {
    const bool overlap = it->off < stage_head + need && stage_head < it->off + it->len;
    if (overlap) CKG_CUDA(cudaEventSynchronize(it->done));
    if (overlap || cudaEventQuery(it->done) == cudaSuccess) {
      cudaEventDestroy(it->done);
      it = stage_used.erase(it);
    } else {
      ++it;
    }
  }
  std::memcpy(stage + stage_head, src, bytes);
  CKG_CUDA(cudaMemcpyAsync(dst, stage + stage_head, bytes, cudaMemcpyHostToDevice, st));
  cudaEvent_t e;
  CKG_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  CKG_CUDA(cudaEventRecord(e, st));
  stage_used.push_back({stage_head, need, e});
  stage_head += need;
}

void Context::trim() {
  int cur = 0;
  cudaGetDevice(&cur);
  if (cur != device) cudaSetDevice(device);
  if (xcache) xcache->trim();
  if (xpool) cudaMemPoolTrimTo(xpool, 0);
  {
    std::lock_guard<std::mutex> lk(aux_mu);
    for (auto& l : aux_lanes)
      if (l && l->pool) cudaMemPoolTrimTo(l->pool, 0);
  }
  cudaMemPool_t def;
  if (cudaDeviceGetDefaultMemPool(&def, device) == cudaSuccess) cudaMemPoolTrimTo(def, 0);
  cudaGetLastError();
  if (cur != device) cudaSetDevice(cur);
}

void Context::trim_all() {
  {
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    for (Context* c : g_ctxs) c->trim();
  }
  {
    std::lock_guard<std::mutex> lk(g_lane_mu);
    for (const Lane* l : g_lanes)
      if (l->pool) cudaMemPoolTrimTo(l->pool, 0);
  }
  cudaGetLastError();
}

Lane& Context::aux_lane(int i) {
  if (i < 0 || i > 1) throw Error(ST_INVALID_PARAMS, "auxiliary lane index out of range");
  std::lock_guard<std::mutex> lk(aux_mu);
  if (!aux_lanes[i]) aux_lanes[i] = std::make_unique<Lane>(device);
  return *aux_lanes[i];
}

void Context::join_transfers() {
  activate();
  if (xfer_in) stream_after(stream, xfer_in->s);
  if (xfer_out) stream_after(stream, xfer_out->s);
}

void Context::sync_transfers() {
  activate();
  if (xfer_in) CKG_CUDA(cudaStreamSynchronize(xfer_in->s));
  if (xfer_out) CKG_CUDA(cudaStreamSynchronize(xfer_out->s));
}

DevBufPtr Context::alloc(size_t words) {
  auto b = std::make_shared<DevBuf>();
  const Lane* ln = tl_lane.ctx == this ? tl_lane.lane : nullptr;
  b->sres = ln ? ln->sres : sres;
  b->device = device;
  b->words = words;
  if (words) {
    auto get = [&] {
      return ln ? cudaMallocFromPoolAsync((void**)&b->p, words * 8, ln->pool, ln->sres->s)
                : cudaMallocAsync((void**)&b->p, words * 8, sres->s);
    };
    cudaError_t e = get();
    if (e == cudaErrorMemoryAllocation) {
      // Free memory may sit cached in another pool (each keeps what it frees): hand the unused
      // blocks of every context's pools and transfer caches back, then try once more.
      cudaGetLastError();
      st_alloc_retries++;
      trim_all();
      e = get();
    }
    if (e != cudaSuccess) throw_cuda(e, "device allocation");
    bounds::track(b->p, words * 8);
  }
  return b;
}

namespace {

// Whether target t of a conversion from `src` can take the FP64-assisted form (kernels.cu,
// k_bconv_f64): V = sum_j y_j w_tj + e (t - [S]_t) + (t - [h]_t) is computed mod 2^64 on the
// integer pipe, its quotient K = V / t is estimated as A = sum_j fl(y_j) fl(w_tj / t) + e fl(..)
// + fl(..) by an FP64 FMA chain, and r = V - rint(A) t must stay inside the signed 64-bit range
// with room to spare. With T_j = y_j w_tj / t < s_j: each term's representation error is at most
// s_j (e1 + e2) (plus e1 e2), where fl(w_tj / t) carries e2 = 2^-53 (3 2^-53 when t >= 2^53, as
// w_tj and t are rounded first) and fl(y_j) e1 = 0 (2^-53 when s_j > 2^53); each of the n + 2
// roundings of the chain is at most half an ulp of A_max = sum_j s_j + 17, the two constant
// terms add 17 2^-52, and rint 1/2. Their sum bounds |K - rint(A)|, and t times it must be at
// most 2^62. `two_stage` is set unless the estimate alone is within 1/2, where r already lies in
// (-t, t).
bool conv_f64_form(const std::vector<HostMod>& mods, const std::vector<uint32_t>& src, uint32_t t, bool* two_stage) {
  const uint64_t q = mods[t].q;
  if (src.empty() || src.size() > (size_t)kMaxSrcF64 || q < (1ULL << 30)) return false;
  const int e2 = q >= (1ULL << 53) ? 3 : 1;
  long double sum = 0, rep = 0;
  for (uint32_t s : src) {
    const long double v = (long double)mods[s].q;
    sum += v;
    rep += v * (e2 + (mods[s].q > (1ULL << 53) ? 1 : 0));
  }
  const long double amax = (sum + 17 + 64) * (1 + ldexpl(1.0L, -40));
  const long double ulp = ldexpl(1.0L, ilogbl(amax) - 52);
  const long double eta = rep * ldexpl(1.0L, -53) + (long double)(src.size() + 2) * ulp / 2 + 17 * ldexpl(1.0L, -52) +
                          ldexpl(1.0L, -30);
  *two_stage = eta >= 0.5L;
  return (eta + 0.5L) * (long double)q <= ldexpl(1.0L, 62);
}

// The inner product's FP64-assisted form for outputs modulo q (kernels.cu k_inner_product):
// with d_j, k_j < q < 2^50 exact in f64, A = sum_j d_j fl(fl(k_j) fl(1/q)) by FMA is within
// delta of V / q (each term's factor carries 2^-52 relative, each of the beta roundings half an
// ulp of A_max = beta q, rint 1/2). Returns the offset ceil(delta) that makes
// x = V - rint(A) q + ceil(delta) q nonnegative, or 0 when A_max >= 2^52 or x could reach 2^53.
uint32_t ip_f64_offset(uint64_t q, uint32_t beta) {
  if (q >= (1ULL << 50)) return 0;
  const long double amax = (long double)beta * q * (1 + ldexpl(1.0L, -40)) + 64;
  if (amax >= ldexpl(1.0L, 52)) return 0;
  const long double ulp = ldexpl(1.0L, ilogbl(amax) - 52);
  const long double delta = (long double)beta * q * ldexpl(1.0L, -52) + beta * ulp / 2 + 0.5L + ldexpl(1.0L, -30);
  const long double off = ceill(delta);
  if ((off + delta) * q >= ldexpl(1.0L, 53)) return 0;
  return (uint32_t)off;
}

void tc_block(const std::vector<HostMod>& mods, const std::vector<uint32_t>& src, const std::vector<uint32_t>& dst,
              std::vector<uint64_t>& w);

// Conversion table (kernels.cuh ConvLayout) for sources `src` -> targets `dst` (global prime
// indices): sum_j y_j [S/s_j]_t - e [S]_t - [h]_t with h = (S-1)/2. Targets that allow it get the
// FP64-assisted record and come first.
std::vector<uint64_t> conv_table(const std::vector<HostMod>& mods, const std::vector<uint32_t>& src,
                                 const std::vector<uint32_t>& dst) {
  std::vector<uint64_t> w;
  const size_t ns = src.size();
  auto bits = [](double v) {
    uint64_t b;
    memcpy(&b, &v, 8);
    return b;
  };
  w.push_back(0);  // FP64-assisted record count, set below
  for (size_t j = 0; j < ns; ++j) {
    const HostMod& m = mods[src[j]];
    uint64_t qhat = 1;
    for (size_t i = 0; i < ns; ++i)
      if (i != j) qhat = m.mul(qhat, mods[src[i]].q % m.q);
    uint64_t qhinv = m.inv(qhat);
    w.push_back(src[j]);
    w.push_back(qhinv);
    w.push_back(m.shoup(qhinv));
    w.push_back(m.q >> 1);
    w.push_back(bits(1.0 / (double)m.q));
  }
  std::vector<std::pair<size_t, bool>> order;  // (output position, two_stage); FP64 records first
  std::vector<size_t> exact;
  for (size_t o = 0; o < dst.size(); ++o) {
    bool two = false;
    if (conv_f64_form(mods, src, dst[o], &two)) order.push_back({o, two});
    else exact.push_back(o);
  }
  w[0] = order.size();
  for (size_t o : exact) order.push_back({o, false});
  for (size_t r = 0; r < order.size(); ++r) {
    const bool f64 = r < w[0];
    const size_t o = order[r].first;
    const uint32_t t = dst[o];
    const HostMod& m = mods[t];
    uint64_t S = 1 % m.q;
    for (uint32_t s : src) S = m.mul(S, mods[s].q % m.q);
    // h = (S - 1)/2 mod t = (S - 1) * 2^-1
    uint64_t h = m.mul(m.sub(S, 1 % m.q), (m.q + 1) / 2);
    const uint64_t r64 = (uint64_t)(((u128)1 << 64) % m.q);
    std::vector<uint64_t> qh(ns);
    for (size_t j = 0; j < ns; ++j) {
      uint64_t qhat = 1 % m.q;
      for (size_t i = 0; i < ns; ++i)
        if (i != j) qhat = m.mul(qhat, mods[src[i]].q % m.q);
      qh[j] = qhat;
    }
    w.push_back(t);
    w.push_back(m.q - S);
    w.push_back(m.q - h);
    w.push_back(m.q);
    if (f64) {
      w.push_back(bits(1.0 / (double)m.q));
      w.push_back(bits((double)(m.q - S) / (double)m.q));
      w.push_back(bits((double)(m.q - h) / (double)m.q));
      w.push_back(o | ((uint64_t)order[r].second << 32));
      for (size_t j = 0; j < ns; ++j) w.push_back(qh[j]);
      for (size_t j = 0; j < ns; ++j) w.push_back(bits((double)qh[j] / (double)m.q));
    } else {
      w.push_back(r64);
      w.push_back(m.shoup(r64));
      w.push_back(m.shoup(1));
      w.push_back(o);
      for (size_t j = 0; j < ns; ++j) w.push_back((qh[j] & ((1ULL << 30) - 1)) | ((qh[j] >> 30) << 32));
      for (size_t j = 0; j < ns; ++j) w.push_back(0);
    }
  }
  tc_block(mods, src, dst, w);
  return w;
}

// The tensor-core block of a conversion table (kernels.cuh ConvLayout, bconv_tc.cu): the
// per-target constants and the byte-split weights. sum_j y_j w_tj = sum_j sum_a y_j[a] 2^(8a) w_tj
// is congruent mod t to sum_b 2^(8b) C_b with C_b = sum_(j,a) y_j[a] W[o, b][j, a], where
// W[o, b][j, a] is byte b of [2^(8a) w_tj]_t: a u8 x u8 -> s32 product of the source bytes (the
// y_j words as stored) with these weight bytes.
void tc_block(const std::vector<HostMod>& mods, const std::vector<uint32_t>& src, const std::vector<uint32_t>& dst,
              std::vector<uint64_t>& w) {
  const size_t ns = src.size(), nd = dst.size();
  while (w.size() % 2) w.push_back(0);
  bool big = true;
  for (uint32_t t : dst) big = big && mods[t].q >= (1ULL << 30);
  if (ns == 0 || ns > (size_t)ConvLayout::kTcMaxSrc || nd == 0 || nd > (size_t)ConvLayout::kTcMaxDst || !big) {
    w.push_back(0);  // no block: the header reads K = N = 0
    w.push_back(0);
    return;
  }
  const int K = ns <= 4 ? 32 : 64;
  const int N = (int)((8 * nd + 15) / 16 * 16);
  w.push_back((uint64_t)K | ((uint64_t)N << 32));
  w.push_back(0);
  std::vector<uint8_t> B((size_t)N * K, 0);
  for (size_t o = 0; o < nd; ++o) {
    const HostMod& m = mods[dst[o]];
    uint64_t S = 1 % m.q;
    for (uint32_t s : src) S = m.mul(S, mods[s].q % m.q);
    const uint64_t h = m.mul(m.sub(S, 1 % m.q), (m.q + 1) / 2);
    auto bits = [](double v) {
      uint64_t b;
      memcpy(&b, &v, 8);
      return b;
    };
    w.push_back(m.q);
    w.push_back(bits(1.0 / (double)m.q));
    w.push_back(m.q - S);
    w.push_back(m.q - h);
    w.push_back(bits((double)(m.q - S)));
    w.push_back(bits((double)(m.q - h)));
    for (size_t j = 0; j < ns; ++j) {
      uint64_t qhat = 1 % m.q;
      for (size_t i = 0; i < ns; ++i)
        if (i != j) qhat = m.mul(qhat, mods[src[i]].q % m.q);
      uint64_t v = qhat;  // [2^(8a) w_tj]_t for a = 0, 1, ...
      for (int a = 0; a < 8; ++a) {
        const int k = (int)(8 * j + a);
        for (int b = 0; b < 8; ++b) {
          const int r = (int)(8 * o + b);
          B[(size_t)(r / 8) * (8 * K) + (k / 16) * 128 + (r % 8) * 16 + (k % 16)] = (uint8_t)(v >> (8 * b));
        }
        v = m.mul(v, 256 % m.q);
      }
    }
  }
  const size_t words = B.size() / 8;
  const size_t at = w.size();
  w.resize(at + words);
  memcpy(w.data() + at, B.data(), B.size());
}

}  // namespace

Context::Context(uint32_t log_n_, const std::vector<uint64_t>& q, const std::vector<uint64_t>& p, uint32_t dnum_,
                 int device_, cudaStream_t st)
    : device(device_), log_n(log_n_) {
  if (log_n < 5 || log_n > 17) throw Error(ST_INVALID_PARAMS, "log_n must be in 5..=17");
  if (q.empty() || p.empty()) throw Error(ST_INVALID_PARAMS, "q and p must be non-empty");
  if (dnum_ == 0 || q.size() % dnum_ != 0) throw Error(ST_INVALID_PARAMS, "dnum must divide the number of q primes");
  if (q.size() / dnum_ > (size_t)kMaxSrc || p.size() > (size_t)kMaxSrc)
    throw Error(ST_INVALID_PARAMS, "at most 16 primes per digit and 16 special primes");
  if (dnum_ > (uint32_t)kMaxDigits) throw Error(ST_INVALID_PARAMS, "at most 16 digits");
  if (q.size() + p.size() > 64) throw Error(ST_INVALID_PARAMS, "at most 64 primes");
  n = 1ULL << log_n;
  nq = q.size();
  k = p.size();
  dnum = dnum_;
  alpha = nq / dnum;
  L = nq - 1;
  primes = q;
  primes.insert(primes.end(), p.begin(), p.end());
  for (size_t i = 0; i < primes.size(); ++i) {
    uint64_t v = primes[i];
    if (v < 3 || v >= (1ULL << 60) || !is_prime(v) || (v - 1) % (2 * n) != 0)
      throw Error(ST_INVALID_PARAMS, "modulus " + std::to_string(v) + " is not an NTT-friendly prime below 2^60");
    for (size_t j = 0; j < i; ++j)
      if (primes[j] == v) throw Error(ST_INVALID_PARAMS, "duplicate modulus " + std::to_string(v));
    mods.emplace_back(v);
  }
  CKG_CUDA(cudaSetDevice(device));
  sres = std::make_shared<StreamRes>();
  sres->device = device;
  if (st) {
    sres->s = st;
  } else {
    CKG_CUDA(cudaStreamCreateWithFlags(&sres->s, cudaStreamNonBlocking));
    sres->own = true;
  }
  {  // keep freed pool memory cached: steady-state ops allocate without driver calls
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
      uint64_t thr = UINT64_MAX;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
  }
  const size_t np = primes.size();
  // per-prime constants
  std::vector<PrimeConst> pc(np);
  std::vector<ulonglong2> twf(np * n), twi(np * n);
  for (size_t i = 0; i < np; ++i) {
    const HostMod& m = mods[i];
    PrimeConst& c = pc[i];
    c.q = m.q;
    c.two_q = 2 * m.q;
    c.b = bit_length(m.q);
    c.mu = (uint64_t)(((u128)1 << (2 * c.b)) / m.q);
    uint64_t psi = minimal_root(n, m), psi_inv = m.inv(psi), ninv = m.inv(n);
    c.ninv = ninv;
    c.ninv_s = m.shoup(ninv);
    uint64_t p = 1, pi = 1;
    for (uint64_t e = 0; e < n; ++e) {
      uint64_t r = bitrev(e, log_n);
      twf[i * n + r] = make_ulonglong2(p, m.shoup(p));
      twi[i * n + r] = make_ulonglong2(pi, m.shoup(pi));
      p = m.mul(p, psi);
      pi = m.mul(pi, psi_inv);
    }
    c.wninv = m.mul(twi[i * n + 1].x, ninv);
    c.wninv_s = m.shoup(c.wninv);
    c.r64 = (uint64_t)(((u128)1 << 64) % m.q);
    c.r64_s = m.shoup(c.r64);
    c.one_s = m.shoup(1);
    c.qd = (double)m.q;
    c.qinv = 1.0 / c.qd;
    c.ninvd = (double)c.ninv;
    c.wninvd = (double)c.wninv;
    c.ip_off = ip_f64_offset(m.q, dnum);
  }
  std::vector<double> twdf(np * n), twdi(np * n);
  for (size_t i = 0; i < np * n; ++i) {
    twdf[i] = (double)twf[i].x;  // exact below 2^53; used only for primes below 2^50
    twdi[i] = (double)twi[i].x;
  }
  CKG_CUDA(cudaMalloc(&d_prime, np * sizeof(PrimeConst)));
  CKG_CUDA(cudaMalloc(&d_tw_fwd, np * n * sizeof(ulonglong2)));
  CKG_CUDA(cudaMalloc(&d_tw_inv, np * n * sizeof(ulonglong2)));
  CKG_CUDA(cudaMemcpy(d_prime, pc.data(), np * sizeof(PrimeConst), cudaMemcpyHostToDevice));
  CKG_CUDA(cudaMemcpy(d_tw_fwd, twf.data(), np * n * sizeof(ulonglong2), cudaMemcpyHostToDevice));
  CKG_CUDA(cudaMemcpy(d_tw_inv, twi.data(), np * n * sizeof(ulonglong2), cudaMemcpyHostToDevice));
  CKG_CUDA(cudaMalloc(&d_twd_fwd, np * n * sizeof(double)));
  CKG_CUDA(cudaMalloc(&d_twd_inv, np * n * sizeof(double)));
  CKG_CUDA(cudaMemcpy(d_twd_fwd, twdf.data(), np * n * sizeof(double), cudaMemcpyHostToDevice));
  CKG_CUDA(cudaMemcpy(d_twd_inv, twdi.data(), np * n * sizeof(double), cudaMemcpyHostToDevice));
  dt = DevTables{d_prime, d_tw_fwd, d_tw_inv, d_twd_fwd, d_twd_inv, (int)log_n};
  // The tensor-core conversion's FP64 quotient needs targets of at least 30 bits, and its tiles
  // 128 coefficients; then every table of <= 8 sources and <= 32 targets carries its block.
  {
    bool big = true;
    for (uint64_t v : primes) big = big && v >= (1ULL << 30);
    dt.bconv_tc = big && log_n >= 7 ? 1 : 0;
  }
  // The TMA-staged column passes are bit-identical but measured slower than the per-tile ones
  // (768-limb transforms: 86 against 69 us per forward and 99 against 81 us per inverse 256-limb
  // column launch): off unless asked for.
  dt.ntt_tma = 0;
  CKG_CUDA(cudaDeviceGetAttribute(&dt.sms, cudaDevAttrMultiProcessorCount, device));

  // conversion tables
  std::vector<uint64_t> conv;
  auto push = [&](const std::vector<uint64_t>& t) {
    if (conv.size() % 2) conv.push_back(0);  // tables start on 16-byte boundaries
    size_t off = conv.size();
    conv.insert(conv.end(), t.begin(), t.end());
    return off;
  };
  modup_off.assign((size_t)nq * dnum, 0);
  moddown_off.assign(nq, 0);
  rescale_off.assign(nq, 0);
  std::vector<uint32_t> pidx;
  for (uint32_t t = 0; t < k; ++t) pidx.push_back(p_prime(t));
  for (uint32_t l = 0; l <= L; ++l) {
    for (uint32_t j = 0; j < digits_at(l); ++j) {
      std::vector<uint32_t> src, dst;
      for (uint32_t i = digit_start(j); i < digit_end(j, l); ++i) src.push_back(i);
      for (uint32_t i = 0; i <= l; ++i)
        if (i < digit_start(j) || i >= digit_end(j, l)) dst.push_back(i);
      dst.insert(dst.end(), pidx.begin(), pidx.end());
      modup_off[(size_t)l * dnum + j] = push(conv_table(mods, src, dst));
    }
    std::vector<uint32_t> qs;
    for (uint32_t i = 0; i <= l; ++i) qs.push_back(i);
    moddown_off[l] = push(conv_table(mods, pidx, qs));
    if (l >= 1) {
      qs.pop_back();
      rescale_off[l] = push(conv_table(mods, {l}, qs));
    }
  }
  CKG_CUDA(cudaMalloc(&d_conv, conv.size() * 8));
  CKG_CUDA(cudaMemcpy(d_conv, conv.data(), conv.size() * 8, cudaMemcpyHostToDevice));
  // finish constants
  for (uint32_t i = 0; i <= L; ++i) {
    const HostMod& m = mods[i];
    uint64_t pm = 1;
    for (uint32_t t = 0; t < k; ++t) pm = m.mul(pm, primes[p_prime(t)] % m.q);
    uint64_t v = m.inv(pm);
    pinv.push_back({v, m.shoup(v)});
  }
  qlinv.assign(nq, {});
  for (uint32_t l = 1; l <= L; ++l)
    for (uint32_t i = 0; i < l; ++i) {
      const HostMod& m = mods[i];
      uint64_t v = m.inv(primes[l] % m.q);
      qlinv[l].push_back({v, m.shoup(v)});
    }
  CKG_CUDA(cudaDeviceSynchronize());
  std::lock_guard<std::mutex> lk(g_ctx_mu);  // last: a constructor that throws registers nothing
  g_ctxs.push_back(this);
}

Context::~Context() {
  {
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    g_ctxs.erase(std::remove(g_ctxs.begin(), g_ctxs.end(), this), g_ctxs.end());
  }
  cudaSetDevice(device);
  cudaStreamSynchronize(stream);
  if (xpool) cudaMemPoolDestroy(xpool);  // released once its last block is freed
  for (auto& u : stage_used) {
    cudaEventSynchronize(u.done);
    cudaEventDestroy(u.done);
  }
  if (stage) cudaFreeHost(stage);
  for (auto& kv : perms) cudaFree(kv.second);
  if (d_xhalf) cudaFree(d_xhalf);
  cudaFree(d_prime);
  cudaFree(d_tw_fwd);
  cudaFree(d_tw_inv);
  cudaFree(d_twd_fwd);
  cudaFree(d_twd_inv);
  cudaFree(d_conv);
}

const uint64_t* Context::x_half() {
  std::lock_guard<std::mutex> lk(mu);
  if (d_xhalf) return d_xhalf;
  std::vector<uint64_t> mono((size_t)(L + 1) * n, 0);
  for (uint32_t i = 0; i <= L; ++i) mono[(size_t)i * n + n / 2] = 1;
  uint64_t* d = nullptr;
  CKG_CUDA(cudaMalloc(&d, mono.size() * 8));
  CKG_CUDA(cudaMemcpy(d, mono.data(), mono.size() * 8, cudaMemcpyHostToDevice));
  std::vector<LimbRef> refs;
  for (uint32_t i = 0; i <= L; ++i) refs.push_back(LimbRef{d + (size_t)i * n, d + (size_t)i * n, i, 0});
  launch_ntt(dt, refs.data(), (int)refs.size(), false, stream);
  CKG_CUDA(cudaStreamSynchronize(stream));  // complete before any stream (lane) reads the cache
  d_xhalf = d;
  return d;
}

const uint32_t* Context::perm(uint64_t elt) {
  std::lock_guard<std::mutex> lk(mu);
  auto it = perms.find(elt);
  if (it != perms.end()) return it->second;
  auto v = galois_perm(n, elt);
  uint32_t* d = nullptr;
  CKG_CUDA(cudaMalloc(&d, n * 4));
  CKG_CUDA(cudaMemcpy(d, v.data(), n * 4, cudaMemcpyHostToDevice));
  perms[elt] = d;
  return d;
}

// -------------------------------------------------------------------------------------

void ntt_limbs(Context& c, const std::vector<LimbRef>& refs, bool inverse) {
  if (!refs.empty()) launch_ntt(c.dt, refs.data(), (int)refs.size(), inverse, c.stream);
}

void ntt_poly(Context& c, const uint64_t* src, uint64_t* dst, uint32_t first_prime, uint32_t count, bool inverse) {
  std::vector<LimbRef> refs(count);
  for (uint32_t i = 0; i < count; ++i) refs[i] = LimbRef{src + i * c.n, dst + i * c.n, first_prime + i, 0};
  ntt_limbs(c, refs, inverse);
}

void rescale_many(Context& c, const std::vector<const uint64_t*>& in, uint32_t l, const std::vector<uint64_t*>& out) {
  const size_t np = in.size(), N = c.n;
  if (!np) return;
  if (l < 1) throw Error(ST_NO_LEVELS_LEFT, "cannot rescale at level 0");
  auto scratch = c.alloc(np * (1 + l) * N);
  // With two-pass transforms (N >= 2^12) the NTT's column pass reads the centred lift of the last
  // limb itself (LimbRef::aux = l + 1); smaller rings run the one-source conversion first.
  const bool fuse_lift = c.log_n >= 12;
  std::vector<LimbRef> refs;
  std::vector<ConvJob> jobs;
  for (size_t i = 0; i < np; ++i) {
    uint64_t* last = scratch->p + i * (1 + l) * N;
    refs.push_back(LimbRef{in[i] + (size_t)l * N, last, l, 0});
    jobs.push_back(ConvJob{last, last + N, c.d_conv + c.rescale_off[l], N, N});
  }
  ntt_limbs(c, refs, true);
  if (!fuse_lift) launch_bconv(c.dt, jobs.data(), (int)jobs.size(), 1, (int)l, c.stream);
  refs.clear();
  std::vector<FinRef> fin;
  for (size_t i = 0; i < np; ++i) {
    const uint64_t* last = scratch->p + i * (1 + l) * N;
    uint64_t* t = scratch->p + i * (1 + l) * N + N;
    for (uint32_t j = 0; j < l; ++j) {
      refs.push_back(LimbRef{last, t + j * N, j, l + 1});
      fin.push_back(FinRef{in[i] + j * N, t + j * N, nullptr, nullptr, out[i] + j * N, c.qlinv[l][j].first,
                           c.qlinv[l][j].second, j, 0});
    }
  }
  launch_ntt_finish(c.dt, fin.data(), (int)fin.size(), c.stream, fuse_lift ? refs.data() : nullptr);
}

void mod_down_many(Context& c, const std::vector<ModDownJob>& jobs, uint32_t l) {
  const size_t nj = jobs.size(), N = c.n, per = c.k + l + 1;
  if (!nj) return;
  auto scratch = c.alloc(nj * per * N);
  std::vector<LimbRef> refs;
  std::vector<ConvJob> conv;
  for (size_t i = 0; i < nj; ++i) {
    uint64_t* pc = scratch->p + i * per * N;
    for (uint32_t t = 0; t < c.k; ++t) refs.push_back(LimbRef{jobs[i].ppart + t * N, pc + t * N, c.p_prime(t), 0});
    conv.push_back(ConvJob{pc, pc + c.k * N, c.d_conv + c.moddown_off[l], N, N});
  }
  ntt_limbs(c, refs, true);
  launch_bconv(c.dt, conv.data(), (int)nj, (int)c.k, (int)(l + 1), c.stream);
  refs.clear();
  std::vector<FinRef> fin;
  for (size_t i = 0; i < nj; ++i) {
    uint64_t* t = scratch->p + i * per * N + c.k * N;
    for (uint32_t j = 0; j <= l; ++j) {
      refs.push_back(LimbRef{t + j * N, t + j * N, j, 0});
      fin.push_back(FinRef{jobs[i].qpart + j * N, t + j * N, jobs[i].add ? jobs[i].add + j * N : nullptr,
                           jobs[i].add_perm, jobs[i].out + j * N, c.pinv[j].first, c.pinv[j].second, j, 0});
    }
  }
  launch_ntt_finish(c.dt, fin.data(), (int)fin.size(), c.stream);
}

size_t conv_limbs(const Context& c, uint32_t l) {
  size_t s = 0;
  for (uint32_t j = 0; j < c.digits_at(l); ++j) s += (l + 1) - (c.digit_end(j, l) - c.digit_start(j)) + c.k;
  return s;
}

size_t conv_offset_limbs(const Context& c, uint32_t l, uint32_t jj) {
  size_t s = 0;
  for (uint32_t j = 0; j < jj; ++j) s += (l + 1) - (c.digit_end(j, l) - c.digit_start(j)) + c.k;
  return s;
}

namespace {

// Global prime index of target t of digit j at level l: data primes outside the digit in
// increasing order, then the special primes.
inline uint32_t target_prime(const Context& c, uint32_t l, uint32_t j, uint32_t t) {
  const uint32_t s = c.digit_start(j), a = c.digit_end(j, l) - s;
  if (t < s) return t;
  if (t < l + 1 - a) return t + a;
  return c.p_prime(t - (l + 1 - a));
}

// ModUp with caller-provided coefficient scratch ((l+1) limbs per input).
void mod_up_into(Context& c, const std::vector<const uint64_t*>& in, uint32_t l, const std::vector<uint64_t*>& conv_out,
                 const std::vector<uint64_t*>& coeff) {
  const size_t N = c.n;
  std::vector<LimbRef> refs;
  for (size_t i = 0; i < in.size(); ++i)
    for (uint32_t j = 0; j <= l; ++j) refs.push_back(LimbRef{in[i] + j * N, coeff[i] + j * N, j, 0});
  ntt_limbs(c, refs, true);
  // group the conversions by shape (a level-clipped last digit differs)
  std::map<std::pair<int, int>, std::vector<ConvJob>> groups;
  for (size_t i = 0; i < in.size(); ++i)
    for (uint32_t j = 0; j < c.digits_at(l); ++j) {
      const uint32_t s = c.digit_start(j), a = c.digit_end(j, l) - s, T = l + 1 - a + c.k;
      groups[{(int)a, (int)T}].push_back(ConvJob{coeff[i] + s * N, conv_out[i] + conv_offset_limbs(c, l, j) * N,
                                                 c.d_conv + c.modup_off[(size_t)l * c.dnum + j], N, N});
    }
  for (auto& g : groups)
    launch_bconv(c.dt, g.second.data(), (int)g.second.size(), g.first.first, g.first.second, c.stream);
  refs.clear();
  for (size_t i = 0; i < in.size(); ++i)
    for (uint32_t j = 0; j < c.digits_at(l); ++j) {
      const uint32_t a = c.digit_end(j, l) - c.digit_start(j), T = l + 1 - a + c.k;
      uint64_t* base = conv_out[i] + conv_offset_limbs(c, l, j) * N;
      for (uint32_t t = 0; t < T; ++t) refs.push_back(LimbRef{base + t * N, base + t * N, target_prime(c, l, j, t), 0});
    }
  ntt_limbs(c, refs, false);
}

}  // namespace

void mod_up_many(Context& c, const std::vector<const uint64_t*>& in, uint32_t l, const std::vector<uint64_t*>& conv_out) {
  if (in.empty()) return;
  auto scratch = c.alloc(in.size() * (l + 1) * c.n);
  std::vector<uint64_t*> coeff;
  for (size_t i = 0; i < in.size(); ++i) coeff.push_back(scratch->p + i * (l + 1) * c.n);
  mod_up_into(c, in, l, conv_out, coeff);
}

size_t key_switch_scratch_words(const Context& c, uint32_t l) {
  // coefficient copy of the input, converted digits, two extended accumulators,
  // ModDown scratch for both accumulators
  return ((l + 1) + conv_limbs(c, l) + 2 * (l + 1 + c.k) + 2 * (c.k + l + 1)) * c.n;
}

namespace {

void check_ks(const Context& c, const KsJob& j, uint32_t l) {
  if (!j.key) throw Error(ST_INVALID_PARAMS, "missing key");
  if (j.key->ctx != &c) throw Error(ST_INVALID_PARAMS, "key is not over this context");
  if (l + 1 > j.key->q_limbs) throw Error(ST_INVALID_PARAMS, "level above the key's maximum level");
  if (c.digits_at(l) > j.key->parts) throw Error(ST_INVALID_PARAMS, "key has too few parts for this level");
}

// Inner product + ModDown of a group of jobs whose digits are in conv[i]; acc buffers and
// ModDown scratch are provided.
void ks_tail(Context& c, const std::vector<KsJob>& jobs, uint32_t l, const std::vector<const uint64_t*>& conv,
             const std::vector<uint64_t*>& acc, const std::vector<uint64_t*>& mdscratch) {
  const size_t N = c.n, ext = l + 1 + c.k;
  std::vector<IpJob> ip;
  for (size_t i = 0; i < jobs.size(); ++i) {
    IpJob jb{};
    jb.level = (int)l;
    jb.ndig = (int)c.digits_at(l);
    jb.key_q = (int)jobs[i].key->q_limbs;
    jb.in = jobs[i].in;
    for (uint32_t j = 0; j < c.digits_at(l); ++j) jb.conv[j] = conv[i] + conv_offset_limbs(c, l, j) * N;
    jb.key = jobs[i].key->buf->p;
    jb.out_b = acc[i];
    jb.out_a = acc[i] + ext * N;
    jb.perm = jobs[i].perm;
    ip.push_back(jb);
  }
  launch_inner_product(c.dt, (int)c.alpha, (int)c.L, (int)c.k, ip.data(), (int)ip.size(), c.stream);
  // ModDown of both accumulators of every job, fused with the additions.
  const size_t per = c.k + l + 1;
  std::vector<LimbRef> refs;
  std::vector<ConvJob> cj;
  for (size_t i = 0; i < jobs.size(); ++i)
    for (int ba = 0; ba < 2; ++ba) {
      const uint64_t* x = acc[i] + ba * ext * N;
      uint64_t* pc = mdscratch[i] + ba * per * N;
      for (uint32_t t = 0; t < c.k; ++t) refs.push_back(LimbRef{x + (l + 1 + t) * N, pc + t * N, c.p_prime(t), 0});
      cj.push_back(ConvJob{pc, pc + c.k * N, c.d_conv + c.moddown_off[l], N, N});
    }
  ntt_limbs(c, refs, true);
  launch_bconv(c.dt, cj.data(), (int)cj.size(), (int)c.k, (int)(l + 1), c.stream);
  refs.clear();
  std::vector<FinRef> fin;
  for (size_t i = 0; i < jobs.size(); ++i)
    for (int ba = 0; ba < 2; ++ba) {
      const uint64_t* x = acc[i] + ba * ext * N;
      uint64_t* t = mdscratch[i] + ba * per * N + c.k * N;
      uint64_t* out = ba == 0 ? jobs[i].out_b : jobs[i].out_a;
      const uint64_t* add = ba == 0 ? jobs[i].add_b : jobs[i].add_a;
      const uint32_t* aperm = ba == 0 ? jobs[i].add_b_perm : nullptr;
      for (uint32_t j = 0; j <= l; ++j) {
        refs.push_back(LimbRef{t + j * N, t + j * N, j, 0});
        fin.push_back(FinRef{x + j * N, t + j * N, add ? add + j * N : nullptr, aperm, out + j * N, c.pinv[j].first,
                             c.pinv[j].second, j, 0});
      }
    }
  launch_ntt_finish(c.dt, fin.data(), (int)fin.size(), c.stream);
}

void ks_group(Context& c, const std::vector<KsJob>& jobs, uint32_t l, uint64_t* scratch) {
  const size_t N = c.n;
  const size_t coeffw = (l + 1) * N, convw = conv_limbs(c, l) * N, accw = 2 * (l + 1 + c.k) * N;
  const size_t mdw = 2 * (c.k + l + 1) * N, per = coeffw + convw + accw + mdw;
  std::vector<const uint64_t*> in, conv;
  std::vector<uint64_t*> coeff, convw_p, acc, md;
  for (size_t i = 0; i < jobs.size(); ++i) {
    uint64_t* base = scratch + i * per;
    coeff.push_back(base);
    convw_p.push_back(base + coeffw);
    acc.push_back(base + coeffw + convw);
    md.push_back(base + coeffw + convw + accw);
    conv.push_back(jobs[i].conv ? jobs[i].conv : base + coeffw);
    if (!jobs[i].conv) in.push_back(jobs[i].in);
  }
  // ModUp for the jobs without precomputed digits
  std::vector<uint64_t*> co, cv;
  for (size_t i = 0; i < jobs.size(); ++i)
    if (!jobs[i].conv) {
      co.push_back(coeff[i]);
      cv.push_back(convw_p[i]);
    }
  if (!in.empty()) mod_up_into(c, in, l, cv, co);
  ks_tail(c, jobs, l, conv, acc, md);
}

}  // namespace

void key_switch_with_scratch(Context& c, const KsJob& job, uint32_t l, uint64_t* scratch) {
  check_ks(c, job, l);
  ks_group(c, {job}, l, scratch);
}

void key_switch_many(Context& c, const std::vector<KsJob>& jobs, uint32_t l) {
  for (auto& j : jobs) check_ks(c, j, l);
  const size_t per = key_switch_scratch_words(c, l);
  // Bound the scratch of one group to about 2 GiB.
  size_t group = std::max<size_t>(1, ((size_t)2 << 30) / (per * 8));
  for (size_t off = 0; off < jobs.size(); off += group) {
    size_t cnt = std::min(group, jobs.size() - off);
    auto scratch = c.alloc(cnt * per);
    std::vector<KsJob> sub(jobs.begin() + off, jobs.begin() + off + cnt);
    ks_group(c, sub, l, scratch->p);
  }
}

}  // namespace ckg
