// Batched, uneven-level execution of evaluator ops (see batch.hpp).
#include <algorithm>
#include <cstring>

#include "batch.hpp"
#include "bounds_refs.hpp"

namespace ckg {

namespace {

// Upper bounds of one chunk: items (the default; Batch::set_chunk_items) and scratch bytes.
// Chunks run one after another on the context's stream and reuse one scratch region.
constexpr size_t kChunkItems = 128;
constexpr size_t kChunkScratchBytes = (size_t)16 << 30;

struct List {
  size_t off = 0;  // byte offset into the descriptor buffer
  int count = 0;
};

// Host-side builder of the descriptor buffer: typed arrays appended at 16-byte alignment.
struct DescBuilder {
  std::vector<unsigned char> bytes;
  template <class T>
  List put(const std::vector<T>& v) {
    List l;
    size_t off = (bytes.size() + 15) & ~(size_t)15;
    bytes.resize(off + v.size() * sizeof(T));
    if (!v.empty()) memcpy(bytes.data() + off, v.data(), v.size() * sizeof(T));
    l.off = off;
    l.count = (int)v.size();
    return l;
  }
};

inline uint32_t target_prime(const Context& c, uint32_t l, uint32_t j, uint32_t t) {
  const uint32_t s = c.digit_start(j), a = c.digit_end(j, l) - s;
  if (t < s) return t;
  if (t < l + 1 - a) return t + a;
  return c.p_prime(t - (l + 1 - a));
}

}  // namespace

struct Batch::Stage {
  List tensor, pmul, gather, intt_in, fwd_conv, ip, intt_p, md_conv, fwd_md, fin_ks, intt_last, rs_conv, fwd_rs,
      fin_rs;
  std::vector<std::pair<int, List>> modup;  // by number of source primes
  std::vector<int> modup_dst;               // the largest target count of each modup list
  int ip_max_limbs = 0, md_dst = 0, rs_dst = 0;
};

Batch::Batch(Evaluator* ev) : ev_(ev), ctx_(ev->ctx()), chunk_items_(kChunkItems) {}

Batch::~Batch() { reset(); }

void Batch::reset() {
  if (exec_) cudaGraphExecDestroy(exec_);
  if (graph_) cudaGraphDestroy(graph_);
  exec_ = nullptr;
  graph_ = nullptr;
  for (auto* s : chunks_) delete s;
  chunks_.clear();
  desc_.reset();
  scratch_.reset();
  built_ = false;
}

void Batch::set_chunk_items(size_t items) {
  if (items < 1 || items > 4096) throw Error(ST_INVALID_PARAMS, "chunk size must be in 1..=4096");
  if (items != chunk_items_) reset();
  chunk_items_ = items;
}

std::vector<Batch::Trial> Batch::autotune(int reps) {
  static const int kWaves[] = {0, 32, 64, 128, 256};
  static const int kChunks[] = {64, 128, 256};
  if (reps < 1 || reps > 100) throw Error(ST_INVALID_PARAMS, "reps must be in 1..=100");
  Context& c = *ctx_;
  c.activate();
  const int wave0 = c.dt.ntt_wave;
  std::vector<Trial> trials;
  cudaEvent_t e0, e1;
  CKG_CUDA(cudaEventCreate(&e0));
  CKG_CUDA(cudaEventCreate(&e1));
  try {
    for (int chunk : kChunks) {
      set_chunk_items((size_t)chunk);
      for (int wave : kWaves) {
        reset();
        c.dt.ntt_wave = wave;
        build();
        CKG_CUDA(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal));
        issue();
        cudaError_t err = cudaStreamEndCapture(c.stream, &graph_);
        if (err != cudaSuccess) throw_cuda(err, "cudaStreamEndCapture");
        CKG_CUDA(cudaGraphInstantiate(&exec_, graph_, 0));
        CKG_CUDA(cudaGraphLaunch(exec_, c.stream));
        CKG_CUDA(cudaEventRecord(e0, c.stream));
        for (int r = 0; r < reps; ++r) CKG_CUDA(cudaGraphLaunch(exec_, c.stream));
        CKG_CUDA(cudaEventRecord(e1, c.stream));
        CKG_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        CKG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        trials.push_back({wave, chunk, ms / reps});
      }
    }
  } catch (...) {
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    reset();
    c.dt.ntt_wave = wave0;
    throw;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  // The fastest trial, unless the default shape (whole-list transforms, kChunkItems per chunk) is
  // within 1% of it: differences that small are run-to-run noise, not a better shape.
  const Trial* best = &trials[0];
  for (const Trial& t : trials)
    if (t.ms < best->ms) best = &t;
  for (const Trial& t : trials)
    if (t.ntt_wave == 0 && t.chunk_items == (int)kChunkItems && t.ms <= best->ms * 1.01) best = &t;
  reset();
  c.dt.ntt_wave = best->ntt_wave;
  chunk_items_ = (size_t)best->chunk_items;
  return trials;
}

Ct Batch::mul_relin_rescale(const Ct& a, const Ct& b, Evaluator* ev) {  // evaluator.rs:463-510
  if (built_) throw Error(ST_INVALID_PARAMS, "batch already built: create a new batch to add ops");
  ev = ev ? ev : ev_;
  if (ev->ctx() != ctx_) throw Error(ST_INVALID_PARAMS, "evaluator is not over this batch's context");
  ev->check_mul_operands(a, b);
  const DevKey& rk = ev->relin_key_checked();
  const uint32_t l = a->level;
  const double s = a->scale * b->scale;
  Item it;
  it.kind = MUL;
  it.ev = ev;
  it.a = a;
  it.b = b;
  it.key = &rk;
  it.out = ev->new_ct(2, l - 1, s / (double)ctx_->primes[l]);
  items_.push_back(it);
  return it.out;
}

Ct Batch::rotate(const Ct& a, int32_t steps, Evaluator* ev) {  // evaluator.rs:534-540
  if (built_) throw Error(ST_INVALID_PARAMS, "batch already built: create a new batch to add ops");
  ev = ev ? ev : ev_;
  if (ev->ctx() != ctx_) throw Error(ST_INVALID_PARAMS, "evaluator is not over this batch's context");
  ev->check_galois_input(a);
  auto e = ev->rotation_elt(steps);
  Item it;
  it.kind = ROT;
  it.ev = ev;
  it.a = a;
  if (!e) {
    it.trivial = true;
    it.out = a;
  } else {
    it.elt = *e;
    it.key = &ev->galois_key(*e);
    it.out = ev->new_ct(2, a->level, a->scale);
  }
  items_.push_back(it);
  return it.out;
}

Ct Batch::mul_plain_rescale(const Ct& a, const Pt& p, Evaluator* ev) {  // evaluator.rs:262-271, 498-510
  if (built_) throw Error(ST_INVALID_PARAMS, "batch already built: create a new batch to add ops");
  ev = ev ? ev : ev_;
  if (ev->ctx() != ctx_) throw Error(ST_INVALID_PARAMS, "evaluator is not over this batch's context");
  ev->check_basis(a);
  ev->check_basis_pt(p);
  if (a->level != p->level) throw Error(ST_LEVEL_MISMATCH, "level mismatch");
  if (a->level == 0) throw Error(ST_NO_LEVELS_LEFT, "no levels left");
  const double s = a->scale * p->scale;
  Item it;
  it.kind = PMUL;
  it.ev = ev;
  it.a = a;
  it.p = p;
  it.out = ev->new_ct(a->ncomp, a->level - 1, s / (double)ctx_->primes[a->level]);
  items_.push_back(it);
  return it.out;
}

size_t Batch::scratch_words(const Context& c, int kind, uint32_t level, uint32_t ncomp) {
  const size_t l = level, k = c.k, ext = l + 1 + k;
  size_t w = 0;
  if (kind != PMUL) {
    w += (kind == MUL ? 3 : 1) * (l + 1);                       // tensor product / gathered c1
    w += (l + 1) + conv_limbs(c, l) + 2 * ext + 2 * (k + l + 1);  // key switch
    if (kind == MUL) w += 2 * (l + 1) + 2 * (1 + l);             // relinearized, rescale
  } else {
    w += ncomp * (l + 1) + ncomp * (1 + l);                      // product, rescale
  }
  return w * c.n;
}

uint64_t Batch::key_switches() const {
  uint64_t n = 0;
  for (auto& it : items_) n += (it.kind == MUL) || (it.kind == ROT && !it.trivial);
  return n;
}

void Batch::build() {
  Context& c = *ctx_;
  const size_t N = c.n, k = c.k;
  // Order: key-switching items sorted by key (so the inner product reads a key once for
  // all of its jobs), then the plaintext products.
  std::vector<size_t> order;
  for (size_t i = 0; i < items_.size(); ++i)
    if (!(items_[i].kind == ROT && items_[i].trivial)) order.push_back(i);
  std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) {
    const Item &a = items_[x], &b = items_[y];
    if ((a.kind == PMUL) != (b.kind == PMUL)) return b.kind == PMUL;
    return a.key < b.key;
  });
  auto item_words = [&](const Item& it) -> size_t { return scratch_words(c, it.kind, it.a->level, it.a->ncomp); };
  // chunks
  std::vector<std::vector<size_t>> chunks;
  size_t cur = 0;
  for (size_t idx : order) {
    const size_t w = item_words(items_[idx]);
    if (chunks.empty() || chunks.back().size() >= chunk_items_ || (cur + w) * 8 > kChunkScratchBytes) {
      chunks.emplace_back();
      cur = 0;
    }
    chunks.back().push_back(idx);
    cur += w;
  }
  size_t scratch_words = 0;
  for (auto& ch : chunks) {
    size_t s = 0;
    for (size_t idx : ch) s += item_words(items_[idx]);
    scratch_words = std::max(scratch_words, s);
  }
  scratch_ = c.alloc(scratch_words);
  DescBuilder db;
  std::vector<Stage> stages(chunks.size());
  for (size_t ci = 0; ci < chunks.size(); ++ci) {
    Stage& S = stages[ci];
    std::vector<TensorRef> tensor;
    std::vector<BinRef> pmul;
    std::vector<GatherRef> gather;
    std::vector<LimbRef> intt_in, fwd_conv, intt_p, fwd_md, intt_last, fwd_rs;
    std::vector<ConvJob> md_conv, rs_conv;
    std::vector<std::vector<ConvJob>> modup(kMaxSrc + 1);
    std::vector<IpJob> ip;
    std::vector<FinRef> fin_ks, fin_rs;
    uint64_t* sp = scratch_->p;
    auto carve = [&](size_t limbs) {
      uint64_t* p = sp;
      sp += limbs * N;
      return p;
    };
    // Rescale by the last prime: INTT of limb l, its centred lift to every other prime, NTT and
    // finish. With two-pass transforms (N >= 2^12) the column pass reads the lift straight from the
    // coefficient-form limb (LimbRef::aux = l + 1), so the lifted limbs are never written out.
    const bool fuse_lift = c.log_n >= 12;
    auto rescale_poly = [&](const uint64_t* poly, uint32_t l, uint64_t* out) {
      uint64_t* last = carve(1 + l);
      uint64_t* T = last + N;
      intt_last.push_back(LimbRef{poly + (size_t)l * N, last, l, 0});
      if (!fuse_lift) rs_conv.push_back(ConvJob{last, T, c.d_conv + c.rescale_off[l], N, N, (int)l, 0});
      for (uint32_t i = 0; i < l; ++i) {
        fwd_rs.push_back(fuse_lift ? LimbRef{last, T + i * N, i, l + 1} : LimbRef{T + i * N, T + i * N, i, 0});
        fin_rs.push_back(FinRef{poly + i * N, T + i * N, nullptr, nullptr, out + i * N, c.qlinv[l][i].first,
                                c.qlinv[l][i].second, i, 0});
      }
    };
    for (size_t idx : chunks[ci]) {
      Item& it = items_[idx];
      const uint32_t l = it.a->level;
      const size_t ext = l + 1 + k;
      if (it.kind == PMUL) {
        uint64_t* prod = carve(it.a->ncomp * (l + 1));
        for (uint32_t cc = 0; cc < it.a->ncomp; ++cc)
          for (uint32_t i = 0; i <= l; ++i)
            pmul.push_back(BinRef{it.a->comp(cc) + i * N, it.p->data() + i * N, prod + (cc * (l + 1) + i) * N, i, 0});
        for (uint32_t cc = 0; cc < it.a->ncomp; ++cc)
          rescale_poly(prod + cc * (l + 1) * N, l, it.out->comp_mut(cc));
        continue;
      }
      const uint64_t* ks_in;
      const uint64_t *add_b, *add_a = nullptr;
      const uint32_t* add_perm = nullptr;
      uint64_t *out_b, *out_a;
      uint64_t* relin = nullptr;
      if (it.kind == MUL) {
        uint64_t* d = carve(3 * (l + 1));
        for (uint32_t i = 0; i <= l; ++i)
          tensor.push_back(TensorRef{it.a->comp(0) + i * N, it.a->comp(1) + i * N, it.b->comp(0) + i * N,
                                     it.b->comp(1) + i * N, d + i * N, d + (l + 1 + i) * N, d + (2 * (l + 1) + i) * N,
                                     i, 0});
        ks_in = d + 2 * (l + 1) * N;
        add_b = d;
        add_a = d + (l + 1) * N;
        relin = carve(2 * (l + 1));
        out_b = relin;
        out_a = relin + (l + 1) * N;
      } else {
        uint64_t* g = carve(l + 1);
        add_perm = c.perm(it.elt);
        for (uint32_t i = 0; i <= l; ++i) gather.push_back(GatherRef{it.a->comp(1) + i * N, g + i * N, add_perm});
        ks_in = g;
        add_b = it.a->comp(0);
        out_b = it.out->comp_mut(0);
        out_a = it.out->comp_mut(1);
      }
      uint64_t* coeff = carve(l + 1);
      uint64_t* conv = carve(conv_limbs(c, l));
      uint64_t* acc = carve(2 * ext);
      uint64_t* md = carve(2 * (k + l + 1));
      for (uint32_t i = 0; i <= l; ++i) intt_in.push_back(LimbRef{ks_in + i * N, coeff + i * N, i, 0});
      IpJob jb{};
      jb.level = (int)l;
      jb.ndig = (int)c.digits_at(l);
      jb.key_q = (int)it.key->q_limbs;
      jb.in = ks_in;
      jb.key = it.key->buf->p;
      jb.out_b = acc;
      jb.out_a = acc + ext * N;
      jb.perm = nullptr;
      for (uint32_t j = 0; j < c.digits_at(l); ++j) {
        const uint32_t s = c.digit_start(j), a = c.digit_end(j, l) - s, T = l + 1 - a + (uint32_t)k;
        uint64_t* base = conv + conv_offset_limbs(c, l, j) * N;
        jb.conv[j] = base;
        modup[a].push_back(
            ConvJob{coeff + s * N, base, c.d_conv + c.modup_off[(size_t)l * c.dnum + j], N, N, (int)T, 0});
        for (uint32_t t = 0; t < T; ++t) fwd_conv.push_back(LimbRef{base + t * N, base + t * N, target_prime(c, l, j, t), 0});
      }
      ip.push_back(jb);
      S.ip_max_limbs = std::max(S.ip_max_limbs, (int)ext);
      const size_t per = k + l + 1;
      for (int ba = 0; ba < 2; ++ba) {
        const uint64_t* x = acc + ba * ext * N;
        uint64_t* pc = md + ba * per * N;
        uint64_t* T = pc + k * N;
        for (uint32_t t = 0; t < k; ++t) intt_p.push_back(LimbRef{x + (l + 1 + t) * N, pc + t * N, c.p_prime(t), 0});
        md_conv.push_back(ConvJob{pc, T, c.d_conv + c.moddown_off[l], N, N, (int)(l + 1), 0});
        const uint64_t* add = ba == 0 ? add_b : add_a;
        const uint32_t* aperm = ba == 0 ? add_perm : nullptr;
        uint64_t* out = ba == 0 ? out_b : out_a;
        for (uint32_t i = 0; i <= l; ++i) {
          fwd_md.push_back(LimbRef{T + i * N, T + i * N, i, 0});
          fin_ks.push_back(FinRef{x + i * N, T + i * N, add ? add + i * N : nullptr, aperm, out + i * N,
                                  c.pinv[i].first, c.pinv[i].second, i, 0});
        }
      }
      if (it.kind == MUL)
        for (int cc = 0; cc < 2; ++cc) rescale_poly(relin + cc * (l + 1) * N, l, it.out->comp_mut(cc));
    }
    if (bounds::enabled()) {  // every entry's buffers, before the lists reach the device
      bounds::refs(tensor.data(), tensor.size(), N, "batch tensor product");
      bounds::refs(pmul.data(), pmul.size(), N, "batch plaintext product");
      bounds::refs(gather.data(), gather.size(), N, "batch Galois gather");
      for (auto* v : {&intt_in, &fwd_conv, &intt_p, &fwd_md, &intt_last, &fwd_rs})
        bounds::refs(v->data(), v->size(), N, "batch NTT limb");
      for (int ns = 1; ns <= kMaxSrc; ++ns) bounds::refs(modup[ns].data(), modup[ns].size(), ns, N, "batch ModUp");
      bounds::refs(md_conv.data(), md_conv.size(), (int)k, N, "batch ModDown");
      bounds::refs(rs_conv.data(), rs_conv.size(), 1, N, "batch rescale lift");
      bounds::refs(ip.data(), ip.size(), (int)c.alpha, (int)k, N, "batch inner product");
      bounds::refs(fin_ks.data(), fin_ks.size(), N, "batch key-switch finish");
      bounds::refs(fin_rs.data(), fin_rs.size(), N, "batch rescale finish");
    }
    S.tensor = db.put(tensor);
    S.pmul = db.put(pmul);
    S.gather = db.put(gather);
    S.intt_in = db.put(intt_in);
    for (int ns = 1; ns <= kMaxSrc; ++ns)
      if (!modup[ns].empty()) {
        S.modup.push_back({ns, db.put(modup[ns])});
        int mx = 0;
        for (const ConvJob& j : modup[ns]) mx = std::max(mx, j.n_dst);
        S.modup_dst.push_back(mx);
      }
    for (const ConvJob& j : md_conv) S.md_dst = std::max(S.md_dst, j.n_dst);
    for (const ConvJob& j : rs_conv) S.rs_dst = std::max(S.rs_dst, j.n_dst);
    S.fwd_conv = db.put(fwd_conv);
    S.ip = db.put(ip);
    S.intt_p = db.put(intt_p);
    S.md_conv = db.put(md_conv);
    S.fwd_md = db.put(fwd_md);
    S.fin_ks = db.put(fin_ks);
    S.intt_last = db.put(intt_last);
    S.rs_conv = db.put(rs_conv);
    S.fwd_rs = db.put(fwd_rs);
    S.fin_rs = db.put(fin_rs);
  }
  // Through the context's pinned staging ring: the host does not wait for work already on
  // the stream, and `db` may go away at once.
  desc_ = c.alloc((db.bytes.size() + 7) / 8);
  c.upload_staged(desc_->p, db.bytes.data(), db.bytes.size());
  for (auto& s : stages) chunks_.push_back(new Stage(s));
  built_ = true;
}

void Batch::issue() {
  Context& c = *ctx_;
  const unsigned char* base = (const unsigned char*)desc_->p;
  auto at = [&](const List& l) { return base + l.off; };
  // every limb a column pass reads is in the scratch, carved in whole limbs
  const LimbRegion reg{scratch_->p, scratch_->words / c.n};
  const LimbRegion* rg = scratch_->p ? &reg : nullptr;
  for (Stage* S : chunks_) {
    launch_tensor_ptr(c.dt, (const TensorRef*)at(S->tensor), S->tensor.count, c.stream);
    launch_binary_ptr(c.dt, (const BinRef*)at(S->pmul), S->pmul.count, 2, c.stream);
    launch_gather_ptr(c.dt, (const GatherRef*)at(S->gather), S->gather.count, c.stream);
    if (S->intt_in.count) launch_ntt_ptr(c.dt, (const LimbRef*)at(S->intt_in), S->intt_in.count, true, c.stream, rg);
    for (size_t g = 0; g < S->modup.size(); ++g)
      launch_bconv_ptr(c.dt, (const ConvJob*)at(S->modup[g].second), S->modup[g].second.count, S->modup[g].first,
                       c.stream, S->modup_dst[g]);
    if (S->fwd_conv.count) launch_ntt_ptr(c.dt, (const LimbRef*)at(S->fwd_conv), S->fwd_conv.count, false, c.stream, rg);
    launch_inner_product_ptr(c.dt, (int)c.alpha, (int)c.L, (int)c.k, (const IpJob*)at(S->ip), S->ip.count,
                             S->ip_max_limbs, c.stream);
    if (S->intt_p.count) launch_ntt_ptr(c.dt, (const LimbRef*)at(S->intt_p), S->intt_p.count, true, c.stream, rg);
    launch_bconv_ptr(c.dt, (const ConvJob*)at(S->md_conv), S->md_conv.count, (int)c.k, c.stream, S->md_dst);
    launch_ntt_finish_ptr(c.dt, (const LimbRef*)at(S->fwd_md), (const FinRef*)at(S->fin_ks), S->fin_ks.count,
                          c.stream, rg);
    if (S->intt_last.count)
      launch_ntt_ptr(c.dt, (const LimbRef*)at(S->intt_last), S->intt_last.count, true, c.stream, rg);
    launch_bconv_ptr(c.dt, (const ConvJob*)at(S->rs_conv), S->rs_conv.count, 1, c.stream, S->rs_dst);
    launch_ntt_finish_ptr(c.dt, (const LimbRef*)at(S->fwd_rs), (const FinRef*)at(S->fin_rs), S->fin_rs.count,
                          c.stream, rg);
  }
}

void Batch::count_ops() {
  for (auto& it : items_) {
    OpCounter d;
    if (it.kind == MUL) {
      d.ct_ct_tensor++;
      d.relins++;
      d.rescales++;
    } else if (it.kind == ROT) {
      d.rotations += it.trivial ? 0 : 1;
    } else {
      d.ct_pt_mults++;
      d.rescales++;
    }
    it.ev->add_counts(d);
  }
}

void Batch::run() {
  ctx_->activate();
  if (!built_) build();
  issue();
  CKG_CUDA(cudaGetLastError());
  count_ops();
}

void Batch::capture_graph() {
  ctx_->activate();
  if (!built_) build();
  if (exec_) return;
  CKG_CUDA(cudaStreamBeginCapture(ctx_->stream, cudaStreamCaptureModeThreadLocal));
  issue();
  cudaError_t e = cudaStreamEndCapture(ctx_->stream, &graph_);
  if (e != cudaSuccess) throw_cuda(e, "cudaStreamEndCapture");
  CKG_CUDA(cudaGraphInstantiate(&exec_, graph_, 0));
}

void Batch::launch_graph() {
  if (!exec_) capture_graph();
  ctx_->activate();
  CKG_CUDA(cudaGraphLaunch(exec_, ctx_->stream));
  count_ops();
}

}  // namespace ckg
