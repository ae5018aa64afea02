// The HeOps evaluator on device-resident ciphertexts. Each method follows the CPU
// Evaluator method of the same name in crates/ckks-train-ckks/src/evaluator.rs (checks in
// the same order, the same errors, f64 scale labels and OpCounter increments) and
// computes bit-identical polynomials with the kernels of kernels.cu.
#include <cmath>
#include <cstring>

#include <type_traits>

#include "evaluator.hpp"

namespace ckg {

namespace {

const double kScaleTolerance = 1.0 / 1024.0;          // evaluator.rs:96
const uint64_t kLabelSearchUlps = 8;                   // evaluator.rs:100
const double kMaxScalarInt = 4611686018427387904.0;   // evaluator.rs:103 (2^62)
const double kMinPlainScale = 1048576.0;               // evaluator.rs:108 (2^20)

void check_level(uint32_t a, uint32_t b) {
  if (a != b) throw Error(ST_LEVEL_MISMATCH, "level mismatch");
}
void check_scale(double a, double b) {  // evaluator.rs:833-839
  if (!(std::fabs(a - b) < kScaleTolerance * std::min(a, b))) throw Error(ST_SCALE_MISMATCH, "scale mismatch");
}
void check_plain_scale(double sp) {  // evaluator.rs:111-119
  if (sp < kMinPlainScale)
    throw Error(ST_INVALID_PARAMS,
                "plaintext scale is below 2^20: the target scale is too small for this ciphertext's scale and level");
}
void check_ct_scale(double s) {  // ciphertext.rs:53-55
  if (!(std::isfinite(s) && s > 0.0)) throw Error(ST_INVALID_PARAMS, "ciphertext scale must be positive and finite");
}

}  // namespace

std::pair<uint32_t, uint32_t> bsgs_split(uint32_t d) {  // linalg.rs:419-424
  uint32_t log_d = __builtin_ctz(d);
  uint32_t baby = 1u << ((log_d + 1) / 2);
  return {baby, d / baby};
}

Evaluator::Evaluator(Context* ctx, KeyPtr relin, std::vector<KeyPtr> galois, EvalConfig cfg)
    : ctx_(ctx), relin_(std::move(relin)), galois_(std::move(galois)), cfg_(cfg) {}

OpCounter Evaluator::counter() const {
  std::lock_guard<std::mutex> lk(mu_);
  return counter_;
}
void Evaluator::reset_counter() { count([](OpCounter& c) { c = OpCounter(); }); }
void Evaluator::add_counts(const OpCounter& o) {
  count([&](OpCounter& c) {
    c.rotations += o.rotations;
    c.relins += o.relins;
    c.ct_ct_tensor += o.ct_ct_tensor;
    c.ct_pt_mults += o.ct_pt_mults;
    c.rescales += o.rescales;
    c.sse_switches += o.sse_switches;
    c.bootstraps += o.bootstraps;
  });
}
std::unique_ptr<Evaluator> Evaluator::fork() const {
  return std::make_unique<Evaluator>(ctx_, relin_, galois_, cfg_);
}
bool Evaluator::has_galois_key(int32_t step) const {
  uint64_t elt = galois_elt(ctx_->n, step);
  for (auto& k : galois_)
    if (k->elt == elt) return true;
  return false;
}

Ct Evaluator::new_ct(uint32_t ncomp, uint32_t level, double scale) {
  check_ct_scale(scale);
  auto c = std::make_shared<CtObj>();
  c->ctx = ctx_;
  c->ncomp = ncomp;
  c->level = level;
  c->scale = scale;
  c->comp_stride = (size_t)(level + 1) * ctx_->n;
  c->buf = ctx_->alloc(ncomp * c->comp_stride);
  return c;
}

Ct Evaluator::upload(const uint64_t* src, bool device_src, uint32_t ncomp, uint32_t level, double scale) {
  if (ncomp < 2) throw Error(ST_INVALID_PARAMS, "a ciphertext needs at least 2 components");
  if (level > ctx_->L) throw Error(ST_INVALID_PARAMS, "level above max_level");
  ctx_->activate();
  Ct c = new_ct(ncomp, level, scale);
  CKG_CUDA(cudaMemcpyAsync(c->buf->p, src, c->buf->words * 8,
                           device_src ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, ctx_->stream));
  return c;
}

Ct Evaluator::upload_overlapped(const uint64_t* host, uint32_t ncomp, uint32_t level, double scale) {
  if (ncomp < 2) throw Error(ST_INVALID_PARAMS, "a ciphertext needs at least 2 components");
  if (level > ctx_->L) throw Error(ST_INVALID_PARAMS, "level above max_level");
  if (!host) throw Error(ST_INVALID_PARAMS, "null host buffer");
  check_ct_scale(scale);
  auto c = std::make_shared<CtObj>();
  c->ctx = ctx_;
  c->ncomp = ncomp;
  c->level = level;
  c->scale = scale;
  c->comp_stride = (size_t)(level + 1) * ctx_->n;
  c->buf = ctx_->upload_overlapped(host, ncomp * c->comp_stride);
  return c;
}

Pt Evaluator::upload_pt_overlapped(const uint64_t* host, uint32_t level, double scale) {
  if (level > ctx_->L) throw Error(ST_INVALID_PARAMS, "level above max_level");
  if (!host) throw Error(ST_INVALID_PARAMS, "null host buffer");
  auto p = std::make_shared<PtObj>();
  p->ctx = ctx_;
  p->level = level;
  p->scale = scale;
  p->buf = ctx_->upload_overlapped(host, (size_t)(level + 1) * ctx_->n);
  return p;
}

std::vector<Ct> Evaluator::upload_overlapped_list(const std::vector<CtUpload>& items) {
  std::vector<Context::HostPart> parts;
  for (const CtUpload& u : items) {
    if (u.ncomp < 2) throw Error(ST_INVALID_PARAMS, "a ciphertext needs at least 2 components");
    if (u.level > ctx_->L) throw Error(ST_INVALID_PARAMS, "level above max_level");
    if (!u.host) throw Error(ST_INVALID_PARAMS, "null host buffer");
    check_ct_scale(u.scale);
    parts.push_back({u.host, (size_t)u.ncomp * (u.level + 1) * ctx_->n});
  }
  std::vector<size_t> off;
  DevBufPtr buf = ctx_->upload_overlapped_list(parts, off);
  std::vector<Ct> out;
  for (size_t i = 0; i < items.size(); ++i) {
    auto c = std::make_shared<CtObj>();
    c->ctx = ctx_;
    c->buf = buf;
    c->offset = off[i];
    c->ncomp = items[i].ncomp;
    c->level = items[i].level;
    c->scale = items[i].scale;
    c->comp_stride = (size_t)(items[i].level + 1) * ctx_->n;
    out.push_back(c);
  }
  return out;
}

std::vector<Pt> Evaluator::upload_pt_overlapped_list(const std::vector<CtUpload>& items) {
  std::vector<Context::HostPart> parts;
  for (const CtUpload& u : items) {
    if (u.level > ctx_->L) throw Error(ST_INVALID_PARAMS, "level above max_level");
    if (!u.host) throw Error(ST_INVALID_PARAMS, "null host buffer");
    parts.push_back({u.host, (size_t)(u.level + 1) * ctx_->n});
  }
  std::vector<size_t> off;
  DevBufPtr buf = ctx_->upload_overlapped_list(parts, off);
  std::vector<Pt> out;
  for (size_t i = 0; i < items.size(); ++i) {
    auto p = std::make_shared<PtObj>();
    p->ctx = ctx_;
    p->buf = buf;
    p->offset = off[i];
    p->level = items[i].level;
    p->scale = items[i].scale;
    out.push_back(p);
  }
  return out;
}

Pt Evaluator::upload_pt(const uint64_t* src, bool device_src, uint32_t level, double scale) {
  if (level > ctx_->L) throw Error(ST_INVALID_PARAMS, "level above max_level");
  ctx_->activate();
  auto p = std::make_shared<PtObj>();
  p->ctx = ctx_;
  p->level = level;
  p->scale = scale;
  p->buf = ctx_->alloc((size_t)(level + 1) * ctx_->n);
  CKG_CUDA(cudaMemcpyAsync(p->buf->p, src, p->buf->words * 8,
                           device_src ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, ctx_->stream));
  return p;
}

void Evaluator::check_basis(const Ct& a) const {
  if (!a || a->ctx != ctx_) throw Error(ST_INVALID_PARAMS, "operand is not over this evaluator's data basis");
}
void Evaluator::check_basis_pt(const Pt& p) const {
  if (!p || p->ctx != ctx_) throw Error(ST_INVALID_PARAMS, "operand is not over this evaluator's data basis");
}

// ---- element-wise ops ----------------------------------------------------------------

namespace {

void binary_comp(Context& c, int op, const uint64_t* a, const uint64_t* b, uint64_t* out, uint32_t limbs,
                 std::vector<BinRef>& refs) {
  for (uint32_t i = 0; i < limbs; ++i) refs.push_back(BinRef{a + i * c.n, b + i * c.n, out + i * c.n, i, 0});
  (void)op;
}

void unary_comp(Context& c, const uint64_t* a, uint64_t* out, uint32_t limbs, std::vector<LimbRef>& refs) {
  for (uint32_t i = 0; i < limbs; ++i) refs.push_back(LimbRef{a + i * c.n, out + i * c.n, i, 0});
}

}  // namespace

Ct Evaluator::add_sub(const Ct& a, const Ct& b, bool sub) {  // evaluator.rs:699-723
  check_basis(a);
  check_basis(b);
  check_level(a->level, b->level);
  check_scale(a->scale, b->scale);
  ctx_->activate();
  const uint32_t limbs = a->level + 1, nc = std::max(a->ncomp, b->ncomp), common = std::min(a->ncomp, b->ncomp);
  Ct r = new_ct(nc, a->level, a->scale);
  std::vector<BinRef> bin;
  for (uint32_t i = 0; i < common; ++i) binary_comp(*ctx_, 0, a->comp(i), b->comp(i), r->comp_mut(i), limbs, bin);
  launch_binary(ctx_->dt, bin.data(), (int)bin.size(), sub ? 1 : 0, ctx_->stream);
  std::vector<LimbRef> cp, ng;
  for (uint32_t i = common; i < a->ncomp; ++i) unary_comp(*ctx_, a->comp(i), r->comp_mut(i), limbs, cp);
  for (uint32_t i = common; i < b->ncomp; ++i) unary_comp(*ctx_, b->comp(i), r->comp_mut(i), limbs, sub ? ng : cp);
  if (!cp.empty()) launch_unary(ctx_->dt, cp.data(), (int)cp.size(), 2, nullptr, nullptr, ctx_->stream);
  if (!ng.empty()) launch_unary(ctx_->dt, ng.data(), (int)ng.size(), 0, nullptr, nullptr, ctx_->stream);
  return r;
}

Ct Evaluator::negate(const Ct& a) {  // evaluator.rs:242-247
  check_basis(a);
  ctx_->activate();
  Ct r = new_ct(a->ncomp, a->level, a->scale);
  std::vector<LimbRef> refs;
  for (uint32_t i = 0; i < a->ncomp; ++i) unary_comp(*ctx_, a->comp(i), r->comp_mut(i), a->level + 1, refs);
  launch_unary(ctx_->dt, refs.data(), (int)refs.size(), 0, nullptr, nullptr, ctx_->stream);
  return r;
}

Ct Evaluator::add_plain(const Ct& a, const Pt& p) {  // evaluator.rs:251-259
  check_basis(a);
  check_basis_pt(p);
  check_level(a->level, p->level);
  check_scale(a->scale, p->scale);
  ctx_->activate();
  const uint32_t limbs = a->level + 1;
  Ct r = new_ct(a->ncomp, a->level, a->scale);
  std::vector<BinRef> bin;
  binary_comp(*ctx_, 0, a->comp(0), p->data(), r->comp_mut(0), limbs, bin);
  launch_binary(ctx_->dt, bin.data(), (int)bin.size(), 0, ctx_->stream);
  std::vector<LimbRef> cp;
  for (uint32_t i = 1; i < a->ncomp; ++i) unary_comp(*ctx_, a->comp(i), r->comp_mut(i), limbs, cp);
  launch_unary(ctx_->dt, cp.data(), (int)cp.size(), 2, nullptr, nullptr, ctx_->stream);
  return r;
}

Ct Evaluator::mul_plain(const Ct& a, const Pt& p) {  // evaluator.rs:262-271
  check_basis(a);
  check_basis_pt(p);
  check_level(a->level, p->level);
  ctx_->activate();
  Ct r = new_ct(a->ncomp, a->level, a->scale * p->scale);
  std::vector<BinRef> bin;
  for (uint32_t i = 0; i < a->ncomp; ++i) binary_comp(*ctx_, 2, a->comp(i), p->data(), r->comp_mut(i), a->level + 1, bin);
  launch_binary(ctx_->dt, bin.data(), (int)bin.size(), 2, ctx_->stream);
  count([](OpCounter& c) { c.ct_pt_mults++; });
  return r;
}

double Evaluator::exact_product_scale(uint32_t level, double target) const {  // evaluator.rs:739-773
  if (level > ctx_->L) throw Error(ST_INVALID_PARAMS, "level exceeds max_level");
  if (!(std::isfinite(target) && target > 0.0))
    throw Error(ST_INVALID_PARAMS, "target scale must be positive and finite");
  if (level == 0) throw Error(ST_NO_LEVELS_LEFT, "no levels left");
  const double q = (double)ctx_->primes[level];
  const double l0 = target * q;
  if (!std::isfinite(l0)) throw Error(ST_INVALID_PARAMS, "target scale times q overflows");
  uint64_t bits;
  memcpy(&bits, &l0, 8);
  for (uint64_t k = 0; k <= kLabelSearchUlps; ++k)
    for (int s = 0; s < 2; ++s) {
      uint64_t b = s == 0 ? bits + k : bits - k;
      double l;
      memcpy(&l, &b, 8);
      if (l / q == target) return l;
    }
  throw Error(ST_SCALE_MISMATCH, "scale mismatch");
}

Ct Evaluator::mul_scalar(const Ct& a, double value, double target) {  // evaluator.rs:361-376, 777-799
  check_basis(a);
  if (!std::isfinite(value)) throw Error(ST_INVALID_PARAMS, "scalar must be finite");
  const double label = exact_product_scale(a->level, target);
  check_plain_scale(label / a->scale);
  const double k = std::round(value * (label / a->scale));
  if (std::fabs(k) >= kMaxScalarInt) throw Error(ST_INVALID_PARAMS, "scalar at this plaintext scale is >= 2^62");
  ctx_->activate();
  Ct r = new_ct(a->ncomp, a->level, label);
  const uint64_t kk = (uint64_t)std::fabs(k);
  ScalarTable st{};
  for (uint32_t i = 0; i <= a->level; ++i) {
    const HostMod& m = ctx_->mods[i];
    uint64_t w = kk % m.q;
    if (k < 0.0 && w) w = m.q - w;  // times |k| then negated, folded into one constant
    st.w[i] = w;
    st.ws[i] = m.shoup(w);
  }
  std::vector<LimbRef> refs;
  for (uint32_t i = 0; i < a->ncomp; ++i) unary_comp(*ctx_, a->comp(i), r->comp_mut(i), a->level + 1, refs);
  launch_scalar(ctx_->dt, refs.data(), (int)refs.size(), st, ctx_->stream);
  count([](OpCounter& c) { c.ct_pt_mults++; });
  return r;
}

Ct Evaluator::mul_plain_to_scale(const Ct& a, const Pt& p, double target) {  // evaluator.rs:393-414
  check_basis(a);
  check_basis_pt(p);
  check_level(a->level, p->level);
  const double label = exact_product_scale(a->level, target);
  check_plain_scale(label / a->scale);
  if (p->scale != label / a->scale) throw Error(ST_SCALE_MISMATCH, "scale mismatch");
  ctx_->activate();
  Ct r = new_ct(a->ncomp, a->level, label);
  std::vector<BinRef> bin;
  for (uint32_t i = 0; i < a->ncomp; ++i) binary_comp(*ctx_, 2, a->comp(i), p->data(), r->comp_mut(i), a->level + 1, bin);
  launch_binary(ctx_->dt, bin.data(), (int)bin.size(), 2, ctx_->stream);
  count([](OpCounter& c) { c.ct_pt_mults++; });
  return r;
}

void Evaluator::check_mul_operands(const Ct& a, const Ct& b) const {  // evaluator.rs:479-496
  check_basis(a);
  check_basis(b);
  if (a->ncomp != 2 || b->ncomp != 2)
    throw Error(ST_INVALID_PARAMS, "multiplication needs 2-component ciphertexts; relinearize first");
  check_level(a->level, b->level);
  if (a->level == 0) throw Error(ST_NO_LEVELS_LEFT, "no levels left");
}

Ct Evaluator::mul_no_relin(const Ct& a, const Ct& b) {  // evaluator.rs:422-439
  check_mul_operands(a, b);
  ctx_->activate();
  Ct r = new_ct(3, a->level, a->scale * b->scale);
  std::vector<TensorRef> refs;
  const size_t N = ctx_->n;
  for (uint32_t i = 0; i <= a->level; ++i)
    refs.push_back(TensorRef{a->comp(0) + i * N, a->comp(1) + i * N, b->comp(0) + i * N, b->comp(1) + i * N,
                             r->comp_mut(0) + i * N, r->comp_mut(1) + i * N, r->comp_mut(2) + i * N, i, 0});
  launch_tensor(ctx_->dt, refs.data(), (int)refs.size(), ctx_->stream);
  count([](OpCounter& c) { c.ct_ct_tensor++; });
  return r;
}

void Evaluator::check_key_basis(const DevKey& k) const {  // evaluator.rs:680-696
  if (k.ctx != ctx_ || k.parts != ctx_->dnum || k.q_limbs != ctx_->L + 1)
    throw Error(ST_INVALID_PARAMS, "key is not over this evaluator's bases");
}

const DevKey& Evaluator::relin_key_checked() const {  // evaluator.rs:470-477
  if (!relin_) throw Error(ST_INVALID_PARAMS, "evaluator has no relinearization key");
  check_key_basis(*relin_);
  return *relin_;
}

Ct Evaluator::relinearize(const Ct& a) {  // evaluator.rs:441-460
  check_basis(a);
  if (a->ncomp != 3) throw Error(ST_INVALID_PARAMS, "relinearize needs a 3-component ciphertext");
  const DevKey& rk = relin_key_checked();
  ctx_->activate();
  Ct r = new_ct(2, a->level, a->scale);
  KsJob j;
  j.in = a->comp(2);
  j.key = &rk;
  j.out_b = r->comp_mut(0);
  j.out_a = r->comp_mut(1);
  j.add_b = a->comp(0);
  j.add_a = a->comp(1);
  key_switch_many(*ctx_, {j}, a->level);
  count([](OpCounter& c) { c.relins++; });
  return r;
}

Ct Evaluator::mul(const Ct& a, const Ct& b) {  // evaluator.rs:463-467
  check_mul_operands(a, b);
  relin_key_checked();
  return relinearize(mul_no_relin(a, b));
}

Ct Evaluator::rescale(const Ct& a) {  // evaluator.rs:498-510
  check_basis(a);
  const uint32_t l = a->level;
  if (l == 0) throw Error(ST_NO_LEVELS_LEFT, "no levels left");
  ctx_->activate();
  Ct r = new_ct(a->ncomp, l - 1, a->scale / (double)ctx_->primes[l]);
  std::vector<const uint64_t*> in;
  std::vector<uint64_t*> out;
  for (uint32_t i = 0; i < a->ncomp; ++i) {
    in.push_back(a->comp(i));
    out.push_back(r->comp_mut(i));
  }
  rescale_many(*ctx_, in, l, out);
  count([](OpCounter& c) { c.rescales++; });
  return r;
}

Ct Evaluator::mod_switch_to_level(const Ct& a, uint32_t level) {  // evaluator.rs:513-525
  check_basis(a);
  if (level > a->level) throw Error(ST_INVALID_PARAMS, "cannot switch a ciphertext up to a higher level");
  auto r = std::make_shared<CtObj>(*a);  // a view: the first level+1 limbs of every component
  r->level = level;
  return r;
}

Ct Evaluator::relabel(const Ct& a, double scale) {  // ops.rs:475-477
  check_basis(a);
  check_ct_scale(scale);
  auto r = std::make_shared<CtObj>(*a);
  r->scale = scale;
  return r;
}

// ---- rotations -----------------------------------------------------------------------

void Evaluator::check_galois_input(const Ct& a) const {  // evaluator.rs:665-676
  check_basis(a);
  if (a->ncomp != 2) throw Error(ST_INVALID_PARAMS, "rotation needs a 2-component ciphertext; relinearize first");
}

std::optional<uint64_t> Evaluator::rotation_elt(int32_t steps) const {  // evaluator.rs:633-638
  const int64_t slots = (int64_t)ctx_->n / 2;
  const int64_t k = (((int64_t)steps % slots) + slots) % slots;
  if (k == 0) return std::nullopt;
  return galois_elt(ctx_->n, (int32_t)k);
}

const DevKey& Evaluator::galois_key(uint64_t elt) const {  // evaluator.rs:648-663
  const uint64_t two_n = 2 * ctx_->n;
  if (elt % 2 == 0 || elt >= two_n)
    throw Error(ST_INVALID_PARAMS, "Galois element " + std::to_string(elt) + " must be odd and < 2N");
  for (auto& k : galois_)
    if (k->elt == elt) {
      check_key_basis(*k);
      return *k;
    }
  throw Error(ST_INVALID_PARAMS, "missing galois key");
}

void Evaluator::check_rotation_keys(const std::vector<int32_t>& steps) const {  // evaluator.rs:621-629
  for (int32_t s : steps) {
    auto e = rotation_elt(s);
    if (e) galois_key(*e);
  }
}

Ct Evaluator::apply_galois(const Ct& a, uint64_t elt) {  // evaluator.rs:640-646, 800-805
  const DevKey& gk = galois_key(elt);
  ctx_->activate();
  const uint32_t* perm = ctx_->perm(elt);
  const uint32_t limbs = a->level + 1;
  Ct r = new_ct(2, a->level, a->scale);
  auto tmp = ctx_->alloc((size_t)limbs * ctx_->n);
  std::vector<LimbRef> refs;
  unary_comp(*ctx_, a->comp(1), tmp->p, limbs, refs);
  launch_unary(ctx_->dt, refs.data(), (int)refs.size(), 3, nullptr, perm, ctx_->stream);  // sigma_g(c1)
  KsJob j;
  j.in = tmp->p;
  j.key = &gk;
  j.out_b = r->comp_mut(0);
  j.out_a = r->comp_mut(1);
  j.add_b = a->comp(0);
  j.add_b_perm = perm;  // + sigma_g(c0)
  key_switch_many(*ctx_, {j}, a->level);
  count([](OpCounter& c) { c.rotations++; });
  return r;
}

std::vector<Ct> Evaluator::rotate_many(const std::vector<std::pair<Ct, int32_t>>& items) {
  // rotate() of each item (same checks, same counts), the key switches of one level as one
  // launch sequence
  for (auto& it : items) check_galois_input(it.first);
  std::vector<Ct> out(items.size());
  std::map<uint32_t, std::vector<size_t>> by_level;
  for (size_t i = 0; i < items.size(); ++i) {
    if (!rotation_elt(items[i].second)) {
      out[i] = items[i].first;
    } else {
      galois_key(*rotation_elt(items[i].second));  // the key exists (before any work)
      by_level[items[i].first->level].push_back(i);
    }
  }
  ctx_->activate();
  uint64_t rotations = 0;
  for (auto& kv : by_level) {
    const uint32_t l = kv.first, limbs = l + 1;
    auto tmp = ctx_->alloc(kv.second.size() * (size_t)limbs * ctx_->n);
    std::vector<KsJob> ks;
    for (size_t k = 0; k < kv.second.size(); ++k) {
      const Ct& a = items[kv.second[k]].first;
      const uint64_t elt = *rotation_elt(items[kv.second[k]].second);
      const uint32_t* perm = ctx_->perm(elt);
      uint64_t* t = tmp->p + k * (size_t)limbs * ctx_->n;
      std::vector<LimbRef> refs;
      unary_comp(*ctx_, a->comp(1), t, limbs, refs);
      launch_unary(ctx_->dt, refs.data(), (int)refs.size(), 3, nullptr, perm, ctx_->stream);  // sigma_g(c1)
      Ct r = new_ct(2, l, a->scale);
      KsJob j;
      j.in = t;
      j.key = &galois_key(elt);
      j.out_b = r->comp_mut(0);
      j.out_a = r->comp_mut(1);
      j.add_b = a->comp(0);
      j.add_b_perm = perm;  // + sigma_g(c0)
      ks.push_back(j);
      out[kv.second[k]] = r;
      rotations++;
    }
    key_switch_many(*ctx_, ks, l);
  }
  count([&](OpCounter& c) { c.rotations += rotations; });
  return out;
}

Ct Evaluator::rotate(const Ct& a, int32_t steps) {  // evaluator.rs:534-540
  check_galois_input(a);
  auto e = rotation_elt(steps);
  if (!e) return a;
  return apply_galois(a, *e);
}

Ct Evaluator::conjugate(const Ct& a) {  // evaluator.rs:547-550
  check_galois_input(a);
  return apply_galois(a, 2 * ctx_->n - 1);
}

std::vector<Ct> Evaluator::hoisted_rotate(const Ct& a, const std::vector<int32_t>& steps) {  // evaluator.rs:572-616
  check_galois_input(a);
  std::vector<Ct> out(steps.size());
  if (!cfg_.hoist) {
    check_rotation_keys(steps);
    for (size_t i = 0; i < steps.size(); ++i) out[i] = rotate(a, steps[i]);
    return out;
  }
  std::vector<std::pair<uint64_t, const DevKey*>> keys(steps.size(), {0, nullptr});
  bool any = false;
  for (size_t i = 0; i < steps.size(); ++i) {
    auto e = rotation_elt(steps[i]);
    if (e) {
      keys[i] = {*e, &galois_key(*e)};
      any = true;
    }
  }
  uint64_t nontrivial = 0;
  if (any) {
    ctx_->activate();
    const uint32_t l = a->level;
    auto conv = ctx_->alloc(conv_limbs(*ctx_, l) * ctx_->n);
    mod_up_many(*ctx_, {a->comp(1)}, l, {conv->p});
    std::vector<KsJob> jobs;
    std::vector<size_t> idx;
    for (size_t i = 0; i < steps.size(); ++i) {
      if (!keys[i].second) continue;
      const uint32_t* perm = ctx_->perm(keys[i].first);
      Ct r = new_ct(2, l, a->scale);
      KsJob j;
      j.in = a->comp(1);
      j.key = keys[i].second;
      j.out_b = r->comp_mut(0);
      j.out_a = r->comp_mut(1);
      j.add_b = a->comp(0);
      j.add_b_perm = perm;
      j.perm = perm;
      j.conv = conv->p;
      jobs.push_back(j);
      out[i] = r;
      nontrivial++;
    }
    key_switch_many(*ctx_, jobs, l);
  }
  for (size_t i = 0; i < steps.size(); ++i)
    if (!keys[i].second) out[i] = a;
  count([&](OpCounter& c) { c.rotations += nontrivial; });
  return out;
}

std::vector<std::vector<Ct>> Evaluator::hoisted_rotate_many(
    const std::vector<std::pair<Ct, std::vector<int32_t>>>& items) {
  // hoisted_rotate() of each item (same checks, results and counts); items at one level share
  // one decomposition launch sequence and one key-switch launch sequence
  bool same = cfg_.hoist && !items.empty();
  for (auto& it : items) same = same && it.first->level == items[0].first->level;
  if (!same) {
    std::vector<std::vector<Ct>> out;
    for (auto& it : items) out.push_back(hoisted_rotate(it.first, it.second));
    return out;
  }
  for (auto& it : items) check_galois_input(it.first);
  std::vector<std::vector<Ct>> out(items.size());
  std::vector<std::vector<std::pair<uint64_t, const DevKey*>>> keys(items.size());
  std::vector<size_t> with;  // items with a nontrivial step
  for (size_t t = 0; t < items.size(); ++t) {
    keys[t].assign(items[t].second.size(), {0, nullptr});
    bool any = false;
    for (size_t i = 0; i < items[t].second.size(); ++i) {
      auto e = rotation_elt(items[t].second[i]);
      if (e) {
        keys[t][i] = {*e, &galois_key(*e)};
        any = true;
      }
    }
    out[t].resize(items[t].second.size());
    if (any) with.push_back(t);
  }
  uint64_t nontrivial = 0;
  if (!with.empty()) {
    ctx_->activate();
    const uint32_t l = items[0].first->level;
    const size_t cl = conv_limbs(*ctx_, l) * ctx_->n;
    auto conv = ctx_->alloc(cl * with.size());
    std::vector<const uint64_t*> ins;
    std::vector<uint64_t*> convs;
    for (size_t k = 0; k < with.size(); ++k) {
      ins.push_back(items[with[k]].first->comp(1));
      convs.push_back(conv->p + k * cl);
    }
    mod_up_many(*ctx_, ins, l, convs);
    std::vector<KsJob> jobs;
    for (size_t k = 0; k < with.size(); ++k) {
      const size_t t = with[k];
      const Ct& a = items[t].first;
      for (size_t i = 0; i < items[t].second.size(); ++i) {
        if (!keys[t][i].second) continue;
        const uint32_t* perm = ctx_->perm(keys[t][i].first);
        Ct r = new_ct(2, l, a->scale);
        KsJob j;
        j.in = a->comp(1);
        j.key = keys[t][i].second;
        j.out_b = r->comp_mut(0);
        j.out_a = r->comp_mut(1);
        j.add_b = a->comp(0);
        j.add_b_perm = perm;
        j.perm = perm;
        j.conv = convs[k];
        jobs.push_back(j);
        out[t][i] = r;
        nontrivial++;
      }
    }
    key_switch_many(*ctx_, jobs, l);
  }
  for (size_t t = 0; t < items.size(); ++t)
    for (size_t i = 0; i < items[t].second.size(); ++i)
      if (!keys[t][i].second) out[t][i] = items[t].first;
  count([&](OpCounter& c) { c.rotations += nontrivial; });
  return out;
}

// ---- BSGS matrix-vector products (crates/ckks-train-ckks/src/linalg.rs:608-893) -------

namespace {

uint32_t entry_level(const Pt& p) { return p->level; }
uint32_t entry_level(const Ct& c) { return c->level; }
double entry_scale(const Pt& p) { return p->scale; }
double entry_scale(const Ct& c) { return c->scale; }

template <class T>
void check_diagonals(Context& c, uint32_t d, uint32_t stride, const std::vector<T>& entries) {
  // Diagonals::from_prerotated (linalg.rs:254-282): shape, stride, one level, one scale.
  if (d == 0 || (d & (d - 1)) || entries.size() != d)
    throw Error(ST_INVALID_PARAMS, "entries for d (d must be a power of two, one entry per diagonal)");
  if (stride == 0 || (c.n / 2) % ((uint64_t)d * stride) != 0)
    throw Error(ST_INVALID_PARAMS, "d * stride must divide the slot count (stride >= 1)");
  for (auto& e : entries)
    if (!e) throw Error(ST_INVALID_PARAMS, "null diagonal entry");
  for (auto& e : entries)
    if (entry_level(e) != entry_level(entries[0])) throw Error(ST_LEVEL_MISMATCH, "level mismatch");
  for (auto& e : entries)
    if (entry_scale(e) != entry_scale(entries[0])) throw Error(ST_SCALE_MISMATCH, "scale mismatch");
}

}  // namespace

std::vector<int32_t> rotation_steps(uint32_t d, uint32_t stride) {  // linalg.rs:433-457
  auto bg = bsgs_split(d);
  std::vector<int32_t> s;
  for (uint32_t k2 = 1; k2 < bg.first; ++k2) s.push_back((int32_t)(k2 * stride));
  for (uint32_t k1 = 1; k1 < bg.second; ++k1) s.push_back((int32_t)(bg.first * k1 * stride));
  return s;
}

template <class T, class MulF, class FinF>
Ct Evaluator::bsgs(uint32_t d, uint32_t stride, const std::vector<T>& entries, const Ct& x, MulF mul, FinF finish) {
  const auto bg = bsgs_split(d);
  const uint32_t baby = bg.first, giant = bg.second;
  const bool share_giant = cfg_.bsgs;
  std::vector<int32_t> steps;
  for (uint32_t k2 = 0; k2 < baby; ++k2) steps.push_back((int32_t)(k2 * stride));
  std::vector<Ct> xs = hoisted_rotate(x, steps);
  Ct acc;
  for (uint32_t k1 = 0; k1 < giant; ++k1) {
    const int64_t shift = (int64_t)baby * k1 * stride;
    Ct block;
    if (!share_giant && shift != 0) {
      for (uint32_t k2 = 0; k2 < baby; ++k2) {
        Ct t = finish(mul(entries[k1 * baby + k2], xs[k2]));
        t = rotate(t, (int32_t)shift);
        block = block ? add(block, t) : t;
      }
    } else {
      Ct inner;
      if constexpr (std::is_same<T, Pt>::value) {  // plaintext diagonals: one fused pass
        std::vector<std::pair<Ct, Pt>> prods;
        for (uint32_t k2 = 0; k2 < baby; ++k2) prods.push_back({xs[k2], entries[k1 * baby + k2]});
        inner = mac_plain(prods);
      } else if (cfg_.lazy_relin) {  // encrypted diagonals, products unrelinearized: one fused pass
        std::vector<std::pair<Ct, Ct>> prods;
        for (uint32_t k2 = 0; k2 < baby; ++k2) prods.push_back({entries[k1 * baby + k2], xs[k2]});
        inner = mac_tensor(prods);
      } else {
        for (uint32_t k2 = 0; k2 < baby; ++k2) {
          Ct t = mul(entries[k1 * baby + k2], xs[k2]);
          inner = inner ? add(inner, t) : t;
        }
      }
      block = finish(inner);
      if (shift != 0) block = rotate(block, (int32_t)shift);
    }
    acc = acc ? add(acc, block) : block;
  }
  return acc;
}

void Evaluator::check_matvec_plain(uint32_t d, uint32_t stride, const std::vector<Pt>& entries, const Ct& x) const {
  check_diagonals(*ctx_, d, stride, entries);
  check_galois_input(x);                       // linalg.rs:608-622
  for (auto& p : entries) check_basis_pt(p);
  for (auto& p : entries)
    if (p->level != x->level) throw Error(ST_LEVEL_MISMATCH, "level mismatch");
  check_rotation_keys(rotation_steps(d, stride));
}

void Evaluator::check_matvec_enc(uint32_t d, uint32_t stride, const std::vector<Ct>& entries, const Ct& x) const {
  check_diagonals(*ctx_, d, stride, entries);
  check_galois_input(x);                       // linalg.rs:642-678
  for (auto& c : entries) check_galois_input(c);
  for (auto& c : entries)
    if (c->level != x->level) throw Error(ST_LEVEL_MISMATCH, "level mismatch");
  check_rotation_keys(rotation_steps(d, stride));
  if (x->level == 0) throw Error(ST_NO_LEVELS_LEFT, "no levels left");
  relin_key_checked();
}

Ct Evaluator::matvec_plain(uint32_t d, uint32_t stride, const std::vector<Pt>& entries, const Ct& x) {
  check_matvec_plain(d, stride, entries, x);
  return bsgs(d, stride, entries, x, [&](const Pt& w, const Ct& xr) { return mul_plain(xr, w); },
              [](const Ct& c) { return c; });
}

Ct Evaluator::matvec_enc(uint32_t d, uint32_t stride, const std::vector<Ct>& entries, const Ct& x) {
  check_matvec_enc(d, stride, entries, x);
  if (cfg_.lazy_relin)
    return bsgs(d, stride, entries, x, [&](const Ct& w, const Ct& xr) { return mul_no_relin(w, xr); },
                [&](const Ct& c) { return relinearize(c); });
  return bsgs(d, stride, entries, x, [&](const Ct& w, const Ct& xr) { return mul(w, xr); },
              [](const Ct& c) { return c; });
}

Ct Evaluator::mac_tensor(const std::vector<std::pair<Ct, Ct>>& terms) {
  const Ct& a0 = terms[0].first;
  const uint32_t level = a0->level;
  ctx_->activate();
  Ct acc;
  for (size_t first = 0; first < terms.size(); first += kMaxMacTensorTerms) {
    const size_t cnt = std::min<size_t>(kMaxMacTensorTerms, terms.size() - first);
    Ct r = new_ct(3, level, a0->scale * terms[0].second->scale);
    MacTensorBatch b{};
    b.count = (int)cnt;
    b.limbs = (int)level + 1;
    b.out0 = r->comp_mut(0);
    b.out1 = r->comp_mut(1);
    b.out2 = r->comp_mut(2);
    for (size_t t = 0; t < cnt; ++t) {
      b.a0[t] = terms[first + t].first->comp(0);
      b.a1[t] = terms[first + t].first->comp(1);
      b.b0[t] = terms[first + t].second->comp(0);
      b.b1[t] = terms[first + t].second->comp(1);
    }
    launch_mac_tensor(ctx_->dt, b, ctx_->stream);
    acc = acc ? add(acc, r) : r;
  }
  count([&](OpCounter& c) { c.ct_ct_tensor += terms.size(); });
  return acc;
}

// The jobs' BSGS products stage by stage (the optimized configuration; operands checked): every
// stage issues one key-switch launch sequence per level for all jobs.
template <class T>
std::vector<Ct> Evaluator::bsgs_batch(const std::vector<MatvecJob<T>>& jobs) {
  constexpr bool kEnc = std::is_same<T, Ct>::value;
  Context& c = *ctx_;
  c.activate();
  const size_t nj = jobs.size(), N = c.n;
  uint64_t rotations = 0, relins = 0;
  std::map<uint32_t, std::vector<size_t>> by_level;
  for (size_t j = 0; j < nj; ++j) by_level[jobs[j].x->level].push_back(j);
  // 1. the hoisted baby rotations x -> rot(x, k2 stride), one ModUp per input (evaluator.rs:572-616)
  std::vector<std::vector<Ct>> xs(nj);
  for (auto& kv : by_level) {
    const uint32_t l = kv.first;
    const size_t per = conv_limbs(c, l) * N;
    constexpr size_t kGroup = 32;  // inputs per ModUp group (bounds the digit buffers)
    for (size_t g0 = 0; g0 < kv.second.size(); g0 += kGroup) {
      std::vector<size_t> need;
      std::vector<const uint64_t*> ins;
      for (size_t u = g0; u < std::min(kv.second.size(), g0 + kGroup); ++u) {
        const size_t j = kv.second[u];
        const uint32_t baby = bsgs_split(jobs[j].d).first;
        xs[j].assign(baby, jobs[j].x);
        bool any = false;
        for (uint32_t k2 = 1; k2 < baby; ++k2) any = any || rotation_elt((int32_t)(k2 * jobs[j].stride)).has_value();
        if (any) {
          need.push_back(j);
          ins.push_back(jobs[j].x->comp(1));
        }
      }
      if (need.empty()) continue;
      auto conv = c.alloc(need.size() * per);
      std::vector<uint64_t*> convs;
      for (size_t i = 0; i < need.size(); ++i) convs.push_back(conv->p + i * per);
      mod_up_many(c, ins, l, convs);
      std::vector<KsJob> ks;
      for (size_t i = 0; i < need.size(); ++i) {
        const MatvecJob<T>& jb = jobs[need[i]];
        const uint32_t baby = bsgs_split(jb.d).first;
        for (uint32_t k2 = 1; k2 < baby; ++k2) {
          auto e = rotation_elt((int32_t)(k2 * jb.stride));
          if (!e) continue;
          const uint32_t* perm = c.perm(*e);
          Ct r = new_ct(2, l, jb.x->scale);
          KsJob k;
          k.in = jb.x->comp(1);
          k.key = &galois_key(*e);
          k.out_b = r->comp_mut(0);
          k.out_a = r->comp_mut(1);
          k.add_b = jb.x->comp(0);
          k.add_b_perm = perm;
          k.perm = perm;
          k.conv = convs[i];
          ks.push_back(k);
          xs[need[i]][k2] = r;
          rotations++;
        }
      }
      key_switch_many(c, ks, l);
    }
  }
  // 2. the inner sums of every giant block (linalg.rs:659-670)
  struct Block {
    size_t job;
    int64_t shift;
    Ct v;
  };
  std::vector<Block> blocks;
  for (size_t j = 0; j < nj; ++j) {
    const auto bg = bsgs_split(jobs[j].d);
    for (uint32_t k1 = 0; k1 < bg.second; ++k1) {
      Ct inner;
      if constexpr (kEnc) {
        std::vector<std::pair<Ct, Ct>> prods;
        for (uint32_t k2 = 0; k2 < bg.first; ++k2) prods.push_back({jobs[j].entries[k1 * bg.first + k2], xs[j][k2]});
        inner = mac_tensor(prods);
      } else {
        std::vector<std::pair<Ct, Pt>> prods;
        for (uint32_t k2 = 0; k2 < bg.first; ++k2) prods.push_back({xs[j][k2], jobs[j].entries[k1 * bg.first + k2]});
        inner = mac_plain(prods);
      }
      blocks.push_back({j, (int64_t)bg.first * k1 * jobs[j].stride, inner});
    }
  }
  xs.clear();
  std::map<uint32_t, std::vector<size_t>> blocks_at;
  for (size_t b = 0; b < blocks.size(); ++b) blocks_at[blocks[b].v->level].push_back(b);
  // 3. relinearize every block (encrypted diagonals, lazy relinearization: evaluator.rs:441-460)
  if constexpr (kEnc) {
    const DevKey& rk = relin_key_checked();
    for (auto& kv : blocks_at) {
      std::vector<KsJob> ks;
      std::vector<Ct> inputs;  // held until the key switches that read them are queued
      for (size_t b : kv.second) {
        const Ct& v = blocks[b].v;
        Ct r = new_ct(2, v->level, v->scale);
        KsJob k;
        k.in = v->comp(2);
        k.key = &rk;
        k.out_b = r->comp_mut(0);
        k.out_a = r->comp_mut(1);
        k.add_b = v->comp(0);
        k.add_a = v->comp(1);
        ks.push_back(k);
        inputs.push_back(v);
        blocks[b].v = r;
        relins++;
      }
      key_switch_many(c, ks, kv.first);
    }
  }
  // 4. the giant rotations of the blocks (evaluator.rs:640-646, 800-805)
  for (auto& kv : blocks_at) {
    const uint32_t l = kv.first;
    std::vector<size_t> rot;
    for (size_t b : kv.second)
      if (blocks[b].shift != 0 && rotation_elt((int32_t)blocks[b].shift)) rot.push_back(b);
    if (rot.empty()) continue;
    const size_t limbs = l + 1;
    auto tmp = c.alloc(rot.size() * limbs * N);
    std::vector<KsJob> ks;
    std::vector<Ct> inputs;  // held until the key switches that read them are queued
    for (size_t i = 0; i < rot.size(); ++i) {
      Block& bl = blocks[rot[i]];
      const uint64_t elt = *rotation_elt((int32_t)bl.shift);
      const uint32_t* perm = c.perm(elt);
      uint64_t* t = tmp->p + i * limbs * N;
      std::vector<LimbRef> refs;
      for (uint32_t q = 0; q < limbs; ++q) refs.push_back(LimbRef{bl.v->comp(1) + q * N, t + q * N, q, 0});
      launch_unary(c.dt, refs.data(), (int)refs.size(), 3, nullptr, perm, c.stream);  // sigma_g(c1)
      Ct r = new_ct(2, l, bl.v->scale);
      KsJob k;
      k.in = t;
      k.key = &galois_key(elt);
      k.out_b = r->comp_mut(0);
      k.out_a = r->comp_mut(1);
      k.add_b = bl.v->comp(0);
      k.add_b_perm = perm;  // + sigma_g(c0)
      ks.push_back(k);
      inputs.push_back(bl.v);
      bl.v = r;
      rotations++;
    }
    key_switch_many(c, ks, l);
  }
  // 5. the sums over the giant blocks
  std::vector<Ct> out(nj);
  for (auto& bl : blocks) out[bl.job] = out[bl.job] ? add(out[bl.job], bl.v) : bl.v;
  count([&](OpCounter& k) {
    k.rotations += rotations;
    k.relins += relins;
  });
  return out;
}

std::vector<Ct> Evaluator::matvec_enc_batch(const std::vector<MatvecJob<Ct>>& jobs) {
  for (auto& j : jobs) check_matvec_enc(j.d, j.stride, j.entries, j.x);
  if (jobs.empty()) return {};
  if (!(cfg_.hoist && cfg_.bsgs && cfg_.lazy_relin)) {
    std::vector<Ct> out;
    for (auto& j : jobs) out.push_back(matvec_enc(j.d, j.stride, j.entries, j.x));
    return out;
  }
  return bsgs_batch(jobs);
}

std::vector<Ct> Evaluator::matvec_plain_batch(const std::vector<MatvecJob<Pt>>& jobs) {
  for (auto& j : jobs) check_matvec_plain(j.d, j.stride, j.entries, j.x);
  if (jobs.empty()) return {};
  if (!(cfg_.hoist && cfg_.bsgs)) {
    std::vector<Ct> out;
    for (auto& j : jobs) out.push_back(matvec_plain(j.d, j.stride, j.entries, j.x));
    return out;
  }
  return bsgs_batch(jobs);
}

}  // namespace ckg
