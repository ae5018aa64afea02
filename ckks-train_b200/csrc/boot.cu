// Bootstrapping on the device (boot.hpp): the evaluator's bootstrap arithmetic, ModRaise
// with SSE, the sparse BSGS sum, CoeffToSlot / SlotToCoeff, the level-optimal Chebyshev
// evaluation, EvalMod and the pipeline.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <optional>
#include <thread>

#include "boot.hpp"

namespace ckg {

namespace {

constexpr double kMinPlainScale = 1048576.0;                            // evaluator.rs:108 (2^20)
constexpr double kMaxConst = 85070591730234615865843651857942052864.0;  // poly.rs:66-67 (2^126)
constexpr double kRelabelTol = 1e-12;                                   // poly.rs:69-71

__int128 rounded_constant(double v) {  // poly.rs:345-353
  const double r = std::round(v);
  if (!(std::isfinite(r) && std::fabs(r) < kMaxConst))
    throw Error(ST_INVALID_PARAMS, "integer constant out of range (|k| < 2^126)");
  return (__int128)r;
}

uint64_t residue(__int128 k, uint64_t q) {  // poly.rs:339-342
  __int128 r = k % (__int128)q;
  if (r < 0) r += q;
  return (uint64_t)r;
}

void check_stride(const Context& c, uint32_t d, uint32_t stride) {  // linalg.rs:523-531
  const uint64_t slots = c.n / 2;
  if (!stride || !d || slots % ((uint64_t)d * stride) != 0)
    throw Error(ST_INVALID_PARAMS, "d * stride must divide the slot count (stride >= 1)");
}

size_t ceil_log2(size_t m) {  // poly.rs:333-336
  size_t p = 1, t = 0;
  while (p < m) {
    p <<= 1;
    ++t;
  }
  return t;
}

}  // namespace

std::vector<int32_t> bsgs_rotation_steps_with_offset(uint32_t d, uint32_t stride, int64_t offset) {
  auto bg = bsgs_split(d);  // linalg.rs:465-497
  std::vector<int32_t> s;
  for (int64_t k2 = 1; k2 < (int64_t)bg.first; ++k2) s.push_back((int32_t)(k2 * stride));
  for (int64_t k1 = 0; k1 < (int64_t)bg.second; ++k1) {
    const int64_t g = (offset + (int64_t)bg.first * k1) * (int64_t)stride;
    if (g != 0) s.push_back((int32_t)g);
  }
  return s;
}

std::vector<int32_t> LinearTransform::rotation_steps() const {  // linear.rs:499-508
  auto s = bsgs_rotation_steps_with_offset(diags.d, diags.stride, diags.offset);
  if (has_second) {
    auto b = bsgs_rotation_steps_with_offset(second.d, second.stride, second.offset);
    s.insert(s.end(), b.begin(), b.end());
  }
  return s;
}

uint32_t BootParams::evalmod_depth() const { return (uint32_t)ceil_log2((size_t)cheb_degree + 1) + double_angle; }

// ---- evaluator ops --------------------------------------------------------------------

void Evaluator::check_boot_input(const Ct& a) const {  // poly.rs:467-471
  check_galois_input(a);
  relin_key_checked();
}

void Evaluator::check_conjugation_key() const {  // evaluator.rs:627-630
  galois_key(2 * ctx_->n - 1);
}

Ct Evaluator::boot_mul_const(const Ct& a, double value, double product_scale) {  // poly.rs:380-400
  check_basis(a);
  const double ratio = product_scale / a->scale;
  if (std::isnan(ratio) || ratio < kMinPlainScale) throw Error(ST_INVALID_PARAMS, "constant scale below 2^20");
  const __int128 k = rounded_constant(value * ratio);
  ctx_->activate();
  Ct r = new_ct(a->ncomp, a->level, product_scale);
  ScalarTable st{};
  for (uint32_t i = 0; i <= a->level; ++i) {
    st.w[i] = residue(k, ctx_->mods[i].q);
    st.ws[i] = ctx_->mods[i].shoup(st.w[i]);
  }
  std::vector<LimbRef> refs;
  for (uint32_t c = 0; c < a->ncomp; ++c)
    for (uint32_t i = 0; i <= a->level; ++i)
      refs.push_back(LimbRef{a->comp(c) + i * ctx_->n, r->comp_mut(c) + i * ctx_->n, i, 0});
  launch_scalar(ctx_->dt, refs.data(), (int)refs.size(), st, ctx_->stream, 0);
  count([](OpCounter& c) { c.ct_pt_mults++; });
  return r;
}

Ct Evaluator::boot_add_const(const Ct& a, double value) {  // poly.rs:404-421
  check_basis(a);
  const __int128 k = rounded_constant(value * a->scale);
  ctx_->activate();
  Ct r = new_ct(a->ncomp, a->level, a->scale);
  ScalarTable st{};
  for (uint32_t i = 0; i <= a->level; ++i) st.w[i] = residue(k, ctx_->mods[i].q);
  std::vector<LimbRef> add, cp;
  for (uint32_t c = 0; c < a->ncomp; ++c)
    for (uint32_t i = 0; i <= a->level; ++i)
      (c == 0 ? add : cp).push_back(LimbRef{a->comp(c) + i * ctx_->n, r->comp_mut(c) + i * ctx_->n, i, 0});
  launch_scalar(ctx_->dt, add.data(), (int)add.size(), st, ctx_->stream, 1);
  launch_unary(ctx_->dt, cp.data(), (int)cp.size(), 2, nullptr, nullptr, ctx_->stream);
  return r;
}

Ct Evaluator::boot_zero(uint32_t level, double scale) {  // poly.rs:436-440
  if (level > ctx_->L) throw Error(ST_INVALID_PARAMS, "level above max_level");
  ctx_->activate();
  Ct r = new_ct(2, level, scale);
  CKG_CUDA(cudaMemsetAsync(r->buf->p, 0, r->buf->words * 8, ctx_->stream));
  return r;
}

Ct Evaluator::mul_by_x_half(const Ct& a) {  // linear.rs:921-936
  check_basis(a);
  ctx_->activate();
  const uint64_t* mono = ctx_->x_half();
  Ct r = new_ct(a->ncomp, a->level, a->scale);
  std::vector<BinRef> bin;
  for (uint32_t c = 0; c < a->ncomp; ++c)
    for (uint32_t i = 0; i <= a->level; ++i)
      bin.push_back(BinRef{a->comp(c) + i * ctx_->n, mono + i * ctx_->n, r->comp_mut(c) + i * ctx_->n, i, 0});
  launch_binary(ctx_->dt, bin.data(), (int)bin.size(), 2, ctx_->stream);
  return r;
}

// Both components raised from level 0 to the top level by the centered lift; limb 0 is
// kept as it is (poly.rs:298-345).
Ct Evaluator::raise_level0(const Ct& a) {
  const uint32_t top = ctx_->L;
  const size_t N = ctx_->n;
  Ct r = new_ct(a->ncomp, top, a->scale);
  auto tmp = ctx_->alloc(a->ncomp * N);
  std::vector<LimbRef> copy, intt, lift, fwd;
  for (uint32_t c = 0; c < a->ncomp; ++c) {
    copy.push_back(LimbRef{a->comp(c), r->comp_mut(c), 0, 0});
    intt.push_back(LimbRef{a->comp(c), tmp->p + c * N, 0, 0});
    for (uint32_t i = 1; i <= top; ++i) {
      lift.push_back(LimbRef{tmp->p + c * N, r->comp_mut(c) + i * N, i, 0});
      fwd.push_back(LimbRef{r->comp_mut(c) + i * N, r->comp_mut(c) + i * N, i, 0});
    }
  }
  launch_unary(ctx_->dt, copy.data(), (int)copy.size(), 2, nullptr, nullptr, ctx_->stream);
  ntt_limbs(*ctx_, intt, true);
  if (!lift.empty()) {
    launch_lift_level0(ctx_->dt, lift.data(), (int)lift.size(), ctx_->stream);
    ntt_limbs(*ctx_, fwd, false);
  }
  return r;
}

namespace {

void check_mod_raise_input(const Evaluator& ev, const Ct& a) {  // modraise.rs:94-107
  if (!ev.owns(a)) throw Error(ST_INVALID_PARAMS, "operand is not over this evaluator's data basis");
  if (a->ncomp != 2) throw Error(ST_INVALID_PARAMS, "mod_raise needs a 2-component ciphertext; relinearize first");
  if (a->level != 0) throw Error(ST_LEVEL_MISMATCH, "level mismatch");
}

void check_sse_key(const Context* c, const DevKey& k, uint32_t parts, uint32_t level) {  // modraise.rs:109-129
  if (k.ctx != c || k.parts != parts || k.q_limbs != level + 1 || k.elt != 0)
    throw Error(ST_INVALID_PARAMS, "SSE keys are not for this evaluator's parameters");
}

}  // namespace

Ct Evaluator::mod_raise(const Ct& a, const DevKey& to_sparse, const DevKey& to_dense) {  // modraise.rs:53-73
  check_mod_raise_input(*this, a);
  check_sse_key(ctx_, to_sparse, 1, 0);
  check_sse_key(ctx_, to_dense, ctx_->dnum, ctx_->L);
  ctx_->activate();
  Ct s = new_ct(2, 0, a->scale);  // (c0 + kb, ka) with (kb, ka) the switch of c1 to s' at level 0
  KsJob j0;
  j0.in = a->comp(1);
  j0.key = &to_sparse;
  j0.out_b = s->comp_mut(0);
  j0.out_a = s->comp_mut(1);
  j0.add_b = a->comp(0);
  key_switch_many(*ctx_, {j0}, 0);
  Ct raised = raise_level0(s);
  Ct r = new_ct(2, ctx_->L, a->scale);  // back to s at the top level
  KsJob j1;
  j1.in = raised->comp(1);
  j1.key = &to_dense;
  j1.out_b = r->comp_mut(0);
  j1.out_a = r->comp_mut(1);
  j1.add_b = raised->comp(0);
  key_switch_many(*ctx_, {j1}, ctx_->L);
  count([](OpCounter& c) { c.sse_switches += 2; });
  return r;
}

Ct Evaluator::mod_raise_main_key(const Ct& a) {  // modraise.rs:82-85
  check_mod_raise_input(*this, a);
  ctx_->activate();
  return raise_level0(a);
}

// ---- sparse BSGS sum: linalg.rs:741-893 --------------------------------------------------

Ct Evaluator::matvec_plain_sum_sparse(const std::vector<std::pair<const SparseDiag*, Ct>>& terms) {
  if (terms.empty()) throw Error(ST_INVALID_PARAMS, "matvec_plain_sum_sparse needs at least one term");
  const SparseDiag& d0 = *terms[0].first;
  const Ct& x0 = terms[0].second;
  const Pt* sp = d0.first();
  for (auto& t : terms) {
    const SparseDiag& diag = *t.first;
    const Ct& x = t.second;
    check_galois_input(x);
    if (diag.d != d0.d || diag.stride != d0.stride || diag.offset != d0.offset)
      throw Error(ST_INVALID_PARAMS, "matvec_plain_sum_sparse terms must share d, stride and offset");
    if (diag.nonzero() == 0) throw Error(ST_INVALID_PARAMS, "a term of matvec_plain_sum_sparse has no nonzero diagonal");
    for (auto& p : diag.entries) {
      if (!p) continue;
      check_basis_pt(p);
      if (p->level != x->level) throw Error(ST_LEVEL_MISMATCH, "level mismatch");
      if (!sp || p->scale != (*sp)->scale) throw Error(ST_SCALE_MISMATCH, "scale mismatch");
    }
    if (x->level != x0->level) throw Error(ST_LEVEL_MISMATCH, "level mismatch");
    if (x->scale != x0->scale) throw Error(ST_SCALE_MISMATCH, "scale mismatch");
    check_stride(*ctx_, diag.d, diag.stride);
    check_rotation_keys(bsgs_rotation_steps_with_offset(diag.d, diag.stride, diag.offset));
  }
  const uint32_t baby = d0.baby, giant = d0.giant, stride = d0.stride;
  const int64_t offset = d0.offset;
  std::vector<std::vector<Ct>> xs;  // xs[t][k2] = rot(x_t, k2 stride) for the baby steps in use
  std::vector<std::vector<uint32_t>> used(terms.size());
  std::vector<std::pair<Ct, std::vector<int32_t>>> hoists;
  for (size_t ti = 0; ti < terms.size(); ++ti) {
    for (uint32_t k2 = 0; k2 < baby; ++k2) {
      bool any = false;
      for (uint32_t k1 = 0; k1 < giant; ++k1) any = any || terms[ti].first->entries[k1 * baby + k2] != nullptr;
      if (any) used[ti].push_back(k2);
    }
    std::vector<int32_t> steps;
    for (uint32_t k2 : used[ti]) steps.push_back((int32_t)(k2 * stride));
    hoists.push_back({terms[ti].second, steps});
  }
  auto rotated = hoisted_rotate_many(hoists);  // every term's baby steps in one launch sequence
  for (size_t ti = 0; ti < terms.size(); ++ti) {
    std::vector<Ct> row(baby);
    for (size_t i = 0; i < used[ti].size(); ++i) row[used[ti][i]] = rotated[ti][i];
    xs.push_back(std::move(row));
  }
  Ct acc;
  // With shared giant steps the giant blocks are independent until their sum: their inner sums
  // first, then every block's giant rotation in one launch sequence (rotate_many), then the sum in
  // block order.
  if (cfg_.bsgs) {
    std::vector<std::pair<Ct, int32_t>> blocks;
    for (uint32_t k1 = 0; k1 < giant; ++k1) {
      const int64_t shift = (offset + (int64_t)baby * k1) * (int64_t)stride;
      std::vector<std::pair<Ct, Pt>> prods;
      for (size_t ti = 0; ti < terms.size(); ++ti)
        for (uint32_t k2 = 0; k2 < baby; ++k2) {
          const Pt& w = terms[ti].first->entries[k1 * baby + k2];
          if (w) prods.push_back({xs[ti][k2], w});
        }
      if (!prods.empty()) blocks.push_back({mac_plain(prods), (int32_t)shift});
    }
    std::vector<std::pair<Ct, int32_t>> to_rotate;
    for (auto& b : blocks)
      if (b.second != 0) to_rotate.push_back(b);
    std::vector<Ct> rotated = rotate_many(to_rotate);
    size_t ri = 0;
    for (auto& b : blocks) {
      const Ct block = b.second != 0 ? rotated[ri++] : b.first;
      acc = acc ? add(acc, block) : block;
    }
    return acc;
  }
  for (uint32_t k1 = 0; k1 < giant; ++k1) {
    const int64_t shift = (offset + (int64_t)baby * k1) * (int64_t)stride;
    Ct block;
    if (!cfg_.bsgs && shift != 0) {
      for (size_t ti = 0; ti < terms.size(); ++ti)
        for (uint32_t k2 = 0; k2 < baby; ++k2) {
          const Pt& w = terms[ti].first->entries[k1 * baby + k2];
          if (!w) continue;
          Ct t = rotate(mul_plain(xs[ti][k2], w), (int32_t)shift);
          block = block ? add(block, t) : t;
        }
    } else {
      std::vector<std::pair<Ct, Pt>> prods;
      for (size_t ti = 0; ti < terms.size(); ++ti)
        for (uint32_t k2 = 0; k2 < baby; ++k2) {
          const Pt& w = terms[ti].first->entries[k1 * baby + k2];
          if (w) prods.push_back({xs[ti][k2], w});
        }
      if (!prods.empty()) {
        Ct inner = mac_plain(prods);
        block = shift != 0 ? rotate(inner, (int32_t)shift) : inner;
      }
    }
    if (block) acc = acc ? add(acc, block) : block;
  }
  return acc;
}

Ct Evaluator::mac_plain(const std::vector<std::pair<Ct, Pt>>& terms) {
  const Ct& x0 = terms[0].first;
  const uint32_t level = x0->level;
  ctx_->activate();
  Ct acc;
  for (size_t first = 0; first < terms.size(); first += kMaxMacTerms) {
    const size_t cnt = std::min<size_t>(kMaxMacTerms, terms.size() - first);
    Ct r = new_ct(2, level, x0->scale * terms[0].second->scale);
    MacBatch b{};
    b.count = (int)cnt;
    b.limbs = (int)level + 1;
    b.out0 = r->comp_mut(0);
    b.out1 = r->comp_mut(1);
    for (size_t t = 0; t < cnt; ++t) {
      b.x0[t] = terms[first + t].first->comp(0);
      b.x1[t] = terms[first + t].first->comp(1);
      b.w[t] = terms[first + t].second->data();
    }
    launch_mac_plain(ctx_->dt, b, ctx_->stream);
    acc = acc ? add(acc, r) : r;
  }
  count([&](OpCounter& c) { c.ct_pt_mults += terms.size(); });
  return acc;
}

// ---- CoeffToSlot / SlotToCoeff: linear.rs:757-937 ---------------------------------------

namespace {

void check_stages(Evaluator& ev, const std::vector<LtPtr>& stages, uint32_t level, double scale) {  // :861-898
  if (stages.empty()) throw Error(ST_INVALID_PARAMS, "no stages");
  double s_in = scale;
  for (size_t k = 0; k < stages.size(); ++k) {
    const LinearTransform& lt = *stages[k];
    if (lt.level + k != level) throw Error(ST_LEVEL_MISMATCH, "level mismatch");
    const double label = ev.exact_product_scale(lt.level, lt.scale);
    const Pt* sp = lt.diags.first();
    if (!sp) throw Error(ST_INVALID_PARAMS, "a stage without diagonals");
    if ((*sp)->scale != label / s_in) throw Error(ST_SCALE_MISMATCH, "scale mismatch");
    if (lt.has_second) {
      if (lt.second.d != lt.diags.d || lt.second.stride != lt.diags.stride || lt.second.offset != lt.diags.offset)
        throw Error(ST_INVALID_PARAMS, "second diagonals of a different layout");
      const Pt* sp2 = lt.second.first();
      if (!sp2 || (*sp2)->scale != (*sp)->scale) throw Error(ST_SCALE_MISMATCH, "scale mismatch");
    }
    ev.check_rotation_keys_pub(lt.rotation_steps());
    s_in = lt.scale;
  }
}

Ct apply_stage(Evaluator& ev, const LinearTransform& lt, const Ct& x, const Ct* x2) {  // :900-919
  std::vector<std::pair<const SparseDiag*, Ct>> terms{{&lt.diags, x}};
  if (lt.has_second && x2) terms.push_back({&lt.second, *x2});
  Ct y = ev.matvec_plain_sum_sparse(terms);
  const double label = ev.exact_product_scale(lt.level, lt.scale);
  if (std::fabs((y->scale - label) / label) > 1e-15) throw Error(ST_SCALE_MISMATCH, "scale mismatch");
  return ev.rescale(ev.relabel(y, label));
}

}  // namespace

std::pair<Ct, Ct> coeff_to_slot(Evaluator& ev, const Ct& ct, const std::vector<LtPtr>& ctos) {  // :776-822
  ev.check_galois_input_pub(ct);
  if (ctos.empty()) throw Error(ST_INVALID_PARAMS, "no stages");
  for (auto& lt : ctos)
    if (lt->direction != DIR_COEFF_TO_SLOT)
      throw Error(ST_INVALID_PARAMS, "coeff_to_slot: a stage of the SlotToCoeff direction");
  bool bad = !ctos.back()->has_second;
  for (size_t i = 0; i + 1 < ctos.size(); ++i) bad = bad || ctos[i]->has_second;
  if (bad) throw Error(ST_INVALID_PARAMS, "coeff_to_slot: only the last stage (and it must) takes the conjugate");
  check_stages(ev, ctos, ct->level, ct->scale);
  ev.check_conjugation_key();
  Ct x = ct;
  for (auto& lt : ctos) {
    if (lt->has_second) {
      Ct xc = ev.conjugate(x);
      x = apply_stage(ev, *lt, x, &xc);
    } else {
      x = apply_stage(ev, *lt, x, nullptr);
    }
  }
  Ct xc = ev.conjugate(x);
  Ct re = ev.add(x, xc);
  Ct im = ev.mul_by_x_half(ev.sub(xc, x));
  return {re, im};
}

Ct slot_to_coeff(Evaluator& ev, const Ct& re, const Ct& im, const std::vector<LtPtr>& stoc) {  // :824-859
  ev.check_galois_input_pub(re);
  ev.check_galois_input_pub(im);
  for (auto& lt : stoc)
    if (lt->direction != DIR_SLOT_TO_COEFF)
      throw Error(ST_INVALID_PARAMS, "slot_to_coeff: a stage of the CoeffToSlot direction");
  bool bad = stoc.empty() || !stoc[0]->has_second;
  for (size_t i = 1; i < stoc.size(); ++i) bad = bad || stoc[i]->has_second;
  if (bad) throw Error(ST_INVALID_PARAMS, "slot_to_coeff: only the first stage (and it must) takes two inputs");
  if (re->level != im->level) throw Error(ST_LEVEL_MISMATCH, "level mismatch");
  if (re->scale != im->scale) throw Error(ST_SCALE_MISMATCH, "scale mismatch");
  check_stages(ev, stoc, re->level, re->scale);
  Ct x = apply_stage(ev, *stoc[0], re, &im);
  for (size_t i = 1; i < stoc.size(); ++i) x = apply_stage(ev, *stoc[i], x, nullptr);
  return x;
}

// ---- Chebyshev: bootstrap/poly.rs:213-714 ------------------------------------------------

namespace {

size_t optimal_split(size_t log_degree) {  // poly.rs:213-222
  int64_t d = (int64_t)log_degree, s = d >> 1;
  const int64_t a = ((int64_t)1 << s) + ((int64_t)1 << (d - s)) + d - s - 3;
  const int64_t b = ((int64_t)1 << (s + 1)) + ((int64_t)1 << std::max<int64_t>(d - s - 1, 0)) + d - s - 4;
  if (a > b) s += 1;
  return (size_t)s;
}

void split_coeffs(const std::vector<double>& p, size_t k, std::vector<double>& q, std::vector<double>& r) {
  const size_t m = p.size() - 1;  // poly.rs:312-330
  r.assign(p.begin(), p.begin() + k);
  q.assign(m - k + 1, 0.0);
  q[0] = p[k];
  for (size_t i = k + 1; i < p.size(); ++i) {
    q[i - k] = 2.0 * p[i];
    r[2 * k - i] -= p[i];
  }
}

Ct add_exact(Evaluator& ev, const Ct& a, const Ct& b, bool sub) {  // poly.rs:428-433
  if (a->scale != b->scale) throw Error(ST_SCALE_MISMATCH, "scale mismatch");
  return sub ? ev.sub(a, b) : ev.add(a, b);
}

Ct relabel_checked(Evaluator& ev, const Ct& ct, double scale) {  // poly.rs:444-449
  if (std::fabs((ct->scale - scale) / scale) > kRelabelTol) throw Error(ST_SCALE_MISMATCH, "scale mismatch");
  return ev.relabel(ct, scale);
}

struct Cheb {  // poly.rs:488-630
  Evaluator& ev;
  size_t top, baby;
  std::map<size_t, Ct> powers;

  void ensure(size_t i) {
    if (powers.count(i)) return;
    const size_t a = (size_t)1 << (ceil_log2(i) - 1);
    const size_t b = i - a, c = 2 * a - i;
    ensure(a);
    ensure(b);
    if (c > 0) ensure(c);
    const Ct& ta0 = powers.at(a);
    const Ct& tb0 = powers.at(b);
    const uint32_t l = std::min(ta0->level, tb0->level);
    Ct ta = ev.mod_switch_to_level(ta0, l);
    Ct tb = ev.mod_switch_to_level(tb0, l);
    Ct prod = ev.relinearize(ev.mul_no_relin(ta, tb));
    prod = add_exact(ev, prod, prod, false);
    if (c == 0) {
      prod = ev.boot_add_const(prod, -1.0);
    } else {
      Ct tc = ev.mod_switch_to_level(powers.at(c), l);
      prod = add_exact(ev, prod, ev.boot_mul_const(tc, 1.0, prod->scale), true);
    }
    powers.emplace(i, ev.rescale(prod));
  }

  std::optional<Ct> rec(const std::vector<double>& p0, size_t tl, double ts) {
    std::optional<size_t> mm;
    for (size_t i = p0.size(); i-- > 0;)
      if (p0[i] != 0.0) {
        mm = i;
        break;
      }
    if (!mm) return std::nullopt;
    const size_t m = *mm;
    std::vector<double> p(p0.begin(), p0.begin() + m + 1);
    if (m == 0 || (m < baby && tl + ceil_log2(m) <= top)) return leaf(p, tl, ts);
    const size_t k = (size_t)1 << (63 - __builtin_clzll(m));
    std::vector<double> q, r;
    split_coeffs(p, k, q, r);
    ensure(k);
    const double s_pow = powers.at(k)->scale;
    const double q_next = (double)ev.ctx()->primes[tl + 1];
    auto qres = rec(q, tl + 1, ts * q_next / s_pow);
    auto rres = rec(r, tl, ts);
    std::optional<Ct> prod;
    if (qres) {
      Ct qc = (*qres)->ncomp == 3 ? ev.relinearize(*qres) : *qres;
      qc = ev.rescale(qc);
      Ct tp = ev.mod_switch_to_level(powers.at(k), (uint32_t)tl);
      prod = relabel_checked(ev, ev.mul_no_relin(qc, tp), ts);
    }
    if (!prod) return rres;
    if (!rres) return prod;
    return add_exact(ev, *prod, *rres, false);
  }

  Ct leaf(const std::vector<double>& p, size_t tl, double ts) {
    std::optional<Ct> acc;
    for (size_t i = 1; i < p.size(); ++i) {
      if (p[i] == 0.0) continue;
      ensure(i);
      Ct t = ev.mod_switch_to_level(powers.at(i), (uint32_t)tl);
      Ct term = ev.boot_mul_const(t, p[i], ts);
      acc = acc ? add_exact(ev, *acc, term, false) : term;
    }
    Ct a = acc ? *acc : ev.boot_zero((uint32_t)tl, ts);
    return p[0] != 0.0 ? ev.boot_add_const(a, p[0]) : a;
  }
};

}  // namespace

Ct eval_chebyshev_to_scale(Evaluator& ev, const Ct& ct, const std::vector<double>& coeffs, double a, double b,
                           double target) {  // poly.rs:655-714
  ev.check_boot_input(ct);
  if (coeffs.size() < 2) throw Error(ST_INVALID_PARAMS, "eval_chebyshev needs degree >= 1 (two coefficients or more)");
  for (double c : coeffs)
    if (!std::isfinite(c)) throw Error(ST_INVALID_PARAMS, "non-finite Chebyshev coefficient");
  if (!(std::isfinite(a) && std::isfinite(b) && a < b))
    throw Error(ST_INVALID_PARAMS, "interval must be finite with a < b");
  if (!(std::isfinite(target) && target > 0.0)) throw Error(ST_INVALID_PARAMS, "target scale must be positive and finite");
  const bool affine = a != -1.0 || b != 1.0;
  const size_t depth = ceil_log2(coeffs.size());
  if (ct->level < depth + (affine ? 1 : 0)) throw Error(ST_NO_LEVELS_LEFT, "no levels left");
  Ct x = ct;
  if (affine) {
    const double alpha = 2.0 / (b - a), beta = -(a + b) / (b - a);
    x = ev.boot_add_const(ev.rescale(ev.mul_scalar(ct, alpha, ct->scale)), beta);
  }
  const size_t top = x->level, tl = top + 1 - depth;
  const double label = ev.exact_product_scale((uint32_t)tl, target);
  Cheb ch{ev, top, (size_t)1 << optimal_split(depth), {}};
  ch.powers.emplace(1, x);
  auto res0 = ch.rec(coeffs, tl, label);
  Ct res = res0 ? *res0 : ev.boot_zero((uint32_t)tl, label);
  if (res->ncomp == 3) res = ev.relinearize(res);
  return ev.rescale(res);
}

Ct eval_mod(Evaluator& ev, const Ct& ct, const BootParams& bp, const std::vector<double>& coeffs) {
  if (bp.k_intervals == 0 || bp.cheb_degree == 0)  // evalmod.rs:147-189
    throw Error(ST_INVALID_PARAMS, "k_intervals and cheb_degree must be positive");
  const uint32_t depth = bp.evalmod_depth();
  if (depth > bp.evalmod_levels) throw Error(ST_INVALID_PARAMS, "EvalMod depth exceeds evalmod_levels");
  if (coeffs.size() != (size_t)bp.cheb_degree + 1)
    throw Error(ST_INVALID_PARAMS, "EvalMod series length is not cheb_degree + 1");
  ev.check_boot_input(ct);
  if (ct->level < depth) throw Error(ST_NO_LEVELS_LEFT, "no levels left");
  const uint32_t r = bp.double_angle;
  std::vector<double> targets(r + 1, ct->scale);
  const uint32_t cheb_out = ct->level - (uint32_t)ceil_log2((size_t)bp.cheb_degree + 1);  // evalmod.rs:210-236
  for (uint32_t i = r; i >= 1; --i) {
    const uint32_t level = cheb_out - (i - 1);
    const double sigma = ev.exact_product_scale(level, targets[i]);
    const double seed = std::sqrt(2.0 * sigma);
    uint64_t bits;
    memcpy(&bits, &seed, 8);
    bool found = false;
    for (uint64_t k = 0; k <= 16 && !found; ++k)
      for (int s = 0; s < 2 && !found; ++s) {
        const uint64_t bb = s == 0 ? bits + k : bits - k;
        double cand;
        memcpy(&cand, &bb, 8);
        try {
          ev.exact_product_scale(level + 1, cand);
          targets[i - 1] = cand;
          found = true;
        } catch (const Error&) {
        }
      }
    if (!found) throw Error(ST_SCALE_MISMATCH, "scale mismatch");
  }
  Ct c = eval_chebyshev_to_scale(ev, ct, coeffs, -1.0, 1.0, targets[0]);
  for (uint32_t i = 1; i < targets.size(); ++i) {  // double angles, poly.rs:721-736
    const double sigma = ev.exact_product_scale(c->level, targets[i]);
    Ct sq = ev.relinearize(ev.mul_no_relin(c, c));
    if (std::fabs((sq->scale / 2.0 - sigma) / sigma) > std::exp2(-40.0)) throw Error(ST_SCALE_MISMATCH, "scale mismatch");
    sq = ev.relabel(sq, sigma);
    c = ev.rescale(ev.boot_add_const(sq, -1.0));
  }
  return c;
}

// ---- the assembled bootstrap: bootstrapper.rs --------------------------------------------

Bootstrapper::Bootstrapper(Context* ctx, const BootParams& bp, std::vector<LtPtr> ctos, std::vector<LtPtr> stoc,
                           std::vector<KeyPtr> galois, KeyPtr to_sparse, KeyPtr to_dense, std::vector<double> coeffs,
                           double evalmod_scale, double stoc_input_scale, double delta)
    : ctx_(ctx),
      bp_(bp),
      ctos_(std::move(ctos)),
      stoc_(std::move(stoc)),
      galois_(std::move(galois)),
      to_sparse_(std::move(to_sparse)),
      to_dense_(std::move(to_dense)),
      coeffs_(std::move(coeffs)),
      evalmod_scale_(evalmod_scale),
      stoc_input_scale_(stoc_input_scale),
      delta_(delta) {
  if (bp_.log_slots + 1 != ctx_->log_n) throw Error(ST_INVALID_PARAMS, "bootstrapping needs full packing");
  const uint32_t used = bp_.ctos_levels + bp_.evalmod_levels + bp_.stoc_levels;
  if (used >= ctx_->L) throw Error(ST_INVALID_PARAMS, "the bootstrap bands leave no compute level");
  if (bp_.evalmod_depth() > bp_.evalmod_levels) throw Error(ST_INVALID_PARAMS, "EvalMod depth exceeds its levels");
  if (ctos_.size() != bp_.ctos_levels || stoc_.size() != bp_.stoc_levels)
    throw Error(ST_INVALID_PARAMS, "stage counts differ from the bootstrap bands");
  if ((bool)to_sparse_ != (bool)to_dense_) throw Error(ST_INVALID_PARAMS, "SSE needs both switching keys");
  for (auto& k : galois_)
    if (!k || k->ctx != ctx_) throw Error(ST_INVALID_PARAMS, "a Galois key is not over this context");
  if (!(std::isfinite(delta_) && delta_ > 0.0)) throw Error(ST_INVALID_PARAMS, "delta must be positive and finite");
}

uint32_t Bootstrapper::output_level() const {
  return ctx_->L - (bp_.ctos_levels + bp_.evalmod_levels + bp_.stoc_levels);
}

namespace {
// `to` waits for the work queued on `from` so far.
void wait_for(cudaStream_t to, cudaStream_t from) {
  cudaEvent_t e;
  CKG_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  cudaError_t err = cudaEventRecord(e, from);
  if (err == cudaSuccess) err = cudaStreamWaitEvent(to, e, 0);
  cudaEventDestroy(e);
  if (err != cudaSuccess) throw_cuda(err, "cudaStreamWaitEvent");
}
}  // namespace

// The real and imaginary EvalMods are independent (the same ops on two ciphertexts): they run
// concurrently, each on one of the context's two auxiliary lanes, issued from two host threads,
// so the small launches of one fill the SMs the other leaves idle. Each keeps its own op order,
// so the results are those of the sequential evaluation; the caller's stream waits for both
// lanes, and the results' buffers are freed on the caller's stream from then on.
std::pair<Ct, Ct> Bootstrapper::eval_mod_pair(Evaluator& inner, const Ct& re_in, const Ct& im_in) {
  Lane& la = ctx_->aux_lane(0);
  Lane& lb = ctx_->aux_lane(1);
  const cudaStream_t caller = ctx_->stream;
  const StreamPtr caller_res = ctx_->cur_sres();
  wait_for(la.sres->s, caller);
  wait_for(lb.sres->s, caller);
  Ct re, im;
  std::exception_ptr err_re, err_im;
  std::thread t([&] {
    try {
      ctx_->activate();
      LaneScope scope(*ctx_, lb);
      im = eval_mod(inner, im_in, bp_, coeffs_);
    } catch (...) {
      err_im = std::current_exception();
    }
  });
  try {
    LaneScope scope(*ctx_, la);
    re = eval_mod(inner, re_in, bp_, coeffs_);
  } catch (...) {
    err_re = std::current_exception();
  }
  t.join();
  wait_for(caller, la.sres->s);  // before anything the caller queues or frees next
  wait_for(caller, lb.sres->s);
  if (err_re) std::rethrow_exception(err_re);
  if (err_im) std::rethrow_exception(err_im);
  re->buf->sres = caller_res;
  im->buf->sres = caller_res;
  return {re, im};
}

Ct Bootstrapper::pipeline(Evaluator& inner, const Ct& ct) {  // bootstrapper.rs:431-473
  Ct raised = to_sparse_ ? inner.mod_raise(ct, *to_sparse_, *to_dense_) : inner.mod_raise_main_key(ct);
  raised = inner.relabel(raised, (double)ctx_->primes[0]);
  auto reim = coeff_to_slot(inner, raised, ctos_);
  auto [re, im] = eval_mod_pair(inner, reim.first, reim.second);
  const uint32_t start = stoc_[0]->level;
  auto to_stoc = [&](const Ct& c) {
    if (c->scale != evalmod_scale_) throw Error(ST_SCALE_MISMATCH, "scale mismatch");
    return inner.relabel(inner.mod_switch_to_level(c, start), stoc_input_scale_);
  };
  return slot_to_coeff(inner, to_stoc(re), to_stoc(im), stoc_);
}

Ct Bootstrapper::bootstrap(Evaluator& ev, const Ct& ct) {  // bootstrapper.rs:385-421
  if (ev.ctx() != ctx_) throw Error(ST_INVALID_PARAMS, "bootstrap: evaluator over other parameters");
  if (!ev.relin_key_present())
    throw Error(ST_INVALID_PARAMS, "bootstrap: the evaluator has no relinearization key (EvalMod needs it)");
  if (!ev.owns(ct)) throw Error(ST_INVALID_PARAMS, "operand is not over this evaluator's data basis");
  if (ct->level != 0) throw Error(ST_INVALID_PARAMS, "bootstrap: input must be at level 0");
  if (ct->scale != delta_) throw Error(ST_SCALE_MISMATCH, "scale mismatch");
  Evaluator inner(ctx_, ev.relin_key(), galois_, EvalConfig{});
  Ct out = pipeline(inner, ct);
  OpCounter done = inner.counter();
  done.bootstraps += 1;
  ev.add_counts(done);
  return out;
}

}  // namespace ckg
