// TEST AND BASELINE INFRASTRUCTURE ONLY -- not part of the product.
//
// Runs the reference's own CUDA kernels (crates/ckks-train-cuda/kernels/{ntt,basis,keyswitch}.cu,
// compiled unmodified from the reference tree, with --fmad=false as the reference's NVRTC
// build passes, crates/ckks-train-cuda/src/device.rs:309-315) through the launch sequences of the
// reference's Rust host code, so the reference's GPU key switch can be timed on the same B200 as
// this library's:
//  - NTT: NttPlan (src/plan.rs:35-80): global stages of 256 threads for distances >= 2048, one
//    shared-memory launch for the rest (forward: global then shared; inverse: shared then the
//    global stages in reverse, src/device.rs:820-870);
//  - key switch: Ks::key_switch = decompose + apply_key (src/ks.rs:335-378): per digit, copy the
//    digit limbs, inverse NTT, basis_convert to the other Q primes and the P primes, forward NTT,
//    copy into Q_l * P order (mod_up_digit, src/basis.rs:480-514); one ks_inner_product over
//    every digit (src/keyswitch.rs:355-421); divide_round_tail of both accumulators (copy the P
//    limbs, inverse NTT, basis_convert P -> Q_l, forward NTT, basis_div_finish; src/basis.rs:455-478).
// Device tables follow src/tables.rs (roots[bitrev(i)] = psi^i with Shoup companions, 7 constants
// per prime) and ConvTable::new (src/basis.rs:251-320). Built by oracle/ref_gpu/Makefile into
// oracle/_ref/libref_gpu.so, which the library never links.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../oracle_core.hpp"

// The reference kernels, each file in its own namespace (their helper functions share names);
// the kernels themselves keep their extern "C" names.
namespace rk_ntt {
#include "ntt.cu"
}
namespace rk_basis {
#include "basis.cu"
}
namespace rk_ks {
#include "keyswitch.cu"
}

namespace {

typedef unsigned long long u64;
constexpr int kNconst = 7;
constexpr unsigned kLogChunk = 11;
constexpr unsigned kGlobalBlock = 256, kElemBlock = 256;

void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

struct DevVec {
  u64* p = nullptr;
  size_t words = 0;
  cudaStream_t st = nullptr;
  DevVec(size_t w, cudaStream_t s) : words(w), st(s) { ck(cudaMallocAsync((void**)&p, w * 8, s), "cudaMallocAsync"); }
  ~DevVec() {
    if (p) cudaFreeAsync(p, st);
  }
  DevVec(const DevVec&) = delete;
  DevVec& operator=(const DevVec&) = delete;
};
typedef std::shared_ptr<DevVec> Buf;

}  // namespace

struct RefCtx {
  unsigned log_n = 0;
  size_t n = 0, nq = 0, np = 0, dnum = 0, alpha = 0;
  std::vector<orc::Modulus> mods;
  cudaStream_t st = nullptr;
  u64 *roots = nullptr, *roots_s = nullptr, *iroots = nullptr, *iroots_s = nullptr, *consts = nullptr;
  std::map<std::vector<uint32_t>, uint32_t*> maps;
  std::map<std::pair<std::vector<uint32_t>, std::vector<uint32_t>>, std::pair<u64*, uint32_t>> tables;
  std::vector<void*> owned;
  // The digit-address lists go through a pinned staging ring (as src/device.rs:138-185 does), so
  // their uploads are asynchronous; a slot is reused once its copy has completed.
  static constexpr int kSlots = 64, kSlotWords = 16;
  u64* pin = nullptr;
  cudaEvent_t slot_done[kSlots] = {};
  bool slot_used[kSlots] = {};
  int next_slot = 0;

  Buf alloc(size_t limbs) { return std::make_shared<DevVec>(limbs * n, st); }
  const uint32_t* limb_map(const std::vector<uint32_t>& primes) {
    auto it = maps.find(primes);
    if (it != maps.end()) return it->second;
    uint32_t* d = nullptr;
    ck(cudaMalloc(&d, primes.size() * 4), "cudaMalloc");
    ck(cudaMemcpy(d, primes.data(), primes.size() * 4, cudaMemcpyHostToDevice), "cudaMemcpy");
    owned.push_back(d);
    maps[primes] = d;
    return d;
  }
  // ConvTable::new (src/basis.rs:251-320): sources, qhat^-1 (values, companions), 1/q as f64
  // bits; per target r: r, [Q]_r (value, companion), h = ([Q]_r - 1) / 2, [Q]_r^-1 (value,
  // companion), then [Q / q_j]_r as (value, companion) per source.
  std::pair<u64*, uint32_t> conv_table(const std::vector<uint32_t>& src, const std::vector<uint32_t>& dst) {
    auto key = std::make_pair(src, dst);
    auto it = tables.find(key);
    if (it != tables.end()) return it->second;
    std::vector<u64> w;
    const size_t k = src.size();
    for (uint32_t s : src) w.push_back(mods[s].q);
    std::vector<orc::Shoup> qhinv;
    for (size_t j = 0; j < k; ++j) {
      const orc::Modulus& m = mods[src[j]];
      uint64_t qhat = 1 % m.q;
      for (size_t i = 0; i < k; ++i)
        if (i != j) qhat = m.mul(qhat, mods[src[i]].q % m.q);
      qhinv.push_back(m.shoup(m.inv_or_throw(qhat)));
    }
    for (auto& s : qhinv) w.push_back(s.w);
    for (auto& s : qhinv) w.push_back(s.ws);
    for (uint32_t s : src) {
      const double inv = 1.0 / (double)mods[s].q;
      u64 b;
      memcpy(&b, &inv, 8);
      w.push_back(b);
    }
    for (uint32_t t : dst) {
      const orc::Modulus& r = mods[t];
      uint64_t qm = 1 % r.q;
      for (uint32_t s : src) qm = r.mul(qm, mods[s].q % r.q);
      const uint64_t h = r.mul(r.sub(qm, 1 % r.q), (r.q + 1) / 2);
      const orc::Shoup qs = r.shoup(qm), inv = r.shoup(r.inv_or_throw(qm));
      w.insert(w.end(), {(u64)r.q, qs.w, qs.ws, h, inv.w, inv.ws});
      for (size_t j = 0; j < k; ++j) {
        uint64_t qhat = 1 % r.q;
        for (size_t i = 0; i < k; ++i)
          if (i != j) qhat = r.mul(qhat, mods[src[i]].q % r.q);
        const orc::Shoup s = r.shoup(qhat);
        w.push_back(s.w);
        w.push_back(s.ws);
      }
    }
    u64* d = nullptr;
    ck(cudaMalloc(&d, w.size() * 8), "cudaMalloc");
    ck(cudaMemcpy(d, w.data(), w.size() * 8, cudaMemcpyHostToDevice), "cudaMemcpy");
    owned.push_back(d);
    return tables[key] = {d, (uint32_t)(k > 1)};
  }

  // NttPlan + the launch loop of src/device.rs:820-870 over `buf` (limbs with primes `primes`).
  void ntt(u64* buf, const std::vector<uint32_t>& primes, bool inverse) {
    const uint32_t* map = limb_map(primes);
    const unsigned limbs = (unsigned)primes.size();
    const unsigned log_chunk = log_n < kLogChunk ? log_n : kLogChunk;
    const dim3 sgrid((unsigned)(n >> log_chunk), limbs), sblock(1u << (log_chunk - 1));
    const size_t smem = (size_t)8 << log_chunk;
    const dim3 ggrid((unsigned)((n / 2 + kGlobalBlock - 1) / kGlobalBlock), limbs), gblock(kGlobalBlock);
    const u64* rt = inverse ? iroots : roots;
    const u64* rs = inverse ? iroots_s : roots_s;
    if (inverse) {
      rk_ntt::ntt_inv_shared<<<sgrid, sblock, smem, st>>>(buf, rt, rs, consts, map, log_n, log_chunk);
      for (unsigned s = log_n - log_chunk; s-- > 0;)
        rk_ntt::ntt_inv_global_stage<<<ggrid, gblock, 0, st>>>(buf, rt, rs, consts, map, log_n, log_n - 1 - s);
    } else {
      for (unsigned s = 0; s < log_n - log_chunk; ++s)
        rk_ntt::ntt_fwd_global_stage<<<ggrid, gblock, 0, st>>>(buf, rt, rs, consts, map, log_n, log_n - 1 - s);
      rk_ntt::ntt_fwd_shared<<<sgrid, sblock, smem, st>>>(buf, rt, rs, consts, map, log_n, log_chunk);
    }
  }
  void copy_limbs(const u64* src, size_t at, u64* dst, size_t dat, size_t count) {
    ck(cudaMemcpyAsync(dst + dat * n, src + at * n, count * n * 8, cudaMemcpyDeviceToDevice, st), "copy");
  }
  void convert(u64* out, const u64* src, const std::vector<uint32_t>& s, const std::vector<uint32_t>& t) {
    auto tab = conv_table(s, t);
    rk_basis::basis_convert<<<dim3((unsigned)((n + kElemBlock - 1) / kElemBlock), 1), kElemBlock, 0, st>>>(
        out, src, tab.first, (unsigned)s.size(), (unsigned)t.size(), log_n, tab.second);
  }
  // divide_round_tail (src/basis.rs:455-478) of a Q_l * P polynomial in NTT form.
  Buf divide_round_tail(const u64* x, const std::vector<uint32_t>& primes, size_t keep) {
    std::vector<uint32_t> head(primes.begin(), primes.begin() + keep), tail(primes.begin() + keep, primes.end());
    Buf src = alloc(tail.size());
    copy_limbs(x, keep, src->p, 0, tail.size());
    ntt(src->p, tail, true);
    Buf t = alloc(keep);
    convert(t->p, src->p, tail, head);
    ntt(t->p, head, false);
    auto tab = conv_table(tail, head);
    rk_basis::basis_div_finish<<<dim3((unsigned)((n + kElemBlock - 1) / kElemBlock), (unsigned)keep), kElemBlock, 0,
                                  st>>>(t->p, x, tab.first, (unsigned)tail.size(), log_n);
    return t;
  }
  // Ks::key_switch (src/ks.rs:335-378) of x (level l, NTT form) with a key of key_q data limbs.
  void key_switch(const u64* x, size_t l, const u64* key, size_t key_q, u64* out_b, u64* out_a) {
    std::vector<uint32_t> qp;
    for (uint32_t i = 0; i <= l; ++i) qp.push_back(i);
    for (uint32_t t = 0; t < np; ++t) qp.push_back((uint32_t)(nq + t));
    std::vector<Buf> digits;
    for (size_t j = 0; j < dnum; ++j) {
      const size_t s = j * alpha, e = std::min((j + 1) * alpha, l + 1);
      if (s > l) break;
      std::vector<uint32_t> sp, tp;
      for (size_t i = s; i < e; ++i) sp.push_back((uint32_t)i);
      for (size_t i = 0; i <= l; ++i)
        if (i < s || i >= e) tp.push_back((uint32_t)i);
      for (uint32_t t = 0; t < np; ++t) tp.push_back((uint32_t)(nq + t));
      Buf src = alloc(sp.size());
      copy_limbs(x, s, src->p, 0, sp.size());
      ntt(src->p, sp, true);
      Buf conv = alloc(tp.size());
      convert(conv->p, src->p, sp, tp);
      ntt(conv->p, tp, false);
      Buf out = alloc(qp.size());
      if (s > 0) copy_limbs(conv->p, 0, out->p, 0, s);
      copy_limbs(x, s, out->p, s, e - s);
      copy_limbs(conv->p, s, out->p, e, tp.size() - s);
      digits.push_back(out);
    }
    const int slot = next_slot;
    next_slot = (next_slot + 1) % kSlots;
    if (slot_used[slot]) ck(cudaEventSynchronize(slot_done[slot]), "staging slot");
    u64* stage = pin + (size_t)slot * kSlotWords;
    for (size_t j = 0; j < digits.size(); ++j) stage[j] = (u64)(uintptr_t)digits[j]->p;
    Buf dp = std::make_shared<DevVec>(digits.size(), st);
    ck(cudaMemcpyAsync(dp->p, stage, digits.size() * 8, cudaMemcpyHostToDevice, st), "ptrs");
    ck(cudaEventRecord(slot_done[slot], st), "event");
    slot_used[slot] = true;
    Buf acc_b = alloc(qp.size()), acc_a = alloc(qp.size());
    rk_ks::ks_inner_product<<<dim3((unsigned)((n + kElemBlock - 1) / kElemBlock), (unsigned)qp.size()), kElemBlock,
                               0, st>>>(acc_b->p, acc_a->p, dp->p, key, consts, limb_map(qp), log_n,
                                        (unsigned)digits.size(), (unsigned)(l + 1), (unsigned)(key_q + np),
                                        (unsigned)(key_q - (l + 1)));
    Buf kb = divide_round_tail(acc_b->p, qp, l + 1);
    Buf ka = divide_round_tail(acc_a->p, qp, l + 1);
    copy_limbs(kb->p, 0, out_b, 0, l + 1);
    copy_limbs(ka->p, 0, out_a, 0, l + 1);
  }
};

namespace {
thread_local std::string g_err;
}

extern "C" {

const char* ref_last_error() { return g_err.c_str(); }

int ref_ctx_create(uint32_t log_n, const uint64_t* q, uint32_t nq, const uint64_t* p, uint32_t np, uint32_t dnum,
                   RefCtx** out) {
  try {
    auto c = std::make_unique<RefCtx>();
    c->log_n = log_n;
    c->n = (size_t)1 << log_n;
    c->nq = nq;
    c->np = np;
    c->dnum = dnum;
    c->alpha = nq / dnum;
    for (uint32_t i = 0; i < nq; ++i) c->mods.emplace_back(q[i]);
    for (uint32_t i = 0; i < np; ++i) c->mods.emplace_back(p[i]);
    ck(cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking), "stream");
    ck(cudaMallocHost((void**)&c->pin, RefCtx::kSlots * RefCtx::kSlotWords * 8), "cudaMallocHost");
    for (auto& e : c->slot_done) ck(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
    const size_t npr = c->mods.size(), n = c->n;
    std::vector<u64> r(npr * n), rs(npr * n), ir(npr * n), irs(npr * n), cs(npr * kNconst);
    for (size_t i = 0; i < npr; ++i) {
      orc::NttTable t(n, c->mods[i]);
      for (size_t k = 0; k < n; ++k) {
        r[i * n + k] = t.roots[k].w;
        rs[i * n + k] = t.roots[k].ws;
        ir[i * n + k] = t.inv_roots[k].w;
        irs[i * n + k] = t.inv_roots[k].ws;
      }
      const orc::u128 ratio = c->mods[i].ratio;  // floor(2^128 / q), src/tables.rs:139-147
      const u64 v[kNconst] = {c->mods[i].q, t.n_inv.w, t.n_inv.ws, t.w_n_inv.w, t.w_n_inv.ws, (u64)ratio,
                              (u64)(ratio >> 64)};
      memcpy(&cs[i * kNconst], v, sizeof v);
    }
    auto up = [&](const std::vector<u64>& h, u64** d) {
      ck(cudaMalloc(d, h.size() * 8), "cudaMalloc");
      ck(cudaMemcpy(*d, h.data(), h.size() * 8, cudaMemcpyHostToDevice), "cudaMemcpy");
      c->owned.push_back(*d);
    };
    up(r, &c->roots);
    up(rs, &c->roots_s);
    up(ir, &c->iroots);
    up(irs, &c->iroots_s);
    up(cs, &c->consts);
    *out = c.release();
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return 1;
  }
}

void ref_ctx_destroy(RefCtx* c) {
  if (!c) return;
  cudaStreamSynchronize(c->st);
  for (void* p : c->owned) cudaFree(p);
  for (auto& e : c->slot_done) cudaEventDestroy(e);
  cudaFreeHost(c->pin);
  cudaStreamDestroy(c->st);
  delete c;
}

void* ref_ctx_stream(RefCtx* c) { return c->st; }

int ref_ntt(RefCtx* c, uint64_t* buf, const uint32_t* primes, uint32_t nlimbs, int inverse) {
  try {
    c->ntt(reinterpret_cast<u64*>(buf), std::vector<uint32_t>(primes, primes + nlimbs), inverse != 0);
    ck(cudaGetLastError(), "launch");
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return 1;
  }
}

int ref_key_switch(RefCtx* c, const uint64_t* in, uint32_t level, const uint64_t* key, uint32_t key_q, uint64_t* out_b,
                   uint64_t* out_a) {
  try {
    c->key_switch(reinterpret_cast<const u64*>(in), level, reinterpret_cast<const u64*>(key), key_q,
                  reinterpret_cast<u64*>(out_b), reinterpret_cast<u64*>(out_a));
    ck(cudaGetLastError(), "launch");
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return 1;
  }
}

int ref_sync(RefCtx* c) {
  cudaError_t e = cudaStreamSynchronize(c->st);
  if (e != cudaSuccess) {
    g_err = cudaGetErrorString(e);
    return 1;
  }
  return 0;
}

}  // extern "C"
