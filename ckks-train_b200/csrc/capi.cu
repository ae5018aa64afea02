// extern "C" entry points of include/ckg.h: handle wrapping, argument checks and the
// translation of C++ errors and CUDA failures into status codes (nothing throws or
// aborts across the boundary).
#include <cstring>
#include <string>

#include "../../include/ckg.h"
#include "bootsetup.hpp"
#include "bounds.hpp"
#include "handles.hpp"
#include "seal.hpp"

using namespace ckg;

static thread_local std::string g_last_error;

void ckg_set_last_error(const char* msg) { g_last_error = msg; }

static int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

#define CKG_API_BEGIN try {
#define CKG_API_END                                                       \
  }                                                                       \
  catch (const Error& e) {                                                \
    return fail(e.code, e.what());                                        \
  }                                                                       \
  catch (const std::bad_alloc&) {                                         \
    return fail(CKG_OOM, "out of host memory");                           \
  }                                                                       \
  catch (const std::invalid_argument& e) {                                \
    return fail(CKG_INVALID_PARAMS, e.what());                            \
  }                                                                       \
  catch (const std::exception& e) {                                       \
    return fail(CKG_DEVICE, std::string("internal error: ") + e.what()); \
  }                                                                       \
  return CKG_OK;

// Launch errors surface here (asynchronous faults at the next synchronisation).
static void check_launch() { CKG_CUDA(cudaGetLastError()); }

static Context& ctx_of(ckg_ctx* c) {
  if (!c || !c->c) throw Error(CKG_INVALID_PARAMS, "null context");
  return *c->c;
}

extern "C" {

const char* ckg_last_error(void) { return g_last_error.c_str(); }
uint32_t ckg_abi_version(void) { return 1; }
uint64_t ckg_launch_count(void) { return g_launches.load(); }

int ckg_primes_for_bits(uint32_t log_n, const uint32_t* q_bits, uint32_t nq, const uint32_t* p_bits, uint32_t np,
                        uint64_t* q_out, uint64_t* p_out) {
  CKG_API_BEGIN
  if (log_n < 1 || log_n > 17) throw Error(CKG_INVALID_PARAMS, "log_n outside [1, 17]");
  if (!nq || !np) throw Error(CKG_INVALID_PARAMS, "q_bits and p_bits must be non-empty");
  std::vector<uint64_t> q, p;
  primes_for_bits(log_n, std::vector<uint32_t>(q_bits, q_bits + nq), std::vector<uint32_t>(p_bits, p_bits + np), q, p);
  memcpy(q_out, q.data(), nq * 8);
  memcpy(p_out, p.data(), np * 8);
  CKG_API_END
}

int ckg_ctx_create(uint32_t log_n, const uint64_t* q, uint32_t nq, const uint64_t* p, uint32_t np, uint32_t dnum,
                   int device, void* stream, ckg_ctx** out) {
  CKG_API_BEGIN
  if (!out) throw Error(CKG_INVALID_PARAMS, "null output");
  auto h = new ckg_ctx;
  try {
    h->c = std::make_unique<Context>(log_n, std::vector<uint64_t>(q, q + nq), std::vector<uint64_t>(p, p + np), dnum,
                                     device, (cudaStream_t)stream);
  } catch (...) {
    delete h;
    throw;
  }
  *out = h;
  CKG_API_END
}

void ckg_ctx_destroy(ckg_ctx* ctx) { delete ctx; }

int ckg_ctx_sync(ckg_ctx* ctx) {
  CKG_API_BEGIN
  Context& c = ctx_of(ctx);
  c.activate();
  CKG_CUDA(cudaStreamSynchronize(c.stream));
  c.sync_transfers();
  const int f = device_fault_take();
  if (f > 0) throw Error(CKG_DEVICE, "a kernel recorded a device fault (code " + std::to_string(f) + ")");
  CKG_API_END
}

int ckg_device_fault(ckg_ctx* ctx, int32_t* code) {
  CKG_API_BEGIN
  ctx_of(ctx).activate();
  *code = device_fault_take();
  CKG_API_END
}

int ckg_ctx_transfer_stats(ckg_ctx* ctx, uint64_t* out, uint32_t n) {
  CKG_API_BEGIN
  if (!out && n) throw Error(CKG_INVALID_PARAMS, "null output");
  Context& c = ctx_of(ctx);
  uint64_t reserved = 0;
  if (c.xpool) {
    unsigned long long v = 0;
    if (cudaMemPoolGetAttribute(c.xpool, cudaMemPoolAttrReservedMemCurrent, &v) == cudaSuccess) reserved = v;
  }
  const uint64_t w[9] = {c.st_upload_calls, c.st_upload_bytes,   c.st_upload_alloc_ns, c.st_upload_copy_ns,
                         reserved,          c.st_download_calls, c.st_download_ns,      c.st_alloc_retries,
                         c.xcache ? c.xcache->waited.load() : 0};
  for (uint32_t i = 0; i < n && i < 9; ++i) out[i] = w[i];
  CKG_API_END
}

int ckg_debug_bounds(int op, uint64_t p, uint64_t bytes) {
  CKG_API_BEGIN
  const void* a = reinterpret_cast<const void*>((uintptr_t)p);
  switch (op) {
    case 0: bounds::set_enabled(bytes != 0); break;
    case 1: bounds::track(a, bytes); break;
    case 2: bounds::untrack(a); break;
    case 3: bounds::check(a, bytes, "checked range"); break;
    default: throw Error(CKG_INVALID_PARAMS, "unknown bounds operation");
  }
  CKG_API_END
}

int ckg_ctx_trim(ckg_ctx* ctx) {
  CKG_API_BEGIN
  ctx_of(ctx).trim();
  CKG_API_END
}

int ckg_host_alloc(uint64_t bytes, void** out) {
  CKG_API_BEGIN
  if (!out) throw Error(CKG_INVALID_PARAMS, "null output");
  *out = nullptr;
  if (!bytes) throw Error(CKG_INVALID_PARAMS, "zero bytes");
  CKG_CUDA(cudaHostAlloc(out, bytes, cudaHostAllocPortable));
  CKG_API_END
}

void ckg_host_free(void* p) {
  if (p) cudaFreeHost(p);
}

int ckg_ctx_join_transfers(ckg_ctx* ctx) {
  CKG_API_BEGIN
  ctx_of(ctx).join_transfers();
  CKG_API_END
}

void* ckg_ctx_stream(ckg_ctx* ctx) { return ctx && ctx->c ? (void*)ctx->c->stream : nullptr; }

// ---- device-buffer primitives ----------------------------------------------------------

static void check_primes(const Context& c, const uint32_t* primes, uint32_t n) {
  for (uint32_t i = 0; i < n; ++i)
    if (primes[i] >= c.primes.size()) throw Error(CKG_INVALID_PARAMS, "prime index out of range");
}

int ckg_ntt(ckg_ctx* ctx, const uint64_t* src, uint64_t* dst, const uint32_t* primes, uint32_t nlimbs, int inverse) {
  CKG_API_BEGIN
  Context& c = ctx_of(ctx);
  check_primes(c, primes, nlimbs);
  c.activate();
  std::vector<LimbRef> refs;
  for (uint32_t i = 0; i < nlimbs; ++i) refs.push_back(LimbRef{src + i * c.n, dst + i * c.n, primes[i], 0});
  ntt_limbs(c, refs, inverse != 0);
  check_launch();
  CKG_API_END
}

int ckg_poly_binary(ckg_ctx* ctx, int op, const uint64_t* a, const uint64_t* b, uint64_t* out, uint32_t first_prime,
                    uint32_t nlimbs) {
  CKG_API_BEGIN
  Context& c = ctx_of(ctx);
  if (op < 0 || op > 2) throw Error(CKG_INVALID_PARAMS, "op must be 0 (add), 1 (sub) or 2 (mul)");
  if (first_prime + nlimbs > c.primes.size()) throw Error(CKG_INVALID_PARAMS, "prime index out of range");
  c.activate();
  std::vector<BinRef> refs;
  for (uint32_t i = 0; i < nlimbs; ++i)
    refs.push_back(BinRef{a + i * c.n, b + i * c.n, out + i * c.n, first_prime + i, 0});
  launch_binary(c.dt, refs.data(), (int)refs.size(), op, c.stream);
  check_launch();
  CKG_API_END
}

int ckg_poly_negate(ckg_ctx* ctx, const uint64_t* a, uint64_t* out, uint32_t first_prime, uint32_t nlimbs) {
  CKG_API_BEGIN
  Context& c = ctx_of(ctx);
  if (first_prime + nlimbs > c.primes.size()) throw Error(CKG_INVALID_PARAMS, "prime index out of range");
  c.activate();
  std::vector<LimbRef> refs;
  for (uint32_t i = 0; i < nlimbs; ++i) refs.push_back(LimbRef{a + i * c.n, out + i * c.n, first_prime + i, 0});
  launch_unary(c.dt, refs.data(), (int)refs.size(), 0, nullptr, nullptr, c.stream);
  check_launch();
  CKG_API_END
}

int ckg_poly_mul_scalar(ckg_ctx* ctx, const uint64_t* a, uint64_t scalar, uint64_t* out, uint32_t first_prime,
                        uint32_t nlimbs) {
  CKG_API_BEGIN
  Context& c = ctx_of(ctx);
  if (first_prime + nlimbs > c.primes.size()) throw Error(CKG_INVALID_PARAMS, "prime index out of range");
  c.activate();
  ScalarTable st{};
  std::vector<LimbRef> refs;
  for (uint32_t i = 0; i < nlimbs; ++i) {
    const uint32_t p = first_prime + i;
    st.w[p] = scalar % c.mods[p].q;
    st.ws[p] = c.mods[p].shoup(st.w[p]);
    refs.push_back(LimbRef{a + i * c.n, out + i * c.n, p, 0});
  }
  launch_scalar(c.dt, refs.data(), (int)refs.size(), st, c.stream);
  check_launch();
  CKG_API_END
}

int ckg_automorphism(ckg_ctx* ctx, const uint64_t* in, uint64_t* out, uint32_t nlimbs, uint64_t galois_elt) {
  CKG_API_BEGIN
  Context& c = ctx_of(ctx);
  if (galois_elt % 2 == 0 || galois_elt >= 2 * c.n) throw Error(CKG_INVALID_PARAMS, "Galois element must be odd and < 2N");
  if (nlimbs > c.primes.size()) throw Error(CKG_INVALID_PARAMS, "too many limbs");
  c.activate();
  const uint32_t* perm = c.perm(galois_elt);
  std::vector<LimbRef> refs;
  for (uint32_t i = 0; i < nlimbs; ++i) refs.push_back(LimbRef{in + i * c.n, out + i * c.n, i, 0});
  launch_unary(c.dt, refs.data(), (int)refs.size(), 3, nullptr, perm, c.stream);
  check_launch();
  CKG_API_END
}

int ckg_rescale(ckg_ctx* ctx, const uint64_t* in, uint32_t level, uint64_t* out) {
  CKG_API_BEGIN
  Context& c = ctx_of(ctx);
  if (level > c.L) throw Error(CKG_INVALID_PARAMS, "level above max_level");
  if (level == 0) throw Error(CKG_NO_LEVELS_LEFT, "cannot rescale at level 0");
  c.activate();
  rescale_many(c, {in}, level, {out});
  check_launch();
  CKG_API_END
}

int ckg_mod_up(ckg_ctx* ctx, const uint64_t* in, uint32_t level, uint32_t digit, uint64_t* out_q, uint64_t* out_p) {
  CKG_API_BEGIN
  Context& c = ctx_of(ctx);
  if (level > c.L) throw Error(CKG_INVALID_PARAMS, "level above max_level");
  if (digit >= c.digits_at(level)) throw Error(CKG_INVALID_PARAMS, "digit out of range for this level");
  c.activate();
  auto conv = c.alloc(conv_limbs(c, level) * c.n);
  mod_up_many(c, {in}, level, {conv->p});
  const uint64_t* base = conv->p + conv_offset_limbs(c, level, digit) * c.n;
  const uint32_t s = c.digit_start(digit), e = c.digit_end(digit, level), a = e - s;
  std::vector<LimbRef> refs;
  uint32_t t = 0;
  for (uint32_t i = 0; i <= level; ++i) {
    if (i >= s && i < e) refs.push_back(LimbRef{in + i * c.n, out_q + i * c.n, i, 0});
    else refs.push_back(LimbRef{base + (t++) * c.n, out_q + i * c.n, i, 0});
  }
  for (uint32_t j = 0; j < c.k; ++j)
    refs.push_back(LimbRef{base + (level + 1 - a + j) * c.n, out_p + j * c.n, c.p_prime(j), 0});
  launch_unary(c.dt, refs.data(), (int)refs.size(), 2, nullptr, nullptr, c.stream);
  check_launch();
  CKG_API_END
}

int ckg_mod_down(ckg_ctx* ctx, const uint64_t* q_part, uint32_t level, const uint64_t* p_part, uint64_t* out) {
  CKG_API_BEGIN
  Context& c = ctx_of(ctx);
  if (level > c.L) throw Error(CKG_INVALID_PARAMS, "level above max_level");
  c.activate();
  mod_down_many(c, {ModDownJob{q_part, p_part, out, nullptr, nullptr}}, level);
  check_launch();
  CKG_API_END
}

static int key_upload(ckg_ctx* ctx, const uint64_t* src, bool device_src, uint32_t parts, uint32_t q_limbs,
                      uint64_t galois_elt, ckg_key** out) {
  CKG_API_BEGIN
  Context& c = ctx_of(ctx);
  if (!parts || parts > c.dnum) throw Error(CKG_INVALID_PARAMS, "key parts must be in 1..=dnum");
  if (!q_limbs || q_limbs > c.L + 1) throw Error(CKG_INVALID_PARAMS, "key data limbs must be in 1..=L+1");
  if (galois_elt && (galois_elt % 2 == 0 || galois_elt >= 2 * c.n))
    throw Error(CKG_INVALID_PARAMS, "Galois element must be odd and < 2N");
  c.activate();
  auto k = std::make_shared<DevKey>();
  k->ctx = &c;
  k->parts = parts;
  k->q_limbs = q_limbs;
  k->elt = galois_elt;
  const size_t words = (size_t)parts * 2 * (q_limbs + c.k) * c.n;
  k->buf = c.alloc(words);
  CKG_CUDA(cudaMemcpyAsync(k->buf->p, src, words * 8, device_src ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                           c.stream));
  CKG_CUDA(cudaStreamSynchronize(c.stream));
  *out = new ckg_key{k};
  CKG_API_END
}

int ckg_key_upload(ckg_ctx* ctx, const uint64_t* host_key, uint32_t parts, uint32_t q_limbs, uint64_t galois_elt,
                   ckg_key** out) {
  return key_upload(ctx, host_key, false, parts, q_limbs, galois_elt, out);
}

int ckg_key_upload_device(ckg_ctx* ctx, const uint64_t* dev_key, uint32_t parts, uint32_t q_limbs, uint64_t galois_elt,
                          ckg_key** out) {
  return key_upload(ctx, dev_key, true, parts, q_limbs, galois_elt, out);
}

void ckg_key_free(ckg_key* key) { delete key; }
uint64_t ckg_key_bytes(const ckg_key* key) { return key && key->k ? key->k->buf->words * 8 : 0; }

int ckg_key_switch(ckg_ctx* ctx, const ckg_key* key, const uint64_t* in, uint32_t level, uint64_t* out_b,
                   uint64_t* out_a) {
  CKG_API_BEGIN
  Context& c = ctx_of(ctx);
  if (!key || !key->k) throw Error(CKG_INVALID_PARAMS, "null key");
  if (level > c.L) throw Error(CKG_INVALID_PARAMS, "level above max_level");
  c.activate();
  KsJob j;
  j.in = in;
  j.key = key->k.get();
  j.out_b = out_b;
  j.out_a = out_a;
  key_switch_many(c, {j}, level);
  check_launch();
  CKG_API_END
}

// ---- evaluator -------------------------------------------------------------------------

static Evaluator& ev_of(ckg_eval* e) {
  if (!e || !e->e) throw Error(CKG_INVALID_PARAMS, "null evaluator");
  return *e->e;
}
static const Ct& ct_of(const ckg_ct* c) {
  if (!c || !c->c) throw Error(CKG_INVALID_PARAMS, "null ciphertext");
  return c->c;
}
static const Pt& pt_of(const ckg_pt* p) {
  if (!p || !p->p) throw Error(CKG_INVALID_PARAMS, "null plaintext");
  return p->p;
}
static int emit(const Ct& c, ckg_ct** out) {
  check_launch();
  *out = new ckg_ct{c};
  return CKG_OK;
}

int ckg_eval_create(ckg_ctx* ctx, const ckg_key* relin, const ckg_key* const* galois, uint32_t ngal, uint32_t flags,
                    ckg_eval** out) {
  CKG_API_BEGIN
  Context& c = ctx_of(ctx);
  std::vector<KeyPtr> g;
  for (uint32_t i = 0; i < ngal; ++i) {
    if (!galois[i] || !galois[i]->k || !galois[i]->k->elt)
      throw Error(CKG_INVALID_PARAMS, "Galois keys need their Galois element");
    g.push_back(galois[i]->k);
  }
  EvalConfig cfg{(flags & CKG_HOIST) != 0, (flags & CKG_BSGS) != 0, (flags & CKG_LAZY_RELIN) != 0};
  *out = new ckg_eval{std::make_unique<Evaluator>(&c, relin ? relin->k : nullptr, g, cfg)};
  CKG_API_END
}

void ckg_eval_destroy(ckg_eval* ev) { delete ev; }

int ckg_eval_fork(const ckg_eval* ev, ckg_eval** out) {
  CKG_API_BEGIN
  if (!ev || !ev->e) throw Error(CKG_INVALID_PARAMS, "null evaluator");
  *out = new ckg_eval{ev->e->fork()};
  CKG_API_END
}

uint32_t ckg_eval_config(const ckg_eval* ev) {
  const EvalConfig& c = ev->e->config();
  return (c.hoist ? CKG_HOIST : 0) | (c.bsgs ? CKG_BSGS : 0) | (c.lazy_relin ? CKG_LAZY_RELIN : 0);
}

void ckg_eval_counter(const ckg_eval* ev, uint64_t out[7]) {
  auto w = ev->e->counter().words();
  memcpy(out, w.data(), 7 * 8);
}
void ckg_eval_reset_counter(ckg_eval* ev) { ev->e->reset_counter(); }
void ckg_eval_add_counts(ckg_eval* ev, const uint64_t c[7]) {
  OpCounter o;
  o.rotations = c[0];
  o.relins = c[1];
  o.ct_ct_tensor = c[2];
  o.ct_pt_mults = c[3];
  o.rescales = c[4];
  o.sse_switches = c[5];
  o.bootstraps = c[6];
  ev->e->add_counts(o);
}
int ckg_eval_has_relin_key(const ckg_eval* ev) { return ev->e->has_relin_key() ? 1 : 0; }
int ckg_eval_has_galois_key(const ckg_eval* ev, int32_t step) { return ev->e->has_galois_key(step) ? 1 : 0; }

int ckg_ct_upload(ckg_eval* ev, const uint64_t* host, uint32_t ncomp, uint32_t level, double scale, ckg_ct** out) {
  CKG_API_BEGIN
  return emit(ev_of(ev).upload(host, false, ncomp, level, scale), out);
  CKG_API_END
}

int ckg_ct_upload_device(ckg_eval* ev, const uint64_t* dev, uint32_t ncomp, uint32_t level, double scale,
                         ckg_ct** out) {
  CKG_API_BEGIN
  return emit(ev_of(ev).upload(dev, true, ncomp, level, scale), out);
  CKG_API_END
}

static void copy_out(const Ct& c, uint64_t* dst, cudaMemcpyKind kind) {
  Context& x = *c->ctx;
  x.activate();
  const size_t words = (size_t)(c->level + 1) * x.n;
  if (c->comp_stride == words) {
    CKG_CUDA(cudaMemcpyAsync(dst, c->comp(0), c->ncomp * words * 8, kind, x.stream));
  } else {
    CKG_CUDA(cudaMemcpy2DAsync(dst, words * 8, c->comp(0), c->comp_stride * 8, words * 8, c->ncomp, kind, x.stream));
  }
}

int ckg_ct_download(const ckg_ct* ct, uint64_t* host) {
  CKG_API_BEGIN
  const Ct& c = ct_of(ct);
  copy_out(c, host, cudaMemcpyDeviceToHost);
  CKG_CUDA(cudaStreamSynchronize(c->ctx->stream));
  CKG_API_END
}

int ckg_ct_download_async(const ckg_ct* ct, uint64_t* host) {
  CKG_API_BEGIN
  copy_out(ct_of(ct), host, cudaMemcpyDeviceToHost);
  CKG_API_END
}

int ckg_ct_download_device(const ckg_ct* ct, uint64_t* dev) {
  CKG_API_BEGIN
  copy_out(ct_of(ct), dev, cudaMemcpyDeviceToDevice);
  CKG_API_END
}

void ckg_ct_info(const ckg_ct* ct, uint32_t* ncomp, uint32_t* level, double* scale) {
  if (ncomp) *ncomp = ct->c->ncomp;
  if (level) *level = ct->c->level;
  if (scale) *scale = ct->c->scale;
}

ckg_ct* ckg_ct_clone(const ckg_ct* ct) { return new ckg_ct{ct->c}; }
void ckg_ct_free(ckg_ct* ct) { delete ct; }
int ckg_eval_owns(const ckg_eval* ev, const ckg_ct* ct) { return ev && ev->e && ct && ev->e->owns(ct->c) ? 1 : 0; }

int ckg_pt_upload(ckg_eval* ev, const uint64_t* host, uint32_t level, double scale, ckg_pt** out) {
  CKG_API_BEGIN
  *out = new ckg_pt{ev_of(ev).upload_pt(host, false, level, scale)};
  check_launch();
  CKG_API_END
}
int ckg_pt_upload_device(ckg_eval* ev, const uint64_t* dev, uint32_t level, double scale, ckg_pt** out) {
  CKG_API_BEGIN
  *out = new ckg_pt{ev_of(ev).upload_pt(dev, true, level, scale)};
  check_launch();
  CKG_API_END
}
int ckg_ct_upload_overlap(ckg_eval* ev, const uint64_t* host, uint32_t ncomp, uint32_t level, double scale,
                          ckg_ct** out) {
  CKG_API_BEGIN
  if (!out) throw Error(CKG_INVALID_PARAMS, "null output");
  return emit(ev_of(ev).upload_overlapped(host, ncomp, level, scale), out);
  CKG_API_END
}

int ckg_pt_upload_overlap(ckg_eval* ev, const uint64_t* host, uint32_t level, double scale, ckg_pt** out) {
  CKG_API_BEGIN
  if (!out) throw Error(CKG_INVALID_PARAMS, "null output");
  *out = new ckg_pt{ev_of(ev).upload_pt_overlapped(host, level, scale)};
  check_launch();
  CKG_API_END
}

int ckg_ct_download_overlap(const ckg_ct* ct, uint64_t* host) {
  CKG_API_BEGIN
  const Ct& c = ct_of(ct);
  if (!host) throw Error(CKG_INVALID_PARAMS, "null host buffer");
  const size_t words = (size_t)(c->level + 1) * c->ctx->n;
  c->ctx->download_overlapped(c->buf, c->comp(0), words, c->comp_stride, c->ncomp, host);
  CKG_API_END
}

int ckg_ct_upload_overlap_list(ckg_eval* ev, uint32_t count, const uint64_t* const* hosts, const uint32_t* ncomp,
                               const uint32_t* levels, const double* scales, ckg_ct** out) {
  CKG_API_BEGIN
  if (count && (!hosts || !ncomp || !levels || !scales || !out)) throw Error(CKG_INVALID_PARAMS, "null list");
  std::vector<Evaluator::CtUpload> items(count);
  for (uint32_t i = 0; i < count; ++i) items[i] = {hosts[i], ncomp[i], levels[i], scales[i]};
  std::vector<Ct> cts = ev_of(ev).upload_overlapped_list(items);
  for (uint32_t i = 0; i < count; ++i) out[i] = new ckg_ct{cts[i]};
  check_launch();
  CKG_API_END
}

int ckg_pt_upload_overlap_list(ckg_eval* ev, uint32_t count, const uint64_t* const* hosts, const uint32_t* levels,
                               const double* scales, ckg_pt** out) {
  CKG_API_BEGIN
  if (count && (!hosts || !levels || !scales || !out)) throw Error(CKG_INVALID_PARAMS, "null list");
  std::vector<Evaluator::CtUpload> items(count);
  for (uint32_t i = 0; i < count; ++i) items[i] = {hosts[i], 0, levels[i], scales[i]};
  std::vector<Pt> pts = ev_of(ev).upload_pt_overlapped_list(items);
  for (uint32_t i = 0; i < count; ++i) out[i] = new ckg_pt{pts[i]};
  check_launch();
  CKG_API_END
}

int ckg_ct_download_overlap_list(uint32_t count, const ckg_ct* const* cts, uint64_t* const* hosts) {
  CKG_API_BEGIN
  if (!count) return CKG_OK;
  if (!cts || !hosts) throw Error(CKG_INVALID_PARAMS, "null list");
  Context* ctx = ct_of(cts[0])->ctx;
  std::vector<Context::DevPart> parts(count);
  for (uint32_t i = 0; i < count; ++i) {
    const Ct& c = ct_of(cts[i]);
    if (!hosts[i]) throw Error(CKG_INVALID_PARAMS, "null host buffer");
    if (c->ctx != ctx) throw Error(CKG_INVALID_PARAMS, "ciphertexts of different contexts in one list");
    const size_t words = (size_t)(c->level + 1) * ctx->n;
    parts[i] = {&c->buf, c->comp(0), words, c->comp_stride, c->ncomp, hosts[i]};
  }
  ctx->download_overlapped_list(parts);
  CKG_API_END
}

void ckg_pt_info(const ckg_pt* pt, uint32_t* level, double* scale) {
  if (level) *level = pt->p->level;
  if (scale) *scale = pt->p->scale;
}
ckg_pt* ckg_pt_clone(const ckg_pt* pt) { return new ckg_pt{pt->p}; }
void ckg_pt_free(ckg_pt* pt) { delete pt; }

#define CKG_BIN(name, method)                                                  \
  int name(ckg_eval* ev, const ckg_ct* a, const ckg_ct* b, ckg_ct** out) {     \
    CKG_API_BEGIN                                                              \
    return emit(ev_of(ev).method(ct_of(a), ct_of(b)), out);                    \
    CKG_API_END                                                                \
  }
#define CKG_UN(name, method)                                  \
  int name(ckg_eval* ev, const ckg_ct* a, ckg_ct** out) {     \
    CKG_API_BEGIN                                             \
    return emit(ev_of(ev).method(ct_of(a)), out);             \
    CKG_API_END                                               \
  }

CKG_BIN(ckg_add, add)
CKG_BIN(ckg_sub, sub)
CKG_BIN(ckg_mul_no_relin, mul_no_relin)
CKG_BIN(ckg_mul, mul)
CKG_UN(ckg_negate, negate)
CKG_UN(ckg_relinearize, relinearize)
CKG_UN(ckg_rescale_ct, rescale)
CKG_UN(ckg_conjugate, conjugate)

int ckg_add_plain(ckg_eval* ev, const ckg_ct* a, const ckg_pt* p, ckg_ct** out) {
  CKG_API_BEGIN
  return emit(ev_of(ev).add_plain(ct_of(a), pt_of(p)), out);
  CKG_API_END
}
int ckg_mul_plain(ckg_eval* ev, const ckg_ct* a, const ckg_pt* p, ckg_ct** out) {
  CKG_API_BEGIN
  return emit(ev_of(ev).mul_plain(ct_of(a), pt_of(p)), out);
  CKG_API_END
}
int ckg_mul_scalar(ckg_eval* ev, const ckg_ct* a, double value, double target_scale, ckg_ct** out) {
  CKG_API_BEGIN
  return emit(ev_of(ev).mul_scalar(ct_of(a), value, target_scale), out);
  CKG_API_END
}
int ckg_mul_plain_to_scale(ckg_eval* ev, const ckg_ct* a, const ckg_pt* p, double target_scale, ckg_ct** out) {
  CKG_API_BEGIN
  return emit(ev_of(ev).mul_plain_to_scale(ct_of(a), pt_of(p), target_scale), out);
  CKG_API_END
}
int ckg_mod_switch_to_level(ckg_eval* ev, const ckg_ct* a, uint32_t level, ckg_ct** out) {
  CKG_API_BEGIN
  return emit(ev_of(ev).mod_switch_to_level(ct_of(a), level), out);
  CKG_API_END
}
int ckg_relabel(ckg_eval* ev, const ckg_ct* a, double scale, ckg_ct** out) {
  CKG_API_BEGIN
  return emit(ev_of(ev).relabel(ct_of(a), scale), out);
  CKG_API_END
}
int ckg_rotate(ckg_eval* ev, const ckg_ct* a, int32_t steps, ckg_ct** out) {
  CKG_API_BEGIN
  return emit(ev_of(ev).rotate(ct_of(a), steps), out);
  CKG_API_END
}

int ckg_hoisted_rotate(ckg_eval* ev, const ckg_ct* a, const int32_t* steps, uint32_t nsteps, ckg_ct** outs) {
  CKG_API_BEGIN
  auto v = ev_of(ev).hoisted_rotate(ct_of(a), std::vector<int32_t>(steps, steps + nsteps));
  check_launch();
  for (size_t i = 0; i < v.size(); ++i) outs[i] = new ckg_ct{v[i]};
  CKG_API_END
}

int ckg_exact_product_scale(const ckg_eval* ev, uint32_t level, double target_scale, double* out) {
  CKG_API_BEGIN
  if (!ev || !ev->e) throw Error(CKG_INVALID_PARAMS, "null evaluator");
  *out = ev->e->exact_product_scale(level, target_scale);
  CKG_API_END
}

int ckg_matvec_plain(ckg_eval* ev, uint32_t d, uint32_t stride, const ckg_pt* const* entries, const ckg_ct* x,
                     ckg_ct** out) {
  CKG_API_BEGIN
  std::vector<Pt> e;
  for (uint32_t i = 0; i < d; ++i) e.push_back(entries[i] ? entries[i]->p : nullptr);
  return emit(ev_of(ev).matvec_plain(d, stride, e, ct_of(x)), out);
  CKG_API_END
}

int ckg_matvec_enc(ckg_eval* ev, uint32_t d, uint32_t stride, const ckg_ct* const* entries, const ckg_ct* x,
                   ckg_ct** out) {
  CKG_API_BEGIN
  std::vector<Ct> e;
  for (uint32_t i = 0; i < d; ++i) e.push_back(entries[i] ? entries[i]->c : nullptr);
  return emit(ev_of(ev).matvec_enc(d, stride, e, ct_of(x)), out);
  CKG_API_END
}

}  // extern "C"

namespace {
template <class T, class H, class F>
std::vector<MatvecJob<T>> matvec_jobs(uint32_t njobs, const uint32_t* d, const uint32_t* stride, const H* const* entries,
                                      const ckg_ct* const* xs, F entry) {
  if (njobs && (!d || !stride || !entries || !xs)) throw Error(CKG_INVALID_PARAMS, "null job arrays");
  std::vector<MatvecJob<T>> jobs(njobs);
  size_t off = 0;
  for (uint32_t i = 0; i < njobs; ++i) {
    jobs[i].d = d[i];
    jobs[i].stride = stride[i];
    for (uint32_t k = 0; k < d[i]; ++k) jobs[i].entries.push_back(entries[off + k] ? entry(entries[off + k]) : nullptr);
    off += d[i];
    jobs[i].x = ct_of(xs[i]);
  }
  return jobs;
}
}  // namespace

extern "C" {

int ckg_matvec_enc_batch(ckg_eval* ev, uint32_t njobs, const uint32_t* d, const uint32_t* stride,
                         const ckg_ct* const* entries, const ckg_ct* const* xs, ckg_ct** outs) {
  CKG_API_BEGIN
  auto jobs = matvec_jobs<Ct>(njobs, d, stride, entries, xs, [](const ckg_ct* e) { return e->c; });
  auto v = ev_of(ev).matvec_enc_batch(jobs);
  check_launch();
  for (size_t i = 0; i < v.size(); ++i) outs[i] = new ckg_ct{v[i]};
  CKG_API_END
}

int ckg_matvec_plain_batch(ckg_eval* ev, uint32_t njobs, const uint32_t* d, const uint32_t* stride,
                           const ckg_pt* const* entries, const ckg_ct* const* xs, ckg_ct** outs) {
  CKG_API_BEGIN
  auto jobs = matvec_jobs<Pt>(njobs, d, stride, entries, xs, [](const ckg_pt* e) { return e->p; });
  auto v = ev_of(ev).matvec_plain_batch(jobs);
  check_launch();
  for (size_t i = 0; i < v.size(); ++i) outs[i] = new ckg_ct{v[i]};
  CKG_API_END
}

// ---- batched execution ------------------------------------------------------------------

static Batch& batch_of(ckg_batch* b) {
  if (!b || !b->b) throw Error(CKG_INVALID_PARAMS, "null batch");
  return *b->b;
}

int ckg_batch_create(ckg_eval* ev, ckg_batch** out) {
  CKG_API_BEGIN
  Evaluator& e = ev_of(ev);
  *out = new ckg_batch{std::make_unique<Batch>(&e), ev};
  CKG_API_END
}

void ckg_batch_destroy(ckg_batch* b) { delete b; }

int ckg_batch_mul_relin_rescale(ckg_batch* b, const ckg_ct* x, const ckg_ct* y, ckg_ct** out) {
  CKG_API_BEGIN
  *out = new ckg_ct{batch_of(b).mul_relin_rescale(ct_of(x), ct_of(y))};
  CKG_API_END
}

int ckg_batch_rotate(ckg_batch* b, const ckg_ct* x, int32_t steps, ckg_ct** out) {
  CKG_API_BEGIN
  *out = new ckg_ct{batch_of(b).rotate(ct_of(x), steps)};
  CKG_API_END
}

int ckg_batch_mul_plain_rescale(ckg_batch* b, const ckg_ct* x, const ckg_pt* p, ckg_ct** out) {
  CKG_API_BEGIN
  *out = new ckg_ct{batch_of(b).mul_plain_rescale(ct_of(x), pt_of(p))};
  CKG_API_END
}

int ckg_batch_run(ckg_batch* b) {
  CKG_API_BEGIN
  batch_of(b).run();
  CKG_API_END
}

int ckg_batch_capture_graph(ckg_batch* b) {
  CKG_API_BEGIN
  batch_of(b).capture_graph();
  CKG_API_END
}

int ckg_batch_launch_graph(ckg_batch* b) {
  CKG_API_BEGIN
  batch_of(b).launch_graph();
  CKG_API_END
}

uint64_t ckg_batch_key_switches(const ckg_batch* b) { return b && b->b ? b->b->key_switches() : 0; }

int ckg_ctx_set_ntt_wave(ckg_ctx* ctx, int32_t limbs) {
  CKG_API_BEGIN
  if (limbs < 0 || limbs > 65536) throw Error(CKG_INVALID_PARAMS, "NTT wave must be in 0..=65536 limbs");
  ctx_of(ctx).dt.ntt_wave = limbs;
  CKG_API_END
}

int32_t ckg_ctx_ntt_wave(ckg_ctx* ctx) { return ctx && ctx->c ? ctx->c->dt.ntt_wave : -1; }

int ckg_ctx_set_bconv_tc(ckg_ctx* ctx, int32_t on) {
  CKG_API_BEGIN
  Context& c = ctx_of(ctx);
  if (on < 0 || on > 2) throw Error(CKG_INVALID_PARAMS, "conversion engine mode must be 0, 1 or 2");
  if (on) {
    bool big = c.log_n >= 7;
    for (uint64_t v : c.primes) big = big && v >= (1ULL << 30);
    if (!big) throw Error(CKG_INVALID_PARAMS, "tensor-core conversion needs N >= 2^7 and primes of at least 30 bits");
  }
  c.dt.bconv_tc = on;
  CKG_API_END
}

int32_t ckg_ctx_bconv_tc(ckg_ctx* ctx) { return ctx && ctx->c ? ctx->c->dt.bconv_tc : -1; }

int ckg_ctx_set_ntt_tma(ckg_ctx* ctx, int32_t on) {
  CKG_API_BEGIN
  ctx_of(ctx).dt.ntt_tma = on ? 1 : 0;
  CKG_API_END
}

int32_t ckg_ctx_ntt_tma(ckg_ctx* ctx) { return ctx && ctx->c ? ctx->c->dt.ntt_tma : -1; }

int ckg_batch_set_chunk_items(ckg_batch* b, int32_t items) {
  CKG_API_BEGIN
  if (items < 1) throw Error(CKG_INVALID_PARAMS, "chunk size must be positive");
  batch_of(b).set_chunk_items((size_t)items);
  CKG_API_END
}

int32_t ckg_batch_chunk_items(const ckg_batch* b) { return b && b->b ? (int32_t)b->b->chunk_items() : -1; }

int ckg_batch_autotune(ckg_batch* b, int32_t reps, int32_t* trials, int32_t max_trials, int32_t* n_trials) {
  CKG_API_BEGIN
  if (!n_trials || (max_trials > 0 && !trials)) throw Error(CKG_INVALID_PARAMS, "null output");
  const auto t = batch_of(b).autotune(reps);
  *n_trials = (int32_t)t.size();
  for (size_t i = 0; i < t.size() && (int32_t)i < max_trials; ++i) {
    trials[3 * i] = t[i].ntt_wave;
    trials[3 * i + 1] = t[i].chunk_items;
    trials[3 * i + 2] = (int32_t)(t[i].ms * 1000.0f + 0.5f);
  }
  CKG_API_END
}

// ---- SEAL wire format -----------------------------------------------------------------------

static uint64_t ring_degree(uint32_t log_n) {
  if (log_n < 1 || log_n > 17) throw Error(CKG_INVALID_PARAMS, "log_n outside [1, 17]");
  return 1ULL << log_n;
}

int ckg_seal_parms_id(uint32_t log_n, const uint64_t* m, uint32_t count, uint64_t out[4]) {
  CKG_API_BEGIN
  if (!out || (count && !m)) throw Error(CKG_INVALID_PARAMS, "null argument");
  const auto id = seal::parms_id(ring_degree(log_n), m, count);
  memcpy(out, id.data(), 32);
  CKG_API_END
}

uint64_t ckg_seal_bytes(uint32_t log_n, uint32_t ncomp, uint32_t level) {
  if (log_n < 1 || log_n > 17) return 0;
  return ncomp ? seal::ct_bytes(1ULL << log_n, ncomp, level + 1) : seal::pt_bytes(1ULL << log_n, level + 1);
}

int ckg_seal_encode(uint32_t log_n, const uint64_t* q, uint32_t nq, const uint64_t* words, uint32_t ncomp,
                    uint32_t level, double scale, uint8_t* out, uint64_t cap, uint64_t* len) {
  CKG_API_BEGIN
  const uint64_t n = ring_degree(log_n);
  if (!q || !words || !len) throw Error(CKG_INVALID_PARAMS, "null argument");
  if (level >= nq) throw Error(CKG_INVALID_PARAMS, "level above max_level");
  if (ncomp > 16) throw Error(CKG_INVALID_PARAMS, "a SEAL ciphertext has at most 16 components");
  *len = ncomp ? seal::ct_bytes(n, ncomp, level + 1) : seal::pt_bytes(n, level + 1);
  if (!out || cap < *len) throw Error(CKG_INVALID_PARAMS, "output buffer holds " + std::to_string(cap) +
                                                              " bytes, the object needs " + std::to_string(*len));
  if (ncomp) seal::encode_ct(n, q, words, ncomp, level, scale, out);
  else seal::encode_pt(n, q, words, level, scale, out);
  CKG_API_END
}

int ckg_seal_decode(uint32_t log_n, const uint64_t* q, uint32_t nq, const uint64_t* p, uint32_t np,
                    const uint8_t* bytes, uint64_t len, int plaintext, uint64_t* words, uint64_t cap,
                    uint64_t* nwords, uint32_t* ncomp, uint32_t* level, double* scale) {
  CKG_API_BEGIN
  const uint64_t n = ring_degree(log_n);
  if (!q || !nq || (np && !p) || !nwords) throw Error(CKG_INVALID_PARAMS, "null argument");
  auto r = plaintext ? seal::decode_pt(n, q, nq, p, np, bytes, len) : seal::decode_ct(n, q, nq, p, np, bytes, len);
  *nwords = r.words.size();
  if (!words || cap < r.words.size())
    throw Error(CKG_INVALID_PARAMS, "output buffer holds " + std::to_string(cap) + " words, the object has " +
                                        std::to_string(r.words.size()));
  memcpy(words, r.words.data(), r.words.size() * 8);
  if (ncomp) *ncomp = r.ncomp;
  if (level) *level = r.level;
  if (scale) *scale = r.scale;
  CKG_API_END
}

static seal::Parsed parse_for(const Context& c, const uint8_t* bytes, uint64_t len, bool plaintext) {
  const uint64_t* q = c.primes.data();
  const uint64_t* p = c.primes.data() + c.nq;
  return plaintext ? seal::decode_pt(c.n, q, c.nq, p, c.k, bytes, len) : seal::decode_ct(c.n, q, c.nq, p, c.k, bytes, len);
}

int ckg_ct_from_seal(ckg_eval* ev, const uint8_t* bytes, uint64_t len, ckg_ct** out) {
  CKG_API_BEGIN
  Evaluator& e = ev_of(ev);
  if (!out) throw Error(CKG_INVALID_PARAMS, "null output");
  auto r = parse_for(*e.ctx(), bytes, len, false);
  return emit(e.upload(r.words.data(), false, r.ncomp, r.level, r.scale), out);
  CKG_API_END
}

int ckg_pt_from_seal(ckg_eval* ev, const uint8_t* bytes, uint64_t len, ckg_pt** out) {
  CKG_API_BEGIN
  Evaluator& e = ev_of(ev);
  if (!out) throw Error(CKG_INVALID_PARAMS, "null output");
  auto r = parse_for(*e.ctx(), bytes, len, true);
  *out = new ckg_pt{e.upload_pt(r.words.data(), false, r.level, r.scale)};
  check_launch();
  CKG_API_END
}

int ckg_ct_to_seal(const ckg_ct* ct, uint8_t* out, uint64_t cap, uint64_t* len) {
  CKG_API_BEGIN
  const Ct& c = ct_of(ct);
  if (!len) throw Error(CKG_INVALID_PARAMS, "null length");
  const Context& x = *c->ctx;
  *len = seal::ct_bytes(x.n, c->ncomp, c->level + 1);
  if (!out || cap < *len) throw Error(CKG_INVALID_PARAMS, "output buffer holds " + std::to_string(cap) +
                                                              " bytes, the ciphertext needs " + std::to_string(*len));
  if (c->ncomp > 16) throw Error(CKG_INVALID_PARAMS, "a SEAL ciphertext has at most 16 components");
  std::vector<uint64_t> words((size_t)c->ncomp * (c->level + 1) * x.n);
  copy_out(c, words.data(), cudaMemcpyDeviceToHost);
  CKG_CUDA(cudaStreamSynchronize(x.stream));
  seal::encode_ct(x.n, x.primes.data(), words.data(), c->ncomp, c->level, c->scale, out);
  CKG_API_END
}

// ---- bootstrapping ------------------------------------------------------------------------

static BootParams boot_params_of(const uint32_t* bp) {
  if (!bp) throw Error(CKG_INVALID_PARAMS, "null boot parameters");
  BootParams b;
  b.log_slots = bp[0];
  b.ctos_levels = bp[1];
  b.evalmod_levels = bp[2];
  b.stoc_levels = bp[3];
  b.k_intervals = bp[4];
  b.cheb_degree = bp[5];
  b.double_angle = bp[6];
  return b;
}

static std::vector<LtPtr> stages_of(const ckg_lt* const* st, uint32_t n) {
  std::vector<LtPtr> v;
  for (uint32_t i = 0; i < n; ++i) {
    if (!st || !st[i] || !st[i]->lt) throw Error(CKG_INVALID_PARAMS, "null stage");
    v.push_back(st[i]->lt);
  }
  return v;
}

int ckg_boot_mul_const(ckg_eval* ev, const ckg_ct* a, double value, double scale, ckg_ct** out) {
  CKG_API_BEGIN
  return emit(ev_of(ev).boot_mul_const(ct_of(a), value, scale), out);
  CKG_API_END
}

int ckg_boot_add_const(ckg_eval* ev, const ckg_ct* a, double value, ckg_ct** out) {
  CKG_API_BEGIN
  return emit(ev_of(ev).boot_add_const(ct_of(a), value), out);
  CKG_API_END
}

int ckg_boot_zero(ckg_eval* ev, uint32_t level, double scale, ckg_ct** out) {
  CKG_API_BEGIN
  return emit(ev_of(ev).boot_zero(level, scale), out);
  CKG_API_END
}

int ckg_boot_relabel(ckg_eval* ev, const ckg_ct* a, double scale, ckg_ct** out) {
  CKG_API_BEGIN
  return emit(ev_of(ev).relabel(ct_of(a), scale), out);
  CKG_API_END
}

int ckg_mul_by_x_half(ckg_eval* ev, const ckg_ct* a, ckg_ct** out) {
  CKG_API_BEGIN
  return emit(ev_of(ev).mul_by_x_half(ct_of(a)), out);
  CKG_API_END
}

int ckg_mod_raise(ckg_eval* ev, const ckg_ct* a, const ckg_key* to_sparse, const ckg_key* to_dense, ckg_ct** out) {
  CKG_API_BEGIN
  if (!to_sparse || !to_sparse->k || !to_dense || !to_dense->k) throw Error(CKG_INVALID_PARAMS, "null SSE key");
  return emit(ev_of(ev).mod_raise(ct_of(a), *to_sparse->k, *to_dense->k), out);
  CKG_API_END
}

int ckg_lt_create(int direction, uint32_t level, double scale, uint32_t d, uint32_t stride, int64_t offset,
                  const ckg_pt* const* entries, const ckg_pt* const* second, ckg_lt** out) {
  CKG_API_BEGIN
  if (!out) throw Error(CKG_INVALID_PARAMS, "null output");
  if (direction != DIR_COEFF_TO_SLOT && direction != DIR_SLOT_TO_COEFF)
    throw Error(CKG_INVALID_PARAMS, "direction must be 0 (CoeffToSlot) or 1 (SlotToCoeff)");
  if (!d || (d & (d - 1))) throw Error(CKG_INVALID_PARAMS, "d must be a power of two");
  if (!(offset <= 0 && offset > -(int64_t)d))
    throw Error(CKG_INVALID_PARAMS, "diagonal offset outside -d < offset <= 0");
  if (!entries) throw Error(CKG_INVALID_PARAMS, "null entries");
  auto lt = std::make_shared<LinearTransform>();
  lt->direction = direction;
  lt->level = level;
  lt->scale = scale;
  auto fill = [&](SparseDiag& sd, const ckg_pt* const* es) {
    auto bg = bsgs_split(d);
    sd.d = d;
    sd.baby = bg.first;
    sd.giant = bg.second;
    sd.stride = stride;
    sd.offset = offset;
    for (uint32_t i = 0; i < d; ++i) sd.entries.push_back(es[i] && es[i]->p ? es[i]->p : Pt());
  };
  fill(lt->diags, entries);
  if (second) {
    lt->has_second = true;
    fill(lt->second, second);
  }
  *out = new ckg_lt{lt};
  CKG_API_END
}

void ckg_lt_free(ckg_lt* lt) { delete lt; }

int ckg_coeff_to_slot(ckg_eval* ev, const ckg_ct* a, const ckg_lt* const* stages, uint32_t n, ckg_ct** re,
                      ckg_ct** im) {
  CKG_API_BEGIN
  auto r = coeff_to_slot(ev_of(ev), ct_of(a), stages_of(stages, n));
  check_launch();
  *re = new ckg_ct{r.first};
  *im = new ckg_ct{r.second};
  CKG_API_END
}

int ckg_slot_to_coeff(ckg_eval* ev, const ckg_ct* re, const ckg_ct* im, const ckg_lt* const* stages, uint32_t n,
                      ckg_ct** out) {
  CKG_API_BEGIN
  return emit(slot_to_coeff(ev_of(ev), ct_of(re), ct_of(im), stages_of(stages, n)), out);
  CKG_API_END
}

int ckg_eval_chebyshev(ckg_eval* ev, const ckg_ct* a, const double* coeffs, uint32_t n, double lo, double hi,
                       double target_scale, ckg_ct** out) {
  CKG_API_BEGIN
  if (!coeffs && n) throw Error(CKG_INVALID_PARAMS, "null coefficients");
  return emit(eval_chebyshev_to_scale(ev_of(ev), ct_of(a), std::vector<double>(coeffs, coeffs + n), lo, hi,
                                      target_scale),
              out);
  CKG_API_END
}

int ckg_eval_mod(ckg_eval* ev, const ckg_ct* a, const uint32_t* bp, const double* coeffs, uint32_t n, ckg_ct** out) {
  CKG_API_BEGIN
  if (!coeffs && n) throw Error(CKG_INVALID_PARAMS, "null coefficients");
  return emit(eval_mod(ev_of(ev), ct_of(a), boot_params_of(bp), std::vector<double>(coeffs, coeffs + n)), out);
  CKG_API_END
}

int ckg_boot_create(ckg_ctx* ctx, const uint32_t* bp, const ckg_lt* const* ctos, uint32_t nctos,
                    const ckg_lt* const* stoc, uint32_t nstoc, const ckg_key* const* galois, uint32_t ngal,
                    const ckg_key* to_sparse, const ckg_key* to_dense, const double* coeffs, uint32_t ncoeffs,
                    const double* scales, ckg_boot** out) {
  CKG_API_BEGIN
  if (!out || !scales || (!coeffs && ncoeffs)) throw Error(CKG_INVALID_PARAMS, "null argument");
  std::vector<KeyPtr> gk;
  for (uint32_t i = 0; i < ngal; ++i) {
    if (!galois || !galois[i] || !galois[i]->k) throw Error(CKG_INVALID_PARAMS, "null Galois key");
    gk.push_back(galois[i]->k);
  }
  KeyPtr ts = to_sparse ? to_sparse->k : KeyPtr(), td = to_dense ? to_dense->k : KeyPtr();
  *out = new ckg_boot{std::make_unique<Bootstrapper>(&ctx_of(ctx), boot_params_of(bp), stages_of(ctos, nctos),
                                                     stages_of(stoc, nstoc), gk, ts, td,
                                                     std::vector<double>(coeffs, coeffs + ncoeffs), scales[0],
                                                     scales[1], scales[2])};
  CKG_API_END
}

void ckg_boot_destroy(ckg_boot* b) { delete b; }

int ckg_bootstrap(ckg_boot* b, ckg_eval* ev, const ckg_ct* a, ckg_ct** out) {
  CKG_API_BEGIN
  if (!b || !b->b) throw Error(CKG_INVALID_PARAMS, "null bootstrapper");
  return emit(b->b->bootstrap(ev_of(ev), ct_of(a)), out);
  CKG_API_END
}

uint32_t ckg_boot_output_level(const ckg_boot* b) { return b && b->b ? b->b->output_level() : 0; }

// ---- bootstrap setup ---------------------------------------------------------------------

int ckg_encode_complex(ckg_eval* ev, const double* values, uint32_t count, double scale, uint32_t level,
                       ckg_pt** out) {
  CKG_API_BEGIN
  if (!values && count) throw Error(CKG_INVALID_PARAMS, "null values");
  Evaluator& e = ev_of(ev);
  e.ctx()->activate();
  Pt p = encode_plaintext(e, values, count, scale, level);
  check_launch();
  *out = new ckg_pt{p};
  CKG_API_END
}

int ckg_encode_complex_host(uint32_t log_n, const uint64_t* q, uint32_t nq, const double* values, uint32_t count,
                            double scale, uint32_t level, uint64_t* out) {
  CKG_API_BEGIN
  if (log_n < 1 || log_n > 17) throw Error(CKG_INVALID_PARAMS, "log_n outside [1, 17]");
  if (!q || !nq || !out || (!values && count)) throw Error(CKG_INVALID_PARAMS, "null argument");
  auto v = encode_complex_coeffs(log_n, q, nq, values, count, scale, level);
  memcpy(out, v.data(), v.size() * 8);
  CKG_API_END
}

int ckg_boot_rotation_steps(const uint32_t* bp, int32_t* out, uint32_t cap, uint32_t* n) {
  CKG_API_BEGIN
  auto st = boot_rotation_steps(boot_params_of(bp));
  if (n) *n = (uint32_t)st.size();
  if (out)
    for (uint32_t i = 0; i < cap && i < st.size(); ++i) out[i] = st[i];
  CKG_API_END
}

int ckg_evalmod_coeffs(const uint32_t* bp, double* out, uint32_t cap) {
  CKG_API_BEGIN
  auto c = evalmod_coeffs(boot_params_of(bp));
  if (!out || cap < c.size()) throw Error(CKG_INVALID_PARAMS, "output holds fewer than cheb_degree + 1 values");
  memcpy(out, c.data(), c.size() * 8);
  CKG_API_END
}

int ckg_boot_plan(const uint32_t* bp, int direction, uint32_t stage, int64_t* info, uint8_t* kept) {
  CKG_API_BEGIN
  if (!info) throw Error(CKG_INVALID_PARAMS, "null output");
  auto plan = plan_boot_stages(boot_params_of(bp), direction);
  if (stage >= plan.size()) throw Error(CKG_INVALID_PARAMS, "stage index out of range");
  const StagePlan& p = plan[stage];
  info[0] = p.d;
  info[1] = p.stride;
  info[2] = p.offset;
  info[3] = p.has_second;
  info[4] = (int64_t)plan.size();
  if (kept)
    for (uint32_t i = 0; i < p.d; ++i) {
      kept[i] = p.kept[i];
      kept[p.d + i] = p.has_second ? p.kept2[i] : 0;
    }
  CKG_API_END
}

int ckg_boot_stage_scales(ckg_ctx* ctx, const uint32_t* bp, double delta, double* out2) {
  CKG_API_BEGIN
  auto s = boot_stage_scales(ctx_of(ctx), boot_params_of(bp), delta);
  out2[0] = s.first;
  out2[1] = s.second;
  CKG_API_END
}

int ckg_boot_encode_stages(ckg_eval* ev, const uint32_t* bp, int direction, double delta, ckg_lt** out,
                           uint32_t cap) {
  CKG_API_BEGIN
  Evaluator& e = ev_of(ev);
  e.ctx()->activate();
  auto st = encode_boot_stages(e, boot_params_of(bp), direction, delta);
  check_launch();
  if (!out || cap < st.size()) throw Error(CKG_INVALID_PARAMS, "output holds fewer handles than stages");
  for (size_t i = 0; i < st.size(); ++i) out[i] = new ckg_lt{st[i]};
  CKG_API_END
}

int ckg_boot_create_encoded(ckg_eval* ev, const uint32_t* bp, double delta, const ckg_key* const* galois,
                            uint32_t ngal, const ckg_key* to_sparse, const ckg_key* to_dense, ckg_boot** out) {
  CKG_API_BEGIN
  if (!out) throw Error(CKG_INVALID_PARAMS, "null output");
  Evaluator& e = ev_of(ev);
  e.ctx()->activate();
  const BootParams b = boot_params_of(bp);
  auto ctos = encode_boot_stages(e, b, DIR_COEFF_TO_SLOT, delta);
  auto stoc = encode_boot_stages(e, b, DIR_SLOT_TO_COEFF, delta);
  check_launch();
  std::vector<KeyPtr> gk;
  for (uint32_t i = 0; i < ngal; ++i) {
    if (!galois || !galois[i] || !galois[i]->k) throw Error(CKG_INVALID_PARAMS, "null Galois key");
    gk.push_back(galois[i]->k);
  }
  auto sc = boot_stage_scales(*e.ctx(), b, delta);
  KeyPtr ts = to_sparse ? to_sparse->k : KeyPtr(), td = to_dense ? to_dense->k : KeyPtr();
  *out = new ckg_boot{std::make_unique<Bootstrapper>(e.ctx(), b, ctos, stoc, gk, ts, td, evalmod_coeffs(b), sc.first,
                                                     sc.second, delta)};
  CKG_API_END
}

// ---- serving loop ------------------------------------------------------------------------

static Server& server_of(const ckg_server* s) {
  if (!s || !s->s) throw Error(CKG_INVALID_PARAMS, "null server");
  return *s->s;
}

int ckg_server_create(ckg_ctx* ctx, uint64_t hbm_budget_bytes, uint32_t max_batch_ks, uint32_t max_inflight,
                      uint32_t flags, ckg_server** out) {
  CKG_API_BEGIN
  if (!out) throw Error(CKG_INVALID_PARAMS, "null output");
  ServerConfig cfg;
  cfg.hbm_budget = hbm_budget_bytes;
  cfg.max_batch_ks = max_batch_ks;
  cfg.max_inflight = max_inflight;
  cfg.eval = EvalConfig{(flags & CKG_HOIST) != 0, (flags & CKG_BSGS) != 0, (flags & CKG_LAZY_RELIN) != 0};
  cfg.boot_lanes = (flags & CKG_SERVE_BOOT_LANES_2) ? 2 : (flags & CKG_SERVE_BOOT_LANE) ? 1 : 0;
  cfg.boot_priority = (flags & CKG_SERVE_LANES_EQUAL_PRIORITY) == 0;
  auto h = new ckg_server{std::make_unique<Server>(&ctx_of(ctx), cfg), hbm_budget_bytes};
  *out = h;
  CKG_API_END
}

void ckg_server_destroy(ckg_server* s) { delete s; }

int ckg_server_add_owner(ckg_server* s, uint32_t* owner) {
  CKG_API_BEGIN
  if (!owner) throw Error(CKG_INVALID_PARAMS, "null output");
  *owner = server_of(s).add_owner();
  CKG_API_END
}

int ckg_server_add_key(ckg_server* s, uint32_t owner, const uint64_t* key, int device_src, uint32_t parts,
                       uint32_t q_limbs, uint64_t galois_elt) {
  CKG_API_BEGIN
  server_of(s).add_key(owner, key, device_src != 0, parts, q_limbs, galois_elt);
  CKG_API_END
}

int ckg_server_add_sse_keys(ckg_server* s, uint32_t owner, const uint64_t* to_sparse, const uint64_t* to_dense,
                            int device_src) {
  CKG_API_BEGIN
  server_of(s).add_sse_keys(owner, to_sparse, to_dense, device_src != 0);
  CKG_API_END
}

int ckg_server_enable_bootstrap(ckg_server* s, const uint32_t* bp, double delta) {
  CKG_API_BEGIN
  server_of(s).enable_bootstrap(boot_params_of(bp), delta);
  check_launch();
  CKG_API_END
}

int ckg_server_submit_bootstrap(ckg_server* s, uint32_t owner, const ckg_ct* a, uint64_t* id) {
  CKG_API_BEGIN
  *id = server_of(s).submit_bootstrap(owner, ct_of(a));
  CKG_API_END
}

int ckg_server_submit_mul(ckg_server* s, uint32_t owner, const ckg_ct* a, const ckg_ct* b, uint64_t* id) {
  CKG_API_BEGIN
  *id = server_of(s).submit_mul(owner, ct_of(a), ct_of(b));
  CKG_API_END
}

int ckg_server_submit_rotate(ckg_server* s, uint32_t owner, const ckg_ct* a, int32_t steps, uint64_t* id) {
  CKG_API_BEGIN
  *id = server_of(s).submit_rotate(owner, ct_of(a), steps);
  CKG_API_END
}

int ckg_server_submit_mul_plain(ckg_server* s, uint32_t owner, const ckg_ct* a, const ckg_pt* p, uint64_t* id) {
  CKG_API_BEGIN
  *id = server_of(s).submit_mul_plain(owner, ct_of(a), pt_of(p));
  CKG_API_END
}

int ckg_server_submit_matvec(ckg_server* s, uint32_t owner, uint32_t d, uint32_t stride, const ckg_pt* const* diag,
                             const ckg_ct* x, uint64_t* id) {
  CKG_API_BEGIN
  if (!diag && d) throw Error(CKG_INVALID_PARAMS, "null diagonals");
  std::vector<Pt> ps;
  for (uint32_t i = 0; i < d; ++i) ps.push_back(pt_of(diag[i]));
  *id = server_of(s).submit_matvec(owner, d, stride, ps, ct_of(x));
  CKG_API_END
}

int ckg_server_result(ckg_server* s, uint64_t id, int64_t timeout_ms, ckg_ct** out, double* times_us) {
  int st = CKG_OK;
  CKG_API_BEGIN
  Ct c;
  std::string err;
  st = server_of(s).result(id, timeout_ms, &c, times_us, &err);
  if (st == CKG_TIMEOUT) return fail(CKG_TIMEOUT, "request still running");
  if (st != CKG_OK) return fail(st, err);
  if (out) *out = new ckg_ct{c};
  CKG_API_END
}

int ckg_server_cancel(ckg_server* s, uint64_t id, int* cancelled) {
  CKG_API_BEGIN
  const bool c = server_of(s).cancel(id);
  if (cancelled) *cancelled = c ? 1 : 0;
  CKG_API_END
}

int ckg_server_drain(ckg_server* s, int64_t timeout_ms) {
  CKG_API_BEGIN
  if (!server_of(s).drain(timeout_ms)) return fail(CKG_TIMEOUT, "requests still running");
  CKG_API_END
}

int ckg_server_stats(const ckg_server* s, uint64_t* out, uint32_t n) {
  CKG_API_BEGIN
  const ServerStats st = server_of(s).stats();
  const uint64_t w[17] = {st.submitted,       st.completed,      st.failed,         st.cancelled,
                          st.batches,         st.multi_owner_batches, st.max_batch_requests, st.key_hits,
                          st.key_misses,      st.key_evictions,  st.key_upload_bytes, st.key_bytes,
                          st.peak_key_bytes,  st.peak_device_bytes, st.budget_waits, st.pending,
                          s->budget};
  for (uint32_t i = 0; i < n && i < 17; ++i) out[i] = w[i];
  CKG_API_END
}

int ckg_server_owner_counter(const ckg_server* s, uint32_t owner, uint64_t* out7) {
  CKG_API_BEGIN
  const auto w = server_of(s).owner_counter(owner).words();
  for (int i = 0; i < 7; ++i) out7[i] = w[i];
  CKG_API_END
}

int ckg_server_inject_upload_failures(ckg_server* s, uint32_t count) {
  CKG_API_BEGIN
  server_of(s).inject_upload_failures(count);
  CKG_API_END
}

}  // extern "C"
