// The evaluator behind the C ABI: the HeOps contract (crates/ckks-train-ckks/src/ops.rs)
// with the checks in the CPU evaluator's order, its errors, f64 scale labels and
// OpCounter increments (crates/ckks-train-ckks/src/evaluator.rs, counter.rs), on
// device-resident ciphertexts. Ciphertexts are immutable and shared: every op returns a
// new one, and clone / relabel / mod_switch_to_level share the input's device buffer.
#pragma once
#include <array>
#include <memory>
#include <mutex>
#include <optional>
#include <vector>

#include "engine.hpp"

namespace ckg {

struct CtObj {
  Context* ctx = nullptr;
  DevBufPtr buf;
  size_t offset = 0;       // words from buf->p to component 0
  size_t comp_stride = 0;  // words between components (>= (level+1) * N)
  uint32_t ncomp = 0;
  uint32_t level = 0;
  double scale = 0;
  const uint64_t* comp(uint32_t i) const { return buf->p + offset + i * comp_stride; }
  uint64_t* comp_mut(uint32_t i) const { return buf->p + offset + i * comp_stride; }
};
typedef std::shared_ptr<const CtObj> Ct;

struct PtObj {
  Context* ctx = nullptr;
  DevBufPtr buf;
  size_t offset = 0;  // words from buf->p to limb 0
  uint32_t level = 0;
  double scale = 0;
  const uint64_t* data() const { return buf->p + offset; }
};
typedef std::shared_ptr<const PtObj> Pt;

struct OpCounter {  // counter.rs:42-58
  uint64_t rotations = 0, relins = 0, ct_ct_tensor = 0, ct_pt_mults = 0, rescales = 0, sse_switches = 0,
           bootstraps = 0;
  std::array<uint64_t, 7> words() const {
    return {rotations, relins, ct_ct_tensor, ct_pt_mults, rescales, sse_switches, bootstraps};
  }
};

struct EvalConfig {  // ops.rs:111-178
  bool hoist = true, bsgs = true, lazy_relin = true;
};

// Plaintext diagonals of a BSGS product with the all-zero entries left out
// (Diagonals<Option<Plaintext>>, linalg.rs:125-380): entry k1 * baby + k2 is diagonal
// offset + baby * k1 + k2 (times `stride`), pre-rotated by its giant step; null = skipped.
struct SparseDiag {
  uint32_t d = 0, baby = 0, giant = 0, stride = 1;
  int64_t offset = 0;
  std::vector<Pt> entries;
  uint32_t nonzero() const {
    uint32_t c = 0;
    for (auto& e : entries) c += e != nullptr;
    return c;
  }
  const Pt* first() const {  // plain_scale() source (linalg.rs:371-373)
    for (auto& e : entries)
      if (e) return &e;
    return nullptr;
  }
};

typedef std::shared_ptr<DevKey> KeyPtr;

// BSGS split of d diagonals into (baby, giant) steps (linalg.rs:419-424) and the rotation
// steps a d-diagonal mat-vec with `stride` needs keys for (linalg.rs:433-457).
std::pair<uint32_t, uint32_t> bsgs_split(uint32_t d);
std::vector<int32_t> rotation_steps(uint32_t d, uint32_t stride);

// One product of a batched BSGS call: W x with d pre-rotated diagonals at `stride` lanes.
template <class T>
struct MatvecJob {
  uint32_t d = 0, stride = 1;
  std::vector<T> entries;
  Ct x;
};

class Evaluator {
 public:
  Evaluator(Context* ctx, KeyPtr relin, std::vector<KeyPtr> galois, EvalConfig cfg);

  Context* ctx() const { return ctx_; }
  const EvalConfig& config() const { return cfg_; }
  OpCounter counter() const;
  void reset_counter();
  void add_counts(const OpCounter& c);
  std::unique_ptr<Evaluator> fork() const;
  bool has_relin_key() const { return (bool)relin_; }
  bool has_galois_key(int32_t step) const;
  bool owns(const Ct& ct) const { return ct && ct->ctx == ctx_; }

  Ct upload(const uint64_t* src, bool device_src, uint32_t ncomp, uint32_t level, double scale);
  Pt upload_pt(const uint64_t* src, bool device_src, uint32_t level, double scale);
  // The same from host memory on the context's upload stream (Context::upload_overlapped).
  Ct upload_overlapped(const uint64_t* host, uint32_t ncomp, uint32_t level, double scale);
  Pt upload_pt_overlapped(const uint64_t* host, uint32_t level, double scale);
  // A list of them in one allocation and one stream dependency; every entry is checked first.
  struct CtUpload {
    const uint64_t* host;
    uint32_t ncomp, level;
    double scale;
  };
  std::vector<Ct> upload_overlapped_list(const std::vector<CtUpload>& items);
  std::vector<Pt> upload_pt_overlapped_list(const std::vector<CtUpload>& items);  // ncomp unused

  Ct add(const Ct& a, const Ct& b) { return add_sub(a, b, false); }
  Ct sub(const Ct& a, const Ct& b) { return add_sub(a, b, true); }
  Ct negate(const Ct& a);
  Ct add_plain(const Ct& a, const Pt& p);
  Ct mul_plain(const Ct& a, const Pt& p);
  Ct mul_scalar(const Ct& a, double value, double target);
  Ct mul_plain_to_scale(const Ct& a, const Pt& p, double target);
  Ct mul_no_relin(const Ct& a, const Ct& b);
  Ct relinearize(const Ct& a);
  Ct mul(const Ct& a, const Ct& b);
  Ct rescale(const Ct& a);
  Ct mod_switch_to_level(const Ct& a, uint32_t level);
  Ct relabel(const Ct& a, double scale);
  Ct rotate(const Ct& a, int32_t steps);
  Ct conjugate(const Ct& a);
  std::vector<Ct> hoisted_rotate(const Ct& a, const std::vector<int32_t>& steps);
  // rotate() of several ciphertexts by their own steps: the key switches of each level as one
  // launch sequence (same results and counts as one rotate() per item)
  std::vector<Ct> rotate_many(const std::vector<std::pair<Ct, int32_t>>& items);
  // hoisted_rotate() of several ciphertexts, each by its own steps: at one level, one
  // decomposition and one key-switch launch sequence for all (same results and counts)
  std::vector<std::vector<Ct>> hoisted_rotate_many(const std::vector<std::pair<Ct, std::vector<int32_t>>>& items);
  double exact_product_scale(uint32_t level, double target) const;
  Ct matvec_plain(uint32_t d, uint32_t stride, const std::vector<Pt>& entries, const Ct& x);
  Ct matvec_enc(uint32_t d, uint32_t stride, const std::vector<Ct>& entries, const Ct& x);
  // Sum over terms of diag_t * x_t with shared giant rotations, skipping null entries and
  // the baby rotations only they would use (linalg.rs:741-799).
  Ct matvec_plain_sum_sparse(const std::vector<std::pair<const SparseDiag*, Ct>>& terms);
  // sum_t mul_plain(x_t, w_t) in one pass (operands checked by the caller: 2 components,
  // one level, equal scales); counts one ct_pt_mults per term as the separate ops would.
  Ct mac_plain(const std::vector<std::pair<Ct, Pt>>& terms);
  // sum_t mul_no_relin(a_t, b_t) in one pass (3 components; operands checked by the caller:
  // 2 components, one level > 0, equal scales); counts one ct_ct_tensor per term.
  Ct mac_tensor(const std::vector<std::pair<Ct, Ct>>& terms);
  // matvec_enc_batch (crates/ckks-train-cuda/src/evaluator.rs:437-520): every job checked as
  // matvec_enc, in order, before any work; results and counts equal those of the jobs run one
  // by one. With the optimized configuration the jobs run stage by stage together: all hoisted
  // baby rotations, all inner sums, all relinearizations, all giant rotations (one key-switch
  // launch sequence per stage and level); other configurations run the jobs one by one.
  std::vector<Ct> matvec_enc_batch(const std::vector<MatvecJob<Ct>>& jobs);
  // The same for plaintext diagonals (matvec_plain per job).
  std::vector<Ct> matvec_plain_batch(const std::vector<MatvecJob<Pt>>& jobs);
  void check_matvec_plain(uint32_t d, uint32_t stride, const std::vector<Pt>& entries, const Ct& x) const;
  void check_matvec_enc(uint32_t d, uint32_t stride, const std::vector<Ct>& entries, const Ct& x) const;

  // BootstrapArithmetic (bootstrap/poly.rs:453-486), ModRaise (bootstrap/modraise.rs) and
  // the exact monomial product of CoeffToSlot (bootstrap/linear.rs:921-936).
  void check_boot_input(const Ct& a) const;
  void check_conjugation_key() const;
  Ct boot_mul_const(const Ct& a, double value, double product_scale);
  Ct boot_add_const(const Ct& a, double value);
  Ct boot_zero(uint32_t level, double scale);
  Ct mul_by_x_half(const Ct& a);
  Ct mod_raise(const Ct& a, const DevKey& to_sparse, const DevKey& to_dense);
  Ct mod_raise_main_key(const Ct& a);
  bool relin_key_present() const { return (bool)relin_; }
  const std::vector<KeyPtr>& galois_keys() const { return galois_; }
  KeyPtr relin_key() const { return relin_; }
  void check_galois_input_pub(const Ct& a) const { check_galois_input(a); }
  void check_rotation_keys_pub(const std::vector<int32_t>& steps) const { check_rotation_keys(steps); }

 private:
  friend class Batch;
  Ct add_sub(const Ct& a, const Ct& b, bool sub);
  Ct new_ct(uint32_t ncomp, uint32_t level, double scale);
  void check_basis(const Ct& a) const;
  void check_basis_pt(const Pt& p) const;
  void check_mul_operands(const Ct& a, const Ct& b) const;
  void check_galois_input(const Ct& a) const;
  const DevKey& relin_key_checked() const;
  const DevKey& galois_key(uint64_t elt) const;
  void check_key_basis(const DevKey& k) const;
  std::optional<uint64_t> rotation_elt(int32_t steps) const;
  void check_rotation_keys(const std::vector<int32_t>& steps) const;
  Ct apply_galois(const Ct& a, uint64_t elt);
  template <class T>
  std::vector<Ct> bsgs_batch(const std::vector<MatvecJob<T>>& jobs);
  Ct raise_level0(const Ct& a);
  template <class F>
  void count(F f) {
    std::lock_guard<std::mutex> lk(mu_);
    f(counter_);
  }
  template <class T, class MulF, class FinF>
  Ct bsgs(uint32_t d, uint32_t stride, const std::vector<T>& entries, const Ct& x, MulF mul, FinF finish);

  Context* ctx_;
  KeyPtr relin_;
  std::vector<KeyPtr> galois_;
  EvalConfig cfg_;
  mutable std::mutex mu_;
  OpCounter counter_;
};

}  // namespace ckg
