// Bootstrapping on the device: CoeffToSlot / SlotToCoeff stages, the level-optimal
// Chebyshev evaluation, EvalMod and the assembled pipeline (ModRaise with sparse-secret
// encapsulation -> CoeffToSlot -> EvalMod x2 -> SlotToCoeff), as the reference's generic
// bootstrap code runs them over its BootstrapArithmetic trait
// (crates/ckks-train-ckks/src/bootstrap/{bootstrapper,linear,poly,evalmod,modraise}.rs).
// Every step is an Evaluator op on the device; the host only walks the recursion and
// computes the f64 scale labels and integer constants, in the reference's operation order,
// so each ciphertext is bit-identical to the CPU bootstrap's.
//
// The encoded stage diagonals, EvalMod's Chebyshev coefficients and the keys are inputs
// (what the reference's Bootstrapper::new prepares on the host).
#pragma once
#include <memory>
#include <vector>

#include "evaluator.hpp"

namespace ckg {

enum Direction { DIR_COEFF_TO_SLOT = 0, DIR_SLOT_TO_COEFF = 1 };

// One CoeffToSlot or SlotToCoeff stage (bootstrap/linear.rs:482-497): diagonals at `level`
// and the exact scale after the stage's rescale; `second` are the diagonals of the
// conjugate (CoeffToSlot's last stage) or of `im` (SlotToCoeff's first stage).
struct LinearTransform {
  int direction = DIR_COEFF_TO_SLOT;
  SparseDiag diags;
  bool has_second = false;
  SparseDiag second;
  uint32_t level = 0;
  double scale = 0;
  std::vector<int32_t> rotation_steps() const;
};
typedef std::shared_ptr<const LinearTransform> LtPtr;

// BSGS rotation steps of a d-diagonal window at `stride` starting at `offset`
// (linalg.rs:465-497).
std::vector<int32_t> bsgs_rotation_steps_with_offset(uint32_t d, uint32_t stride, int64_t offset);

struct BootParams {  // bootstrap/params.rs:35-66
  uint32_t log_slots = 15, ctos_levels = 4, evalmod_levels = 7, stoc_levels = 4;
  uint32_t k_intervals = 13, cheb_degree = 127, double_angle = 0;
  uint32_t evalmod_depth() const;  // params.rs:123-126
};

std::pair<Ct, Ct> coeff_to_slot(Evaluator& ev, const Ct& ct, const std::vector<LtPtr>& ctos);
Ct slot_to_coeff(Evaluator& ev, const Ct& re, const Ct& im, const std::vector<LtPtr>& stoc);
Ct eval_chebyshev_to_scale(Evaluator& ev, const Ct& ct, const std::vector<double>& coeffs, double a, double b,
                           double target);
// EvalMod with the series `coeffs` (evalmod_coeffs(bp) of the reference).
Ct eval_mod(Evaluator& ev, const Ct& ct, const BootParams& bp, const std::vector<double>& coeffs);

class Bootstrapper {
 public:
  // `galois`: the rotation keys of the stages and the conjugation key; `to_sparse` /
  // `to_dense`: the SSE keys (both null: mod-raise under the main key); `delta`: the
  // preset scale a bootstrap input must carry.
  Bootstrapper(Context* ctx, const BootParams& bp, std::vector<LtPtr> ctos, std::vector<LtPtr> stoc,
               std::vector<KeyPtr> galois, KeyPtr to_sparse, KeyPtr to_dense, std::vector<double> coeffs,
               double evalmod_scale, double stoc_input_scale, double delta);
  // bootstrapper.rs:385-421: from a level-0 ciphertext at scale delta to output_level() at
  // delta; the run's counts plus one `bootstraps` are added to ev's counter.
  Ct bootstrap(Evaluator& ev, const Ct& ct);
  uint32_t output_level() const;
  Context* ctx() const { return ctx_; }

 private:
  Ct pipeline(Evaluator& inner, const Ct& ct);
  std::pair<Ct, Ct> eval_mod_pair(Evaluator& inner, const Ct& re, const Ct& im);
  Context* ctx_;
  BootParams bp_;
  std::vector<LtPtr> ctos_, stoc_;
  std::vector<KeyPtr> galois_;
  KeyPtr to_sparse_, to_dense_;
  std::vector<double> coeffs_;
  double evalmod_scale_, stoc_input_scale_, delta_;
};

}  // namespace ckg
