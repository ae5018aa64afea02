// Host-side bootstrap setup: what the reference's Bootstrapper::new prepares before any
// bootstrap runs (crates/ckks-train-ckks/src/bootstrap/bootstrapper.rs:250-290) -- the
// special-DFT stage matrices of CoeffToSlot and SlotToCoeff (bootstrap/linear.rs:78-455),
// adapted to the slot order with the folded factor and encoded at their levels and exact
// diagonal scales (linear.rs:512-677, linalg.rs:334-369, encoder.rs:215-283), the rotation
// steps they need, and the EvalMod Chebyshev series (bootstrap/evalmod.rs:58-96,
// bootstrap/poly.rs:90-140). The f64 steps follow the reference's operation order (num-complex
// 0.4 formulas, the C library's sin/cos/exp2/log2/pow/hypot), so every encoded diagonal has
// the reference's integer coefficients. Key generation is not here: keys come from the owner.
#pragma once
#include <cstdint>
#include <vector>

#include "boot.hpp"

namespace ckg {

// encode_complex (encoder.rs:215-283): the integer coefficients of `values` (re, im pairs,
// at most N/2 of them) at `scale`, reduced mod q_0..q_level (`primes` holds the nq data
// primes), coefficient form, limb-major. Host only.
std::vector<uint64_t> encode_complex_coeffs(uint32_t log_n, const uint64_t* primes, uint32_t nq, const double* values,
                                           size_t count, double scale, uint32_t level);

// Layout of one encoded stage without its values: the BSGS window and which pre-rotated
// entries are stored (non-zero) for the main and the second input. Host only.
struct StagePlan {
  uint32_t d = 0, stride = 0;
  int64_t offset = 0;
  bool has_second = false;
  std::vector<bool> kept, kept2;
};
std::vector<StagePlan> plan_boot_stages(const BootParams& bp, int direction);
// The same as a device plaintext (NTT form).
Pt encode_plaintext(Evaluator& ev, const double* values, size_t count, double scale, uint32_t level);

// galois_steps_for over both transforms (linear.rs:432-450): sorted, deduplicated, nonzero.
std::vector<int32_t> boot_rotation_steps(const BootParams& bp);

// evalmod_coeffs (evalmod.rs:58-96): degree cheb_degree series on [-1, 1].
std::vector<double> evalmod_coeffs(const BootParams& bp);

// stage_specs (bootstrapper.rs:207-230) + encode_stages (linear.rs:595-652) for one direction.
std::vector<LtPtr> encode_boot_stages(Evaluator& ev, const BootParams& bp, int direction, double delta);

// (evalmod_scale, stoc_input_scale) of stage_specs.
std::pair<double, double> boot_stage_scales(const Context& c, const BootParams& bp, double delta);

}  // namespace ckg
