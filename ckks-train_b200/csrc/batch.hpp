// Batched execution of many evaluator ops at uneven levels in one launch sequence.
//
// A Batch collects HMult+relinearize+rescale, rotation and plaintext-multiply+rescale ops
// on ciphertexts of any levels, with the evaluator's checks at enqueue time. Running it
// issues one launch per stage for all ops of a chunk (tensor products, Galois gathers,
// INTT, ModUp conversions, NTT, key inner products, ModDown, rescale), each over work lists
// resident in device memory, and can be captured once into a CUDA graph and replayed.
// Every result is bit-identical to the same op run on its own (the same kernels compute
// each ciphertext independently), and the OpCounter advances as the per-op calls would.
#pragma once
#include <vector>

#include "evaluator.hpp"

namespace ckg {

class Batch {
 public:
  explicit Batch(Evaluator* ev);
  ~Batch();

  // Each op is checked by, draws its keys from and is counted on `ev` (default: the
  // batch's evaluator), so one batch can serve the ops of several key owners.
  Ct mul_relin_rescale(const Ct& a, const Ct& b, Evaluator* ev = nullptr);
  Ct rotate(const Ct& a, int32_t steps, Evaluator* ev = nullptr);
  Ct mul_plain_rescale(const Ct& a, const Pt& p, Evaluator* ev = nullptr);

  void run();           // queues the whole batch on the context's stream
  void capture_graph(); // captures run()'s launches into a CUDA graph (once)
  void launch_graph();  // replays the graph
  uint64_t key_switches() const;
  size_t size() const { return items_.size(); }

  // Tuning. The chunk size (ops per launch sequence; default 128) applies at the next build
  // and drops a built batch and its graph. autotune() times every (NTT limb wave, chunk size)
  // pair of the grid below on this batch's own ops (`reps` graph replays each, after one
  // warm-up; no OpCounter change), leaves the fastest wave on the context and the fastest chunk
  // size on the batch (unbuilt), and returns every trial.
  struct Trial {
    int ntt_wave;
    int chunk_items;
    float ms;
  };
  void set_chunk_items(size_t items);
  size_t chunk_items() const { return chunk_items_; }
  std::vector<Trial> autotune(int reps);

  enum Kind { MUL = 0, ROT = 1, PMUL = 2 };
  // Device working words of one op (its share of the batch scratch) on a level-`level`,
  // `ncomp`-component input.
  static size_t scratch_words(const Context& c, int kind, uint32_t level, uint32_t ncomp);

 private:
  struct Item {
    Kind kind;
    Evaluator* ev = nullptr;
    Ct a, b, out;
    Pt p;
    uint64_t elt = 0;
    const DevKey* key = nullptr;
    bool trivial = false;  // rotation by a multiple of the slot count: out = a
  };
  struct Stage;  // device work lists of one chunk
  void build();
  void issue();
  void count_ops();
  void reset();  // drops the graph, work lists and scratch (the ops stay)

  Evaluator* ev_;
  Context* ctx_;
  std::vector<Item> items_;
  bool built_ = false;
  size_t chunk_items_;
  DevBufPtr scratch_;
  DevBufPtr desc_;
  std::vector<Stage*> chunks_;
  cudaGraph_t graph_ = nullptr;
  cudaGraphExec_t exec_ = nullptr;
};

}  // namespace ckg
