#pragma once
#include <vector>

#include "ctx.h"
#include "fetd.h"

namespace temf {

// Schedule choices of the merged multi-model sweeps (picked by the autotuner).
struct BatchTuning {
  int order = 0;      // task merge: 0 proportional interleave, 1 level-aligned, 2 model after model
  int grid_pct = 100; // resident CTAs used, percent of what fits
};

struct BatchStats {
  double ms_total = 0, ms_factor = 0, ms_steps = 0, ms_tune = 0;
  int steps = 0;           // lockstep steps
  int64_t launches = 0;
  int64_t solves = 0;      // merged forward+backward sweep pairs
  std::vector<double> tune_ms;  // per candidate (order x grid), when tuned in this run
};

struct Batch {
  std::vector<temf_ctx*> models;
  int device = 0;
  cudaStream_t stream = nullptr;
  BatchTuning tune;
  bool tuned = false;
  BatchStats stats;
  std::vector<RunResult> results;
};

// Run the adaptive FETD loop (adap_euler) of every model in lockstep: each
// model keeps its own dt schedule, factors and accept/reject decisions; the
// triangular solves of all models of a step run as one merged forward and
// one merged backward persistent kernel.  Pulse types 1 and 2, one RHS each.
// `autotune` times the candidate schedules on the first step's factors and
// keeps the fastest (also stored in B.tune for later runs).
void run_batch(Batch& B, const RunOptions& o, bool autotune);

}  // namespace temf
