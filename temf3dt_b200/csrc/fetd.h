#pragma once
#include <vector>

#include "ctx.h"

namespace temf {

struct RunOptions {
  int step_dvsi = 0;            // sp_division
  int step_dble = 0;            // sp_double
  int step_dblesize = 2;        // sp_dblesize
  double time_maximum = 0.0;    // time_maximum
  // Reproduce the build that wrote the shipped LINUX/*.field files: after an
  // accepted dt-doubling trial it restarted BDF2 from all_e(idx - sp_dblesize)
  // and advanced the time by one more old step than src/FETD_FWD.f90:1350,1405.
  int legacy_linux = 0;
  int use_graphs = 1;           // capture full dt segments as CUDA graphs
  const int* forced = nullptr;  // per trial: 1 accept, 0 reject, <0 own decision (test hook)
  int n_forced = 0;
  int max_steps = 0;            // 0: run to time_maximum
  int record_every = 0;         // >0: record the solve graph + checkpoints for the adjoint
};

struct RunResult {
  std::vector<int> steps;
  std::vector<double> times, dts;
  std::vector<double> samples;  // rows x nrec x 6 : (ex,ey,ez, dBx/dt,dBy/dt,dBz/dt)
  std::vector<double> trial_err;
  std::vector<int> trial_acc;
  double ms_factor = 0, ms_steps = 0, ms_total = 0;
  int n_factor = 0, n_solve = 0;
  int64_t launches = 0;
};

// dI/dt of the source waveform (time_const_p, src/FETD_UTILITY.f90:1050-1078)
double time_const_p(int source_type, int pulse_type, double t, double t0, double cur);
// receiver samples of x into trace row (row_base[0] + k)
void launch_receivers_row(temf_ctx& c, const double* x, int nrhs, const int* row_base, int k, double* trace,
                          cudaStream_t st);

// Adaptive BDF2 time loop (adap_euler, src/FETD_FWD.f90:1229-1464) on the GPU.
// Pulse type 3 runs the DC pass first (time_solver, :1212-1215).
void run_fetd(temf_ctx& c, const RunOptions& opt, RunResult& res);

}  // namespace temf
