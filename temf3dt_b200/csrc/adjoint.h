#pragma once
#include <vector>

#include "ctx.h"

namespace temf {

struct AdjointResult {
  double ms_total = 0, ms_factor = 0;
  int n_nodes = 0, n_blocks = 0, n_factor = 0;
  int64_t launches = 0;
};

// Reverse sweep over the solve graph recorded by the last run.
//   dJ_dsamples: rows x nrec x 6 (E, dB/dt per receiver and output row)
//   tet_cell:    cell of each tet, 0-based, -1 outside the inversion grid
// Writes grad_cell[ncell] = dJ/dlog(sigma_c) and, if non-null,
// grad_tet[n_tets] = dJ/dsigma_t.
void run_adjoint(temf_ctx& c, const double* dJ_dsamples, int rows, const int* tet_cell, int ncell,
                 double* grad_cell, double* grad_tet, AdjointResult& res);

}  // namespace temf
