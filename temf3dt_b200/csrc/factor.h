#pragma once
#include "ctx.h"

namespace temf {
constexpr int kSnCols = 64;     // maximum supernode width (columns per panel)
constexpr int kUpdTile = 64;    // update tile edge

void build_factor_plan(temf_ctx& c);
// Doubles of one factor slot: the panels, then the scaled diagonal blocks.
inline int64_t slot_len(const temf_ctx& c) { return c.sym.stored + c.fplan.dsc_len; }
// Numeric LL^T of A = 3 M + 2 dt K into `slot`.  Returns 0 or the 1-based
// (original numbering) column of the first non-positive pivot.
int numeric_factor(temf_ctx& c, int slot, double dt);
// General form: L = LL^T factor of a*X + b*Y where X, Y are values on the
// permuted full pattern (device arrays).  Same return convention.
int numeric_factor_values(temf_ctx& c, int slot, const double* X, double a, const double* Y, double b);
// The same in two halves: enqueue every kernel on the context's stream, then
// (finish) wait for the stream and read the pivot status.  Factorisations of
// different contexts can run concurrently between the two calls.
void launch_factor(temf_ctx& c, int slot, double dt);
// indefinite: A = L S L^T with S = diag(+-1) (the reference's mtype -2 retry)
void launch_factor_values(temf_ctx& c, int slot, const double* X, double a, const double* Y, double b,
                          bool indefinite = false);
int finish_factor(temf_ctx& c, int slot);
// numeric_factor_values, and when A is not positive definite the indefinite
// factorisation into the same slot: returns 0 (LL^T) or the first
// non-positive pivot column (original numbering, 1-based) with a valid
// indefinite factor.
int numeric_factor_values_fallback(temf_ctx& c, int slot, const double* X, double a, const double* Y, double b);
}  // namespace temf
