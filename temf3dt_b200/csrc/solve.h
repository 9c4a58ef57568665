#pragma once
#include <string>
#include <vector>

#include "ctx.h"

namespace temf {
// One model's view for the persistent sweeps: its schedule, factor and
// right-hand side.  The single-model kernels build it from their arguments;
// the multi-model kernels read one per task from a device array.
struct SweepView {
  const SolveTask* tasks;
  const int* sn_first;
  const int64_t* rows_ptr;
  const int* sn_rows;
  const int64_t* Lptr;
  double* const* Lbase;
  double* x;
  const int* tgt_ptr;      // forward: supernodes each task's rows feed; backward: owners of its rows
  const int* tgt;
  const int* expect;       // forward: chunk tasks feeding each supernode
  const int* nchunk;       // backward: row chunks per supernode
  const int64_t* part_off; // backward: partial-sum offsets
  double* part;
  int* sync;               // ready | ydone | cdone | xdone (nsn each) | counters
  int nsn;
  int ntask;
  // ready-queue scheduling (null queue: tasks are claimed in schedule order)
  int* queue;              // ntask slots: task + 1 once ready, 0 before
  int* qhead;              // pop counter
  int* qtail;              // push counter
  const int* diag_task;    // per supernode: index of its diagonal task in this sweep
  const int* dep_ptr;      // backward: per supernode, the tasks waiting for its x
  const int* dep;
  const int* need;         // backward: per task, completions it waits for
  int* cnt;                // backward: per task, completions so far
  int q_lo, q_hi;          // tasks [q_lo, q_hi) go through the queue, the rest are claimed in order
  int tag;                 // model id << 24 when several models share one queue (0 otherwise)
  int spin = 0;            // iterations a device wait may spin before it gives up (0: the default)
  double* bacc = nullptr;  // backward, one column: chunk partial sums accumulated per column (FP64 atomics)
  // single column: offsets (from the panel base) of the factor's scaled copies
  // of the diagonal blocks (unit lower triangle, reciprocal diagonal); null:
  // the tasks read the blocks from the panels
  const int64_t* Dptr = nullptr;
};

void build_solve_plan(temf_ctx& c);
// Host check of a symbolic analysis: supernode structure, then the sweep
// schedules replayed (both chunk heights; claim order and ready queue).
// Empty string, or the violation.
std::string check_schedules(const Symbolic& S);
void ensure_update_buffer(temf_ctx& c, int nrhs);

// x (device, permuted order, row-major n x nrhs) is overwritten: b -> A^{-1} b.
// `Lbase` points at a device word holding the panel base of the factor to use
// (an indirection so captured graphs can follow the factor slot).
// sgn != null: the factor is indefinite, L S L^T with S = diag(sgn) (applied
// between the sweeps).
void launch_solve(temf_ctx& c, double* const* Lbase, double* x, int nrhs, cudaStream_t st,
                  const double* sgn = nullptr);
// r = b - A x for the matrix factored in fs (permuted order, nrhs columns row-major)
void launch_residual(temf_ctx& c, const FactorSlot& fs, const double* x, const double* b, double* r, int nrhs,
                     cudaStream_t st);
// kernels launch_solve issues for nrhs columns
int solve_launch_count(const temf_ctx& c, int nrhs);
// Single right-hand side, every scratch word supplied by the caller: `sync`
// (4*nsn+4 ints, cleared here), `part` (part_len doubles), `err` (one int).
void launch_solve_scratch(temf_ctx& c, double* const* Lbase, double* x, int* sync, double* part, int* err,
                          cudaStream_t st);
// Timeout flag of the persistent solve kernels (0 = fine; 1..4 = which wait
// gave up).  Reading it synchronises the stream.
int solve_error_flag(temf_ctx& c);
void clear_solve_error_flag(temf_ctx& c);

// y = M (4 e2 - e3) for nrhs columns (row-major), permuted order.
void launch_bdf_rhs(temf_ctx& c, const double* e2, const double* e3, double* y, int nrhs, cudaStream_t st);
// y[src_idx] -= coef_dev[0] * src_coef   (source term of sys_right)
void launch_source(temf_ctx& c, const double* coef_dev, double* y, int nrhs, cudaStream_t st);
// receiver samples of x: out[rec*6 + q] = sum_j W[rec][q][j] x[edge_j]
void launch_receivers(temf_ctx& c, const double* x, int nrhs, double* out, cudaStream_t st);
// ||a-b||^2 and ||b||^2 per RHS column -> out[2*nrhs] (deterministic);
// `out` must hold two_error_len(nrhs) doubles (the tail is block partials).
inline size_t two_error_len(int nrhs) { return (size_t)(1 + 296) * 2 * nrhs; }
void launch_two_error(temf_ctx& c, const double* a, const double* b, int nrhs, double* out, cudaStream_t st);
// plain y = M x (full symmetric)
void launch_spmv(temf_ctx& c, const double* M, const double* x, double* y, int nrhs, cudaStream_t st);

// Many models at once: views of one model's sweeps (the forward view carries
// the forward schedule, the backward view the backward one; `sync` is that
// model's 4*nsn+4 words, cleared by the caller before each solve), the
// number of CTAs the merged kernels keep resident, and the launch of one
// forward and one backward merged sweep over (model, task) lists.  counters:
// two claim counters, cleared by the caller; err: timeout word.
SweepView fwd_view(temf_ctx& c, double* const* Lbase, double* x, int* sync);
SweepView bwd_view(temf_ctx& c, double* const* Lbase, double* x, int* sync);
int models_grid(bool forward);
// Autotuner of the sweeps' ready-queue split level (the supernodes below it
// are scheduled through the queue, the ones above are claimed in order with
// their panels prefetched): times one solve of nrhs columns with the factor
// in `slot` per candidate and keeps the fastest.  Returns the chosen level.
int tune_solve(temf_ctx& c, int slot, int nrhs);
// The single-column plan set explicitly: subtree level (0: none) and queue
// split level; checked on the host first.
void set_tree_plan(temf_ctx& c, int level, int split, bool leaders);
// Profiling aid: one single-column solve of b (permuted order) in `slot` with
// a per-task timeline (8 words per task; see solve.cu).
void solve_timeline(temf_ctx& c, int slot, const double* b_perm, int64_t cap, unsigned long long* out,
                    int* n_fwd, int* n_bwd);
// Merged sweeps with a shared ready queue: order_f/order_b list the models'
// in-order (above-split) tasks; the views carry the shared queues (forward
// and backward), each model's own queue range and completion counts; qlim_f,
// qlim_b = queued tasks of the active models.  counters: 2 claim counters.
void launch_solve_models(int nf, const int2* order_f, const SweepView* vf, int nb, const int2* order_b,
                         const SweepView* vb, const int* active, int* counters, int* err, int grid_f, int grid_b,
                         int qlim_f, int qlim_b, cudaStream_t st);
// queue ranges [0, f_hi) (forward) and [b_lo, nb) (backward) of a context's
// single-column schedule, and its initially ready queued tasks
void queue_ranges(const temf_ctx& c, int& f_hi, int& b_lo);
void queue_init_lists(const temf_ctx& c, std::vector<int>& finit, std::vector<int>& binit);
}  // namespace temf
