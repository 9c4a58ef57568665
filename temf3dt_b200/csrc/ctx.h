// The library context: mesh, media, assembled matrices, symbolic plan,
// factor slots and the state of a running FETD simulation.
#pragma once
#include <memory>
#include <string>
#include <vector>

#include "common.h"
#include "symbolic.h"

namespace temf {

// Permuted full-symmetric CSR of the step-matrix pattern plus the list of
// element-matrix entries that sum into each nonzero (deterministic assembly).
struct Pattern {
  int n = 0;
  int64_t nnz = 0;
  std::vector<int> rowptr;       // n+1 (int32: nnz < 2^31 is checked)
  std::vector<int> col;          // nnz, ascending per row
  std::vector<int> contrib_ptr;  // nnz+1
  std::vector<int> contrib_idx;  // packed element entry: k * n_tets + t, k in [0,21)
};

// One entry of the factor update schedule: a 64x64 tile (rows i0.., cols j0..)
// of the Schur update L21 * L21^T of supernode s (indices into its row list),
// summed over the m = mj & 15 supernodes s-m+1 .. s (a run of column blocks
// of one wider supernode), restricted to columns j < mj >> 4 when that is > 0.
struct UpdTile {
  int s;
  int i0;
  int j0;
  int mj;
};

struct FactorPlan {
  // device copies of the supernode partition
  DBuf<int> sn_first, sn_parent, sn_rows, level_sn;
  DBuf<int64_t> sn_rows_ptr, sn_Lptr;
  std::vector<int> level_ptr;  // host
  // A -> L load map (lower triangle incl. diagonal of the permuted CSR)
  DBuf<int> a2l_src;           // CSR position
  DBuf<int64_t> a2l_dst;       // offset into the panels
  int64_t n_a2l = 0;
  // update scatter metadata
  DBuf<int> row_grp;           // per below-diagonal row entry: global target-group id
  DBuf<int> grp_target, grp_shift;
  DBuf<int64_t> grp_relind;    // rel index of row 0 of the source (tables shared by the blocks of a run)
  DBuf<int> relind;
  DBuf<UpdTile> tiles;
  std::vector<int64_t> tile_level_ptr;  // host, nlevels+1
  DBuf<int2> trsm;             // (supernode, first row) chunks of the row solves
  std::vector<int64_t> trsm_level_ptr;
  int64_t n_trsm = 0;
  int64_t n_relind = 0;
  int64_t n_tiles = 0;
  int n_runs = 0;              // runs of column blocks whose updates are summed
  // The single-column sweeps' copy of each diagonal block, after the panels in
  // the same slot allocation: c x c column-major, row i scaled by 1/L_ii
  // (unit lower triangle below the diagonal) and 1/L_ii on the diagonal.
  DBuf<int64_t> sn_Dptr;       // per supernode: offset of its copy (from the panel base)
  int64_t dsc_len = 0;         // doubles of all copies
};

// A task of the persistent triangular-solve kernels: the diagonal block of
// supernode s (kind 0) or rows [r0, r1) of its below-diagonal panel (kind 1).
struct SolveTask {
  int s;
  int kind;
  int r0;
  int r1;
};

// Ready-queue scheduling of a pair of sweep schedules: diagonal task per
// supernode (forward, backward), backward dependants and completion counts,
// initially ready tasks (stored as task + 1), and the per-solve queue words
// [fq: n_ftask][bq: n_btask][bcnt: n_btask][fhead, bhead, ftail, btail].
// The queue serves the supernodes below `split` (levels from the leaves); the
// tasks above it are claimed in schedule order with their panels prefetched
// before the dependency waits (forward tasks [0, f_hi), backward [b_lo, nb)
// are queued).
struct QueuePlan {
  DBuf<int> fdiag, bdiag, bdep_ptr, bdep, bneed, finit, binit, qtails;
  int n_finit = 0, n_binit = 0;
  int split = 0, f_hi = 0, b_lo = 0;
  bool tuned = false;
  std::vector<double> tune_ms;  // per candidate split, when tuned
  std::vector<int> tune_split;
  DBuf<int> qbuf;
};

// Single-column sweeps with the bottom of the tree cut into whole subtrees:
// the supernodes below `level` form disjoint subtrees (contiguous index ranges
// [first, root] of the postordered supernodes), each swept by one warp with
// no waits (k_fwd_subtrees before, k_bwd_subtrees after the task kernels);
// the task schedules and their ready-queue data cover the supernodes at or
// above `level` only.  level 0: no subtrees (the full schedules).
struct TreePlan {
  int level = 0;
  bool leaders = true;         // runs of column blocks above the queue split swept by one leader task
  int ntree = 0;
  DBuf<int2> trees;            // (first, root) per subtree, most stored panel values first
  DBuf<SolveTask> ftask, btask;
  int n_ftask = 0, n_btask = 0;
  DBuf<int> ftgt_ptr, ftgt, fexpect, btgt_ptr, btgt;
  QueuePlan q;
  DBuf<double> bacc;           // backward: per column, the sum of its supernode's chunk partials
  bool tuned = false;
  std::vector<int> tune_level;  // per candidate (level, split) when tuned; splits and times in q
};

struct SolvePlan {
  int64_t u_len = 0;           // sum over supernodes of the rows below the diagonal block
  // persistent schedules (tasks in an order where every wait targets an earlier task)
  DBuf<SolveTask> ftask, btask;
  int n_ftask = 0, n_btask = 0;
  DBuf<int> ftgt_ptr, ftgt;    // per forward task: supernodes whose columns its rows feed
  DBuf<int> fexpect;           // per supernode: forward chunk tasks feeding it
  DBuf<int> btgt_ptr, btgt;    // per backward task: supernodes owning its rows (solved first)
  DBuf<int> nchunk;            // per supernode: row chunks of its panel
  DBuf<int64_t> part_off;      // per supernode: offset of its backward partial sums
  int64_t part_len = 0;
  QueuePlan q1;                // ready-queue data of the schedules above
  // the same schedules with 64-row chunks for blocks of up to 64 right-hand sides
  DBuf<SolveTask> mftask, mbtask;
  int n_mftask = 0, n_mbtask = 0;
  DBuf<int> mftgt_ptr, mftgt, mfexpect, mbtgt_ptr, mbtgt, mnchunk;
  DBuf<int64_t> macc_off;      // per supernode with >= 2 chunks: row offset of its c x 64 accumulator
  int64_t macc_len = 0;
  QueuePlan qm;
  TreePlan tree;               // the single-column sweeps of temf_solve / temf_run
  DBuf<int> sync;              // ready | ydone | cdone | xdone (nsn each) | counters
  int nsn = 0;
};

struct FactorSlot {
  DBuf<double> L;
  bool valid = false;
  double dt = 0.0;
  int status = 0;
  // the matrix factored, a X + b Y on the permuted full pattern (device
  // arrays that outlive the factor: the iterative refinement applies it)
  const double* X = nullptr;
  const double* Y = nullptr;
  double a = 0.0, b = 0.0;
  // indefinite mode (the reference's mtype -2 retry): A = L S L^T, S = diag(sgn)
  bool indefinite = false;
  int perturbed = 0;          // pivots perturbed to +-tau
  DBuf<double> sgn;           // n, permuted order
};

struct Source {
  int nrhs = 0;
  int source_type = 1, pulse_type = 1;
  double t0 = 0.0, current = 0.0;
  // per RHS column: source entries (permuted edge index, drc*len)
  std::vector<int> ptr;        // nrhs+1
  std::vector<int> idx;        // permuted unknown index
  std::vector<int> rhs_col;    // which RHS column each entry belongs to
  std::vector<double> coef;    // drc * edge length
  DBuf<int> d_idx, d_col;
  DBuf<double> d_coef;
};

struct Receivers {
  int nrec = 0;
  std::vector<int> rec_tet;    // 0-based
  std::vector<int> rec_rhs;    // RHS column each receiver reads
  std::vector<double> xyz;     // nrec*3
  DBuf<int> d_edges;           // nrec*6 permuted unknown indices
  DBuf<int> d_rhs;
  DBuf<double> d_w;            // nrec*36: rows (ex,ey,ez,dx,dy,dz) x 6 edges, tet_drc folded in
  std::vector<double> w_host;  // same, copied back (n_arr/d_arr for checks)
};

// Record of a forward run for the adjoint: the solve graph (each node:
// dt, source scalar, the two history nodes it reads), the node each output row
// reports, and checkpoints of the last W node states taken before the first
// node of every block (every `every` nodes and wherever dt changes).
struct AdjointRecord {
  int every = 0;                 // 0: recording off
  bool valid = false;
  int W = 0;                     // history window (states a node may read, counted back)
  std::vector<double> dt, coef;  // per node k = 1..N at index k-1
  std::vector<int> a, b;
  std::vector<int> row_node;
  std::vector<int> ck_first;     // first node of each block
  std::vector<std::unique_ptr<DBuf<double>>> ck;  // W states: nodes ck_first-W .. ck_first-1
};

// Whole-mesh field dumps of the next temf_run (vtkout, src/FETD_FWD.f90:1642-1864):
// at every output row E and D at the tet centroids, B accumulated as D * dt,
// and a snapshot of E, D, B at the first row at or after each time.
struct MeshFieldPlan {
  std::vector<double> times;  // vtkout times (at most 30)
  std::vector<int> done;      // per time: its snapshot was taken in the last run
  DBuf<int> edges;            // per tet its 6 edges in the permuted order
  DBuf<double> b;             // tets x 3
  DBuf<double> snap;          // times x tets x 9 (E, D, B)
  DBuf<int> trig;             // per trace row: bit i = the row takes snapshot i
  DBuf<double> dt;            // [0]: the rows' dt
  int n() const { return (int)times.size(); }
};

}  // namespace temf

struct temf_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  // mesh (0-based, row-major per tet)
  int n_nodes = 0, n_tets = 0, n_edges = 0;
  std::vector<double> xyz;       // n_nodes*3
  std::vector<int> tet_vex;      // n_tets*4
  std::vector<int> edg_vex;      // n_edges*2
  std::vector<int> tet_edg;      // n_tets*6
  std::vector<int> tet_drc;      // n_tets*6
  std::vector<double> sig, mu;   // per tet
  // anisotropic media: per tet row-major 3 x 3 conductivity tensor and the
  // curl-curl tensor (elementwise reciprocal of the permeability tensor)
  bool aniso = false;
  std::vector<double> sig9, tm9;
  // first-order absorbing boundary: 4 face bits per tet (0: PEC, no term)
  int bound_cond = 0;
  std::vector<unsigned char> face_mask;
  bool have_mesh = false, have_media = false;
  // symbolic + pattern
  temf::SymbolicOptions sym_opt;
  temf::Symbolic sym;
  temf::Pattern pat;
  bool analysed = false;
  // device mesh / matrices
  temf::DBuf<double> d_xyz, d_sig, d_mu, d_sig9, d_tm9;
  temf::DBuf<unsigned char> d_face_mask;
  temf::DBuf<int> d_tet_vex, d_tet_drc;
  temf::DBuf<int> d_rowptr, d_col, d_contrib_ptr, d_contrib_idx;
  temf::DBuf<double> d_elemM, d_elemK, d_M, d_K;
  bool assembled = false;
  temf::FactorPlan fplan;
  temf::SolvePlan splan;
  temf::FactorSlot slots[2];
  temf::DBuf<int> d_status;      // device status words (pivot failure etc.)
  temf::Source src;
  temf::Receivers rec;
  // scratch vectors
  temf::DBuf<double> d_part;     // backward partial sums (part_len), or block accumulators (macc_len * 64)
  temf::AdjointRecord adj;
  temf::MeshFieldPlan mf;
  int u_nrhs = 0;
  // device waits of the sweeps: iterations before a wait gives up (0: the
  // default, about a second); inject_wait: the next single-column solve waits
  // once on a count that nothing completes (failure-detection test)
  int spin_limit = 0;
  int inject_wait = 0;
};
