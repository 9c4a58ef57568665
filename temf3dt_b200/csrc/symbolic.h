// Host-side symbolic analysis of the FETD step matrix  A(dt) = 3 M_sigma + 2 dt K.
//
// The pattern of A does not depend on dt (every entry of M and K comes from
// the same per-tetrahedron 6x6 blocks, src/FETD_FWD.f90:642-662), so the
// ordering, elimination tree and supernode partition are computed once per
// mesh and reused by every refactorisation at a dt-doubling point.  This
// replaces the reorder + symbolic part of PARDISO phase 12
// (src/FETD_UTILITY.f90:912-917) whose ordering the reference leaves at MKL's
// default (iparm = 0, :909-910).
#pragma once
#include <algorithm>
#include <cstdint>
#include <exception>
#include <memory>
#include <system_error>
#include <thread>
#include <vector>
#include <string>

namespace temf {

struct SymbolicOptions {
  int leaf_size = 96;          // nested-dissection leaf size
  int max_sn_cols = 64;        // supernodes are split into column blocks of at most this width
  bool amalgamate = true;      // relaxed supernode amalgamation
  int amalg_level = 2;         // 1: merge while the zero fraction stays small; 2: merge small supernodes harder;
                               // 3: also merge up to 64 columns at 25 % zeros (fewer bottom tasks)
  int threads = 0;             // host threads for the ordering (0: $TEMF_HOST_THREADS, else all cores);
                               // the result does not depend on it
};

struct Symbolic {
  int n = 0;
  std::vector<int> perm;        // perm[new] = old
  std::vector<int> iperm;       // iperm[old] = new
  // supernode partition (on the permuted matrix)
  int nsn = 0;
  std::vector<int> sn_first;        // nsn+1: first column of each supernode
  std::vector<int> sn_parent;       // parent supernode or -1
  std::vector<int64_t> sn_rows_ptr; // nsn+1: offsets of the below-diagonal row lists
  std::vector<int> sn_rows;         // below-diagonal rows (permuted indices, ascending)
  std::vector<int64_t> sn_Lptr;     // nsn+1: panel offsets in doubles; panel = (c+r) x c, column-major
  std::vector<int> col2sn;          // n
  std::vector<int> sn_level;        // bottom-up level (leaves = 0)
  int nlevels = 0;
  std::vector<int> level_ptr;       // nlevels+1
  std::vector<int> level_sn;        // supernodes grouped by level
  // statistics
  int64_t nnzL = 0;                 // nonzeros of L held by the supernodes (incl. amalgamation zeros)
  int64_t nnzL_exact = 0;           // structural nonzeros of L (sum of column counts)
  int64_t stored = 0;               // doubles stored in the panels
  double flops = 0.0;               // factor flops (mul+add counted as 2)
  double t_order = 0, t_etree = 0, t_colcount = 0, t_super = 0;
};

// Nested-dissection ordering on the symmetric graph (xadj/adj without the
// diagonal) using recursive coordinate bisection with vertex separators.
// Returns perm[new] = old.  Independent halves are ordered by up to
// `threads` host threads (0: $TEMF_HOST_THREADS, else all cores); the
// ordering is the same for any count.
std::vector<int> nested_dissection(int n, const int64_t* xadj, const int* adj,
                                   const double* xyz, int leaf_size, int threads = 0);

// Runs of column blocks: the supernodes that come from splitting one wider
// supernode into blocks of at most max_sn_cols columns.  q and q + 1 are
// consecutive blocks when q's parent is q + 1 and q's rows are exactly q + 1's
// columns followed by q + 1's rows.  run_first[s] = the first block of s's
// (maximal) run.
std::vector<int> block_run_first(const Symbolic& S);

// Update groups of the numeric factorisation.  The below-diagonal rows of a
// supernode s fall into runs owned by one ancestor t each (a group); the
// update of s scatters its rows i >= j (j = the group's first row) into t's
// panel at
//     column (sn_rows[j'] - first column of t), row rel[grp_rel[g] + i] - grp_shift[g].
// One relative-index table serves all the groups of s whose targets are
// blocks of one run T (t_0 .. t_e): it holds, for the rows of s from the
// first one owned by T, their positions in t_0's panel; a block t_q of the
// run shares the same order shifted by grp_shift = (first column of t_q) -
// (first column of t_0), since each block's rows are the later blocks'
// columns followed by the last block's rows.
struct UpdateGroups {
  std::vector<int> row_grp;      // per entry of Symbolic::sn_rows: its group
  std::vector<int> grp_target;   // per group: t
  std::vector<int> grp_shift;    // per group: first column of t - first column of its run's first block
  std::vector<int64_t> grp_rel;  // per group: rel index of row 0 of s (the table's start minus its first row)
  std::unique_ptr<int[]> rel;    // relative positions (uninitialised storage, all written)
  int64_t n_rel = 0;
};

// Builds the update groups with up to `threads` host threads (0:
// $TEMF_HOST_THREADS, else all cores); the result does not depend on the
// count.  Throws if a row of s is missing from its ancestor's structure.
void update_groups(const Symbolic& S, UpdateGroups& G, int threads = 0);
// Host check of the update groups: every row a supernode's update scatters
// lands on that row of its target panel.  Empty string, or the violation.
std::string check_update_groups(const Symbolic& S);

// Host threads to use for a request (0: $TEMF_HOST_THREADS, else the cores
// this process may run on, bounded by the cgroup CPU quota, at most 64).
int host_threads(int requested);

// Runs work(k) for k = 0 .. n-1: k >= 1 on new threads where one can be
// created, the rest on the calling thread; rethrows the first exception
// after all have finished.
template <class F>
void parallel_for_each(int n, F&& work) {
  std::vector<std::exception_ptr> failed(std::max(n, 1));
  std::vector<std::thread> pool;
  pool.reserve(std::max(n - 1, 0));
  std::vector<int> here{0};
  for (int k = 1; k < n; ++k) {
    try {
      pool.emplace_back([&work, &failed, k] {
        try {
          work(k);
        } catch (...) {
          failed[k] = std::current_exception();
        }
      });
    } catch (const std::system_error&) {
      here.push_back(k);
    }
  }
  for (int k : here) {
    if (k >= n) break;
    try {
      work(k);
    } catch (...) {
      failed[k] = std::current_exception();
    }
  }
  for (std::thread& t : pool) t.join();
  for (const std::exception_ptr& e : failed)
    if (e) std::rethrow_exception(e);
}

// Full symbolic analysis.  (xadj, adj) is the symmetric pattern of A in the
// original numbering without the diagonal; xyz gives a point per unknown
// (edge midpoints) for the geometric bisection.
void analyse(int n, const int64_t* xadj, const int* adj, const double* xyz,
             const SymbolicOptions& opt, Symbolic& out);

}  // namespace temf
