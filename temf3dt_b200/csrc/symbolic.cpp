// Nested dissection + elimination tree + supernodes for the FETD step matrix.
// See symbolic.h for what this replaces in the reference.
#include "symbolic.h"

#include <sched.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <numeric>
#include <stdexcept>
#include <thread>

namespace temf {

namespace {

double now_s() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

// ---------------------------------------------------------------------------
// Nested dissection by recursive coordinate bisection.
//
// For a subset, each coordinate axis is sorted once and the vertex separator
// of EVERY split position k (left = the k lowest along the axis) is counted in
// one pass: a left vertex is on the left boundary for the splits
// rank < k <= max neighbour rank, a right vertex on the right boundary for
// min neighbour rank < k <= rank; difference arrays turn those intervals into
// counts for all k.  The split with the smallest boundary among balanced ones
// (35-65 %) wins; the smaller-side boundary becomes the separator.  Each
// subset is ordered: left part, right part, separator (separators are
// eliminated last, forming the top of the elimination tree).  The ordering
// is built in place: a subset's range of the vertex array ends as its order.
//
// The two halves of a split are ordered by separate threads when both are
// large.  They share no edge (the separator covers every cut edge), so a
// thread writes stamp/rank only for its own vertices and reads them only for
// its own vertices and finished separators; subset ids come from one atomic
// counter, so they are unique and the result does not depend on the number
// of threads.
// ---------------------------------------------------------------------------
struct NDState {
  int n;
  const int64_t* xadj;
  const int* adj;
  const double* xyz;
  int leaf;
  std::vector<int> stamp;   // subset id a vertex currently belongs to
  std::vector<int> rank;    // rank along the axis being evaluated
  std::atomic<int> next_id{1};
  std::atomic<int> spare_threads{0};
};

constexpr int kNdParallelMin = 20000;       // smallest half handed to another thread
constexpr int kNdAxisParallelMin = 200000;  // smallest subset whose three axes run in parallel

struct Split {
  int axis = -1;
  int k = 0;          // left = the k lowest
  int sep = -1;
  bool left = true;   // separator taken from the left boundary
  double cost = 0;
};

// v sorted along `axis`, ties by vertex id (keys gathered once, not per comparison).
void sort_along(const NDState& S, int* v, int m, int axis) {
  std::vector<std::pair<double, int>> key(m);
  for (int i = 0; i < m; ++i) key[i] = {S.xyz[3 * (int64_t)v[i] + axis], v[i]};
  std::sort(key.begin(), key.end());
  for (int i = 0; i < m; ++i) v[i] = key[i].second;
}

int take_threads(NDState& S, int want) {
  int k = S.spare_threads.load();
  while (k > 0 && !S.spare_threads.compare_exchange_weak(k, k - std::min(k, want))) {}
  return std::min(k, want);
}

// Evaluate all split positions along `axis` for the subset stamped `id`;
// leaves v sorted along the axis and rank[v[i]] = i.
void eval_axis(const NDState& S, int* v, int m, int axis, int id, int* rank, Split& best) {
  sort_along(S, v, m, axis);
  for (int i = 0; i < m; ++i) rank[v[i]] = i;
  std::vector<int> dl(m + 2, 0), dr(m + 2, 0);
  for (int i = 0; i < m; ++i) {
    const int u = v[i];
    int mx = -1, mn = m;
    for (int64_t p = S.xadj[u]; p < S.xadj[u + 1]; ++p) {
      const int w = S.adj[p];
      if (S.stamp[w] != id) continue;
      const int rw = rank[w];
      mx = std::max(mx, rw);
      mn = std::min(mn, rw);
    }
    if (mx > i) { dl[i + 1] += 1; dl[mx + 1] -= 1; }   // left boundary for k in (i, mx]
    if (mn < i) { dr[mn + 1] += 1; dr[i + 1] -= 1; }   // right boundary for k in (mn, i]
  }
  const int lo = std::max(1, (int)(0.35 * m)), hi = std::min(m - 1, (int)(0.65 * m));
  int bl = 0, br = 0;
  for (int k = 0; k <= hi; ++k) {
    bl += dl[k];
    br += dr[k];
    if (k < lo) continue;
    const int sep = std::min(bl, br);
    const double cost = sep + 1e-3 * m * std::fabs((double)k / m - 0.5);
    if (best.sep < 0 || cost < best.cost) {
      best.axis = axis; best.k = k; best.sep = sep; best.left = bl <= br; best.cost = cost;
    }
  }
}

// The best split of the three axes; the first axis wins ties.  Large subsets
// evaluate the axes on copies of v in parallel (private rank arrays).
Split best_split(NDState& S, int* v, int m) {
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int i = 0; i < m; ++i)
    for (int a = 0; a < 3; ++a) {
      double x = S.xyz[3 * (int64_t)v[i] + a];
      lo[a] = std::min(lo[a], x); hi[a] = std::max(hi[a], x);
    }
  const int id = S.next_id++;
  for (int i = 0; i < m; ++i) S.stamp[v[i]] = id;
  Split cand[3];
  const int extra = m >= kNdAxisParallelMin ? take_threads(S, 2) : 0;
  if (extra == 0) {
    for (int a = 0; a < 3; ++a)
      if (hi[a] > lo[a]) eval_axis(S, v, m, a, id, S.rank.data(), cand[a]);
  } else {
    // axis 0 here; axes 1 and 2 on one or two other threads
    std::vector<int> va(v, v + m), vb(extra == 2 ? m : 0);
    std::vector<int> ra(S.n), rb(extra == 2 ? S.n : 0);
    if (extra == 2) std::copy(v, v + m, vb.begin());
    try {
      parallel_for_each(1 + extra, [&](int k) {
        if (k == 0) {
          if (hi[0] > lo[0]) eval_axis(S, v, m, 0, id, S.rank.data(), cand[0]);
        } else if (k == 1) {
          if (hi[1] > lo[1]) eval_axis(S, va.data(), m, 1, id, ra.data(), cand[1]);
          if (extra == 1 && hi[2] > lo[2]) eval_axis(S, va.data(), m, 2, id, ra.data(), cand[2]);
        } else if (hi[2] > lo[2]) {
          eval_axis(S, vb.data(), m, 2, id, rb.data(), cand[2]);
        }
      });
    } catch (...) {
      S.spare_threads.fetch_add(extra);
      throw;
    }
    S.spare_threads.fetch_add(extra);
  }
  Split best;
  for (int a = 0; a < 3; ++a)
    if (cand[a].sep >= 0 && (best.sep < 0 || cand[a].cost < best.cost)) best = cand[a];
  return best;
}

void nd_rec(NDState& S, int* v, int m) {
  if (m <= S.leaf) return;
  const Split best = best_split(S, v, m);
  if (best.axis < 0) return;  // all points coincide: give up splitting
  // re-sort along the chosen axis (v holds the order of an axis tried)
  const int id = S.next_id++;
  sort_along(S, v, m, best.axis);
  for (int i = 0; i < m; ++i) { S.rank[v[i]] = i; S.stamp[v[i]] = id; }
  // Minimum vertex cover of the bipartite graph of cut edges (Koenig): maximum
  // matching between the left boundary BL and the right boundary BR, then the
  // alternating search from unmatched BL vertices; cover = (BL \ Z) u (BR n Z).
  // It is never larger than either boundary.
  std::vector<int> BL, BR;
  for (int i = 0; i < m; ++i) {
    const int u = v[i];
    const bool on_left = i < best.k;
    for (int64_t p = S.xadj[u]; p < S.xadj[u + 1]; ++p) {
      const int w = S.adj[p];
      if (S.stamp[w] == id && ((S.rank[w] < best.k) != on_left)) {
        (on_left ? BL : BR).push_back(u);
        break;
      }
    }
  }
  // local indices: BL -> [0, nbl), BR -> [0, nbr) via `pos` (reuse rank storage after the cut is fixed)
  std::vector<int> pos_of(BL.size() + BR.size());
  std::vector<char> in_cover;
  {
    const int nbl = (int)BL.size(), nbr = (int)BR.size();
    std::vector<int> lidx(m, -1);  // by rank
    for (int q = 0; q < nbl; ++q) lidx[S.rank[BL[q]]] = q;
    for (int q = 0; q < nbr; ++q) lidx[S.rank[BR[q]]] = q;
    std::vector<int> gptr(nbl + 1, 0), gadj;
    for (int q = 0; q < nbl; ++q) {
      const int u = BL[q];
      for (int64_t p = S.xadj[u]; p < S.xadj[u + 1]; ++p) {
        const int w = S.adj[p];
        if (S.stamp[w] == id && S.rank[w] >= best.k) gadj.push_back(lidx[S.rank[w]]);
      }
      gptr[q + 1] = (int)gadj.size();
    }
    std::vector<int> mL(nbl, -1), mR(nbr, -1);
    for (int q = 0; q < nbl; ++q)  // greedy start
      for (int e = gptr[q]; e < gptr[q + 1]; ++e)
        if (mR[gadj[e]] < 0) { mL[q] = gadj[e]; mR[gadj[e]] = q; break; }
    std::vector<int> seen(nbl, -1), stackv, stacke, parentR(nbr, -1);
    int budget = 200 * (nbl + nbr) + 100000;  // bounded work; fall back to the greedy matching
    for (int q0 = 0; q0 < nbl && budget > 0; ++q0) {
      if (mL[q0] >= 0) continue;
      // iterative DFS for an augmenting path from q0
      stackv.assign(1, q0); stacke.assign(1, gptr[q0]);
      seen[q0] = q0;
      int found = -1;
      while (!stackv.empty() && found < 0 && budget-- > 0) {
        const int q = stackv.back();
        int& e = stacke.back();
        if (e >= gptr[q + 1]) { stackv.pop_back(); stacke.pop_back(); continue; }
        const int rr = gadj[e++];
        const int nq = mR[rr];
        if (nq < 0) { parentR[rr] = q; found = rr; break; }
        if (seen[nq] == q0) continue;
        seen[nq] = q0;
        parentR[rr] = q;
        stackv.push_back(nq);
        stacke.push_back(gptr[nq]);
      }
      if (found >= 0) {  // flip the path
        int rr = found;
        while (true) {
          const int q = parentR[rr];
          const int prev = mL[q];
          mL[q] = rr; mR[rr] = q;
          if (q == q0) break;
          rr = prev;
        }
      }
    }
    // Koenig: Z = vertices reachable from unmatched BL by alternating paths
    std::vector<char> zl(nbl, 0), zr(nbr, 0);
    std::vector<int> queue;
    for (int q = 0; q < nbl; ++q)
      if (mL[q] < 0) { zl[q] = 1; queue.push_back(q); }
    for (size_t h = 0; h < queue.size(); ++h) {
      const int q = queue[h];
      for (int e = gptr[q]; e < gptr[q + 1]; ++e) {
        const int rr = gadj[e];
        if (zr[rr] || mL[q] == rr) continue;
        zr[rr] = 1;
        const int nq = mR[rr];
        if (nq >= 0 && !zl[nq]) { zl[nq] = 1; queue.push_back(nq); }
      }
    }
    in_cover.assign(m, 0);  // by rank
    int cover = 0;
    for (int q = 0; q < nbl; ++q) if (!zl[q]) { in_cover[S.rank[BL[q]]] = 1; ++cover; }
    for (int q = 0; q < nbr; ++q) if (zr[q]) { in_cover[S.rank[BR[q]]] = 1; ++cover; }
    // keep the plain boundary if the cover is not smaller (e.g. budget ran out)
    const int plain = std::min(nbl, nbr);
    if (cover >= plain) {
      std::fill(in_cover.begin(), in_cover.end(), 0);
      const bool use_left = nbl <= nbr;
      for (int u : (use_left ? BL : BR)) in_cover[S.rank[u]] = 1;
    }
  }
  std::vector<int> L, R, Sp;
  L.reserve(best.k + 1); R.reserve(m - best.k + 1);
  for (int i = 0; i < m; ++i) {
    const int u = v[i];
    if (in_cover[i]) Sp.push_back(u);
    else if (i < best.k) L.push_back(u);
    else R.push_back(u);
  }
  std::copy(L.begin(), L.end(), v);
  std::copy(R.begin(), R.end(), v + L.size());
  std::copy(Sp.begin(), Sp.end(), v + L.size() + R.size());
  const int nl = (int)L.size(), nr = (int)R.size();
  { std::vector<int>().swap(L); std::vector<int>().swap(R); std::vector<int>().swap(Sp); }
  const bool fork = std::min(nl, nr) >= kNdParallelMin && take_threads(S, 1) == 1;
  if (!fork) {
    nd_rec(S, v, nl);
    nd_rec(S, v + nl, nr);
    return;
  }
  try {
    parallel_for_each(2, [&](int k) {
      if (k == 0) nd_rec(S, v + nl, nr);
      else nd_rec(S, v, nl);
    });
  } catch (...) {
    S.spare_threads.fetch_add(1);
    throw;
  }
  S.spare_threads.fetch_add(1);
}

// Column counts of L for a postordered elimination tree (children before
// parents, every subtree a contiguous index range), by the method of
// Gilbert, Ng & Peyton, "An efficient algorithm to compute row and column
// counts for sparse Cholesky factorization" (SIAM J. Matrix Anal. Appl.
// 15(4), 1994).  cc[j] = #{i : L(i,j) != 0} = #{i : j in T_i}, where the row
// subtree T_i is the union of the tree paths from every k < i with
// A(i,k) != 0 (and from i itself) up to i.  With weights w and
// cc[j] = sum of w over the subtree of j, one row subtree contributes
//   +1 at each of its leaves k_1 < ... < k_m,
//   -1 at lca(k_{t-1}, k_t) for t >= 2, and -1 at parent(i):
// every node of T_i then sums to 1 and every other node to 0.  Columns are
// visited in increasing order; k is a leaf of T_i iff no earlier column of
// row i lies in k's subtree, i.e. the last one seen is below first(k); the
// lca of the previous leaf and k is the lowest ancestor of the previous
// leaf not yet finished (a column is finished, and its set joined to its
// parent's, once all its entries are visited), found with path compression.
std::vector<int64_t> column_counts(int n, const int64_t* xadj, const int* adj, const std::vector<int>& perm,
                                   const std::vector<int>& iperm, const std::vector<int>& parent) {
  std::vector<int64_t> w(n, 0);
  std::vector<int> first(n), size(n, 1);
  for (int j = 0; j < n; ++j)
    if (parent[j] >= 0) size[parent[j]] += size[j];
  for (int j = 0; j < n; ++j) first[j] = j - size[j] + 1;
  std::vector<int> last_seen(n, -1), prev_leaf(n, -1), anc(n);
  std::iota(anc.begin(), anc.end(), 0);
  for (int k = 0; k < n; ++k) {
    if (first[k] == k) w[k] += 1;           // an etree leaf: T_k = {k}
    if (parent[k] >= 0) w[parent[k]] -= 1;  // the root correction of T_k
    const int ok = perm[k];
    for (int64_t p = xadj[ok]; p < xadj[ok + 1]; ++p) {
      const int i = iperm[adj[p]];
      if (i <= k) continue;
      const bool leaf = last_seen[i] < first[k];
      last_seen[i] = k;
      if (!leaf) continue;
      w[k] += 1;
      const int pl = prev_leaf[i];
      prev_leaf[i] = k;
      if (pl < 0) continue;
      int q = pl;
      while (anc[q] != q) q = anc[q];
      for (int x = pl; x != q;) {
        const int nx = anc[x];
        anc[x] = q;
        x = nx;
      }
      w[q] -= 1;
    }
    if (parent[k] >= 0) anc[k] = parent[k];
  }
  for (int j = 0; j < n; ++j)
    if (parent[j] >= 0) w[parent[j]] += w[j];
  return w;
}

}  // namespace

int host_threads(int requested) {
  if (requested > 0) return requested;
  const char* env = std::getenv("TEMF_HOST_THREADS");
  if (env && std::atoi(env) > 0) return std::atoi(env);
  int n = (int)std::max(1u, std::thread::hardware_concurrency());
  cpu_set_t set;
  if (sched_getaffinity(0, sizeof(set), &set) == 0) n = std::max(1, CPU_COUNT(&set));
  // a container's CPU quota (cgroup v2 cpu.max: "quota period" or "max period")
  if (FILE* f = std::fopen("/sys/fs/cgroup/cpu.max", "r")) {
    char q[32] = {0};
    long long period = 0;
    if (std::fscanf(f, "%31s %lld", q, &period) == 2 && std::strcmp(q, "max") != 0 && period > 0)
      n = std::min(n, std::max(1, (int)(std::atoll(q) / period)));
    std::fclose(f);
  }
  return std::min(n, 64);
}

std::vector<int> block_run_first(const Symbolic& S) {
  const int nsn = S.nsn;
  std::vector<int> first(nsn);
  for (int s = 0; s < nsn; ++s) first[s] = s;
  for (int q = 0; q + 1 < nsn; ++q) {
    if (S.sn_parent[q] != q + 1) continue;
    const int f1 = S.sn_first[q + 1], c1 = S.sn_first[q + 2] - f1;
    const int64_t b0 = S.sn_rows_ptr[q], r0 = S.sn_rows_ptr[q + 1] - b0;
    const int64_t b1 = S.sn_rows_ptr[q + 1], r1 = S.sn_rows_ptr[q + 2] - b1;
    if (r0 != c1 + r1) continue;
    bool ok = true;
    for (int k = 0; k < c1 && ok; ++k) ok = S.sn_rows[b0 + k] == f1 + k;
    if (!ok || !std::equal(S.sn_rows.begin() + b0 + c1, S.sn_rows.begin() + b0 + r0, S.sn_rows.begin() + b1))
      continue;
    first[q + 1] = first[q];
  }
  return first;
}

void update_groups(const Symbolic& S, UpdateGroups& G, int threads) {
  const int nsn = S.nsn;
  const std::vector<int> run_first = block_run_first(S);
  std::vector<int> run_last(nsn);  // last block of each run, indexed by any block
  for (int s = nsn - 1; s >= 0; --s)
    run_last[s] = (s + 1 < nsn && run_first[s + 1] == run_first[s]) ? run_last[s + 1] : s;
  auto owner = [&](int64_t rp, int64_t j) { return S.col2sn[S.sn_rows[rp + j]]; };
  // pass 1: groups and relative positions per supernode (one table per target run)
  std::vector<int64_t> goff(nsn + 1, 0), roff(nsn + 1, 0);
  for (int s = 0; s < nsn; ++s) {
    const int64_t rp = S.sn_rows_ptr[s], r = S.sn_rows_ptr[s + 1] - rp;
    int64_t ng = 0, nr = 0;
    int last_run = -1;
    for (int64_t j = 0; j < r;) {
      const int t = owner(rp, j);
      int64_t j2 = j;
      while (j2 < r && owner(rp, j2) == t) ++j2;
      ++ng;
      if (run_first[t] != last_run) {  // a new table from row j
        nr += r - j;
        last_run = run_first[t];
      }
      j = j2;
    }
    goff[s + 1] = goff[s] + ng;
    roff[s + 1] = roff[s] + nr;
  }
  const int64_t ngrp = goff[nsn];
  if (ngrp > INT32_MAX) throw std::runtime_error("too many update groups for int32 indices");
  G.row_grp.assign(S.sn_rows.size(), 0);
  G.grp_target.assign(ngrp, 0);
  G.grp_shift.assign(ngrp, 0);
  G.grp_rel.assign(ngrp, 0);
  G.n_rel = roff[nsn];
  G.rel.reset(new int[std::max<int64_t>(G.n_rel, 1)]);
  // pass 2: fill, supernode ranges of about equal work per thread
  auto fill = [&](int s0, int s1) {
    for (int s = s0; s < s1; ++s) {
      const int64_t rp = S.sn_rows_ptr[s], r = S.sn_rows_ptr[s + 1] - rp;
      int64_t g = goff[s], q = roff[s];
      int last_run = -1;
      int64_t table = 0;  // rel index of row 0 of s in the current table
      for (int64_t j = 0; j < r;) {
        const int t = owner(rp, j);
        int64_t j2 = j;
        while (j2 < r && owner(rp, j2) == t) ++j2;
        const int t0 = run_first[t];
        if (t0 != last_run) {
          // positions of rows j..r-1 in the panel of the run's first block t0:
          // its columns, the later blocks' columns, then the last block's rows
          const int te = run_last[t0];
          const int f0 = S.sn_first[t0], fend = S.sn_first[te + 1];
          const int* tb = S.sn_rows.data() + S.sn_rows_ptr[te];
          const int64_t tr = S.sn_rows_ptr[te + 1] - S.sn_rows_ptr[te];
          table = q - j;
          int64_t k = 0;
          for (int64_t i = j; i < r; ++i) {
            const int gi = S.sn_rows[rp + i];
            if (gi < fend) {
              G.rel[q++] = gi - f0;
              continue;
            }
            while (k < tr && tb[k] < gi) ++k;
            if (k >= tr || tb[k] != gi) throw std::runtime_error("symbolic structure inconsistent (update row)");
            G.rel[q++] = (int)((fend - f0) + k);
          }
          last_run = t0;
        }
        G.grp_target[g] = t;
        G.grp_shift[g] = S.sn_first[t] - S.sn_first[t0];
        G.grp_rel[g] = table;
        for (int64_t jj = j; jj < j2; ++jj) G.row_grp[rp + jj] = (int)g;
        ++g;
        j = j2;
      }
    }
  };
  const int nt = (int)std::min<int64_t>(host_threads(threads), std::max<int64_t>(1, G.n_rel / 4000000));
  if (nt <= 1) {
    fill(0, nsn);
    return;
  }
  std::vector<int> cut(nt + 1, nsn);
  cut[0] = 0;
  for (int k = 1, s = 0; k < nt; ++k) {
    const int64_t target = G.n_rel * k / nt;
    while (s < nsn && roff[s] < target) ++s;
    cut[k] = s;
  }
  parallel_for_each(nt, [&](int k) { fill(cut[k], cut[k + 1]); });
}

std::string check_update_groups(const Symbolic& S) {
  UpdateGroups G;
  try {
    update_groups(S, G);
  } catch (const std::exception& e) {
    return e.what();
  }
  for (int s = 0; s < S.nsn; ++s) {
    const int64_t rp = S.sn_rows_ptr[s], r = S.sn_rows_ptr[s + 1] - rp;
    for (int64_t j = 0; j < r; ++j) {
      const int g = G.row_grp[rp + j];
      const int t = G.grp_target[g];
      if (S.col2sn[S.sn_rows[rp + j]] != t) return "a row's group targets another supernode";
      if (j > 0 && G.row_grp[rp + j - 1] == g) continue;
      // rows i >= j of s land on their own rows of t's panel
      const int ft = S.sn_first[t], ct = S.sn_first[t + 1] - ft;
      const int* tb = S.sn_rows.data() + S.sn_rows_ptr[t];
      const int64_t tr = S.sn_rows_ptr[t + 1] - S.sn_rows_ptr[t];
      for (int64_t i = j; i < r; ++i) {
        const int64_t pos = (int64_t)G.rel[G.grp_rel[g] + i] - G.grp_shift[g];
        const int gi = S.sn_rows[rp + i];
        const int at = pos < 0 ? -1 : pos < ct ? ft + (int)pos : (pos - ct < tr ? tb[pos - ct] : -1);
        if (at != gi) return "an update row scatters to the wrong row of its target panel";
      }
    }
  }
  return std::string();
}

std::vector<int> nested_dissection(int n, const int64_t* xadj, const int* adj,
                                   const double* xyz, int leaf_size, int threads) {
  NDState S;
  S.n = n; S.xadj = xadj; S.adj = adj; S.xyz = xyz; S.leaf = std::max(leaf_size, 4);
  S.stamp.assign(n, 0);
  S.rank.assign(n, 0);
  threads = host_threads(threads);
  S.spare_threads = std::max(0, threads - 1);
  std::vector<int> v(n);
  std::iota(v.begin(), v.end(), 0);
  nd_rec(S, v.data(), n);
  return v;
}

void analyse(int n, const int64_t* xadj, const int* adj, const double* xyz,
             const SymbolicOptions& opt, Symbolic& out) {
  out = Symbolic();
  out.n = n;
  double t0 = now_s();
  std::vector<int> perm = nested_dissection(n, xadj, adj, xyz, opt.leaf_size, opt.threads);
  std::vector<int> iperm(n);
  for (int i = 0; i < n; ++i) iperm[perm[i]] = i;
  double t1 = now_s();
  out.t_order = t1 - t0;

  // --- elimination tree of the permuted matrix (Liu, with path compression) ---
  auto etree_of = [&](const std::vector<int>& pm, const std::vector<int>& ipm,
                      std::vector<int>& parent) {
    parent.assign(n, -1);
    std::vector<int> anc(n, -1);
    for (int j = 0; j < n; ++j) {
      int oj = pm[j];
      for (int64_t p = xadj[oj]; p < xadj[oj + 1]; ++p) {
        int i = ipm[adj[p]];
        if (i >= j) continue;
        // walk from i to the root of its current subtree, compressing to j
        while (i != -1 && i < j) {
          int next = anc[i];
          anc[i] = j;
          if (next == -1) { parent[i] = j; break; }
          i = next;
        }
      }
    }
  };
  std::vector<int> parent;
  etree_of(perm, iperm, parent);
  // postorder (children in increasing order), iterative
  {
    std::vector<int> head(n, -1), nxt(n, -1), post;
    post.reserve(n);
    for (int j = n - 1; j >= 0; --j) {
      if (parent[j] != -1) { nxt[j] = head[parent[j]]; head[parent[j]] = j; }
    }
    std::vector<int> stack;
    for (int r = 0; r < n; ++r) {
      if (parent[r] != -1) continue;
      stack.push_back(r);
      while (!stack.empty()) {
        int p = stack.back();
        int c = head[p];
        if (c == -1) { stack.pop_back(); post.push_back(p); }
        else { head[p] = nxt[c]; stack.push_back(c); }
      }
    }
    std::vector<int> perm2(n);
    for (int k = 0; k < n; ++k) perm2[k] = perm[post[k]];
    perm.swap(perm2);
    for (int i = 0; i < n; ++i) iperm[perm[i]] = i;
    etree_of(perm, iperm, parent);
  }
  double t2 = now_s();
  out.t_etree = t2 - t1;

  // --- column counts (Gilbert, Ng & Peyton 1994, near-linear in nnz(A)) ---
  std::vector<int64_t> cc = column_counts(n, xadj, adj, perm, iperm, parent);
  double t3 = now_s();
  out.t_colcount = t3 - t2;
  out.nnzL_exact = 0;
  for (int j = 0; j < n; ++j) out.nnzL_exact += cc[j];

  // --- fundamental supernodes ---
  std::vector<int> nchild(n, 0);
  for (int j = 0; j < n; ++j) if (parent[j] != -1) nchild[parent[j]]++;
  std::vector<int> fs_first;
  fs_first.push_back(0);
  for (int j = 1; j < n; ++j) {
    bool merge = parent[j - 1] == j && cc[j - 1] == cc[j] + 1 && nchild[j] == 1;
    if (!merge) fs_first.push_back(j);
  }
  fs_first.push_back(n);
  int nfs = (int)fs_first.size() - 1;
  std::vector<int> fcol2sn(n);
  for (int s = 0; s < nfs; ++s)
    for (int j = fs_first[s]; j < fs_first[s + 1]; ++j) fcol2sn[j] = s;
  std::vector<int> fs_parent(nfs, -1);
  for (int s = 0; s < nfs; ++s) {
    int l = fs_first[s + 1] - 1;
    if (parent[l] != -1) fs_parent[s] = fcol2sn[parent[l]];
  }
  // below-diagonal row count of each fundamental supernode: cc[last]-1
  std::vector<int64_t> fs_r(nfs);
  for (int s = 0; s < nfs; ++s) fs_r[s] = cc[fs_first[s + 1] - 1] - 1;

  // --- relaxed amalgamation (merge a supernode with the child that precedes it) ---
  // merged[s] = representative; processed in increasing order (children first).
  std::vector<int> rep_first(nfs), rep_c(nfs);
  std::vector<int64_t> rep_r(nfs), rep_zeros(nfs, 0);
  std::vector<char> absorbed(nfs, 0);
  std::vector<int> into(nfs);
  std::iota(into.begin(), into.end(), 0);
  auto find = [&](int s) {
    int r = s;
    while (into[r] != r) r = into[r];
    while (into[s] != r) { int nx = into[s]; into[s] = r; s = nx; }
    return r;
  };
  for (int s = 0; s < nfs; ++s) {
    rep_first[s] = fs_first[s];
    rep_c[s] = fs_first[s + 1] - fs_first[s];
    rep_r[s] = fs_r[s];
  }
  if (opt.amalgamate) {
    std::vector<int> owner(n);  // last column of a fundamental supernode -> that supernode
    for (int s = 0; s < nfs; ++s) owner[fs_first[s + 1] - 1] = s;
    for (int p = 0; p < nfs; ++p) {
      while (true) {
        int f = rep_first[p];
        if (f == 0) break;
        int s = find(owner[f - 1]);
        if (s == p || fs_parent[s] < 0 || find(fs_parent[s]) != p) break;
        int64_t c1 = rep_c[s], r1 = rep_r[s], c2 = rep_c[p], r2 = rep_r[p];
        int64_t c = c1 + c2;
        int64_t nz_s = c1 * (c1 + 1) / 2 + c1 * r1;
        int64_t nz_p = c2 * (c2 + 1) / 2 + c2 * r2;
        int64_t nz_m = c * (c + 1) / 2 + c * r2;
        int64_t zeros = nz_m - nz_s - nz_p + rep_zeros[s] + rep_zeros[p];
        double zf = (double)zeros / (double)nz_m;
        bool ok = opt.amalg_level >= 3
                      ? (c <= 16) || (c <= 32 && zf < 0.4) || (c <= 64 && zf < 0.25) || (c <= 256 && zf < 0.05)
                  : opt.amalg_level == 2
                      ? (c <= 16) || (c <= 32 && zf < 0.3) || (c <= 64 && zf < 0.15) || (c <= 256 && zf < 0.05)
                      : (c <= 4) || (c <= 16 && zf < 0.8) || (c <= 48 && zf < 0.1) || (c <= 256 && zf < 0.05);
        if (!ok) break;
        absorbed[s] = 1;
        into[s] = p;
        rep_first[p] = rep_first[s];
        rep_c[p] = (int)c;
        rep_zeros[p] = zeros;
      }
    }
  }
  // live supernodes in column order
  std::vector<int> live;
  for (int s = 0; s < nfs; ++s) if (!absorbed[s]) live.push_back(s);
  // map fundamental supernode -> live supernode that absorbed it
  std::vector<int> fs2live(nfs, -1);
  {
    int li = 0;
    for (int s = 0; s < nfs; ++s) {
      while (li < (int)live.size() && rep_first[live[li]] + rep_c[live[li]] <= fs_first[s]) ++li;
      fs2live[s] = li;
    }
  }
  int nlive = (int)live.size();
  std::vector<int> lfirst(nlive + 1);
  for (int i = 0; i < nlive; ++i) lfirst[i] = rep_first[live[i]];
  lfirst[nlive] = n;
  std::vector<int> lcol2sn(n);
  for (int i = 0; i < nlive; ++i)
    for (int j = lfirst[i]; j < lfirst[i + 1]; ++j) lcol2sn[j] = i;

  // --- row structures of the live supernodes ---
  // struct_below(S) = rows > last(S) of: A's columns in S, and struct_below of children.
  std::vector<int64_t> lrows_ptr(nlive + 1, 0);
  std::vector<int> lrows;
  std::vector<int> lparent(nlive, -1);
  {
    std::vector<std::vector<int>> children(nlive);
    std::vector<int> mark(n, -1);
    std::vector<int> buf;
    lrows.reserve((size_t)n * 8);
    // children are known only after parents are found; compute in increasing order.
    for (int s = 0; s < nlive; ++s) {
      int f = lfirst[s], l = lfirst[s + 1] - 1;
      buf.clear();
      for (int j = f; j <= l; ++j) {
        int oj = perm[j];
        for (int64_t p = xadj[oj]; p < xadj[oj + 1]; ++p) {
          int i = iperm[adj[p]];
          if (i > l && mark[i] != s) { mark[i] = s; buf.push_back(i); }
        }
      }
      for (int c : children[s]) {
        for (int64_t p = lrows_ptr[c]; p < lrows_ptr[c + 1]; ++p) {
          int i = lrows[p];
          if (i > l && mark[i] != s) { mark[i] = s; buf.push_back(i); }
        }
      }
      std::sort(buf.begin(), buf.end());
      lrows_ptr[s + 1] = lrows_ptr[s] + (int64_t)buf.size();
      lrows.insert(lrows.end(), buf.begin(), buf.end());
      if (!buf.empty()) {
        lparent[s] = lcol2sn[buf[0]];
        children[lparent[s]].push_back(s);
      }
    }
  }

  // --- split wide supernodes into column blocks of at most max_sn_cols ---
  const int CB = std::max(1, opt.max_sn_cols);
  std::vector<int> sfirst;
  std::vector<int> sorig;  // live supernode each block came from
  for (int s = 0; s < nlive; ++s) {
    for (int f = lfirst[s]; f < lfirst[s + 1]; f += CB) { sfirst.push_back(f); sorig.push_back(s); }
  }
  int nsn = (int)sfirst.size();
  sfirst.push_back(n);
  out.nsn = nsn;
  out.sn_first = sfirst;
  out.col2sn.assign(n, 0);
  for (int s = 0; s < nsn; ++s)
    for (int j = sfirst[s]; j < sfirst[s + 1]; ++j) out.col2sn[j] = s;
  out.sn_rows_ptr.assign(nsn + 1, 0);
  out.sn_parent.assign(nsn, -1);
  {
    int64_t total = 0;
    for (int s = 0; s < nsn; ++s) {
      int o = sorig[s];
      int lastcol_orig = lfirst[o + 1] - 1;
      int l = sfirst[s + 1] - 1;
      total += (lastcol_orig - l) + (lrows_ptr[o + 1] - lrows_ptr[o]);
    }
    out.sn_rows.reserve(total);
    for (int s = 0; s < nsn; ++s) {
      int o = sorig[s];
      int lastcol_orig = lfirst[o + 1] - 1;
      int l = sfirst[s + 1] - 1;
      for (int j = l + 1; j <= lastcol_orig; ++j) out.sn_rows.push_back(j);
      for (int64_t p = lrows_ptr[o]; p < lrows_ptr[o + 1]; ++p) out.sn_rows.push_back(lrows[p]);
      out.sn_rows_ptr[s + 1] = (int64_t)out.sn_rows.size();
      if (out.sn_rows_ptr[s + 1] > out.sn_rows_ptr[s])
        out.sn_parent[s] = out.col2sn[out.sn_rows[out.sn_rows_ptr[s]]];
    }
  }
  // panels, statistics, levels
  out.sn_Lptr.assign(nsn + 1, 0);
  out.sn_level.assign(nsn, 0);
  out.nnzL = 0; out.flops = 0; out.stored = 0;
  for (int s = 0; s < nsn; ++s) {
    int64_t c = sfirst[s + 1] - sfirst[s];
    int64_t r = out.sn_rows_ptr[s + 1] - out.sn_rows_ptr[s];
    out.sn_Lptr[s + 1] = out.sn_Lptr[s] + (c + r) * c;
    out.nnzL += c * (c + 1) / 2 + c * r;
    double cd = (double)c, rd = (double)r;
    out.flops += cd * cd * cd / 3.0 + cd * cd * rd + cd * rd * rd;
  }
  out.stored = out.sn_Lptr[nsn];
  int maxlev = 0;
  for (int s = 0; s < nsn; ++s) {
    int p = out.sn_parent[s];
    if (p >= 0) {
      if (p <= s) throw std::runtime_error("supernodal tree is not postordered");
      out.sn_level[p] = std::max(out.sn_level[p], out.sn_level[s] + 1);
    }
    maxlev = std::max(maxlev, out.sn_level[s]);
  }
  out.nlevels = nsn ? maxlev + 1 : 0;
  out.level_ptr.assign(out.nlevels + 1, 0);
  for (int s = 0; s < nsn; ++s) out.level_ptr[out.sn_level[s] + 1]++;
  for (int l = 0; l < out.nlevels; ++l) out.level_ptr[l + 1] += out.level_ptr[l];
  out.level_sn.assign(nsn, 0);
  {
    std::vector<int> fill(out.level_ptr.begin(), out.level_ptr.end() - 1);
    for (int s = 0; s < nsn; ++s) out.level_sn[fill[out.sn_level[s]]++] = s;
  }
  out.perm = perm;
  out.iperm = iperm;
  out.t_super = now_s() - t3;
}

}  // namespace temf
