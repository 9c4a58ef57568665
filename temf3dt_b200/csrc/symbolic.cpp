// Nested dissection + elimination tree + supernodes for the FETD step matrix.
// See symbolic.h for what this replaces in the reference.
#include "symbolic.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <numeric>
#include <stdexcept>

namespace temf {

namespace {

double now_s() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

// ---------------------------------------------------------------------------
// Nested dissection by recursive coordinate bisection.
//
// A subset is split at the median of one coordinate axis; the vertex
// separator is the boundary of the smaller-boundary side.  The axis with the
// smallest separator is kept.  Each subset is ordered: left part, right part,
// separator (so separators are eliminated last, forming the top of the tree).
// ---------------------------------------------------------------------------
struct NDState {
  int n;
  const int64_t* xadj;
  const int* adj;
  const double* xyz;
  int leaf;
  std::vector<int> stamp;   // subset id a vertex currently belongs to
  std::vector<signed char> side;
  std::vector<int> order;   // output: new -> old
  std::vector<double> key;
  int next_id = 1;
};

// Separator size when the subset v[0..m) is split at the median along `axis`.
// On return side[] holds 0/1 for the chosen split and `use_left` says which
// boundary is smaller.
int try_split(NDState& S, int* v, int m, int axis, int id, bool& use_left) {
  const int half = m / 2;
  std::nth_element(v, v + half, v + m, [&](int a, int b) {
    double ka = S.xyz[3 * (int64_t)a + axis], kb = S.xyz[3 * (int64_t)b + axis];
    return ka < kb || (ka == kb && a < b);
  });
  for (int i = 0; i < half; ++i) { S.side[v[i]] = 0; S.stamp[v[i]] = id; }
  for (int i = half; i < m; ++i) { S.side[v[i]] = 1; S.stamp[v[i]] = id; }
  int bl = 0, br = 0;
  for (int i = 0; i < m; ++i) {
    int u = v[i];
    int su = S.side[u];
    for (int64_t p = S.xadj[u]; p < S.xadj[u + 1]; ++p) {
      int w = S.adj[p];
      if (S.stamp[w] == id && S.side[w] != su) {
        if (su == 0) ++bl; else ++br;
        break;
      }
    }
  }
  use_left = bl <= br;
  return use_left ? bl : br;
}

void nd_rec(NDState& S, int* v, int m) {
  if (m <= S.leaf) {
    // leaf: order by a coordinate sweep (keeps the leaf block banded)
    for (int i = 0; i < m; ++i) S.order.push_back(v[i]);
    return;
  }
  int best_axis = 0, best_sep = -1;
  bool best_left = true;
  // extent per axis
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int i = 0; i < m; ++i)
    for (int a = 0; a < 3; ++a) {
      double x = S.xyz[3 * (int64_t)v[i] + a];
      lo[a] = std::min(lo[a], x); hi[a] = std::max(hi[a], x);
    }
  for (int axis = 0; axis < 3; ++axis) {
    if (hi[axis] <= lo[axis]) continue;
    bool ul;
    int id = S.next_id++;
    int sep = try_split(S, v, m, axis, id, ul);
    if (best_sep < 0 || sep < best_sep) { best_sep = sep; best_axis = axis; best_left = ul; }
  }
  if (best_sep < 0) {  // all points coincide: give up splitting
    for (int i = 0; i < m; ++i) S.order.push_back(v[i]);
    return;
  }
  bool ul;
  int id = S.next_id++;
  try_split(S, v, m, best_axis, id, ul);
  (void)ul;
  const int sep_side = best_left ? 0 : 1;
  // classify: separator = vertices on sep_side with a neighbour on the other side
  std::vector<int> L, R, Sp;
  L.reserve(m / 2 + 1); R.reserve(m / 2 + 1);
  for (int i = 0; i < m; ++i) {
    int u = v[i];
    int su = S.side[u];
    bool is_sep = false;
    if (su == sep_side) {
      for (int64_t p = S.xadj[u]; p < S.xadj[u + 1]; ++p) {
        int w = S.adj[p];
        if (S.stamp[w] == id && S.side[w] != su) { is_sep = true; break; }
      }
    }
    if (is_sep) Sp.push_back(u);
    else if (su == 0) L.push_back(u);
    else R.push_back(u);
  }
  std::copy(L.begin(), L.end(), v);
  std::copy(R.begin(), R.end(), v + L.size());
  std::copy(Sp.begin(), Sp.end(), v + L.size() + R.size());
  const int nl = (int)L.size(), nr = (int)R.size(), ns = (int)Sp.size();
  { std::vector<int>().swap(L); std::vector<int>().swap(R); std::vector<int>().swap(Sp); }
  nd_rec(S, v, nl);
  nd_rec(S, v + nl, nr);
  for (int i = 0; i < ns; ++i) S.order.push_back(v[nl + nr + i]);
}

}  // namespace

std::vector<int> nested_dissection(int n, const int64_t* xadj, const int* adj,
                                   const double* xyz, int leaf_size) {
  NDState S;
  S.n = n; S.xadj = xadj; S.adj = adj; S.xyz = xyz; S.leaf = std::max(leaf_size, 4);
  S.stamp.assign(n, 0);
  S.side.assign(n, 0);
  S.order.reserve(n);
  std::vector<int> v(n);
  std::iota(v.begin(), v.end(), 0);
  nd_rec(S, v.data(), n);
  if ((int)S.order.size() != n) throw std::runtime_error("nested dissection lost vertices");
  return S.order;
}

void analyse(int n, const int64_t* xadj, const int* adj, const double* xyz,
             const SymbolicOptions& opt, Symbolic& out) {
  out = Symbolic();
  out.n = n;
  double t0 = now_s();
  std::vector<int> perm = nested_dissection(n, xadj, adj, xyz, opt.leaf_size);
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

  // --- column counts by row subtrees (O(nnz(L))) ---
  std::vector<int64_t> cc(n, 0);
  {
    std::vector<int> mark(n, -1);
    for (int i = 0; i < n; ++i) {
      mark[i] = i;
      cc[i] += 1;
      int oi = perm[i];
      for (int64_t p = xadj[oi]; p < xadj[oi + 1]; ++p) {
        int k = iperm[adj[p]];
        if (k >= i) continue;
        while (mark[k] != i) {
          mark[k] = i;
          cc[k] += 1;
          k = parent[k];
        }
      }
    }
  }
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
        bool ok = (c <= 4) || (c <= 16 && zf < 0.8) || (c <= 48 && zf < 0.1) ||
                  (c <= 256 && zf < 0.05);
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
