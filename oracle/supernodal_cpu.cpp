// CPU supernodal Cholesky of the FETD step matrix A(dt) = 3 M_sigma + 2 dt K:
// the host-core stand-in for the reference's MKL PARDISO path
// (pardiso_direct_1/2, src/FETD_UTILITY.f90:879-957), used only as the timed
// CPU baseline and checked against the SuperLU slots of fetd_oracle.py.  It is
// test infrastructure, never part of the GPU product path.
//
// It shares the product's host analysis (nested dissection, elimination tree,
// supernodes: temf3dt_b200/csrc/symbolic.cpp), so both sides factor the same
// matrix in the same order.  The product splits supernodes into 64-column
// blocks for the GPU; here the blocks of one supernode (consecutive blocks
// whose rows are the next block's columns followed by its rows) are merged
// back, so wide separators are factored by dense BLAS calls on whole panels.
//
// Numeric factorisation is right-looking, level by level (leaves first):
// dpotrf on the diagonal block, dtrsm for the rows below, then the Schur
// update L21 L21^T, computed by dgemm in column tiles and scattered into the
// ancestors.  Levels with many supernodes run them on OpenMP threads with
// single-threaded BLAS (atomic scatter); levels with few run them one at a
// time as tiled factorisations on all threads, with a threaded scatter (a
// supernode's groups and tiles write disjoint target columns).  The solves follow the same
// levels: forward y_s = L11^-1 y_s, y[rows] -= L21 y_s; backward
// x_s = L11^-T (y_s - L21^T x[rows]).
//
// BLAS/LAPACK come from the caller as Fortran-ABI function pointers (the
// OpenBLAS that scipy ships), together with that library's thread-count
// setter: BLAS runs single-threaded inside OpenMP loops (its own threads,
// spinning between calls, stalled the OpenMP barriers on a full machine).
#include <omp.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../temf3dt_b200/csrc/symbolic.h"

namespace {

typedef void (*dgemm_f)(const char*, const char*, const int*, const int*, const int*, const double*, const double*,
                        const int*, const double*, const int*, const double*, double*, const int*);
typedef void (*dtrsm_f)(const char*, const char*, const char*, const char*, const int*, const int*, const double*,
                        const double*, const int*, double*, const int*);
typedef void (*dpotrf_f)(const char*, const int*, double*, const int*, int*);
typedef void (*dgemv_f)(const char*, const int*, const int*, const double*, const double*, const int*, const double*,
                        const int*, const double*, double*, const int*);
typedef void (*dtrsv_f)(const char*, const char*, const char*, const int*, const double*, const int*, double*,
                        const int*);
typedef void (*setthreads_f)(int);

constexpr int kTile = 256;  // column tile of the Schur update

struct Super {
  int first = 0, c = 0;      // columns first .. first + c - 1
  int64_t rp = 0, r = 0;     // rows[rp .. rp + r): rows below the diagonal block, ascending
  int64_t off = 0;           // panel (c + r) x c, column-major, at L + off
  int parent = -1;
};

struct Solver {
  int n = 0;
  int threads = 1;
  dgemm_f gemm = nullptr;
  dtrsm_f trsm = nullptr;
  dpotrf_f potrf = nullptr;
  dgemv_f gemv = nullptr;
  dtrsv_f trsv = nullptr;
  setthreads_f set_threads = nullptr;
  std::vector<int> perm, iperm;  // perm[new] = old
  std::vector<Super> sn;
  std::vector<int> rows, col2sn;
  std::vector<int> level_ptr, level_sn;
  int64_t stored = 0;
  double flops = 0;
  // upper CSR entries of M_sigma and K (old numbering) -> panel offsets
  std::vector<int64_t> posB, posC;
  std::vector<double> valB, valC;
  std::unique_ptr<double[]> L[2];
  int status[2] = {0, 0};
  std::string err;
};

void blas_threads(Solver& S, int t) {
  if (S.set_threads) S.set_threads(t);
}

// position of global row i inside the panel of supernode t (i >= first(t))
int64_t panel_row(const Solver& S, int t, int i) {
  const Super& T = S.sn[t];
  if (i < T.first + T.c) return i - T.first;
  const int* b = S.rows.data() + T.rp;
  const int* e = b + T.r;
  const int* p = std::lower_bound(b, e, i);
  if (p == e || *p != i) throw std::runtime_error("row missing from its supernode's structure");
  return T.c + (p - b);
}

void build(Solver& S, const temf::Symbolic& Y) {
  // merge consecutive blocks s, s+1 when rows(s) = columns(s+1) ++ rows(s+1)
  const int nb = Y.nsn;
  std::vector<int> start;
  for (int s = 0; s < nb;) {
    start.push_back(s);
    int e = s;
    while (e + 1 < nb) {
      const int64_t r0 = Y.sn_rows_ptr[e], r = Y.sn_rows_ptr[e + 1] - r0;
      const int f1 = Y.sn_first[e + 1], c1 = Y.sn_first[e + 2] - f1;
      const int64_t q0 = Y.sn_rows_ptr[e + 1], q = Y.sn_rows_ptr[e + 2] - q0;
      if (r != c1 + q) break;
      bool same = true;
      for (int k = 0; k < c1 && same; ++k) same = Y.sn_rows[r0 + k] == f1 + k;
      for (int64_t k = 0; k < q && same; ++k) same = Y.sn_rows[r0 + c1 + k] == Y.sn_rows[q0 + k];
      if (!same) break;
      ++e;
    }
    s = e + 1;
  }
  start.push_back(nb);
  const int ns = (int)start.size() - 1;
  S.sn.assign(ns, Super());
  S.col2sn.assign(S.n, 0);
  S.rows.clear();
  int64_t off = 0;
  for (int k = 0; k < ns; ++k) {
    Super& T = S.sn[k];
    const int last = start[k + 1] - 1;
    T.first = Y.sn_first[start[k]];
    T.c = Y.sn_first[last + 1] - T.first;
    T.rp = (int64_t)S.rows.size();
    T.r = Y.sn_rows_ptr[last + 1] - Y.sn_rows_ptr[last];
    S.rows.insert(S.rows.end(), Y.sn_rows.begin() + Y.sn_rows_ptr[last], Y.sn_rows.begin() + Y.sn_rows_ptr[last + 1]);
    T.off = off;
    off += (T.c + T.r) * (int64_t)T.c;
    for (int j = T.first; j < T.first + T.c; ++j) S.col2sn[j] = k;
    const double c = T.c, r = (double)T.r;
    S.flops += c * c * c / 3.0 + c * c * r + c * r * r;
  }
  S.stored = off;
  std::vector<int> level(ns, 0);
  int nlev = 0;
  for (int k = 0; k < ns; ++k) {
    Super& T = S.sn[k];
    if (T.r > 0) {
      T.parent = S.col2sn[S.rows[T.rp]];
      if (T.parent <= k) throw std::runtime_error("supernodes are not in postorder");
      level[T.parent] = std::max(level[T.parent], level[k] + 1);
    }
    nlev = std::max(nlev, level[k] + 1);
  }
  S.level_ptr.assign(nlev + 1, 0);
  for (int k = 0; k < ns; ++k) S.level_ptr[level[k] + 1]++;
  for (int l = 0; l < nlev; ++l) S.level_ptr[l + 1] += S.level_ptr[l];
  S.level_sn.assign(ns, 0);
  std::vector<int> fill(S.level_ptr.begin(), S.level_ptr.end() - 1);
  for (int k = 0; k < ns; ++k) S.level_sn[fill[level[k]]++] = k;
  // largest first inside a level, so the dynamic schedule ends on small ones
  auto work = [&](int k) {
    const double c = S.sn[k].c, r = (double)S.sn[k].r;
    return c * c * c / 3.0 + c * c * r + c * r * r;
  };
  for (int l = 0; l < nlev; ++l)
    std::stable_sort(S.level_sn.begin() + S.level_ptr[l], S.level_sn.begin() + S.level_ptr[l + 1],
                     [&](int a, int b) { return work(a) > work(b); });
}

// panel offset of the lower-triangle entry (row a, column b) of the permuted matrix, a >= b
int64_t entry_pos(const Solver& S, int a, int b) {
  const int t = S.col2sn[b];
  const Super& T = S.sn[t];
  return T.off + (int64_t)(b - T.first) * (T.c + T.r) + panel_row(S, t, a);
}

// Schur update of supernode s into its ancestors; `par`: threads over
// (group, tile) pairs (one supernode at a time), else serial with atomics.
// False if a row of s is missing from an ancestor's structure.
bool schur(Solver& S, double* L, int s, bool par, bool atomic) {
  const Super& T = S.sn[s];
  if (T.r == 0) return true;
  const int ld = T.c + (int)T.r;
  const double* P = L + T.off;
  const int* R = S.rows.data() + T.rp;
  const int r = (int)T.r;
  struct Work { int t, j, j2, jt0, jt1; int64_t relo; };
  std::vector<Work> work;
  std::vector<int> rel;  // per group: positions of rows j .. r-1 in t's panel
  for (int j = 0; j < r;) {
    const int t = S.col2sn[R[j]];
    const Super& U = S.sn[t];
    int j2 = j;
    while (j2 < r && R[j2] < U.first + U.c) ++j2;
    const int64_t relo = (int64_t)rel.size();
    const int* tb = S.rows.data() + U.rp;
    int64_t k = 0;
    for (int i = j; i < r; ++i) {
      if (R[i] < U.first + U.c) {
        rel.push_back(R[i] - U.first);
        continue;
      }
      while (k < U.r && tb[k] < R[i]) ++k;
      if (k >= U.r || tb[k] != R[i]) return false;
      rel.push_back((int)(U.c + k));
    }
    for (int jt0 = j; jt0 < j2; jt0 += kTile) work.push_back({t, j, j2, jt0, std::min(jt0 + kTile, j2), relo});
    j = j2;
  }
  auto one = [&](const Work& w, std::vector<double>& W) {
    const int m = r - w.jt0, k = w.jt1 - w.jt0;
    W.resize((size_t)m * k);
    const double one_ = 1.0, zero = 0.0;
    S.gemm("N", "T", &m, &k, &T.c, &one_, P + T.c + w.jt0, &ld, P + T.c + w.jt0, &ld, &zero, W.data(), &m);
    const Super& U = S.sn[w.t];
    const int ldt = U.c + (int)U.r;
    const int* rl = rel.data() + w.relo;
    for (int jj = w.jt0; jj < w.jt1; ++jj) {
      double* Pt = L + U.off + (int64_t)(R[jj] - U.first) * ldt;
      const double* Wc = W.data() + (size_t)(jj - w.jt0) * m;
      for (int ii = jj; ii < r; ++ii) {
        const double v = Wc[ii - w.jt0];
        double* dst = Pt + rl[ii - w.j];
        if (atomic) {
#pragma omp atomic
          *dst -= v;
        } else {
          *dst -= v;
        }
      }
    }
  };
  if (par) {
#pragma omp parallel
    {
      std::vector<double> W;
#pragma omp for schedule(dynamic, 1)
      for (int64_t q = 0; q < (int64_t)work.size(); ++q) one(work[q], W);
    }
  } else {
    std::vector<double> W;
    for (const Work& w : work) one(w, W);
  }
  return true;
}

// dense part of supernode s: L11 = chol(A11), L21 = A21 L11^-T.  Returns 0 or
// the 1-based (new-numbering) column of the first non-positive pivot.
int factor_panel(Solver& S, double* L, int s) {
  const Super& T = S.sn[s];
  const int ld = T.c + (int)T.r;
  double* P = L + T.off;
  int info = 0;
  S.potrf("L", &T.c, P, &ld, &info);
  if (info != 0) return T.first + info;
  if (T.r > 0) {
    const int r = (int)T.r;
    const double one = 1.0;
    S.trsm("R", "L", "T", "N", &r, &T.c, &one, P, &ld, P + T.c, &ld);
  }
  return 0;
}

// The same for one large supernode on all threads: a tiled right-looking
// Cholesky of its (c + r) x c panel with single-threaded BLAS per tile
// (dpotrf on a diagonal tile, dtrsm on the row chunks below it, dgemm on the
// trailing tiles), which scales where a threaded dpotrf does not.
int factor_panel_tiled(Solver& S, double* L, int s) {
  const Super& T = S.sn[s];
  const int ld = T.c + (int)T.r, h = ld;
  double* P = L + T.off;
  const double one = 1.0, mone = -1.0;
  struct Pair { int i0, j0; };
  std::vector<Pair> pairs;
  for (int k0 = 0; k0 < T.c; k0 += kTile) {
    const int kc = std::min(kTile, T.c - k0);
    int info = 0;
    double* D = P + (int64_t)k0 * ld + k0;
    S.potrf("L", &kc, D, &ld, &info);
    if (info != 0) return T.first + k0 + info;
    const int below = h - k0 - kc;
    const int nchunk = (below + kTile - 1) / kTile;
#pragma omp parallel for schedule(dynamic, 1)
    for (int q = 0; q < nchunk; ++q) {
      const int i0 = k0 + kc + q * kTile, m = std::min(kTile, h - i0);
      S.trsm("R", "L", "T", "N", &m, &kc, &one, D, &ld, P + (int64_t)k0 * ld + i0, &ld);
    }
    pairs.clear();
    for (int j0 = k0 + kc; j0 < T.c; j0 += kTile)
      for (int i0 = j0; i0 < h; i0 += kTile) pairs.push_back({i0, j0});
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t q = 0; q < (int64_t)pairs.size(); ++q) {
      const int i0 = pairs[q].i0, j0 = pairs[q].j0;
      const int m = std::min(kTile, h - i0), n = std::min(kTile, T.c - j0);
      S.gemm("N", "T", &m, &n, &kc, &mone, P + (int64_t)k0 * ld + i0, &ld, P + (int64_t)k0 * ld + j0, &ld, &one,
             P + (int64_t)j0 * ld + i0, &ld);
    }
  }
  return 0;
}

int factor(Solver& S, int slot, double dt) {
  omp_set_num_threads(S.threads);  // the thread count is per process; another handle may have changed it
  double* L = S.L[slot].get();
  // zero the panels on all threads: faster, and on a multi-socket host the
  // pages are spread over the memory nodes of the threads that use them
  const int64_t chunk = 1 << 17;
#pragma omp parallel for schedule(static)
  for (int64_t q = 0; q < (S.stored + chunk - 1) / chunk; ++q)
    std::memset(L + q * chunk, 0, sizeof(double) * (size_t)std::min(chunk, S.stored - q * chunk));
  const int64_t nb = (int64_t)S.posB.size(), nc = (int64_t)S.posC.size();
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < nb; ++k) L[S.posB[k]] += 3.0 * S.valB[k];
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < nc; ++k) L[S.posC[k]] += 2.0 * dt * S.valC[k];
  const int nlev = (int)S.level_ptr.size() - 1;
  int bad = 0;
  for (int l = 0; l < nlev && !bad; ++l) {
    const int q0 = S.level_ptr[l], q1 = S.level_ptr[l + 1];
    if (q1 - q0 >= S.threads) {
      int lbad = 0, broken = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(max : lbad, broken)
      for (int q = q0; q < q1; ++q) {
        const int s = S.level_sn[q];
        const int st = factor_panel(S, L, s);
        if (st) {
          lbad = std::max(lbad, st);
          continue;
        }
        if (!schur(S, L, s, false, true)) broken = 1;
      }
      if (broken) throw std::runtime_error("update row missing from the ancestor");
      bad = lbad;
    } else {
      for (int q = q0; q < q1 && !bad; ++q) {
        const int s = S.level_sn[q];
        bad = factor_panel_tiled(S, L, s);
        if (bad) break;
        if (!schur(S, L, s, true, false)) throw std::runtime_error("update row missing from the ancestor");
      }
    }
  }
  S.status[slot] = bad ? S.perm[bad - 1] + 1 : 0;
  return S.status[slot];
}

// y[0..m) += alpha A x, A m x n (column-major, lda), on all threads: row chunks
void par_gemv_n(const Solver& S, int m, int n, double alpha, const double* A, int lda, const double* x, double* y) {
  const int inc = 1;
  const double one = 1.0;
  const int nchunk = (m + 1023) / 1024;
#pragma omp parallel for schedule(dynamic, 1)
  for (int q = 0; q < nchunk; ++q) {
    const int i0 = q * 1024, mi = std::min(1024, m - i0);
    S.gemv("N", &mi, &n, &alpha, A + i0, &lda, x, &inc, &one, y + i0, &inc);
  }
}

// y[0..n) += alpha A^T x, A m x n, on all threads: column chunks
void par_gemv_t(const Solver& S, int m, int n, double alpha, const double* A, int lda, const double* x, double* y) {
  const int inc = 1;
  const double one = 1.0;
  const int nchunk = (n + 63) / 64;
#pragma omp parallel for schedule(dynamic, 1)
  for (int q = 0; q < nchunk; ++q) {
    const int j0 = q * 64, nj = std::min(64, n - j0);
    S.gemv("T", &m, &nj, &alpha, A + (int64_t)j0 * lda, &lda, x, &inc, &one, y + j0, &inc);
  }
}

// Levels with one supernode solve its diagonal block in column tiles, the
// matrix-vector products in between split over the threads; other levels
// run their supernodes on the threads.  BLAS stays single-threaded.
void solve(Solver& S, int slot, const double* b, double* x) {
  omp_set_num_threads(S.threads);
  const double* L = S.L[slot].get();
  std::vector<double> y(S.n), z;
  for (int i = 0; i < S.n; ++i) y[i] = b[S.perm[i]];
  const int nlev = (int)S.level_ptr.size() - 1;
  const int inc = 1;
  const double one = 1.0, zero = 0.0, mone = -1.0;
  // forward, leaves first
  for (int l = 0; l < nlev; ++l) {
    const int q0 = S.level_ptr[l], q1 = S.level_ptr[l + 1];
    if (q1 - q0 == 1) {
      const Super& T = S.sn[S.level_sn[q0]];
      const int ld = T.c + (int)T.r, h = ld;
      const double* P = L + T.off;
      z.assign(h, 0.0);
      std::copy(y.begin() + T.first, y.begin() + T.first + T.c, z.begin());
      for (int k0 = 0; k0 < T.c; k0 += kTile) {
        const int kc = std::min(kTile, T.c - k0), m = h - k0 - kc;
        S.trsv("L", "N", "N", &kc, P + (int64_t)k0 * ld + k0, &ld, z.data() + k0, &inc);
        if (m > 0) par_gemv_n(S, m, kc, -1.0, P + (int64_t)k0 * ld + k0 + kc, ld, z.data() + k0, z.data() + k0 + kc);
      }
      std::copy(z.begin(), z.begin() + T.c, y.begin() + T.first);
      const int* R = S.rows.data() + T.rp;
      for (int64_t i = 0; i < T.r; ++i) y[R[i]] += z[T.c + i];
      continue;
    }
#pragma omp parallel
    {
      std::vector<double> tmp;
#pragma omp for schedule(dynamic, 4)
      for (int q = q0; q < q1; ++q) {
        const Super& T = S.sn[S.level_sn[q]];
        const int ld = T.c + (int)T.r, r = (int)T.r;
        const double* P = L + T.off;
        S.trsv("L", "N", "N", &T.c, P, &ld, y.data() + T.first, &inc);
        if (r == 0) continue;
        tmp.resize(r);
        S.gemv("N", &r, &T.c, &one, P + T.c, &ld, y.data() + T.first, &inc, &zero, tmp.data(), &inc);
        const int* R = S.rows.data() + T.rp;
        for (int i = 0; i < r; ++i) {
#pragma omp atomic
          y[R[i]] -= tmp[i];
        }
      }
    }
  }
  // backward, root first
  for (int l = nlev - 1; l >= 0; --l) {
    const int q0 = S.level_ptr[l], q1 = S.level_ptr[l + 1];
    if (q1 - q0 == 1) {
      const Super& T = S.sn[S.level_sn[q0]];
      const int ld = T.c + (int)T.r, r = (int)T.r;
      const double* P = L + T.off;
      double* zs = y.data() + T.first;
      if (r > 0) {
        z.resize(r);
        const int* R = S.rows.data() + T.rp;
        for (int i = 0; i < r; ++i) z[i] = y[R[i]];
        par_gemv_t(S, r, T.c, -1.0, P + T.c, ld, z.data(), zs);
      }
      const int ntile = (T.c + kTile - 1) / kTile;
      for (int k = ntile - 1; k >= 0; --k) {
        const int k0 = k * kTile, kc = std::min(kTile, T.c - k0);
        S.trsv("L", "T", "N", &kc, P + (int64_t)k0 * ld + k0, &ld, zs + k0, &inc);
        if (k0 > 0) par_gemv_t(S, kc, k0, -1.0, P + k0, ld, zs + k0, zs);
      }
      continue;
    }
#pragma omp parallel
    {
      std::vector<double> g;
#pragma omp for schedule(dynamic, 4)
      for (int q = q0; q < q1; ++q) {
        const Super& T = S.sn[S.level_sn[q]];
        const int ld = T.c + (int)T.r, r = (int)T.r;
        const double* P = L + T.off;
        if (r > 0) {
          g.resize(r);
          const int* R = S.rows.data() + T.rp;
          for (int i = 0; i < r; ++i) g[i] = y[R[i]];
          S.gemv("T", &r, &T.c, &mone, P + T.c, &ld, g.data(), &inc, &one, y.data() + T.first, &inc);
        }
        S.trsv("L", "T", "N", &T.c, P, &ld, y.data() + T.first, &inc);
      }
    }
  }
  for (int i = 0; i < S.n; ++i) x[S.perm[i]] = y[i];
}

}  // namespace

extern "C" {

// n unknowns; M_sigma and K as 0-based upper CSR (row pointers int64,
// columns int32, old numbering); xyz(3, n) a point per unknown for the
// ordering; blas[6] = dgemm, dtrsm, dpotrf, dgemv, dtrsv (Fortran ABI) and
// the BLAS thread-count setter (may be null).  Returns a handle or null.
void* sncpu_create(int n, const long long* bp, const int* bi, const double* bv, const long long* cp, const int* ci,
                   const double* cv, const double* xyz, void* const* blas, int threads, double* stats) {
  Solver* S = new Solver();
  try {
    S->n = n;
    S->gemm = (dgemm_f)blas[0];
    S->trsm = (dtrsm_f)blas[1];
    S->potrf = (dpotrf_f)blas[2];
    S->gemv = (dgemv_f)blas[3];
    S->trsv = (dtrsv_f)blas[4];
    S->set_threads = (setthreads_f)blas[5];
    S->threads = std::max(1, std::min(threads, 64));
    omp_set_num_threads(S->threads);
    blas_threads(*S, 1);  // all parallelism is OpenMP's: BLAS threads would compete with it
    // symmetric adjacency (no diagonal) of the union of both patterns
    std::vector<std::vector<int>> nb(n);
    for (int pass = 0; pass < 2; ++pass) {
      const long long* p = pass ? cp : bp;
      const int* ix = pass ? ci : bi;
      for (int i = 0; i < n; ++i)
        for (long long q = p[i]; q < p[i + 1]; ++q) {
          const int j = ix[q];
          if (j == i) continue;
          nb[i].push_back(j);
          nb[j].push_back(i);
        }
    }
    std::vector<int64_t> xadj(n + 1, 0);
    std::vector<int> adj;
    for (int i = 0; i < n; ++i) {
      std::sort(nb[i].begin(), nb[i].end());
      nb[i].erase(std::unique(nb[i].begin(), nb[i].end()), nb[i].end());
      adj.insert(adj.end(), nb[i].begin(), nb[i].end());
      xadj[i + 1] = (int64_t)adj.size();
      std::vector<int>().swap(nb[i]);
    }
    temf::SymbolicOptions o;
    temf::Symbolic Y;
    temf::analyse(n, xadj.data(), adj.data(), xyz, o, Y);
    S->perm = Y.perm;
    S->iperm = Y.iperm;
    build(*S, Y);
    for (int pass = 0; pass < 2; ++pass) {
      const long long* p = pass ? cp : bp;
      const int* ix = pass ? ci : bi;
      const double* v = pass ? cv : bv;
      std::vector<int64_t>& pos = pass ? S->posC : S->posB;
      std::vector<double>& val = pass ? S->valC : S->valB;
      pos.resize(p[n]);
      val.assign(v, v + p[n]);
      for (int i = 0; i < n; ++i)
        for (long long q = p[i]; q < p[i + 1]; ++q) {
          int a = S->iperm[i], b = S->iperm[ix[q]];
          if (a < b) std::swap(a, b);
          pos[q] = entry_pos(*S, a, b);
        }
    }
    if (stats) {
      stats[0] = (double)S->sn.size();
      stats[1] = (double)S->level_ptr.size() - 1;
      stats[2] = (double)S->stored;
      stats[3] = S->flops;
    }
    return S;
  } catch (const std::exception& e) {
    delete S;
    return nullptr;
  }
}

void sncpu_destroy(void* h) { delete static_cast<Solver*>(h); }

// factor A(dt) = 3 M_sigma + 2 dt K into slot 0/1: 0, the 1-based (original
// numbering) column of the first non-positive pivot, or -1 on error
int sncpu_factor(void* h, int slot, double dt) {
  Solver* S = static_cast<Solver*>(h);
  if (!S || slot < 0 || slot > 1) return -1;
  try {
    if (!S->L[slot]) S->L[slot].reset(new double[std::max<int64_t>(S->stored, 1)]);
    return factor(*S, slot, dt);
  } catch (const std::exception& e) {
    S->err = e.what();
    return -1;
  }
}

int sncpu_solve(void* h, int slot, const double* b, double* x) {
  Solver* S = static_cast<Solver*>(h);
  if (!S || slot < 0 || slot > 1 || !S->L[slot] || S->status[slot] != 0) return -1;
  solve(*S, slot, b, x);
  return 0;
}

// y = A x for a CSR matrix (int32 row pointers and columns) on the
// solver's threads: the mkl_sparse_d_mv of the BDF2 right-hand side
// (src/FETD_FWD.f90:1427), which MKL runs threaded
void sncpu_spmv(void* h, int n, const int* ptr, const int* col, const double* val, const double* x, double* y) {
  Solver* S = static_cast<Solver*>(h);
  if (S) omp_set_num_threads(S->threads);
#pragma omp parallel for schedule(static, 4096)
  for (int i = 0; i < n; ++i) {
    double a = 0.0;
    for (int p = ptr[i]; p < ptr[i + 1]; ++p) a += val[p] * x[col[p]];
    y[i] = a;
  }
}

void sncpu_release(void* h, int slot) {
  Solver* S = static_cast<Solver*>(h);
  if (S && slot >= 0 && slot <= 1) S->L[slot].reset();
}

}  // extern "C"
