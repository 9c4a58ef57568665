// Adjoint gradient of the FETD run with respect to the conductivities.
//
// The reference has no readable adjoint (its inversion module ships only as
// compiled objects); this follows the mathematics of the forward run.  With
// the accept/reject decisions of the adaptive schedule fixed, every solve of
// the run is a node k of a graph:
//
//     A_k x_k = M (4 x_{a_k} - x_{b_k}) - c_k s,      A_k = 3 M + 2 dt_k K,
//
// (sys_right and the BDF2 history of adap_euler, src/FETD_FWD.f90:1312-1421,
// 1466-1511).  For a misfit J of the receiver samples, the adjoint states are
//
//     A_k l_k = -dJ/dx_k + M (4 sum_{a_j = k} l_j - sum_{b_j = k} l_j)
//
// (A_k is symmetric, so the forward factor serves), and
//
//     dJ/dsigma_t = sum_k l_k^T M_t (3 x_k - 4 x_{a_k} + x_{b_k}),
//
// with M_t the unit-conductivity mass matrix of tet t.
//
// B200 design.  The forward run records the graph (host) and, every `every`
// nodes and wherever dt changes, a checkpoint of the W states the next block
// can read.  The reverse sweep walks the blocks backwards: one factorisation
// per run of equal dt, a recompute of the block's states from its checkpoint
// (same kernels as the forward step), then per node one SpMV, one sparse
// subtraction of dJ/dx, one pair of persistent triangular-solve kernels and
// one gradient kernel (a thread per tet: six lambda and eighteen state
// gathers against the 21 packed unit-mass entries precomputed once, folded
// into a per-tet accumulator -- deterministic, no atomics).  The per-cell
// reduction sum_{t in c} sigma_t G_t runs on the host in FP64.
#include <algorithm>
#include <map>

#include "adjoint.h"
#include "element.cuh"
#include "factor.h"
#include "solve.h"

namespace temf {

__global__ void __launch_bounds__(128) k_unit_mass(int T, const double* __restrict__ xyz,
                                                   const int* __restrict__ tet_vex, const int* __restrict__ tet_drc,
                                                   double* __restrict__ Mu) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= T) return;
  double X[4][3];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int v = tet_vex[4 * (int64_t)t + k];
#pragma unroll
    for (int a = 0; a < 3; ++a) X[k][a] = xyz[3 * (int64_t)v + a];
  }
  double M21[21];
  unit_elements(X, M21, nullptr);
  double s[6];
#pragma unroll
  for (int j = 0; j < 6; ++j) s[j] = (double)tet_drc[6 * (int64_t)t + j];
#pragma unroll
  for (int i = 0; i < 6; ++i)
#pragma unroll
    for (int j = i; j < 6; ++j) {
      const int k = packed_upper(i, j);
      Mu[(int64_t)k * T + t] = s[i] * s[j] * M21[k];
    }
}

// G[t] += lam[te]^T Mu_t (3 xk - 4 xa + xb)[te]
__global__ void __launch_bounds__(128) k_grad_tets(int T, const int* __restrict__ te, const double* __restrict__ Mu,
                                                   const double* __restrict__ lam, const double* __restrict__ xk,
                                                   const double* __restrict__ xa, const double* __restrict__ xb,
                                                   double* __restrict__ G) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= T) return;
  double l[6], w[6];
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    const int e = te[(int64_t)j * T + t];
    l[j] = lam[e];
    w[j] = 3.0 * xk[e] - 4.0 * xa[e] + xb[e];
  }
  double acc = 0.0;
#pragma unroll
  for (int i = 0; i < 6; ++i)
#pragma unroll
    for (int j = i; j < 6; ++j) {
      const double m = Mu[(int64_t)packed_upper(i, j) * T + t];
      acc += (i == j) ? m * l[i] * w[i] : m * (l[i] * w[j] + l[j] * w[i]);
    }
  G[t] += acc;
}

constexpr int kMaxTerms = 8;
struct LinComb {
  const double* x[kMaxTerms];
  int m;
};

// y = sum of the listed vectors
__global__ void k_sum_vectors(int n, LinComb L, double* __restrict__ y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double s = 0.0;
  for (int q = 0; q < L.m; ++q) s += L.x[q][i];
  y[i] = s;
}

// y[idx[q]] -= val[q]   (indices distinct)
__global__ void k_sub_sparse(int cnt, const int* __restrict__ idx, const double* __restrict__ val,
                             double* __restrict__ y) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < cnt) y[idx[q]] -= val[q];
}

__global__ void k_set_ptr_adj(double** p, double* v) { *p = v; }

void run_adjoint(temf_ctx& c, const double* dJ, int rows, const int* tet_cell, int ncell, double* grad_cell,
                 double* grad_tet, AdjointResult& res) {
  AdjointRecord& A = c.adj;
  if (!A.valid) throw StateError("no recorded run: enable recording before temf_run");
  if (c.aniso) throw StateError("the adjoint gradient covers isotropic conductivities");
  if ((int)A.row_node.size() != rows) throw ArgError("dJ has a different number of rows than the recorded run");
  res = AdjointResult();
  cudaStream_t st = c.stream;
  const int n = c.n_edges, T = c.n_tets, N = (int)A.dt.size(), W = A.W, nrec = c.rec.nrec;
  const int nb = (int)A.ck_first.size();
  res.n_nodes = N;
  res.n_blocks = nb;
  for (int k = 1; k <= N; ++k)
    if (k - A.a[k - 1] > W || k - A.b[k - 1] > W || A.a[k - 1] >= k || A.b[k - 1] >= k)
      throw StateError("recorded graph reads beyond the checkpoint window");

  // children of each node (l_j with a_j = k or b_j = k)
  std::vector<std::vector<int>> kid_a(N + 1), kid_b(N + 1);
  for (int j = 1; j <= N; ++j) {
    kid_a[A.a[j - 1]].push_back(j);
    kid_b[A.b[j - 1]].push_back(j);
  }
  for (int k = 1; k <= N; ++k)
    if ((int)kid_a[k].size() > kMaxTerms || (int)kid_b[k].size() > kMaxTerms)
      throw StateError("recorded graph: a node has too many dependants");

  // dJ/dx_k on the receiver edges (permuted numbering), merged per node
  std::vector<std::map<int, double>> gx(N + 1);
  for (int i = 0; i < rows; ++i) {
    const int k = A.row_node[i];
    if (k == 0) continue;  // the initial state is fixed
    for (int r = 0; r < nrec; ++r) {
      const int t = c.rec.rec_tet[r];
      for (int j = 0; j < 6; ++j) {
        double v = 0.0;
        for (int q = 0; q < 6; ++q) v += dJ[((size_t)i * nrec + r) * 6 + q] * c.rec.w_host[r * 36 + q * 6 + j];
        gx[k][c.sym.iperm[c.tet_edg[6LL * t + j]]] += v;
      }
    }
  }
  std::vector<int> gptr(N + 2, 0), gidx;
  std::vector<double> gval;
  for (int k = 1; k <= N; ++k) {
    for (auto& e : gx[k]) { gidx.push_back(e.first); gval.push_back(e.second); }
    gptr[k + 1] = (int)gidx.size();
  }
  DBuf<int> d_gidx;
  DBuf<double> d_gval, d_coef;
  d_gidx.upload(gidx.data(), gidx.size(), st);
  d_gval.upload(gval.data(), gval.size(), st);
  d_coef.upload(A.coef.data(), A.coef.size(), st);

  // permuted tet edges [6][T] and unit mass [21][T]
  std::vector<int> te((size_t)6 * T);
  for (int t = 0; t < T; ++t)
    for (int j = 0; j < 6; ++j) te[(size_t)j * T + t] = c.sym.iperm[c.tet_edg[6LL * t + j]];
  DBuf<int> d_te;
  DBuf<double> d_Mu, d_G;
  d_te.upload(te.data(), te.size(), st);
  d_Mu.alloc((size_t)21 * T);
  d_G.alloc(T);
  TEMF_CUDA(cudaMemsetAsync(d_G.p, 0, d_G.bytes(), st));

  int maxlen = 1;
  for (int b = 0; b < nb; ++b) {
    const int f = A.ck_first[b], e = (b + 1 < nb) ? A.ck_first[b + 1] : N + 1;
    maxlen = std::max(maxlen, e - f);
  }
  DBuf<double> S, Lam, va, vb, zero;
  S.alloc((size_t)(W + maxlen) * n);        // checkpoint window + block states
  Lam.alloc((size_t)(W + 1) * n);           // l_j, j % (W + 1)
  va.alloc(n);
  vb.alloc(n);
  zero.alloc(n);
  TEMF_CUDA(cudaMemsetAsync(zero.p, 0, zero.bytes(), st));
  DBuf<double*> lp;
  lp.alloc(1);
  ensure_update_buffer(c, 1);
  if (c.slots[0].L.n < (size_t)slot_len(c)) c.slots[0].L.alloc(slot_len(c));
  k_set_ptr_adj<<<1, 1, 0, st>>>(lp.p, c.slots[0].L.p);
  TEMF_CHECK_LAUNCH();
  clear_solve_error_flag(c);

  cudaEvent_t e0, e1, f0, f1;
  TEMF_CUDA(cudaEventCreate(&e0));
  TEMF_CUDA(cudaEventCreate(&e1));
  TEMF_CUDA(cudaEventCreate(&f0));
  TEMF_CUDA(cudaEventCreate(&f1));
  TEMF_CUDA(cudaEventRecord(e0, st));
  k_unit_mass<<<ceil_div(T, 128), 128, 0, st>>>(T, c.d_xyz.p, c.d_tet_vex.p, c.d_tet_drc.p, d_Mu.p);
  TEMF_CHECK_LAUNCH();
  res.launches += 1;

  const int gb = ceil_div(n, 256);
  auto vecsum = [&](const std::vector<int>& kids, DBuf<double>& scratch) -> const double* {
    if (kids.empty()) return zero.p;
    if (kids.size() == 1) return Lam.p + (size_t)(kids[0] % (W + 1)) * n;
    LinComb L;
    L.m = (int)kids.size();
    for (int q = 0; q < L.m; ++q) L.x[q] = Lam.p + (size_t)(kids[q] % (W + 1)) * n;
    k_sum_vectors<<<gb, 256, 0, st>>>(n, L, scratch.p);
    TEMF_CHECK_LAUNCH();
    res.launches += 1;
    return scratch.p;
  };

  double cur_dt = -1.0;
  for (int b = nb - 1; b >= 0; --b) {
    const int f = A.ck_first[b], e = (b + 1 < nb) ? A.ck_first[b + 1] : N + 1;
    const double dt = A.dt[f - 1];
    if (dt != cur_dt) {
      TEMF_CUDA(cudaEventRecord(f0, st));
      const int stt = numeric_factor(c, 0, dt);
      TEMF_CUDA(cudaEventRecord(f1, st));
      TEMF_CUDA(cudaEventSynchronize(f1));
      float ms = 0;
      TEMF_CUDA(cudaEventElapsedTime(&ms, f0, f1));
      res.ms_factor += ms;
      res.n_factor += 1;
      res.launches += 2 + 2 * (int64_t)c.sym.nlevels;
      if (stt != 0) throw StateError("non-positive pivot in the adjoint factorisation");
      cur_dt = dt;
    }
    // node j's state lives in S slot j - (f - W)
    auto X = [&](int j) { return S.p + (size_t)(j - (f - W)) * n; };
    TEMF_CUDA(cudaMemcpyAsync(S.p, A.ck[b]->p, (size_t)W * n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    for (int j = f; j < e; ++j) {
      if (A.dt[j - 1] != dt) throw StateError("recorded block mixes step sizes");
      launch_bdf_rhs(c, X(A.a[j - 1]), X(A.b[j - 1]), X(j), 1, st);
      res.launches += 1;
      if (A.coef[j - 1] != 0.0) { launch_source(c, d_coef.p + (j - 1), X(j), 1, st); res.launches += 1; }
      launch_solve(c, lp.p, X(j), 1, st);
      res.launches += 2;
    }
    for (int k = e - 1; k >= f; --k) {
      const double* pa = vecsum(kid_a[k], va);
      const double* pb = vecsum(kid_b[k], vb);
      double* lk = Lam.p + (size_t)(k % (W + 1)) * n;
      launch_bdf_rhs(c, pa, pb, lk, 1, st);
      res.launches += 1;
      const int cnt = gptr[k + 1] - gptr[k];
      if (cnt) {
        k_sub_sparse<<<ceil_div(cnt, 128), 128, 0, st>>>(cnt, d_gidx.p + gptr[k], d_gval.p + gptr[k], lk);
        TEMF_CHECK_LAUNCH();
        res.launches += 1;
      }
      launch_solve(c, lp.p, lk, 1, st);
      res.launches += 2;
      k_grad_tets<<<ceil_div(T, 128), 128, 0, st>>>(T, d_te.p, d_Mu.p, lk, X(k), X(A.a[k - 1]), X(A.b[k - 1]),
                                                     d_G.p);
      TEMF_CHECK_LAUNCH();
      res.launches += 1;
    }
  }
  std::vector<double> G(T);
  TEMF_CUDA(cudaMemcpyAsync(G.data(), d_G.p, (size_t)T * sizeof(double), cudaMemcpyDeviceToHost, st));
  TEMF_CUDA(cudaEventRecord(e1, st));
  TEMF_CUDA(cudaEventSynchronize(e1));
  float ms = 0;
  TEMF_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  res.ms_total = ms;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaEventDestroy(f0);
  cudaEventDestroy(f1);
  c.slots[0].valid = false;
  if (const int fl = solve_error_flag(c))
    throw StateError("a triangular-solve wait timed out in the adjoint sweep (code " + std::to_string(fl) + ")");
  if (grad_cell) std::fill(grad_cell, grad_cell + ncell, 0.0);
  for (int t = 0; t < T; ++t) {
    if (grad_tet) grad_tet[t] = G[t];
    if (grad_cell && tet_cell) {
      const int cc = tet_cell[t];
      if (cc >= 0 && cc < ncell) grad_cell[cc] += c.sig[t] * G[t];
    }
  }
}

}  // namespace temf
