// K1: first-order Nedelec element assembly of the sigma-mass (M) and the
// curl-curl (K) matrices on the GPU.
//
// Reference: mesh_process, src/FETD_FWD.f90:588-711 (serial loop over tets,
// upper-triangle COO with orientation signs, MKL COO->CSR with duplicates
// summed); element integrals f_kind_iso (:826-851) and e_kind_iso (:797-824);
// geometric coefficients (:245-281).
//
// B200 design: one thread per tetrahedron computes the simplex gradients from
// the four vertices (the reference precomputes a,b,c,d on the host) and the 21
// upper entries of both 6x6 element matrices, orientation signs folded in,
// written structure-of-arrays so a warp's stores coalesce.  A second kernel,
// one thread per nonzero of the permuted symmetric CSR, sums the element
// entries listed for that nonzero in a fixed order -- the COO duplicate sum
// without atomics, so the assembled matrices are bitwise reproducible.
#include <algorithm>
#include <numeric>

#include "assemble.h"

namespace temf {

// local edge j joins local vertices IND_TET[j][0] -> IND_TET[j][1] (src/FETD_FWD.f90:23)
__constant__ int c_ind_tet[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {3, 1}, {2, 3}};

__host__ __device__ inline int packed_upper(int i, int j) {  // i <= j < 6
  return i * 6 - (i * (i - 1)) / 2 + (j - i);
}

// Gradients g_k = (b_k, c_k, d_k) and V, written as differences from the first
// vertex (the cofactor expansion of the reference's 3x3 determinants after
// subtracting one row from the others; same values up to rounding).
__device__ inline void tet_gradients(const double X[4][3], double g[4][3], double& vol) {
  // D(u,w; p,q,r) = det [[1,u_p,w_p],[1,u_q,w_q],[1,u_r,w_r]]
  auto D = [&](int u, int w, int p, int q, int r) {
    return (X[q][u] - X[p][u]) * (X[r][w] - X[p][w]) - (X[r][u] - X[p][u]) * (X[q][w] - X[p][w]);
  };
  const int rest[4][3] = {{1, 2, 3}, {0, 2, 3}, {0, 1, 3}, {0, 1, 2}};
  const double sa[4] = {1.0, -1.0, 1.0, -1.0};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int p = rest[k][0], q = rest[k][1], r = rest[k][2];
    g[k][0] = -sa[k] * D(1, 2, p, q, r);  // b_k
    g[k][1] = sa[k] * D(0, 2, p, q, r);   // c_k
    g[k][2] = -sa[k] * D(0, 1, p, q, r);  // d_k
  }
  const double ax = X[1][0] - X[0][0], ay = X[1][1] - X[0][1], az = X[1][2] - X[0][2];
  const double bx = X[2][0] - X[0][0], by = X[2][1] - X[0][1], bz = X[2][2] - X[0][2];
  const double cx = X[3][0] - X[0][0], cy = X[3][1] - X[0][1], cz = X[3][2] - X[0][2];
  vol = (ax * (by * cz - bz * cy) - ay * (bx * cz - bz * cx) + az * (bx * cy - by * cx)) / 6.0;
}

__global__ void __launch_bounds__(128) k_element_matrices(
    int n_tets, const double* __restrict__ xyz, const int* __restrict__ tet_vex,
    const int* __restrict__ tet_drc, const double* __restrict__ sig, const double* __restrict__ mu,
    double* __restrict__ elemM, double* __restrict__ elemK) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_tets) return;
  double X[4][3];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int v = tet_vex[4 * (int64_t)t + k];
#pragma unroll
    for (int a = 0; a < 3; ++a) X[k][a] = xyz[3 * (int64_t)v + a];
  }
  double g[4][3], vol;
  tet_gradients(X, g, vol);
  double len[6], cr[6][3], s[6];
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    const int p = c_ind_tet[j][0], q = c_ind_tet[j][1];
    const double dx = X[p][0] - X[q][0], dy = X[p][1] - X[q][1], dz = X[p][2] - X[q][2];
    len[j] = sqrt(dx * dx + dy * dy + dz * dz);
    cr[j][0] = g[p][1] * g[q][2] - g[q][1] * g[p][2];
    cr[j][1] = g[q][0] * g[p][2] - g[p][0] * g[q][2];
    cr[j][2] = g[p][0] * g[q][1] - g[q][0] * g[p][1];
    s[j] = (double)tet_drc[6 * (int64_t)t + j];
  }
  double gram[4][4];
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int l = 0; l < 4; ++l) gram[k][l] = g[k][0] * g[l][0] + g[k][1] * g[l][1] + g[k][2] * g[l][2];
  const double sv = sig[t], inv_mu = 1.0 / mu[t];
  const double v6 = 6.0 * vol;
  const double fM = sv / (720.0 * vol);
  const double fK = inv_mu * 4.0 * vol / (v6 * v6 * v6 * v6);
#pragma unroll
  for (int i = 0; i < 6; ++i) {
#pragma unroll
    for (int j = i; j < 6; ++j) {
      const int pi = c_ind_tet[i][0], qi = c_ind_tet[i][1];
      const int pj = c_ind_tet[j][0], qj = c_ind_tet[j][1];
      // f_kind_iso bracket (src/FETD_FWD.f90:843-844)
      const double br = gram[qi][qj] * (1.0 + (pi == pj)) - gram[pi][qj] * (1.0 + (qi == pj)) -
                        gram[qi][pj] * (1.0 + (pi == qj)) + gram[pi][pj] * (1.0 + (qi == qj));
      const double ll = len[i] * len[j];
      const double sgn = s[i] * s[j];
      const double dots = cr[i][0] * cr[j][0] + cr[i][1] * cr[j][1] + cr[i][2] * cr[j][2];
      const int k = packed_upper(i, j);
      elemM[(int64_t)k * n_tets + t] = sgn * (ll * fM * br);
      elemK[(int64_t)k * n_tets + t] = sgn * (ll * fK * dots);
    }
  }
}

__global__ void __launch_bounds__(256) k_gather_nonzeros(
    int64_t nnz, const int* __restrict__ cptr, const int* __restrict__ cidx,
    const double* __restrict__ elemM, const double* __restrict__ elemK,
    double* __restrict__ M, double* __restrict__ K) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nnz) return;
  double m = 0.0, k = 0.0;
  for (int q = cptr[p]; q < cptr[p + 1]; ++q) {
    const int e = cidx[q];
    m += elemM[e];
    k += elemK[e];
  }
  M[p] = m;
  K[p] = k;
}

// ---------------------------------------------------------------------------
// Host: adjacency and permuted pattern with contribution lists
// ---------------------------------------------------------------------------
static void edge_incidence(const temf_ctx& c, std::vector<int64_t>& iptr, std::vector<int>& inc) {
  const int n = c.n_edges, T = c.n_tets;
  iptr.assign(n + 1, 0);
  for (int64_t q = 0; q < 6LL * T; ++q) iptr[c.tet_edg[q] + 1]++;
  for (int e = 0; e < n; ++e) iptr[e + 1] += iptr[e];
  inc.assign(6LL * T, 0);
  std::vector<int64_t> fill(iptr.begin(), iptr.end() - 1);
  for (int64_t q = 0; q < 6LL * T; ++q) inc[fill[c.tet_edg[q]]++] = (int)q;  // q = 6*t + local
}

void build_adjacency(const temf_ctx& c, std::vector<int64_t>& xadj, std::vector<int>& adj) {
  const int n = c.n_edges;
  std::vector<int64_t> iptr;
  std::vector<int> inc;
  edge_incidence(c, iptr, inc);
  std::vector<int> mark(n, -1);
  xadj.assign(n + 1, 0);
  adj.clear();
  adj.reserve((size_t)n * 16);
  for (int e = 0; e < n; ++e) {
    mark[e] = e;
    for (int64_t q = iptr[e]; q < iptr[e + 1]; ++q) {
      const int t = inc[q] / 6;
      for (int b = 0; b < 6; ++b) {
        const int f = c.tet_edg[6LL * t + b];
        if (mark[f] != e) { mark[f] = e; adj.push_back(f); }
      }
    }
    xadj[e + 1] = (int64_t)adj.size();
  }
}

void build_pattern(const temf_ctx& c, const std::vector<int>& perm, const std::vector<int>& iperm,
                   Pattern& P) {
  const int n = c.n_edges, T = c.n_tets;
  std::vector<int64_t> iptr;
  std::vector<int> inc;
  edge_incidence(c, iptr, inc);
  P.n = n;
  P.rowptr.assign(n + 1, 0);
  P.col.clear();
  P.contrib_ptr.clear();
  P.contrib_idx.clear();
  P.contrib_ptr.push_back(0);
  std::vector<int> slot(n, -1);  // new column -> local entry index within the current row
  struct Ent { int col; std::vector<int> c; };
  std::vector<int> cols;
  std::vector<std::vector<int>> contr;
  std::vector<int> order;
  for (int r = 0; r < n; ++r) {
    const int e = perm[r];
    cols.clear();
    for (auto& v : contr) v.clear();
    int m = 0;
    for (int64_t q = iptr[e]; q < iptr[e + 1]; ++q) {
      const int t = inc[q] / 6, a = inc[q] % 6;
      for (int b = 0; b < 6; ++b) {
        const int cn = iperm[c.tet_edg[6LL * t + b]];
        int k = slot[cn];
        if (k < 0) {
          k = m++;
          slot[cn] = k;
          cols.push_back(cn);
          if ((int)contr.size() < m) contr.emplace_back();
        }
        const int i = std::min(a, b), j = std::max(a, b);
        contr[k].push_back(packed_upper(i, j) * T + t);
      }
    }
    order.resize(m);
    std::iota(order.begin(), order.end(), 0);
    std::sort(order.begin(), order.end(), [&](int x, int y) { return cols[x] < cols[y]; });
    for (int k : order) {
      P.col.push_back(cols[k]);
      for (int v : contr[k]) P.contrib_idx.push_back(v);
      P.contrib_ptr.push_back((int)P.contrib_idx.size());
    }
    for (int k = 0; k < m; ++k) slot[cols[k]] = -1;
    P.rowptr[r + 1] = (int)P.col.size();
    if ((int64_t)P.col.size() > (int64_t)INT32_MAX - 64) throw ArgError("matrix too large for int32 CSR");
  }
  P.nnz = (int64_t)P.col.size();
}

void upload_mesh(temf_ctx& c) {
  cudaStream_t s = c.stream;
  c.d_xyz.upload(c.xyz.data(), c.xyz.size(), s);
  c.d_tet_vex.upload(c.tet_vex.data(), c.tet_vex.size(), s);
  c.d_tet_drc.upload(c.tet_drc.data(), c.tet_drc.size(), s);
}

void upload_media(temf_ctx& c) {
  c.d_sig.upload(c.sig.data(), c.sig.size(), c.stream);
  c.d_mu.upload(c.mu.data(), c.mu.size(), c.stream);
}

void upload_pattern(temf_ctx& c) {
  cudaStream_t s = c.stream;
  c.d_rowptr.upload(c.pat.rowptr.data(), c.pat.rowptr.size(), s);
  c.d_col.upload(c.pat.col.data(), c.pat.col.size(), s);
  c.d_contrib_ptr.upload(c.pat.contrib_ptr.data(), c.pat.contrib_ptr.size(), s);
  c.d_contrib_idx.upload(c.pat.contrib_idx.data(), c.pat.contrib_idx.size(), s);
  c.d_elemM.alloc(21LL * c.n_tets);
  c.d_elemK.alloc(21LL * c.n_tets);
  c.d_M.alloc(c.pat.nnz);
  c.d_K.alloc(c.pat.nnz);
}

void launch_assembly(temf_ctx& c) {
  const int T = c.n_tets;
  k_element_matrices<<<ceil_div(T, 128), 128, 0, c.stream>>>(T, c.d_xyz.p, c.d_tet_vex.p, c.d_tet_drc.p,
                                                             c.d_sig.p, c.d_mu.p, c.d_elemM.p, c.d_elemK.p);
  TEMF_CHECK_LAUNCH();
  const int64_t nnz = c.pat.nnz;
  k_gather_nonzeros<<<ceil_div(nnz, 256), 256, 0, c.stream>>>(nnz, c.d_contrib_ptr.p, c.d_contrib_idx.p,
                                                              c.d_elemM.p, c.d_elemK.p, c.d_M.p, c.d_K.p);
  TEMF_CHECK_LAUNCH();
}

}  // namespace temf
