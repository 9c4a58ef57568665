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
#include <climits>
#include <exception>
#include <numeric>
#include <thread>

#include "assemble.h"
#include "element.cuh"

namespace temf {

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
  double M21[21], K21[21];
  unit_elements(X, M21, K21);
  double s[6];
#pragma unroll
  for (int j = 0; j < 6; ++j) s[j] = (double)tet_drc[6 * (int64_t)t + j];
  const double sv = sig[t], inv_mu = 1.0 / mu[t];
#pragma unroll
  for (int i = 0; i < 6; ++i) {
#pragma unroll
    for (int j = i; j < 6; ++j) {
      const int k = packed_upper(i, j);
      const double sgn = s[i] * s[j];
      elemM[(int64_t)k * n_tets + t] = sgn * (sv * M21[k]);
      elemK[(int64_t)k * n_tets + t] = sgn * (inv_mu * K21[k]);
    }
  }
}

// The same for anisotropic media: per tet the conductivity tensor S and the
// curl-curl tensor Tm (row-major, 9 doubles each).
__global__ void __launch_bounds__(128) k_element_matrices_aniso(
    int n_tets, const double* __restrict__ xyz, const int* __restrict__ tet_vex,
    const int* __restrict__ tet_drc, const double* __restrict__ sig9, const double* __restrict__ tm9,
    double* __restrict__ elemM, double* __restrict__ elemK) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_tets) return;
  double X[4][3], S[9], Tm[9];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int v = tet_vex[4 * (int64_t)t + k];
#pragma unroll
    for (int a = 0; a < 3; ++a) X[k][a] = xyz[3 * (int64_t)v + a];
  }
#pragma unroll
  for (int a = 0; a < 9; ++a) {
    S[a] = sig9[9 * (int64_t)t + a];
    Tm[a] = tm9[9 * (int64_t)t + a];
  }
  double M21[21], K21[21];
  aniso_elements(X, S, Tm, M21, K21);
  double s[6];
#pragma unroll
  for (int j = 0; j < 6; ++j) s[j] = (double)tet_drc[6 * (int64_t)t + j];
#pragma unroll
  for (int i = 0; i < 6; ++i) {
#pragma unroll
    for (int j = i; j < 6; ++j) {
      const int k = packed_upper(i, j);
      const double sgn = s[i] * s[j];
      elemM[(int64_t)k * n_tets + t] = sgn * M21[k];
      elemK[(int64_t)k * n_tets + t] = sgn * K21[k];
    }
  }
}

// First-order absorbing boundary: for each tet with boundary faces (bits of
// face_mask), add the faces' integrals (times sqrt(1.257e-6 / 8.85e-12),
// orientation signs folded in) to its sigma-mass entries -- b_mat + w_mat of
// mesh_process (src/FETD_FWD.f90:635-640).
__global__ void __launch_bounds__(128) k_boundary_terms(int n_tets, const double* __restrict__ xyz,
                                                        const int* __restrict__ tet_vex,
                                                        const int* __restrict__ tet_drc,
                                                        const unsigned char* __restrict__ face_mask,
                                                        double* __restrict__ elemM) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_tets) return;
  const unsigned mask = face_mask[t];
  if (!mask) return;
  double X[4][3];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int v = tet_vex[4 * (int64_t)t + k];
#pragma unroll
    for (int a = 0; a < 3; ++a) X[k][a] = xyz[3 * (int64_t)v + a];
  }
  double W[6][6];
#pragma unroll
  for (int i = 0; i < 6; ++i)
#pragma unroll
    for (int j = 0; j < 6; ++j) W[i][j] = 0.0;
  for (int f = 0; f < 4; ++f) {
    if (!(mask & (1u << f))) continue;
    double P[3][3], F[3][3];
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int a = 0; a < 3; ++a) P[k][a] = X[face_vertex(f, k)][a];
    face_integral(P, F);
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
      for (int k = 0; k < 3; ++k) W[face_edge(f, j)][face_edge(f, k)] += face_dir(f, j) * face_dir(f, k) * F[j][k];
  }
  const double z0 = sqrt(1.257e-6 / 8.85e-12);
  double s[6];
#pragma unroll
  for (int j = 0; j < 6; ++j) s[j] = (double)tet_drc[6 * (int64_t)t + j];
#pragma unroll
  for (int i = 0; i < 6; ++i)
#pragma unroll
    for (int j = i; j < 6; ++j) elemM[(int64_t)packed_upper(i, j) * n_tets + t] += s[i] * s[j] * (W[i][j] * z0);
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

// Rows of the permuted pattern are independent: each host thread builds a
// contiguous row range into its own arrays, which are then concatenated, so
// the result is the same for any thread count.
void build_pattern(const temf_ctx& c, const std::vector<int>& perm, const std::vector<int>& iperm,
                   Pattern& P) {
  const int n = c.n_edges, T = c.n_tets;
  if (21LL * T > (int64_t)INT32_MAX) throw ArgError("mesh too large: element entries k * n_tets + t exceed int32");
  std::vector<int64_t> iptr;
  std::vector<int> inc;
  edge_incidence(c, iptr, inc);
  struct Part {
    std::vector<int> rowlen, col, cnt, idx;  // per row: entries; per entry: contributions
  };
  auto rows = [&](int r0, int r1, Part& out) {
    std::vector<int> slot(n, -1);  // new column -> local entry index within the current row
    std::vector<int> cols;
    std::vector<std::vector<int>> contr;
    std::vector<int> order;
    for (int r = r0; r < r1; ++r) {
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
        out.col.push_back(cols[k]);
        out.cnt.push_back((int)contr[k].size());
        out.idx.insert(out.idx.end(), contr[k].begin(), contr[k].end());
      }
      for (int k = 0; k < m; ++k) slot[cols[k]] = -1;
      out.rowlen.push_back(m);
    }
  };
  const int nt = std::max(1, std::min(host_threads(0), n / 50000));
  std::vector<Part> parts(nt);
  parallel_for_each(nt, [&](int k) { rows((int)((int64_t)n * k / nt), (int)((int64_t)n * (k + 1) / nt), parts[k]); });
  int64_t nnz = 0, ncontr = 0;
  for (const Part& q : parts) {
    nnz += (int64_t)q.col.size();
    ncontr += (int64_t)q.idx.size();
  }
  if (nnz > (int64_t)INT32_MAX - 64 || ncontr > (int64_t)INT32_MAX - 64)
    throw ArgError("matrix too large for int32 CSR");
  P.n = n;
  P.nnz = nnz;
  P.rowptr.assign(n + 1, 0);
  P.col.clear();
  P.col.reserve(nnz);
  P.contrib_ptr.assign(1, 0);
  P.contrib_ptr.reserve(nnz + 1);
  P.contrib_idx.clear();
  P.contrib_idx.reserve(ncontr);
  int r = 0;
  for (Part& q : parts) {
    for (int len : q.rowlen) {
      P.rowptr[r + 1] = P.rowptr[r] + len;
      ++r;
    }
    P.col.insert(P.col.end(), q.col.begin(), q.col.end());
    for (int k : q.cnt) P.contrib_ptr.push_back(P.contrib_ptr.back() + k);
    P.contrib_idx.insert(P.contrib_idx.end(), q.idx.begin(), q.idx.end());
    std::vector<int>().swap(q.rowlen);
    std::vector<int>().swap(q.col);
    std::vector<int>().swap(q.cnt);
    std::vector<int>().swap(q.idx);
  }
}

void upload_mesh(temf_ctx& c) {
  cudaStream_t s = c.stream;
  c.d_xyz.upload(c.xyz.data(), c.xyz.size(), s);
  c.d_tet_vex.upload(c.tet_vex.data(), c.tet_vex.size(), s);
  c.d_tet_drc.upload(c.tet_drc.data(), c.tet_drc.size(), s);
}

void upload_media(temf_ctx& c) {
  if (c.aniso) {
    c.d_sig9.upload(c.sig9.data(), c.sig9.size(), c.stream);
    c.d_tm9.upload(c.tm9.data(), c.tm9.size(), c.stream);
  } else {
    c.d_sig.upload(c.sig.data(), c.sig.size(), c.stream);
    c.d_mu.upload(c.mu.data(), c.mu.size(), c.stream);
  }
}

void boundary_face_mask(const temf_ctx& c, std::vector<unsigned char>& mask) {
  // faces that belong to one tet; on a convex mesh these are the faces
  // surface_integral's plane test finds (src/FETD_FWD.f90:928-950)
  static const int fv[4][3] = {{0, 2, 1}, {3, 1, 2}, {0, 3, 2}, {0, 1, 3}};
  const int T = c.n_tets;
  struct Face {
    int a, b, c;
    int64_t q;  // 4 * tet + local face
  };
  std::vector<Face> faces((size_t)4 * T);
  for (int t = 0; t < T; ++t)
    for (int f = 0; f < 4; ++f) {
      int v[3] = {c.tet_vex[4LL * t + fv[f][0]], c.tet_vex[4LL * t + fv[f][1]], c.tet_vex[4LL * t + fv[f][2]]};
      std::sort(v, v + 3);
      faces[4LL * t + f] = {v[0], v[1], v[2], 4LL * t + f};
    }
  std::sort(faces.begin(), faces.end(), [](const Face& x, const Face& y) {
    return x.a != y.a ? x.a < y.a : (x.b != y.b ? x.b < y.b : x.c < y.c);
  });
  mask.assign(T, 0);
  for (size_t i = 0; i < faces.size();) {
    size_t j = i + 1;
    while (j < faces.size() && faces[j].a == faces[i].a && faces[j].b == faces[i].b && faces[j].c == faces[i].c) ++j;
    if (j - i == 1) mask[faces[i].q / 4] |= (unsigned char)(1u << (faces[i].q % 4));
    i = j;
  }
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
  if (c.aniso) {
    k_element_matrices_aniso<<<ceil_div(T, 128), 128, 0, c.stream>>>(T, c.d_xyz.p, c.d_tet_vex.p, c.d_tet_drc.p,
                                                                     c.d_sig9.p, c.d_tm9.p, c.d_elemM.p, c.d_elemK.p);
  } else {
    k_element_matrices<<<ceil_div(T, 128), 128, 0, c.stream>>>(T, c.d_xyz.p, c.d_tet_vex.p, c.d_tet_drc.p,
                                                               c.d_sig.p, c.d_mu.p, c.d_elemM.p, c.d_elemK.p);
  }
  TEMF_CHECK_LAUNCH();
  if (c.bound_cond != 0) {
    k_boundary_terms<<<ceil_div(T, 128), 128, 0, c.stream>>>(T, c.d_xyz.p, c.d_tet_vex.p, c.d_tet_drc.p,
                                                             c.d_face_mask.p, c.d_elemM.p);
    TEMF_CHECK_LAUNCH();
  }
  const int64_t nnz = c.pat.nnz;
  k_gather_nonzeros<<<ceil_div(nnz, 256), 256, 0, c.stream>>>(nnz, c.d_contrib_ptr.p, c.d_contrib_idx.p,
                                                              c.d_elemM.p, c.d_elemK.p, c.d_M.p, c.d_K.p);
  TEMF_CHECK_LAUNCH();
}

}  // namespace temf
