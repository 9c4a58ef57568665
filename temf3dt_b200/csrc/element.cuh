#pragma once
// Per-tetrahedron Nedelec element integrals shared by the assembly and the
// adjoint-gradient kernels.
//
// f_kind_iso (src/FETD_FWD.f90:826-851): F_ij = l_i l_j / (720 V) *
//   [g_qi.g_qj (1+d(pi,pj)) - g_pi.g_qj (1+d(qi,pj)) - g_qi.g_pj (1+d(pi,qj)) + g_pi.g_pj (1+d(qi,qj))]
// e_kind_iso (src/FETD_FWD.f90:797-824): E_ij = 4 l_i l_j V / (6V)^4 (g_pi x g_qi).(g_pj x g_qj)
// with g_k = (b_k, c_k, d_k) the cofactor gradients and (p_j, q_j) the local
// vertex pair of edge j (ind_tet, src/FETD_FWD.f90:23).  Both matrices are
// returned as 21 packed upper entries, without the material factor and
// without the orientation signs.
namespace temf {

__host__ __device__ inline int packed_upper(int i, int j) {  // i <= j < 6
  return i * 6 - (i * (i - 1)) / 2 + (j - i);
}

// local edge j joins local vertices ind_tet(j,0) -> ind_tet(j,1):
// (0,1) (0,2) (0,3) (1,2) (3,1) (2,3)
__host__ __device__ __forceinline__ int ind_tet(int j, int k) {
  return (k == 0) ? (j == 4 ? 3 : (j < 3 ? 0 : (j == 3 ? 1 : 2)))
                  : (j == 0 ? 1 : (j == 1 ? 2 : (j == 2 ? 3 : (j == 3 ? 2 : (j == 4 ? 1 : 3)))));
}

// Gradients g_k = (b_k, c_k, d_k) and V, written as differences from the first
// vertex (the cofactor expansion of the reference's 3x3 determinants after
// subtracting one row from the others; same values up to rounding).
__host__ __device__ inline void tet_gradients(const double X[4][3], double g[4][3], double& vol) {
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

// vtk_field_save (src/FETD_FWD.f90:1670-1711) for one tet: E and D of the
// edge values ev[j] (orientation signs applied) at the centroid, where every
// barycentric coordinate is 1/4:
//   E = sum_j ev_j l_j (lam_p g_q - lam_q g_p) / (6V)^2 with lam = 6V / 4,
//   D = sum_j ev_j 2 l_j (g_p x g_q) / (6V)^2.
__host__ __device__ inline void centroid_fields(const double X[4][3], const double ev[6], double E[3], double D[3]) {
  double g[4][3], vol;
  tet_gradients(X, g, vol);
  const double v6 = 6.0 * vol;
  const double inv2 = 1.0 / (v6 * v6), lam = 0.25 * v6;
  for (int k = 0; k < 3; ++k) E[k] = D[k] = 0.0;
  for (int j = 0; j < 6; ++j) {
    const int p = ind_tet(j, 0), q = ind_tet(j, 1);
    const double dx = X[p][0] - X[q][0], dy = X[p][1] - X[q][1], dz = X[p][2] - X[q][2];
    const double s = sqrt(dx * dx + dy * dy + dz * dz) * inv2 * ev[j];
    for (int k = 0; k < 3; ++k) E[k] += s * (lam * g[q][k] - lam * g[p][k]);
    D[0] += 2.0 * s * (g[p][1] * g[q][2] - g[q][1] * g[p][2]);
    D[1] += 2.0 * s * (g[q][0] * g[p][2] - g[p][0] * g[q][2]);
    D[2] += 2.0 * s * (g[p][0] * g[q][1] - g[q][0] * g[p][1]);
  }
}

// Unit-material mass (M21) and curl-curl (K21) element matrices; either
// output may be null.
__device__ inline void unit_elements(const double X[4][3], double* M21, double* K21) {
  double g[4][3], vol;
  tet_gradients(X, g, vol);
  double len[6], cr[6][3];
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    const int p = ind_tet(j, 0), q = ind_tet(j, 1);
    const double dx = X[p][0] - X[q][0], dy = X[p][1] - X[q][1], dz = X[p][2] - X[q][2];
    len[j] = sqrt(dx * dx + dy * dy + dz * dz);
    cr[j][0] = g[p][1] * g[q][2] - g[q][1] * g[p][2];
    cr[j][1] = g[q][0] * g[p][2] - g[p][0] * g[q][2];
    cr[j][2] = g[p][0] * g[q][1] - g[q][0] * g[p][1];
  }
  double gram[4][4];
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int l = 0; l < 4; ++l) gram[k][l] = g[k][0] * g[l][0] + g[k][1] * g[l][1] + g[k][2] * g[l][2];
  const double v6 = 6.0 * vol;
  const double fM = 1.0 / (720.0 * vol);
  const double fK = 4.0 * vol / (v6 * v6 * v6 * v6);
#pragma unroll
  for (int i = 0; i < 6; ++i) {
#pragma unroll
    for (int j = i; j < 6; ++j) {
      const int pi = ind_tet(i, 0), qi = ind_tet(i, 1);
      const int pj = ind_tet(j, 0), qj = ind_tet(j, 1);
      const double br = gram[qi][qj] * (1.0 + (pi == pj)) - gram[pi][qj] * (1.0 + (qi == pj)) -
                        gram[qi][pj] * (1.0 + (pi == qj)) + gram[pi][pj] * (1.0 + (qi == qj));
      const double ll = len[i] * len[j];
      const double dots = cr[i][0] * cr[j][0] + cr[i][1] * cr[j][1] + cr[i][2] * cr[j][2];
      const int k = packed_upper(i, j);
      if (M21) M21[k] = ll * fM * br;
      if (K21) K21[k] = ll * fK * dots;
    }
  }
}

// Anisotropic media (f_kind_ani, src/FETD_FWD.f90:884-912; e_kind_ani,
// :853-882): the mass bracket with g_k . S g_l in place of g_k . g_l, and the
// curl-curl term (curl N_i) . Tm (curl N_j) V, where S is the conductivity
// tensor and Tm the tensor mesh_process passes for mu (the elementwise
// reciprocal of the permeability tensor, :624-633).  Row-major 3 x 3 inputs;
// 21 packed upper entries out, without orientation signs.
__device__ inline void aniso_elements(const double X[4][3], const double* S, const double* Tm, double* M21,
                                      double* K21) {
  double g[4][3], vol;
  tet_gradients(X, g, vol);
  double len[6], cr[6][3];
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    const int p = ind_tet(j, 0), q = ind_tet(j, 1);
    const double dx = X[p][0] - X[q][0], dy = X[p][1] - X[q][1], dz = X[p][2] - X[q][2];
    len[j] = sqrt(dx * dx + dy * dy + dz * dz);
    cr[j][0] = g[p][1] * g[q][2] - g[q][1] * g[p][2];
    cr[j][1] = g[q][0] * g[p][2] - g[p][0] * g[q][2];
    cr[j][2] = g[p][0] * g[q][1] - g[q][0] * g[p][1];
  }
  double H[4][4];
#pragma unroll
  for (int l = 0; l < 4; ++l) {
    double sg[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) sg[a] = S[3 * a] * g[l][0] + S[3 * a + 1] * g[l][1] + S[3 * a + 2] * g[l][2];
#pragma unroll
    for (int k = 0; k < 4; ++k) H[k][l] = g[k][0] * sg[0] + g[k][1] * sg[1] + g[k][2] * sg[2];
  }
  double tc[6][3];
#pragma unroll
  for (int j = 0; j < 6; ++j)
#pragma unroll
    for (int a = 0; a < 3; ++a) tc[j][a] = Tm[3 * a] * cr[j][0] + Tm[3 * a + 1] * cr[j][1] + Tm[3 * a + 2] * cr[j][2];
  const double v6 = 6.0 * vol;
  const double fM = 1.0 / (vol * 720.0);
  const double fK = 4.0 * vol / (v6 * v6 * v6 * v6);
#pragma unroll
  for (int i = 0; i < 6; ++i) {
#pragma unroll
    for (int j = i; j < 6; ++j) {
      const int pi = ind_tet(i, 0), qi = ind_tet(i, 1);
      const int pj = ind_tet(j, 0), qj = ind_tet(j, 1);
      const double br = H[qi][qj] * (1.0 + (pi == pj)) - H[pi][qj] * (1.0 + (qi == pj)) -
                        H[qi][pj] * (1.0 + (pi == qj)) + H[pi][pj] * (1.0 + (qi == qj));
      const double ll = len[i] * len[j];
      const double dots = cr[i][0] * tc[j][0] + cr[i][1] * tc[j][1] + cr[i][2] * tc[j][2];
      const int k = packed_upper(i, j);
      M21[k] = ll * fM * br;
      K21[k] = ll * fK * dots;
    }
  }
}

// First-order absorbing boundary (surface_integral, src/FETD_FWD.f90:914-1007):
// local face f of a tet has vertices face_vertex(f, 0..2) and edges
// face_edge(f, 0..2) with directions face_dir(f, 0..2) (ind_tri, ind_edg,
// ind_dir, :24-26).  face_integral is triangle_int + f_int_2d as written.
__device__ __forceinline__ int face_vertex(int f, int k) {
  const int t[4][3] = {{0, 2, 1}, {3, 1, 2}, {0, 3, 2}, {0, 1, 3}};
  return t[f][k];
}
__device__ __forceinline__ int face_edge(int f, int k) {
  const int t[4][3] = {{3, 0, 1}, {3, 5, 4}, {5, 1, 2}, {4, 2, 0}};
  return t[f][k];
}
__device__ __forceinline__ double face_dir(int f, int k) { return (k == 2 || f == 1) ? 1.0 : -1.0; }

__device__ inline void face_integral(const double P[3][3], double F[3][3]) {
  double d21[3], d31[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    d21[a] = P[1][a] - P[0][a];
    d31[a] = P[2][a] - P[0][a];
  }
  const double u2 = sqrt(d21[0] * d21[0] + d21[1] * d21[1] + d21[2] * d21[2]);
  const double u3 = (d31[0] * d21[0] + d31[1] * d21[1] + d31[2] * d21[2]) / u2;
  const double l31 = sqrt(d31[0] * d31[0] + d31[1] * d31[1] + d31[2] * d31[2]);
  const double r = u3 / l31;
  const double v3 = sqrt(1.0 - r * r) * l31;
  const double x[3] = {0.0, u2, u3}, y[3] = {0.0, 0.0, v3};
  const double len[3] = {hypot(x[0] - x[1], y[0] - y[1]), hypot(x[1] - x[2], y[1] - y[2]),
                         hypot(x[2] - x[0], y[2] - y[0])};
  const double area = 0.5 * (x[0] * (y[1] - y[2]) - y[0] * (x[1] - x[2]) + 1.0 * (x[1] * y[2] - x[2] * y[1]));
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const double v = 6.0 * (y[i] - y[2]) * (y[j] - y[2]) - 2.0 * (y[i] + y[j] - 2.0 * y[2]) * (y[0] + y[1] - 2.0 * y[2]) +
                       (y[0] - y[2]) * (y[0] - y[2]) + (y[1] - y[2]) * (y[1] - y[2]) + (y[0] - y[2]) * (y[1] - y[2]) +
                       6.0 * (x[i] - x[2]) * (x[j] - x[2]) - 2.0 * (x[i] + x[j] - 2.0 * x[2]) * (x[0] + x[1] - 2.0 * x[2]) +
                       (x[0] - x[2]) * (x[0] - x[2]) + (x[1] - x[2]) * (x[1] - x[2]) + (x[0] - x[2]) * (x[1] - x[2]);
      F[i][j] = v * len[i] * len[j] / 24.0 / area;
    }
}

}  // namespace temf
