// K4 + K5 + K6 + K7: per-step kernels of the FETD time loop.
//
//  * K5  r = M_sigma (4 e^n - e^{n-1}) - 2 dt s(t): the BDF2 right-hand side,
//        src/FETD_FWD.f90:1425-1428 (mkl_sparse_d_mv with the symmetric-upper
//        descriptor, :1191-1193; sys_right :1466-1511).  Full symmetric CSR,
//        eight lanes per row with shuffle reductions, vectors in the
//        fill-reducing order so no permutation happens per step.
//  * K4  x = A^{-1} r with the supernodal factor: PARDISO phase 33,
//        src/FETD_UTILITY.f90:938-957.  Forward substitution by bottom-up
//        levels, backward by top-down levels, one CTA per supernode; the
//        below-diagonal coupling of the forward sweep goes through a per-supernode
//        update buffer that the consumer gathers in a fixed order, so the solve
//        is deterministic (no atomics).
//  * K6  ||a - b||^2 and ||b||^2 for the dt-doubling test (two_error,
//        src/FETD_UTILITY.f90:578-599), fixed-order block reduction.
//  * K7  receiver E and dB/dt from the six edge values of the receiver's
//        tetrahedron (solution_output, src/FETD_FWD.f90:1532-1540).
#include <algorithm>

#include "factor.h"
#include "solve.h"

namespace temf {

constexpr int kSolveThreads = 128;

// ---------------------------------------------------------------------------
// forward:  L y = b  (one level)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kSolveThreads) k_fwd_level(
    const int* __restrict__ level_sn, const int* __restrict__ sn_first,
    const int64_t* __restrict__ rows_ptr, const int64_t* __restrict__ Lptr, double* const* Lbase,
    const int64_t* __restrict__ in_ptr, const int64_t* __restrict__ in_idx,
    const int64_t* __restrict__ uoff, double* __restrict__ u, double* __restrict__ x, int nrhs) {
  constexpr int CB = kSnCols;
  __shared__ double D[CB][CB + 1];
  extern __shared__ double ys[];  // [c][nrhs]
  const int s = level_sn[blockIdx.x];
  const int f = sn_first[s];
  const int c = sn_first[s + 1] - f;
  const int64_t r = rows_ptr[s + 1] - rows_ptr[s];
  const int64_t ld = c + r;
  const double* P = *Lbase + Lptr[s];
  const int tid = threadIdx.x;
  for (int idx = tid; idx < c * c; idx += blockDim.x) {
    const int j = idx / c, i = idx % c;
    if (i >= j) D[i][j] = P[(int64_t)j * ld + i];
  }
  for (int idx = tid; idx < c * nrhs; idx += blockDim.x) {
    const int k = idx / nrhs, col = idx % nrhs;
    double v = x[(int64_t)(f + k) * nrhs + col];
    for (int64_t q = in_ptr[f + k]; q < in_ptr[f + k + 1]; ++q) v -= u[in_idx[q] * nrhs + col];
    ys[idx] = v;
  }
  __syncthreads();
  if (nrhs == 1) {
    if (tid < 32) {
      const int lane = tid;
      double y0 = lane < c ? ys[lane] : 0.0;
      double y1 = lane + 32 < c ? ys[lane + 32] : 0.0;
      for (int j = 0; j < c; ++j) {
        const double v = __shfl_sync(0xffffffffu, j < 32 ? y0 : y1, j & 31);
        const double yj = v / D[j][j];
        if (lane == (j & 31)) { if (j < 32) y0 = yj; else y1 = yj; }
        if (lane > j && lane < c) y0 -= D[lane][j] * yj;
        if (lane + 32 > j && lane + 32 < c) y1 -= D[lane + 32][j] * yj;
      }
      if (lane < c) ys[lane] = y0;
      if (lane + 32 < c) ys[lane + 32] = y1;
    }
  } else {
    for (int j = 0; j < c; ++j) {
      for (int col = tid; col < nrhs; col += blockDim.x) ys[j * nrhs + col] /= D[j][j];
      __syncthreads();
      for (int idx = tid; idx < (c - j - 1) * nrhs; idx += blockDim.x) {
        const int k = j + 1 + idx / nrhs, col = idx % nrhs;
        ys[k * nrhs + col] -= D[k][j] * ys[j * nrhs + col];
      }
      __syncthreads();
    }
  }
  __syncthreads();
  for (int idx = tid; idx < c * nrhs; idx += blockDim.x) x[(int64_t)f * nrhs + idx] = ys[idx];
  // u_s = L21 y_s
  double* us = u + uoff[s] * nrhs;
  for (int64_t i = tid; i < r; i += blockDim.x) {
    for (int col = 0; col < nrhs; ++col) {
      double acc = 0.0;
      for (int j = 0; j < c; ++j) acc += P[(int64_t)j * ld + c + i] * ys[j * nrhs + col];
      us[i * nrhs + col] = acc;
    }
  }
}

// ---------------------------------------------------------------------------
// backward:  L^T x = y  (one level, top-down)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kSolveThreads) k_bwd_level(
    const int* __restrict__ level_sn, const int* __restrict__ sn_first,
    const int64_t* __restrict__ rows_ptr, const int* __restrict__ sn_rows,
    const int64_t* __restrict__ Lptr, double* const* Lbase, double* __restrict__ x, int nrhs) {
  constexpr int CB = kSnCols;
  __shared__ double D[CB][CB + 1];
  extern __shared__ double zs[];  // [c][nrhs]
  const int s = level_sn[blockIdx.x];
  const int f = sn_first[s];
  const int c = sn_first[s + 1] - f;
  const int64_t rp = rows_ptr[s];
  const int64_t r = rows_ptr[s + 1] - rp;
  const int64_t ld = c + r;
  const double* P = *Lbase + Lptr[s];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
  for (int idx = tid; idx < c * c; idx += blockDim.x) {
    const int j = idx / c, i = idx % c;
    if (i >= j) D[i][j] = P[(int64_t)j * ld + i];
  }
  for (int idx = tid; idx < c * nrhs; idx += blockDim.x) zs[idx] = x[(int64_t)f * nrhs + idx];
  __syncthreads();
  // z_j -= sum_i L21[i][j] x[rows_i]
  for (int j = warp; j < c; j += nw) {
    const double* colp = P + (int64_t)j * ld + c;
    for (int col = 0; col < nrhs; ++col) {
      double acc = 0.0;
      for (int64_t i = lane; i < r; i += 32) acc += colp[i] * x[(int64_t)sn_rows[rp + i] * nrhs + col];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
      if (lane == 0) zs[j * nrhs + col] -= acc;
    }
  }
  __syncthreads();
  if (nrhs == 1) {
    if (tid < 32) {
      double z0 = lane < c ? zs[lane] : 0.0;
      double z1 = lane + 32 < c ? zs[lane + 32] : 0.0;
      for (int j = c - 1; j >= 0; --j) {
        const double v = __shfl_sync(0xffffffffu, j < 32 ? z0 : z1, j & 31);
        const double xj = v / D[j][j];
        if (lane == (j & 31)) { if (j < 32) z0 = xj; else z1 = xj; }
        if (lane < j) z0 -= D[j][lane] * xj;
        if (lane + 32 < j) z1 -= D[j][lane + 32] * xj;
      }
      if (lane < c) zs[lane] = z0;
      if (lane + 32 < c) zs[lane + 32] = z1;
    }
  } else {
    for (int j = c - 1; j >= 0; --j) {
      for (int col = tid; col < nrhs; col += blockDim.x) zs[j * nrhs + col] /= D[j][j];
      __syncthreads();
      for (int idx = tid; idx < j * nrhs; idx += blockDim.x) {
        const int k = idx / nrhs, col = idx % nrhs;
        zs[k * nrhs + col] -= D[j][k] * zs[j * nrhs + col];
      }
      __syncthreads();
    }
  }
  __syncthreads();
  for (int idx = tid; idx < c * nrhs; idx += blockDim.x) x[(int64_t)f * nrhs + idx] = zs[idx];
}

// ---------------------------------------------------------------------------
// SpMV-type kernels
// ---------------------------------------------------------------------------
// y = M (4 e2 - e3), eight lanes per row
__global__ void __launch_bounds__(256) k_bdf_rhs(int n, const int* __restrict__ rowptr,
                                                 const int* __restrict__ col, const double* __restrict__ M,
                                                 const double* __restrict__ e2, const double* __restrict__ e3,
                                                 double* __restrict__ y) {
  const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int row = (int)(gid >> 3);
  const int sub = (int)(gid & 7);
  double acc = 0.0;
  if (row < n) {
    const int p1 = rowptr[row + 1];
    for (int p = rowptr[row] + sub; p < p1; p += 8) {
      const int j = __ldg(col + p);
      acc += __ldg(M + p) * (4.0 * __ldg(e2 + j) - __ldg(e3 + j));
    }
  }
  acc += __shfl_down_sync(0xffffffffu, acc, 4, 8);
  acc += __shfl_down_sync(0xffffffffu, acc, 2, 8);
  acc += __shfl_down_sync(0xffffffffu, acc, 1, 8);
  if (row < n && sub == 0) y[row] = acc;
}

// multi-column variants: one thread per (row, column)
__global__ void k_bdf_rhs_multi(int n, int nrhs, const int* __restrict__ rowptr, const int* __restrict__ col,
                                const double* __restrict__ M, const double* __restrict__ e2,
                                const double* __restrict__ e3, double* __restrict__ y) {
  const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (int64_t)n * nrhs) return;
  const int row = (int)(gid / nrhs), cc = (int)(gid % nrhs);
  double acc = 0.0;
  for (int p = rowptr[row]; p < rowptr[row + 1]; ++p) {
    const int64_t j = (int64_t)col[p] * nrhs + cc;
    acc += M[p] * (4.0 * e2[j] - e3[j]);
  }
  y[gid] = acc;
}

__global__ void k_spmv_multi(int n, int nrhs, const int* __restrict__ rowptr, const int* __restrict__ col,
                             const double* __restrict__ M, const double* __restrict__ x, double* __restrict__ y) {
  const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (int64_t)n * nrhs) return;
  const int row = (int)(gid / nrhs), cc = (int)(gid % nrhs);
  double acc = 0.0;
  for (int p = rowptr[row]; p < rowptr[row + 1]; ++p) acc += M[p] * x[(int64_t)col[p] * nrhs + cc];
  y[gid] = acc;
}

__global__ void k_source(int nent, const int* __restrict__ idx, const int* __restrict__ rcol,
                         const double* __restrict__ coef, const double* __restrict__ scal, int nrhs,
                         double* __restrict__ y) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nent) return;
  y[(int64_t)idx[q] * nrhs + rcol[q]] -= scal[0] * coef[q];
}

__global__ void k_receivers(int nrec, const int* __restrict__ edges, const int* __restrict__ rrhs,
                            const double* __restrict__ w, const double* __restrict__ x, int nrhs,
                            double* __restrict__ out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nrec * 6) return;
  const int rec = t / 6, q = t % 6;
  double acc = 0.0;
#pragma unroll
  for (int j = 0; j < 6; ++j) acc += w[rec * 36 + q * 6 + j] * x[(int64_t)edges[rec * 6 + j] * nrhs + rrhs[rec]];
  out[t] = acc;
}

constexpr int kErrBlocks = 296;
__global__ void __launch_bounds__(256) k_err_partial(int64_t n, int nrhs, const double* __restrict__ a,
                                                     const double* __restrict__ b, double* __restrict__ part) {
  // part[(block * nrhs + col) * 2 + {0,1}]
  __shared__ double sa[256], sb[256];
  for (int col = 0; col < nrhs; ++col) {
    double da = 0.0, db = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
      const double bv = b[i * nrhs + col];
      const double d = a[i * nrhs + col] - bv;
      da += d * d;
      db += bv * bv;
    }
    sa[threadIdx.x] = da;
    sb[threadIdx.x] = db;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
      if (threadIdx.x < o) { sa[threadIdx.x] += sa[threadIdx.x + o]; sb[threadIdx.x] += sb[threadIdx.x + o]; }
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      part[((int64_t)blockIdx.x * nrhs + col) * 2 + 0] = sa[0];
      part[((int64_t)blockIdx.x * nrhs + col) * 2 + 1] = sb[0];
    }
    __syncthreads();
  }
}

__global__ void k_err_final(int nblocks, int nrhs, const double* __restrict__ part, double* __restrict__ out) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= nrhs) return;
  double da = 0.0, db = 0.0;
  for (int b = 0; b < nblocks; ++b) {
    da += part[((int64_t)b * nrhs + col) * 2 + 0];
    db += part[((int64_t)b * nrhs + col) * 2 + 1];
  }
  out[2 * col] = da;
  out[2 * col + 1] = db;
}

// ---------------------------------------------------------------------------
// host
// ---------------------------------------------------------------------------
void build_solve_plan(temf_ctx& c) {
  const Symbolic& S = c.sym;
  SolvePlan& P = c.splan;
  const int n = S.n, nsn = S.nsn;
  std::vector<int64_t> uoff(nsn + 1, 0);
  for (int s = 0; s < nsn; ++s) uoff[s + 1] = uoff[s] + (S.sn_rows_ptr[s + 1] - S.sn_rows_ptr[s]);
  P.u_len = uoff[nsn];
  std::vector<int64_t> in_ptr(n + 1, 0);
  for (size_t q = 0; q < S.sn_rows.size(); ++q) in_ptr[S.sn_rows[q] + 1]++;
  for (int i = 0; i < n; ++i) in_ptr[i + 1] += in_ptr[i];
  std::vector<int64_t> in_idx(S.sn_rows.size());
  std::vector<int64_t> fill(in_ptr.begin(), in_ptr.end() - 1);
  for (int s = 0; s < nsn; ++s)
    for (int64_t q = S.sn_rows_ptr[s]; q < S.sn_rows_ptr[s + 1]; ++q)
      in_idx[fill[S.sn_rows[q]]++] = uoff[s] + (q - S.sn_rows_ptr[s]);
  P.uoff.upload(uoff.data(), uoff.size(), c.stream);
  P.in_ptr.upload(in_ptr.data(), in_ptr.size(), c.stream);
  P.in_idx.upload(in_idx.data(), in_idx.size(), c.stream);
  TEMF_CUDA(cudaStreamSynchronize(c.stream));
}

void ensure_update_buffer(temf_ctx& c, int nrhs) {
  const size_t need = (size_t)std::max<int64_t>(c.splan.u_len, 1) * nrhs;
  if (c.d_u.n < need) c.d_u.alloc(need);
}

static size_t solve_smem(int nrhs) { return (size_t)kSnCols * nrhs * sizeof(double); }

void launch_solve(temf_ctx& c, double* const* Lbase, double* x, int nrhs, cudaStream_t st) {
  const Symbolic& S = c.sym;
  FactorPlan& F = c.fplan;
  SolvePlan& P = c.splan;
  ensure_update_buffer(c, nrhs);
  const size_t smem = solve_smem(nrhs);
  if (smem > 48 * 1024) {
    TEMF_CUDA(cudaFuncSetAttribute(k_fwd_level, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    TEMF_CUDA(cudaFuncSetAttribute(k_bwd_level, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  }
  for (int l = 0; l < S.nlevels; ++l) {
    const int cnt = S.level_ptr[l + 1] - S.level_ptr[l];
    if (!cnt) continue;
    k_fwd_level<<<cnt, kSolveThreads, smem, st>>>(F.level_sn.p + S.level_ptr[l], F.sn_first.p, F.sn_rows_ptr.p,
                                                  F.sn_Lptr.p, Lbase, P.in_ptr.p, P.in_idx.p, P.uoff.p, c.d_u.p, x,
                                                  nrhs);
    TEMF_CHECK_LAUNCH();
  }
  for (int l = S.nlevels - 1; l >= 0; --l) {
    const int cnt = S.level_ptr[l + 1] - S.level_ptr[l];
    if (!cnt) continue;
    k_bwd_level<<<cnt, kSolveThreads, smem, st>>>(F.level_sn.p + S.level_ptr[l], F.sn_first.p, F.sn_rows_ptr.p,
                                                  F.sn_rows.p, F.sn_Lptr.p, Lbase, x, nrhs);
    TEMF_CHECK_LAUNCH();
  }
}

void launch_bdf_rhs(temf_ctx& c, const double* e2, const double* e3, double* y, int nrhs, cudaStream_t st) {
  const int n = c.pat.n;
  if (nrhs == 1) {
    k_bdf_rhs<<<ceil_div((int64_t)n * 8, 256), 256, 0, st>>>(n, c.d_rowptr.p, c.d_col.p, c.d_M.p, e2, e3, y);
  } else {
    k_bdf_rhs_multi<<<ceil_div((int64_t)n * nrhs, 256), 256, 0, st>>>(n, nrhs, c.d_rowptr.p, c.d_col.p, c.d_M.p,
                                                                       e2, e3, y);
  }
  TEMF_CHECK_LAUNCH();
}

void launch_spmv(temf_ctx& c, const double* M, const double* x, double* y, int nrhs, cudaStream_t st) {
  const int n = c.pat.n;
  k_spmv_multi<<<ceil_div((int64_t)n * nrhs, 256), 256, 0, st>>>(n, nrhs, c.d_rowptr.p, c.d_col.p, M, x, y);
  TEMF_CHECK_LAUNCH();
}

void launch_source(temf_ctx& c, const double* coef_dev, double* y, int nrhs, cudaStream_t st) {
  const int nent = (int)c.src.idx.size();
  if (!nent) return;
  k_source<<<ceil_div(nent, 128), 128, 0, st>>>(nent, c.src.d_idx.p, c.src.d_col.p, c.src.d_coef.p, coef_dev,
                                                nrhs, y);
  TEMF_CHECK_LAUNCH();
}

void launch_receivers(temf_ctx& c, const double* x, int nrhs, double* out, cudaStream_t st) {
  const int nrec = c.rec.nrec;
  if (!nrec) return;
  k_receivers<<<ceil_div(nrec * 6, 128), 128, 0, st>>>(nrec, c.rec.d_edges.p, c.rec.d_rhs.p, c.rec.d_w.p, x, nrhs,
                                                      out);
  TEMF_CHECK_LAUNCH();
}

void launch_two_error(temf_ctx& c, const double* a, const double* b, int nrhs, double* out, cudaStream_t st) {
  // partials live right after the 2*nrhs outputs: the caller provides `out`
  // with room for (1 + kErrBlocks) * 2 * nrhs doubles (see two_error_len()).
  double* partials = out + 2 * nrhs;
  k_err_partial<<<kErrBlocks, 256, 0, st>>>(c.pat.n, nrhs, a, b, partials);
  TEMF_CHECK_LAUNCH();
  k_err_final<<<ceil_div(nrhs, 64), 64, 0, st>>>(kErrBlocks, nrhs, partials, out);
  TEMF_CHECK_LAUNCH();
}

}  // namespace temf
