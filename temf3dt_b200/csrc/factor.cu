// K2 + K3: step-matrix formation and supernodal numeric Cholesky on the GPU.
//
// Replaces mkl_add_3 + mkl_to_csr (src/FETD_FWD.f90:2006-2039, 1974-2004)
// and the numeric part of PARDISO phase 12 (src/FETD_UTILITY.f90:912-917,
// mtype 2 = real SPD).  A(dt) = 0*A_eps + 3*M_sigma + 2*dt*K is formed
// directly into the supernodal panels (the pattern is dt-independent).
//
// Schedule: bottom-up levels of the supernodal elimination tree.  Per level:
//   k_potrf      : one CTA per supernode: dense Cholesky of the (<=64 x 64)
//                  diagonal block in shared memory;
//   k_trsm       : the below-diagonal rows solved against it, 128 rows per
//                  CTA (one row per thread, in registers);
//   k_update     : the Schur update L21 L21^T of every supernode of the level,
//                  in 64x64 tiles on the FP64 tensor cores (DMMA
//                  mma.sync.m8n8k4.f64), scattered into the ancestor panels
//                  through precomputed relative indices.  Several supernodes
//                  of one level may update the same ancestor entry, so the
//                  scatter of such levels uses FP64 atomics
//                  (red.global.add.f64); a level holding a single supernode
//                  (the dense top of the tree, where most flops are) writes
//                  with plain read-modify-write.
// Pivot failures are reported through a status word (first failing column),
// never by trapping.
#include <algorithm>
#include <climits>

#include "factor.h"

namespace temf {

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------
__global__ void k_load_A(int64_t n, const int* __restrict__ src, const int64_t* __restrict__ dst,
                         const double* __restrict__ M, double a, const double* __restrict__ K, double b,
                         double* __restrict__ L) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const int p = src[q];
  L[dst[q]] = a * M[p] + (K ? b * K[p] : 0.0);
}

constexpr int kFacThreads = 128;

// Dense Cholesky of the (<= 64 x 64) diagonal block of each supernode of a level.
//
// sgn != null: the indefinite mode, A = L S L^T with S = diag(+-1) (sgn, in
// the permuted order) and L_kk = sqrt(|d_k|) > 0, the sign of the pivot d_k in
// s_k.  A pivot that cancels below kPivotTol of its column's diagonal entry
// as the block's elimination starts (or is not finite) is perturbed to that
// size (static pivot perturbation, counted in status[2]); the iterative
// refinement of the solves recovers the accuracy.  The first non-positive
// pivot is recorded in status[0] in both modes.
constexpr double kPivotTol = 1e-13;

__global__ void __launch_bounds__(kFacThreads) k_potrf(
    const int* __restrict__ level_sn, const int* __restrict__ sn_first,
    const int64_t* __restrict__ rows_ptr, const int64_t* __restrict__ Lptr, double* __restrict__ L,
    int* __restrict__ status, double* __restrict__ sgn, const int64_t* __restrict__ Dptr) {
  constexpr int CB = kSnCols;
  __shared__ double D[CB][CB + 1];
  __shared__ double diag[CB];  // L_kk, written into D after the loop
  __shared__ double d0[CB];
  const int s = level_sn[blockIdx.x];
  const int f = sn_first[s];
  const int c = sn_first[s + 1] - f;
  const int64_t r = rows_ptr[s + 1] - rows_ptr[s];
  const int64_t ld = c + r;
  double* P = L + Lptr[s];
  const int tid = threadIdx.x;
  for (int idx = tid; idx < c * c; idx += blockDim.x) {
    const int j = idx / c, i = idx % c;
    D[i][j] = (i >= j) ? P[(int64_t)j * ld + i] : 0.0;
  }
  __syncthreads();
  if (tid < c) d0[tid] = fabs(D[tid][tid]);
  __syncthreads();
  // Right-looking, two barriers per column: every thread derives the pivot
  // from the same shared value (the diagonal itself is written at the end),
  // the column is scaled, then the trailing triangle is updated on a 8 x 16
  // thread grid.
  const int tx = tid & 15, ty = tid >> 4;
  for (int k = 0; k < c; ++k) {
    const double a = D[k][k];
    double d = a, s = 1.0;
    bool perturbed = false;
    if (sgn) {
      s = d < 0.0 ? -1.0 : 1.0;
      d = fabs(d);
      const double tau = kPivotTol * (d0[k] > 0.0 ? d0[k] : 1.0);
      if (!(d >= tau) || !(d <= 1e300)) {  // cancelled, NaN or infinite pivot: perturb
        d = tau;
        perturbed = true;
      }
    } else if (!(d > 0.0)) {
      d = 1.0;  // continue with 1; the factor is reported invalid
    }
    const double lkk = sqrt(d);
    if (tid == 0) {
      if (!(a > 0.0)) atomicMin(status, f + k + 1);  // non-positive or NaN pivot: record
      if (perturbed) atomicAdd(status + 2, 1);
      if (sgn) sgn[f + k] = s;
      diag[k] = lkk;
    }
    const double inv = 1.0 / (lkk * s);
    for (int i = k + 1 + tid; i < c; i += blockDim.x) D[i][k] *= inv;
    __syncthreads();
    for (int ii = k + 1 + ty; ii < c; ii += 8) {
      const double lik = D[ii][k] * s;
      for (int jj = k + 1 + tx; jj <= ii; jj += 16) D[ii][jj] -= lik * D[jj][k];
    }
    __syncthreads();
  }
  if (tid < c) {
    D[tid][tid] = diag[tid];
    d0[tid] = 1.0 / diag[tid];
  }
  __syncthreads();
  // the panel's block, and the sweeps' copy: row i scaled by 1/L_ii, 1/L_ii on
  // the diagonal, zeros above (c x c, column-major)
  double* Q = L + Dptr[s];
  for (int idx = tid; idx < c * c; idx += blockDim.x) {
    const int j = idx / c, i = idx % c;
    if (i >= j) P[(int64_t)j * ld + i] = D[i][j];
    Q[idx] = i > j ? D[i][j] * d0[i] : (i == j ? d0[i] : 0.0);
  }
}

// Below-diagonal rows of the level's supernodes, kTrsmRows rows per CTA:
// x L11^T = a, forward substitution per row in registers.
struct TrsmChunk {
  int s;
  int r0;
};
constexpr int kTrsmRows = kFacThreads;

// Indefinite mode (sgn != null): L21 = A21 L11^{-T} S11.
__global__ void __launch_bounds__(kFacThreads) k_trsm(const TrsmChunk* __restrict__ chunks,
                                                      const int* __restrict__ sn_first,
                                                      const int64_t* __restrict__ rows_ptr,
                                                      const int64_t* __restrict__ Lptr, double* __restrict__ L,
                                                      const double* __restrict__ sgn) {
  constexpr int CB = kSnCols;
  __shared__ double D[CB][CB + 1];
  const TrsmChunk ch = chunks[blockIdx.x];
  const int s = ch.s;
  const int f = sn_first[s];
  const int c = sn_first[s + 1] - f;
  const int64_t r = rows_ptr[s + 1] - rows_ptr[s];
  const int64_t ld = c + r;
  double* P = L + Lptr[s];
  const int tid = threadIdx.x;
  for (int idx = tid; idx < c * c; idx += blockDim.x) {
    const int j = idx / c, i = idx % c;
    if (i >= j) D[i][j] = P[(int64_t)j * ld + i];
  }
  __syncthreads();
  const int64_t i = ch.r0 + tid;
  if (i >= r) return;
  double x[CB];
#pragma unroll
  for (int j = 0; j < CB; ++j) x[j] = (j < c) ? P[(int64_t)j * ld + c + i] : 0.0;
#pragma unroll
  for (int j = 0; j < CB; ++j) {
    if (j < c) {
      double v = x[j];
#pragma unroll
      for (int k = 0; k < j; ++k) v -= x[k] * D[j][k];
      x[j] = v / D[j][j];
    }
  }
  if (sgn) {
#pragma unroll
    for (int j = 0; j < CB; ++j)
      if (j < c) x[j] *= sgn[f + j];
  }
#pragma unroll
  for (int j = 0; j < CB; ++j)
    if (j < c) P[(int64_t)j * ld + c + i] = x[j];
}

__device__ __forceinline__ void dmma_8x8x4(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

constexpr int kLdsU = kUpdTile + 8;  // 72 doubles: two 128-byte wavefronts per fragment load

// Bulk global -> shared copies on the TMA engine (cp.async.bulk, this GPU's
// own memory, each CTA its own copy), completed on an mbarrier: one instruction per
// panel column segment instead of one 8-byte copy per element.  Addresses
// and sizes must be multiples of 16 bytes: a segment that starts at an odd
// double is copied from one double earlier (its rows then start at offset 1
// of the shared row), and the size is rounded up to 16 bytes -- at most one
// double past the segment, which stays inside the slot allocation (the
// panels are followed by the scaled diagonal copies).
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* b, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, unsigned bytes) {
  asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
  asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.shared::cta.b64 st, [%0];\n}\n" ::"r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* b, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void bulk_g2s(void* dst, const double* src, unsigned bytes, uint64_t* b) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   smem_u32(dst)),
               "l"(__cvta_generic_to_global(src)), "r"(bytes), "r"(smem_u32(b))
               : "memory");
}
// Bounded wait for a phase of the copy barrier: gives up after ~seconds and
// reports through the error word (the factor is then refused by the host).
constexpr int kCopySpinLimit = 1 << 22;
__device__ __forceinline__ void mbar_wait(uint64_t* b, unsigned parity, int* err) {
  for (int it = 0; !mbar_try_wait(b, parity); ++it) {
    if (it > kCopySpinLimit) {
      atomicExch(err, 1);
      return;
    }
    if (it > 64) __nanosleep(32);
  }
}

// Schur update tiles.  A tile (s, i0, j0, members m, column limit jl) holds
// C = sum over the m supernodes q = s-m+1 .. s of L21_q[rows beyond] *
// L21_q[rows beyond]^T for the 64 x 64 block (i0.., j0..) of s's row list:
// m > 1 for the column blocks of one wider supernode (a run), whose updates
// beyond the run are summed in one pass (K = the run's columns, each member's
// rows beyond the run are the rows of s, at offset r_q - r_s of its list);
// m = 1 otherwise.  jl > 0 restricts the tile to columns j < jl (inside a run,
// a member updates the later members' columns only).  C is scattered into the
// ancestors' panels through the relative indices of s.  The K loop runs over
// 16-column chunks of the members, double-buffered: the next chunk's bulk
// copies (one per column segment of A and of B: 32 per chunk, issued by warp
// 0) are in flight while the DMMA tiles consume the current one (37 KB of
// shared memory: five CTAs per SM, by registers, where 32-column chunks
// allowed three).
constexpr int kUpdChunk = 16;
constexpr int kUpdMaxMembers = 8;

__global__ void __launch_bounds__(128, 5) k_update(
    const UpdTile* __restrict__ tiles, const int* __restrict__ sn_first,
    const int64_t* __restrict__ rows_ptr, const int* __restrict__ sn_rows,
    const int64_t* __restrict__ Lptr, const int* __restrict__ row_grp,
    const int* __restrict__ grp_target, const int* __restrict__ grp_shift,
    const int64_t* __restrict__ grp_relind, const int* __restrict__ relind, double* __restrict__ L,
    int use_atomics, const double* __restrict__ sgn, int* __restrict__ err) {
  extern __shared__ __align__(128) double sm[];
  __shared__ __align__(8) uint64_t mbar[2];
  __shared__ unsigned char shift[2][2][kUpdChunk];  // per buffer, operand, row: offset of the segment's first row
  // [buffer][A | B][kUpdChunk][kLdsU]
  auto As = [&](int buf) { return sm + (size_t)buf * 2 * kUpdChunk * kLdsU; };
  auto Bs = [&](int buf) { return sm + (size_t)buf * 2 * kUpdChunk * kLdsU + kUpdChunk * kLdsU; };
  const UpdTile tile = tiles[blockIdx.x];
  const int s = tile.s;
  const int m = tile.mj & 15;
  const int jl = tile.mj >> 4;
  const int64_t rp = rows_ptr[s];
  const int r = (int)(rows_ptr[s + 1] - rp);
  const int tid = threadIdx.x;
  // K chunks of kUpdChunk columns over the members in order; a cursor
  // (member, first column) for the chunk being copied and one for the chunk
  // being multiplied
  int nch = 0;
  for (int u = 0; u < m; ++u) {
    const int q = s - m + 1 + u;
    nch += (sn_first[q + 1] - sn_first[q] + kUpdChunk - 1) / kUpdChunk;
  }
  int cp_q = s - m + 1, cp_k0 = 0, mm_q = s - m + 1, mm_k0 = 0;
  auto advance = [&](int& q, int& k0) {
    k0 += kUpdChunk;
    if (k0 >= sn_first[q + 1] - sn_first[q]) {
      ++q;
      k0 = 0;
    }
  };
  auto issue = [&](int buf) {
    const int q = cp_q, k0 = cp_k0;
    advance(cp_q, cp_k0);
    const int fq = sn_first[q];
    const int cq = sn_first[q + 1] - fq;
    const int rq = (int)(rows_ptr[q + 1] - rows_ptr[q]);
    const int64_t ldq = cq + rq;
    const double* P = L + Lptr[q] + cq + (rq - r);  // row 0 of the rows beyond the run
    if (tid < 2 * kUpdChunk) {  // warp 0: one segment each (operand A rows i0.., B rows j0..)
      const int op = tid / kUpdChunk, k = tid % kUpdChunk, kk = k0 + k;
      const int g0 = op == 0 ? tile.i0 : tile.j0;
      double* row = (op == 0 ? As(buf) : Bs(buf)) + k * kLdsU;
      if (kk < cq && g0 < r) {
        const double* src = P + (int64_t)kk * ldq + g0;
        const int n = min(kUpdTile, r - g0);  // rows past r only feed outputs that are not scattered
        const int o = (__cvta_generic_to_global(src) & 15) ? 1 : 0;
        const unsigned bytes = (unsigned)(((n + o) * 8 + 15) & ~15);
        shift[buf][op][k] = (unsigned char)o;
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        mbar_expect_tx(&mbar[buf], bytes);
        bulk_g2s(row, src - o, bytes, &mbar[buf]);
      } else {  // past the member's columns: a zero row
        shift[buf][op][k] = 0;
        for (int ii = 0; ii < kUpdTile; ++ii) row[ii] = 0.0;
      }
      __syncwarp();
      if (tid == 0) mbar_arrive(&mbar[buf]);
    }
  };
  const int warp = tid >> 5, lane = tid & 31;
  const int wr = (warp >> 1) * 32, wc = (warp & 1) * 32;
  const int g = lane >> 2, qd = lane & 3;
  double acc[4][4][2];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
  if (tid == 0) {
    mbar_init(&mbar[0], 1);
    mbar_init(&mbar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  unsigned phases = 0u;  // bit b: parity of buffer b's next phase
  issue(0);
  for (int ch = 0; ch < nch; ++ch) {
    const int buf = ch & 1;
    if (ch + 1 < nch) issue(buf ^ 1);
    mbar_wait(&mbar[buf], (phases >> buf) & 1u, err);
    phases ^= 1u << buf;
    __syncthreads();
    double* A = As(buf);
    const double* B = Bs(buf);
    if (sgn) {  // indefinite mode: A22 -= L21 S11 L21^T
      const int fq = sn_first[mm_q];
      const int cq = sn_first[mm_q + 1] - fq;
      for (int idx = tid; idx < kUpdChunk * kUpdTile; idx += blockDim.x) {
        const int k = idx / kUpdTile, ii = idx % kUpdTile;
        if (mm_k0 + k < cq) A[k * kLdsU + shift[buf][0][k] + ii] *= sgn[fq + mm_k0 + k];
      }
      __syncthreads();
    }
    advance(mm_q, mm_k0);
#pragma unroll 2
    for (int k0 = 0; k0 < kUpdChunk; k0 += 4) {
      double fa[4], fb[4];
      const int sa = shift[buf][0][k0 + qd], sb = shift[buf][1][k0 + qd];
#pragma unroll
      for (int a = 0; a < 4; ++a) fa[a] = A[(k0 + qd) * kLdsU + sa + wr + a * 8 + g];
#pragma unroll
      for (int b = 0; b < 4; ++b) fb[b] = B[(k0 + qd) * kLdsU + sb + wc + b * 8 + g];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) dmma_8x8x4(acc[a][b][0], acc[a][b][1], fa[a], fb[b]);
    }
    __syncthreads();  // the buffer is refilled by the next issue
  }
  // scatter-subtract into the ancestors
  const int jend = jl > 0 ? min(jl, r) : r;
#pragma unroll
  for (int b = 0; b < 4; ++b) {
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const int j = tile.j0 + wc + b * 8 + 2 * qd + e;
      if (j >= jend) continue;
      const int grp = row_grp[rp + j];
      const int t = grp_target[grp];
      const int ft = sn_first[t];
      const int ct = sn_first[t + 1] - ft;
      const int64_t ldt = ct + (rows_ptr[t + 1] - rows_ptr[t]);
      double* dstcol = L + Lptr[t] + (int64_t)(sn_rows[rp + j] - ft) * ldt - grp_shift[grp];
      const int* rel = relind + grp_relind[grp];
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        const int i = tile.i0 + wr + a * 8 + g;
        if (i < r && i >= j) {
          // one supernode per level: every target entry has a single writer
          if (use_atomics) atomicAdd(dstcol + rel[i], -acc[a][b][e]);
          else dstcol[rel[i]] -= acc[a][b][e];
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// host plan
// ---------------------------------------------------------------------------
// Runs of the factor's Schur updates: up to `max_members` consecutive
// supernodes that are the column blocks of one wider supernode -- each the
// parent of the previous, and each one's rows exactly the next block's
// columns followed by the next block's rows.  run_end[s] = the last member
// of s's run (s itself outside runs).
std::vector<int> update_runs(const Symbolic& S, int max_members) {
  const int nsn = S.nsn;
  const std::vector<int> run_first = block_run_first(S);
  std::vector<int> end(nsn);
  for (int s = 0; s < nsn;) {
    int e = s;
    while (e - s + 1 < max_members && e + 1 < nsn && run_first[e + 1] == run_first[s]) ++e;
    for (int q = s; q <= e; ++q) end[q] = e;
    s = e + 1;
  }
  return end;
}

void build_factor_plan(temf_ctx& c) {
  const Symbolic& S = c.sym;
  FactorPlan& F = c.fplan;
  cudaStream_t st = c.stream;
  F.sn_first.upload(S.sn_first.data(), S.sn_first.size(), st);
  F.sn_parent.upload(S.sn_parent.data(), S.sn_parent.size(), st);
  F.sn_rows.upload(S.sn_rows.data(), S.sn_rows.size(), st);
  F.sn_rows_ptr.upload(S.sn_rows_ptr.data(), S.sn_rows_ptr.size(), st);
  F.sn_Lptr.upload(S.sn_Lptr.data(), S.sn_Lptr.size(), st);
  F.level_sn.upload(S.level_sn.data(), S.level_sn.size(), st);
  F.level_ptr = S.level_ptr;

  auto width = [&](int s) { return S.sn_first[s + 1] - S.sn_first[s]; };
  auto nrows = [&](int s) { return (int64_t)(S.sn_rows_ptr[s + 1] - S.sn_rows_ptr[s]); };
  {  // the sweeps' scaled copies of the diagonal blocks, after the panels
    std::vector<int64_t> dp(S.nsn + 1);
    int64_t o = S.stored;
    for (int s = 0; s < S.nsn; ++s) {
      dp[s] = o;
      o += (int64_t)width(s) * width(s);
    }
    dp[S.nsn] = o;
    F.dsc_len = o - S.stored;
    F.sn_Dptr.upload(dp.data(), dp.size(), st);
  }
  // position of global row i in the panel of supernode t (i >= first column of t)
  auto panel_row = [&](int t, int i) -> int64_t {
    const int ft = S.sn_first[t], ct = width(t);
    if (i < ft + ct) return i - ft;
    const int* b = S.sn_rows.data() + S.sn_rows_ptr[t];
    const int* e = S.sn_rows.data() + S.sn_rows_ptr[t + 1];
    const int* p = std::lower_bound(b, e, i);
    if (p == e || *p != i) throw StateError("symbolic structure inconsistent (row not in ancestor)");
    return ct + (p - b);
  };

  // A -> L map
  {
    std::vector<int> src;
    std::vector<int64_t> dst;
    const Pattern& P = c.pat;
    for (int i = 0; i < P.n; ++i) {
      for (int p = P.rowptr[i]; p < P.rowptr[i + 1]; ++p) {
        const int j = P.col[p];
        if (j > i) break;
        const int s = S.col2sn[j];
        const int64_t ld = width(s) + nrows(s);
        src.push_back(p);
        dst.push_back(S.sn_Lptr[s] + (int64_t)(j - S.sn_first[s]) * ld + panel_row(s, i));
      }
    }
    F.n_a2l = (int64_t)src.size();
    F.a2l_src.upload(src.data(), src.size(), st);
    F.a2l_dst.upload(dst.data(), dst.size(), st);
  }
  // update groups + relative indices (host threads; see symbolic.h)
  {
    UpdateGroups G;
    update_groups(S, G);
    F.n_relind = G.n_rel;
    F.row_grp.upload(G.row_grp.data(), G.row_grp.size(), st);
    F.grp_target.upload(G.grp_target.data(), G.grp_target.size(), st);
    F.grp_shift.upload(G.grp_shift.data(), G.grp_shift.size(), st);
    F.grp_relind.upload(G.grp_rel.data(), G.grp_rel.size(), st);
    F.relind.upload(G.rel.get(), (size_t)G.n_rel, st);
    TEMF_CUDA(cudaStreamSynchronize(st));  // G's host arrays go out of scope
  }
  // row chunks of the triangular solves per level
  {
    std::vector<TrsmChunk> ch;
    std::vector<int64_t> lp(S.nlevels + 1, 0);
    for (int l = 0; l < S.nlevels; ++l) {
      for (int q = S.level_ptr[l]; q < S.level_ptr[l + 1]; ++q) {
        const int s = S.level_sn[q];
        const int r = (int)nrows(s);
        for (int r0 = 0; r0 < r; r0 += kTrsmRows) ch.push_back({s, r0});
      }
      lp[l + 1] = (int64_t)ch.size();
    }
    F.trsm_level_ptr = lp;
    F.n_trsm = (int64_t)ch.size();
    F.trsm.upload(reinterpret_cast<const int2*>(ch.data()), ch.size(), st);
  }
  // tiles per level, with runs of column blocks summed (see k_update)
  {
    const std::vector<int> run_end = update_runs(S, kUpdMaxMembers);
    F.n_runs = 0;
    std::vector<UpdTile> tiles;
    F.tile_level_ptr.assign(S.nlevels + 1, 0);
    for (int l = 0; l < S.nlevels; ++l) {
      for (int q = S.level_ptr[l]; q < S.level_ptr[l + 1]; ++q) {
        const int s = S.level_sn[q];
        const int r = (int)nrows(s);
        const int e = run_end[s];
        if (e != s) {
          // a run member before its last: only the later members' columns
          const int g = S.sn_first[e + 1] - S.sn_first[s + 1];
          for (int tj = 0; tj * kUpdTile < g; ++tj)
            for (int ti = tj; ti * kUpdTile < r; ++ti) tiles.push_back({s, ti * kUpdTile, tj * kUpdTile, 1 | (g << 4)});
          continue;
        }
        int m = 1;  // members of the run ending at s
        while (s - m >= 0 && run_end[s - m] == s) ++m;
        if (m > 1) ++F.n_runs;
        const int nt = ceil_div(r, kUpdTile);
        for (int ti = 0; ti < nt; ++ti)
          for (int tj = 0; tj <= ti; ++tj) tiles.push_back({s, ti * kUpdTile, tj * kUpdTile, m});
      }
      F.tile_level_ptr[l + 1] = (int64_t)tiles.size();
    }
    F.n_tiles = (int64_t)tiles.size();
    F.tiles.upload(tiles.data(), tiles.size(), st);
  }
  TEMF_CUDA(cudaStreamSynchronize(st));
}

int numeric_factor(temf_ctx& c, int slot, double dt) {
  // A(dt) = 0*A_eps + 3*M_sigma + 2*dt*K  (mkl_add_3 at src/FETD_FWD.f90:1288,1354)
  return numeric_factor_values(c, slot, c.d_M.p, 3.0, c.d_K.p, 2.0 * dt);
}

int numeric_factor_values(temf_ctx& c, int slot, const double* X, double a, const double* Y, double b) {
  launch_factor_values(c, slot, X, a, Y, b);
  return finish_factor(c, slot);
}

int numeric_factor_values_fallback(temf_ctx& c, int slot, const double* X, double a, const double* Y, double b) {
  const int st = numeric_factor_values(c, slot, X, a, Y, b);
  if (st <= 0) return st;
  // not positive definite: refactor in the indefinite mode (the reference
  // retries PARDISO with mtype -2, src/FETD_UTILITY.f90:923-935)
  launch_factor_values(c, slot, X, a, Y, b, true);
  finish_factor(c, slot);
  return st;
}

int finish_factor(temf_ctx& c, int slot) {
  FactorSlot& fs = c.slots[slot];
  int words[4] = {0, 0, 0, 0};
  TEMF_CUDA(cudaMemcpyAsync(words, c.d_status.p, 4 * sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  TEMF_CUDA(cudaStreamSynchronize(c.stream));
  if (words[3] != 0) {
    fs.valid = false;
    throw StateError("a factor update's panel copies did not complete (bounded wait timed out)");
  }
  const int status = words[0];
  fs.perturbed = fs.indefinite ? words[2] : 0;
  if (status != INT_MAX) {
    // the first non-positive pivot (original numbering); an indefinite-mode
    // factor is valid nonetheless
    fs.status = c.sym.perm[status - 1] + 1;
    fs.valid = fs.indefinite;
    return fs.status;
  }
  fs.valid = true;
  fs.status = 0;
  return 0;
}

void launch_factor(temf_ctx& c, int slot, double dt) {
  launch_factor_values(c, slot, c.d_M.p, 3.0, c.d_K.p, 2.0 * dt);
}

void launch_factor_values(temf_ctx& c, int slot, const double* X, double a, const double* Y, double b,
                          bool indefinite) {
  const Symbolic& S = c.sym;
  FactorPlan& F = c.fplan;
  FactorSlot& fs = c.slots[slot];
  cudaStream_t st = c.stream;
  if (fs.L.n < (size_t)slot_len(c)) fs.L.alloc(slot_len(c));
  TEMF_CUDA(cudaMemsetAsync(fs.L.p, 0, S.stored * sizeof(double), st));
  int init[3] = {INT_MAX, 0, 0};
  TEMF_CUDA(cudaMemcpyAsync(c.d_status.p, &init[0], sizeof(int), cudaMemcpyHostToDevice, st));
  TEMF_CUDA(cudaMemcpyAsync(c.d_status.p + 2, &init[2], sizeof(int), cudaMemcpyHostToDevice, st));
  TEMF_CUDA(cudaMemcpyAsync(c.d_status.p + 3, &init[1], sizeof(int), cudaMemcpyHostToDevice, st));  // copy waits
  fs.X = X;
  fs.a = a;
  fs.Y = Y;
  fs.b = b;
  fs.indefinite = indefinite;
  double* sgn = nullptr;
  if (indefinite) {
    if (fs.sgn.n < (size_t)S.n) fs.sgn.alloc(S.n);
    sgn = fs.sgn.p;
  }
  if (F.n_a2l) {
    k_load_A<<<ceil_div(F.n_a2l, 256), 256, 0, st>>>(F.n_a2l, F.a2l_src.p, F.a2l_dst.p, X, a, Y, b, fs.L.p);
    TEMF_CHECK_LAUNCH();
  }
  const size_t upd_smem = 2 * 2 * kUpdChunk * kLdsU * sizeof(double);
  TEMF_CUDA(cudaFuncSetAttribute(k_update, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)upd_smem));
  for (int l = 0; l < S.nlevels; ++l) {
    const int cnt = S.level_ptr[l + 1] - S.level_ptr[l];
    if (cnt > 0) {
      k_potrf<<<cnt, kFacThreads, 0, st>>>(F.level_sn.p + S.level_ptr[l], F.sn_first.p, F.sn_rows_ptr.p,
                                           F.sn_Lptr.p, fs.L.p, c.d_status.p, sgn, F.sn_Dptr.p);
      TEMF_CHECK_LAUNCH();
    }
    const int64_t c0 = F.trsm_level_ptr[l], c1 = F.trsm_level_ptr[l + 1];
    if (c1 > c0) {
      k_trsm<<<(unsigned)(c1 - c0), kFacThreads, 0, st>>>(reinterpret_cast<const TrsmChunk*>(F.trsm.p) + c0,
                                                          F.sn_first.p, F.sn_rows_ptr.p, F.sn_Lptr.p, fs.L.p, sgn);
      TEMF_CHECK_LAUNCH();
    }
    const int64_t t0 = F.tile_level_ptr[l], t1 = F.tile_level_ptr[l + 1];
    if (t1 > t0) {
      if (t1 - t0 > INT_MAX) throw StateError("too many update tiles in one level");
      k_update<<<(unsigned)(t1 - t0), 128, upd_smem, st>>>(F.tiles.p + t0, F.sn_first.p, F.sn_rows_ptr.p,
                                                          F.sn_rows.p, F.sn_Lptr.p, F.row_grp.p, F.grp_target.p,
                                                          F.grp_shift.p, F.grp_relind.p, F.relind.p, fs.L.p,
                                                          cnt > 1 ? 1 : 0, sgn, c.d_status.p + 3);
      TEMF_CHECK_LAUNCH();
    }
  }
  fs.dt = b * 0.5;
  fs.valid = false;
}

}  // namespace temf
