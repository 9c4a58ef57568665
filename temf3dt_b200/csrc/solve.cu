// K4 + K5 + K6 + K7: per-step kernels of the FETD time loop.
//
//  * K5  r = M_sigma (4 e^n - e^{n-1}) - 2 dt s(t): the BDF2 right-hand side,
//        src/FETD_FWD.f90:1425-1428 (mkl_sparse_d_mv with the symmetric-upper
//        descriptor, :1191-1193; sys_right :1466-1511).  Full symmetric CSR,
//        eight lanes per row with shuffle reductions, vectors in the
//        fill-reducing order so no permutation happens per step.
//  * K4  x = A^{-1} r with the supernodal factor: PARDISO phase 33,
//        src/FETD_UTILITY.f90:938-957.  Two persistent, dependency-driven
//        kernels (forward, backward): tasks are the diagonal blocks and the
//        128-row chunks of every supernode panel, claimed in an order in which
//        every wait targets an earlier task, so no level barriers and no
//        per-level launches; every wait is bounded and reports a timeout
//        through an error word instead of hanging.  The forward sweep pushes
//        row-chunk updates into the right-hand side with FP64 atomics; the
//        backward sweep reduces in a fixed order.
//  * K6  ||a - b||^2 and ||b||^2 for the dt-doubling test (two_error,
//        src/FETD_UTILITY.f90:578-599), fixed-order block reduction.
//  * K7  receiver E and dB/dt from the six edge values of the receiver's
//        tetrahedron (solution_output, src/FETD_FWD.f90:1532-1540).
#include <algorithm>

#include "factor.h"
#include "solve.h"

namespace temf {

constexpr int kSolveThreads = 128;
constexpr int kChunkRows = 128;        // rows of a panel handled by one task (= threads per CTA)
constexpr int kChunkRowsMulti = 64;    // rows per task when solving blocks of right-hand sides
constexpr int kMultiCols = 64;         // right-hand sides per block
constexpr int kSpinLimit = 1 << 22;    // bounded waits: ~seconds, then the error flag (default)

// Optional per-task timeline of the single-model sweeps (profiling aid; null
// unless temf_solve_timeline is running): per task start, dependency
// satisfied, end (global ns timer) and SM id.
__device__ unsigned long long* g_timeline_f = nullptr;
__device__ unsigned long long* g_timeline_b = nullptr;
__device__ __forceinline__ unsigned long long gtime() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ unsigned smid() {
  unsigned r;
  asm volatile("mov.u32 %0, %%smid;" : "=r"(r));
  return r;
}

// 8-byte asynchronous global -> shared copy (L1-allocating: only for data
// no CTA writes during the sweep, i.e. the factor panels)
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Bounded wait until *flag >= target (written by other CTAs of the same
// kernel).  Polls tightly first, then with a short sleep.  On timeout the
// error word is set and the wait gives up, so the kernel always terminates;
// the host reports the error.
__device__ __forceinline__ int spin_limit(const SweepView& V) { return V.spin > 0 ? V.spin : kSpinLimit; }
__device__ __forceinline__ void wait_geq(const int* flag, int target, int* err, int code, int limit) {
  const volatile int* f = flag;
  int it = 0;
  while (*f < target) {
    if (++it > limit) {
      atomicExch(err, code);
      break;
    }
    if (it > 256) __nanosleep(32);
  }
  __threadfence();
}

// One warp solves the c x c diagonal block for one right-hand side; lane l
// holds rows l (v0) and 32 + l (v1).  Columns are taken eight at a time:
// their eight current values are broadcast, every lane solves the 8 x 8
// block redundantly, the owners take their rows' results and every lane
// updates its rows beyond the block.  Each row receives exactly the updates
// of column-by-column substitution, one FMA each, in the same column order,
// so the result is the same to the bit; the dependent chain per column is one
// FMA and one multiply instead of a shuffle round trip.
__device__ __forceinline__ void diag_solve_fwd_warp(const double (*D)[kSnCols + 1], const double* rinv, double& v0,
                                                    double& v1, int c) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int k0 = 0; k0 < kSnCols; k0 += 8) {
    if (k0 < c) {  // warp-uniform
      double y[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) y[i] = __shfl_sync(0xffffffffu, k0 < 32 ? v0 : v1, (k0 + i) & 31);
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        if (k0 + i < c) {
          double t = y[i];
#pragma unroll
          for (int j = 0; j < i; ++j) t -= D[k0 + i][k0 + j] * y[j];
          y[i] = t * rinv[k0 + i];
        }
      }
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        if (lane == ((k0 + i) & 31) && k0 + i < c) {
          if (k0 < 32) v0 = y[i];
          else v1 = y[i];
        }
      }
      if (k0 < 32 && lane >= k0 + 8 && lane < c) {
#pragma unroll
        for (int j = 0; j < 8; ++j) v0 -= D[lane][k0 + j] * y[j];
      }
      if (lane + 32 >= k0 + 8 && lane + 32 < c) {
#pragma unroll
        for (int j = 0; j < 8; ++j) v1 -= D[lane + 32][k0 + j] * y[j];
      }
    }
  }
}
// L^T x = z, columns from the last: the same blocking, eight at a time from
// the top, every row updated in descending column order as in the
// column-by-column substitution.
__device__ __forceinline__ void diag_solve_bwd_warp(const double (*D)[kSnCols + 1], const double* rinv, double& v0,
                                                    double& v1, int c) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int k0 = kSnCols - 8; k0 >= 0; k0 -= 8) {
    if (k0 < c) {  // warp-uniform
      double x[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) x[i] = __shfl_sync(0xffffffffu, k0 < 32 ? v0 : v1, (k0 + i) & 31);
#pragma unroll
      for (int i = 7; i >= 0; --i) {
        if (k0 + i < c) {
          double t = x[i];
#pragma unroll
          for (int j = 7; j > i; --j)
            if (k0 + j < c) t -= D[k0 + j][k0 + i] * x[j];
          x[i] = t * rinv[k0 + i];
        }
      }
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        if (lane == ((k0 + i) & 31) && k0 + i < c) {
          if (k0 < 32) v0 = x[i];
          else v1 = x[i];
        }
      }
      if (lane < k0 && lane < c) {
#pragma unroll
        for (int j = 7; j >= 0; --j)
          if (k0 + j < c) v0 -= D[k0 + j][lane] * x[j];
      }
      if (k0 >= 32 && lane + 32 < k0 && lane + 32 < c) {
#pragma unroll
        for (int j = 7; j >= 0; --j)
          if (k0 + j < c) v1 -= D[k0 + j][lane + 32] * x[j];
      }
    }
  }
}

// The same blocking on the factor's scaled copy of the block: D holds the
// unit lower triangle L_ij / L_ii below its diagonal.  Forward: L y = b is
// D y = b / L_ii, so each unknown is its scaled right-hand side minus the
// scaled products of the unknowns before it -- one FMA per column on the
// dependent chain (FP64 latency is about 23 cycles on sm_100a, a shuffle
// about 26), against an FMA and a multiply with the unscaled block.
// Backward: L^T x = z is D^T w = z with w_i = L_ii x_i; the caller scales w.
__device__ __forceinline__ void unit_solve_fwd_warp(const double (*D)[kSnCols + 1], double& v0, double& v1, int c) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int k0 = 0; k0 < kSnCols; k0 += 8) {
    if (k0 < c) {  // warp-uniform
      double y[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) y[i] = __shfl_sync(0xffffffffu, k0 < 32 ? v0 : v1, (k0 + i) & 31);
#pragma unroll
      for (int i = 1; i < 8; ++i) {
        if (k0 + i < c) {
#pragma unroll
          for (int j = 0; j < i; ++j) y[i] -= D[k0 + i][k0 + j] * y[j];
        }
      }
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        if (lane == ((k0 + i) & 31) && k0 + i < c) {
          if (k0 < 32) v0 = y[i];
          else v1 = y[i];
        }
      }
      if (k0 < 32 && lane >= k0 + 8 && lane < c) {
#pragma unroll
        for (int j = 0; j < 8; ++j) v0 -= D[lane][k0 + j] * y[j];
      }
      if (lane + 32 >= k0 + 8 && lane + 32 < c) {
#pragma unroll
        for (int j = 0; j < 8; ++j) v1 -= D[lane + 32][k0 + j] * y[j];
      }
    }
  }
}
__device__ __forceinline__ void unit_solve_bwd_warp(const double (*D)[kSnCols + 1], double& v0, double& v1, int c) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int k0 = kSnCols - 8; k0 >= 0; k0 -= 8) {
    if (k0 < c) {  // warp-uniform
      double x[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) x[i] = __shfl_sync(0xffffffffu, k0 < 32 ? v0 : v1, (k0 + i) & 31);
#pragma unroll
      for (int i = 6; i >= 0; --i) {
        if (k0 + i < c) {
#pragma unroll
          for (int j = 7; j > i; --j)
            if (k0 + j < c) x[i] -= D[k0 + j][k0 + i] * x[j];
        }
      }
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        if (lane == ((k0 + i) & 31) && k0 + i < c) {
          if (k0 < 32) v0 = x[i];
          else v1 = x[i];
        }
      }
      if (lane < k0 && lane < c) {
#pragma unroll
        for (int j = 7; j >= 0; --j)
          if (k0 + j < c) v0 -= D[k0 + j][lane] * x[j];
      }
      if (k0 >= 32 && lane + 32 < k0 && lane + 32 < c) {
#pragma unroll
        for (int j = 7; j >= 0; --j)
          if (k0 + j < c) v1 -= D[k0 + j][lane + 32] * x[j];
      }
    }
  }
}

// Dense lower-triangular solve of the c x c diagonal block held in D (shared)
// for nrhs columns of ys (row-major c x nrhs), forward (L y = b) or backward
// (L^T x = z).  nrhs == 1 runs in one warp (the blocked substitution above).
__device__ void diag_solve(const double (*D)[kSnCols + 1], const double* rinv, double* ys, int c, int nrhs,
                           bool forward, bool scaled = false) {
  const int tid = threadIdx.x;
  if (nrhs == 1 && scaled) {  // D: the factor's scaled copy; rinv: 1 / L_ii
    if (tid < 32) {
      const int lane = tid;
      double v0 = lane < c ? ys[lane] : 0.0;
      double v1 = lane + 32 < c ? ys[lane + 32] : 0.0;
      if (forward) {
        v0 *= lane < c ? rinv[lane] : 0.0;
        v1 *= lane + 32 < c ? rinv[lane + 32] : 0.0;
        unit_solve_fwd_warp(D, v0, v1, c);
      } else {
        unit_solve_bwd_warp(D, v0, v1, c);
        v0 *= lane < c ? rinv[lane] : 0.0;
        v1 *= lane + 32 < c ? rinv[lane + 32] : 0.0;
      }
      if (lane < c) ys[lane] = v0;
      if (lane + 32 < c) ys[lane + 32] = v1;
    }
    __syncthreads();
    return;
  }
  if (nrhs == 1) {
    if (tid < 32) {
      const int lane = tid;
      double v0 = lane < c ? ys[lane] : 0.0;
      double v1 = lane + 32 < c ? ys[lane + 32] : 0.0;
      if (forward) diag_solve_fwd_warp(D, rinv, v0, v1, c);
      else diag_solve_bwd_warp(D, rinv, v0, v1, c);
      if (lane < c) ys[lane] = v0;
      if (lane + 32 < c) ys[lane + 32] = v1;
    }
    __syncthreads();
    return;
  }
  if (forward) {
    for (int j = 0; j < c; ++j) {
      for (int col = tid; col < nrhs; col += blockDim.x) ys[j * nrhs + col] *= rinv[j];
      __syncthreads();
      for (int idx = tid; idx < (c - j - 1) * nrhs; idx += blockDim.x) {
        const int k = j + 1 + idx / nrhs, col = idx % nrhs;
        ys[k * nrhs + col] -= D[k][j] * ys[j * nrhs + col];
      }
      __syncthreads();
    }
  } else {
    for (int j = c - 1; j >= 0; --j) {
      for (int col = tid; col < nrhs; col += blockDim.x) ys[j * nrhs + col] *= rinv[j];
      __syncthreads();
      for (int idx = tid; idx < j * nrhs; idx += blockDim.x) {
        const int k = idx / nrhs, col = idx % nrhs;
        ys[k * nrhs + col] -= D[j][k] * ys[j * nrhs + col];
      }
      __syncthreads();
    }
  }
}

// Lower triangle of the diagonal block into D with asynchronous copies
// (issued before a dependency wait; coalesced per column), and the
// reciprocals of its diagonal once the copies have landed.
__device__ __forceinline__ void load_diag_start(double (*D)[kSnCols + 1], const double* P, int c, int64_t ld) {
  for (int idx = threadIdx.x; idx < c * c; idx += blockDim.x) {
    const int j = idx / c, i = idx - j * c;
    if (i >= j) cp_async8(&D[i][j], P + (int64_t)j * ld + i);
  }
}
__device__ __forceinline__ void load_diag_finish(double (*D)[kSnCols + 1], double* rinv, int c, bool scaled = false) {
  cp_async_wait_all();
  __syncthreads();
  if ((int)threadIdx.x < c) rinv[threadIdx.x] = scaled ? D[threadIdx.x][threadIdx.x] : 1.0 / D[threadIdx.x][threadIdx.x];
  __syncthreads();
}
// the factor's scaled copy of the block (c x c, column-major), lower triangle
__device__ __forceinline__ void load_diag_start_scaled(double (*D)[kSnCols + 1], const double* Q, int c) {
  for (int idx = threadIdx.x; idx < c * c; idx += blockDim.x) {
    const int j = idx / c, i = idx - j * c;
    if (i >= j) cp_async8(&D[i][j], Q + idx);
  }
}
// single column: the scaled copy when the view has one, else the panel's block
__device__ __forceinline__ void load_diag_start_1(double (*D)[kSnCols + 1], const SweepView& V, const double* Lb, int s,
                                                  const double* P, int c, int64_t ld) {
  if (V.Dptr) load_diag_start_scaled(D, Lb + V.Dptr[s], c);
  else load_diag_start(D, P, c, ld);
}

// Row-chunk products, single right-hand side.  The panel values are loaded
// into registers by pre_* (before any dependency wait: the factor does not
// depend on it) and consumed by the matching fin_*.
struct FwdRegs {
  double v[kSnCols];
};
__device__ __forceinline__ void pre_fwd(FwdRegs& R, const double* Pc, int c, int64_t ld, int i, bool on) {
#pragma unroll
  for (int j = 0; j < kSnCols; ++j) R.v[j] = (on && j < c) ? __ldg(Pc + (int64_t)j * ld + i) : 0.0;
}
__device__ __forceinline__ double fin_fwd(const FwdRegs& R, const double* ys, int c) {
  double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
#pragma unroll
  for (int j = 0; j < kSnCols; j += 4) {
    a0 += R.v[j] * (j < c ? ys[j] : 0.0);
    a1 += R.v[j + 1] * (j + 1 < c ? ys[j + 1] : 0.0);
    a2 += R.v[j + 2] * (j + 2 < c ? ys[j + 2] : 0.0);
    a3 += R.v[j + 3] * (j + 3 < c ? ys[j + 3] : 0.0);
  }
  return (a0 + a1) + (a2 + a3);
}

// Sum over the 32 lanes of each of the 32 per-lane values a[0..31]: lane l
// ends with the sum of a[l] (31 shuffles: each step halves the live values).
__device__ __forceinline__ double lane_transpose_sum(double a[32]) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) {
    const bool up = (lane & o) != 0;
#pragma unroll
    for (int k = 0; k < o; ++k) {
      const double send = up ? a[k] : a[k + o];
      const double keep = up ? a[k + o] : a[k];
      a[k] = keep + __shfl_xor_sync(0xffffffffu, send, o);
    }
  }
  return a[0];
}

// Backward chunk products, single right-hand side: the chunk is loaded as in
// the forward sweep (thread = row, its c panel values in registers, loads
// coalesced along each column); each thread scales its row by z_row and the
// per-column sums over the warp's 32 rows come out of two transposing
// shuffle reductions, one value per lane and column: seg[warp][j].  The
// consumers add the four warps' sums in a fixed order.
__device__ __forceinline__ void bwd_row_sums(FwdRegs& R, double zi, double (*seg)[kSnCols]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < kSnCols; ++j) R.v[j] *= zi;
  seg[warp][lane] = lane_transpose_sum(R.v);
  seg[warp][32 + lane] = lane_transpose_sum(R.v + 32);
}

// Ready queue: a task is appended once every task it depends on has finished
// (the finishing task that completes its count appends it), and CTAs pop
// tasks in the order they became ready, so no CTA holds a task that is still
// waiting for its inputs.  Slots hold task + 1 (0 = not yet written).
__device__ __forceinline__ bool in_queue(const SweepView& V, int task) {
  return V.queue != nullptr && task >= V.q_lo && task < V.q_hi;
}
__device__ __forceinline__ void q_push(const SweepView& V, int task) {
  if (!in_queue(V, task)) return;  // claimed in schedule order instead
  const int pos = atomicAdd(V.qtail, 1);
  atomicExch(V.queue + pos, (V.tag | task) + 1);
}
// Forward: one more input for each supernode in tgt[k0, k1); the queued
// diagonal tasks whose inputs are then complete are pushed.  Four entries
// per thread at a time, so the round trips of their atomics overlap.
__device__ __forceinline__ void count_inputs(const SweepView& V, int k0, int k1) {
  int* ready = V.sync;
  const int nt = blockDim.x;
  for (int k = k0 + (int)threadIdx.x; k < k1; k += 4 * nt) {
    int o[4], d[4], ex[4], old[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) o[u] = k + u * nt < k1 ? V.tgt[k + u * nt] : -1;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      d[u] = o[u] >= 0 ? V.diag_task[o[u]] : -1;
      ex[u] = o[u] >= 0 ? V.expect[o[u]] : 0;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) old[u] = o[u] >= 0 ? atomicAdd(ready + o[u], 1) : -1;
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (o[u] >= 0 && in_queue(V, d[u]) && old[u] == ex[u] - 1) q_push(V, d[u]);
  }
}
// Backward: one completion for each task in dep[k0, k1) (an owner of its
// rows is solved); the queued tasks whose count is then complete are pushed.
__device__ __forceinline__ void count_owner_done(const SweepView& V, int k0, int k1) {
  const int nt = blockDim.x;
  for (int k = k0 + (int)threadIdx.x; k < k1; k += 4 * nt) {
    int d[4], nd[4], old[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      d[u] = k + u * nt < k1 ? V.dep[k + u * nt] : -1;
      if (d[u] >= 0 && !in_queue(V, d[u])) d[u] = -1;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) nd[u] = d[u] >= 0 ? V.need[d[u]] : 0;
#pragma unroll
    for (int u = 0; u < 4; ++u) old[u] = d[u] >= 0 ? atomicAdd(V.cnt + d[u], 1) : -1;
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (d[u] >= 0 && old[u] == nd[u] - 1) q_push(V, d[u]);
  }
}

// thread 0 only: next ready task, or -1 when all ntask tasks are handed out
// (or a wait timed out: error word set)
__device__ __forceinline__ int q_pop(int* qhead, const int* queue, int limit, int* err, int spin) {
  const int idx = atomicAdd(qhead, 1);
  if (idx >= limit) return -1;
  const volatile int* slot = queue + idx;
  int it = 0, v;
  while ((v = *slot) == 0) {
    if (++it > spin) {
      atomicExch(err, 5);
      return -1;
    }
    if (it > 256) __nanosleep(64);
  }
  __threadfence();
  return v - 1;
}

// Next task of this CTA (every thread gets it; -1 when done).  Two phases:
// the queue range through the ready queue, and the other tasks claimed in
// schedule order from `counter` (with dependency waits).  Forward sweeps run
// the queue phase first (their queue range is the bottom of the tree, at the
// start of the schedule), backward sweeps last.  Without a queue every task
// is claimed in order.
__device__ __forceinline__ int next_task(const SweepView& V, int* counter, bool queue_first, int* err, int& phase,
                                         int* sh) {
  for (;;) {
    const bool use_q = (phase == 0) == queue_first;
    if (threadIdx.x == 0) {
      int t = -1;
      if (use_q) {
        if (V.queue) t = q_pop(V.qhead, V.queue, V.q_hi - V.q_lo, err, spin_limit(V));
      } else {
        const bool front = V.queue == nullptr || V.q_lo > 0;  // static tasks before the queue range
        const int lo = front ? 0 : V.q_hi, hi = V.queue == nullptr ? V.ntask : (front ? V.q_lo : V.ntask);
        const int i = atomicAdd(counter, 1);
        t = lo + i < hi ? lo + i : -1;
      }
      *sh = t;
    }
    __syncthreads();
    const int t = *sh;
    __syncthreads();
    if (t >= 0) return t;
    if (phase == 1) return -1;
    phase = 1;
  }
}

// ---------------------------------------------------------------------------
// forward  L y = b : persistent, dependency driven
//   diagonal task of s (with its first row chunk): wait until every chunk that
//     touches s's columns has landed, solve with L11, publish y_s, then push
//     -L21[0..128) y_s into the right-hand side of those rows (FP64 atomics:
//     the rows belong to ancestors that have not been solved yet) and bump the
//     ready counter of each supernode owning one of the rows;
//   chunk task (s, r0..r1), r0 >= 128: wait for y_s, push the same way.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void fwd_task(const SweepView& V, int t, const double* Lb, int nrhs, int* err,
                                         double (*D)[kSnCols + 1], double* rinv, double* ys,
                                         unsigned long long* stamp = nullptr) {
  int* ready = V.sync;
  int* ydone = V.sync + V.nsn;
  double* x = V.x;
  const int tid = threadIdx.x;
  const SolveTask T = V.tasks[t];
  const int s = T.s;
  const int f = V.sn_first[s];
  const int c = V.sn_first[s + 1] - f;
  const int64_t rp = V.rows_ptr[s];
  const int64_t r = V.rows_ptr[s + 1] - rp;
  const int64_t ld = c + r;
  const double* P = Lb + V.Lptr[s];
  const double* Pc = P + c;
  const int i = T.r0 + tid;
  const bool row_on = i < T.r1;
  FwdRegs R;
  if (nrhs == 1) pre_fwd(R, Pc, c, ld, i, row_on);
  const int row_i = row_on ? V.sn_rows[rp + i] : 0;  // the row this thread pushes to (read before the wait)
  const bool queued = in_queue(V, t);
  // this thread's target supernode with its diagonal task and input count,
  // read before the wait (a chunk of at most blockDim rows feeds at most
  // blockDim supernodes: one entry per thread)
  int tg_o = -1, tg_d = -1, tg_ex = 0;
  if (V.queue && T.r1 > T.r0) {
    const int k = V.tgt_ptr[t] + tid;
    if (k < V.tgt_ptr[t + 1]) {
      tg_o = V.tgt[k];
      tg_d = V.diag_task[tg_o];
      tg_ex = V.expect[tg_o];
    }
  }
  const bool sc = nrhs == 1 && V.Dptr != nullptr;
  if (T.kind == 0) {
    if (sc) load_diag_start_scaled(D, Lb + V.Dptr[s], c);
    else load_diag_start(D, P, c, ld);
    if (tid == 0 && !queued) wait_geq(ready + s, V.expect[s], err, 1, spin_limit(V));
    __syncthreads();
    if (stamp && tid == 0) *stamp = gtime();
    for (int idx = tid; idx < c * nrhs; idx += blockDim.x) ys[idx] = __ldcg(x + (int64_t)f * nrhs + idx);
    load_diag_finish(D, rinv, c, sc);
    diag_solve(D, rinv, ys, c, nrhs, true, sc);
    for (int idx = tid; idx < c * nrhs; idx += blockDim.x) x[(int64_t)f * nrhs + idx] = ys[idx];
    // y_s is published together with the first chunk's pushes below: one fence for both
  } else {
    if (tid == 0 && !queued) wait_geq(ydone + s, 1, err, 2, spin_limit(V));
    __syncthreads();
    if (stamp && tid == 0) *stamp = gtime();
    for (int idx = tid; idx < c * nrhs; idx += blockDim.x) ys[idx] = __ldcg(x + (int64_t)f * nrhs + idx);
    __syncthreads();
  }
  if (T.r1 > T.r0) {
    if (nrhs == 1) {
      if (row_on) atomicAdd(x + row_i, -fin_fwd(R, ys, c));
    } else if (row_on) {
      double* dst = x + (int64_t)row_i * nrhs;
      for (int col = 0; col < nrhs; ++col) {
        double a = 0.0;
        for (int j = 0; j < c; ++j) a += __ldg(Pc + (int64_t)j * ld + i) * ys[j * nrhs + col];
        atomicAdd(dst + col, -a);
      }
    }
  }
  __threadfence();
  __syncthreads();
  if (T.kind == 0) {
    if (tid == 0) atomicExch(ydone + s, 1);
    if (V.queue) {  // y_s is out: the other row chunks of s are ready (they follow this task)
      const int nx = max(1, (int)((r + kChunkRows - 1) / kChunkRows)) - 1;
      for (int k = tid; k < nx; k += blockDim.x) q_push(V, t + 1 + k);
    }
  }
  if (T.r1 > T.r0) {
    if (V.queue) {
      if (tg_o >= 0) {
        const int old = atomicAdd(ready + tg_o, 1);
        if (in_queue(V, tg_d) && old == tg_ex - 1) q_push(V, tg_d);
      }
      count_inputs(V, V.tgt_ptr[t] + (int)blockDim.x, V.tgt_ptr[t + 1]);  // longer lists (none expected)
    } else if (tid == 0) {
      for (int q = V.tgt_ptr[t]; q < V.tgt_ptr[t + 1]; ++q) atomicAdd(ready + V.tgt[q], 1);
    }
  }
}

__global__ void __launch_bounds__(kSolveThreads) k_fwd_persistent(
    int ntask, const SolveTask* __restrict__ tasks, const int* __restrict__ sn_first,
    const int64_t* __restrict__ rows_ptr, const int* __restrict__ sn_rows, const int64_t* __restrict__ Lptr,
    double* const* Lbase, double* x, int nrhs, const int* __restrict__ tgt_ptr, const int* __restrict__ tgt,
    const int* __restrict__ expect, int* sync, int nsn, int* err) {
  __shared__ double D[kSnCols][kSnCols + 1];
  __shared__ double rinv[kSnCols];
  extern __shared__ double ys[];  // c x nrhs
  __shared__ int task_id;
  int* counter = sync + 4 * nsn;
  const SweepView V{tasks, sn_first, rows_ptr, sn_rows, Lptr, Lbase, x, tgt_ptr, tgt, expect,
                    nullptr, nullptr, nullptr, sync, nsn, ntask};
  const double* Lb = *Lbase;
  for (;;) {
    if (threadIdx.x == 0) task_id = atomicAdd(counter, 1);
    __syncthreads();
    const int t = task_id;
    __syncthreads();
    if (t >= ntask) break;
    unsigned long long* rec = g_timeline_f ? g_timeline_f + 4 * (size_t)t : nullptr;
    if (rec && threadIdx.x == 0) rec[0] = gtime();
    fwd_task(V, t, Lb, nrhs, err, D, rinv, ys, rec ? rec + 1 : nullptr);
    if (rec && threadIdx.x == 0) { rec[2] = gtime(); rec[3] = smid(); }
  }
}

// ---------------------------------------------------------------------------
// backward  L^T x = y : persistent, dependency driven, top-down
//   chunk task (s, r0..r1), r0 >= 128: wait for the supernodes owning those
//     rows, stage x[rows] in shared memory, write the chunk's partial sums
//     p_j = sum_i L21[i][j] x[rows_i];
//   diagonal task of s (with its first chunk): wait for the other chunks and
//     the owners of the first chunk's rows, z = y_s - partials (fixed order,
//     so the backward sweep is deterministic), solve with L11^T, publish x_s.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void bwd_task(const SweepView& V, int t, const double* Lb, int nrhs, int* err,
                                         double (*D)[kSnCols + 1], double* rinv, double (*seg)[kSnCols],
                                         double* zs, unsigned long long* stamp = nullptr) {
  int* cdone = V.sync + 2 * V.nsn;
  int* xdone = V.sync + 3 * V.nsn;
  double* x = V.x;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
  const SolveTask T = V.tasks[t];
  const int s = T.s;
  const int f = V.sn_first[s];
  const int c = V.sn_first[s + 1] - f;
  const int64_t rp = V.rows_ptr[s];
  const int64_t r = V.rows_ptr[s + 1] - rp;
  const int64_t ld = c + r;
  const double* P = Lb + V.Lptr[s];
  const int nr = T.r1 - T.r0;
  FwdRegs R;
  if (nrhs == 1 && nr > 0) pre_fwd(R, P + c, c, ld, T.r0 + tid, tid < nr);
  // one chunk row per thread for a single column: its index read before the wait
  const int row_t = (nrhs == 1 && tid < nr) ? V.sn_rows[rp + T.r0 + tid] : 0;
  const bool sc = nrhs == 1 && V.Dptr != nullptr;
  if (T.kind == 0) {
    if (sc) load_diag_start_scaled(D, Lb + V.Dptr[s], c);
    else load_diag_start(D, P, c, ld);
  }
  const bool queued = in_queue(V, t);
  // Diagonal task, one column: y_s (written by the forward sweep only) is read
  // before any wait, and the column sums of the other chunks once their count
  // is complete, while the owner of the first chunk's rows is still awaited
  // (on the top chain that owner is the block just above, finished last).
  const bool pre = T.kind == 0 && nrhs == 1 && V.bacc != nullptr;
  const bool more = V.nchunk[s] > 1;
  double y_pre = 0.0, acc_pre = 0.0;
  if (pre && tid < c) y_pre = __ldcg(x + f + tid);
  // the chunk's rows need their owners' x; the diagonal task also its other chunks
  if (!queued) {  // one polling thread per owner (and one for the chunk count)
    const int q0 = V.tgt_ptr[t], nq = V.tgt_ptr[t + 1] - q0;
    if (pre) {
      if (tid == blockDim.x - 1) wait_geq(cdone + s, V.nchunk[s] - (nr > 0 ? 1 : 0), err, 4, spin_limit(V));
      __syncthreads();
      if (tid < c && more) acc_pre = __ldcg(V.bacc + f + tid);
    }
    for (int q = tid; q < nq; q += blockDim.x) wait_geq(xdone + V.tgt[q0 + q], 1, err, 3, spin_limit(V));
    if (!pre && T.kind == 0 && tid == blockDim.x - 1)
      wait_geq(cdone + s, V.nchunk[s] - (nr > 0 ? 1 : 0), err, 4, spin_limit(V));
  } else if (pre && tid < c && more) {
    acc_pre = __ldcg(V.bacc + f + tid);
  }
  __syncthreads();
  if (stamp && tid == 0) *stamp = gtime();
  double* zx = zs + (T.kind == 0 ? kSnCols * nrhs : 0);  // chunk rows live after the diagonal block
  if (nr > 0) {
    if (nrhs == 1) {  // nr <= blockDim.x: one row per thread
      bwd_row_sums(R, tid < nr ? __ldcg(x + row_t) : 0.0, seg);
    } else {
      for (int idx = tid; idx < nr * nrhs; idx += blockDim.x) {
        const int ii = idx / nrhs, col = idx % nrhs;
        zx[idx] = __ldcg(x + (int64_t)V.sn_rows[rp + T.r0 + ii] * nrhs + col);
      }
    }
    __syncthreads();
  }
  if (T.kind == 1) {
    const int chunk = T.r0 / kChunkRows;
    double* pp = V.part + (V.part_off[s] + (int64_t)chunk * c) * nrhs;
    if (nrhs == 1 && V.bacc) {  // one accumulator per column: the diagonal task reads c values
      for (int j = tid; j < c; j += blockDim.x)
        atomicAdd(V.bacc + f + j, (seg[0][j] + seg[1][j]) + (seg[2][j] + seg[3][j]));
    } else if (nrhs == 1) {
      for (int j = tid; j < c; j += blockDim.x) pp[j] = (seg[0][j] + seg[1][j]) + (seg[2][j] + seg[3][j]);
    } else {
      for (int j = warp; j < c; j += nw) {
        const double* colp = P + (int64_t)j * ld + c + T.r0;
        for (int col = 0; col < nrhs; ++col) {
          double acc = 0.0;
          for (int ii = lane; ii < nr; ii += 32) acc += __ldg(colp + ii) * zx[ii * nrhs + col];
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
          if (lane == 0) pp[j * nrhs + col] = acc;
        }
      }
    }
    __threadfence();
    __syncthreads();
    if (tid == 0) {
      atomicAdd(cdone + s, 1);
      if (V.queue) {
        const int d = V.diag_task[s];
        if (in_queue(V, d) && atomicAdd(V.cnt + d, 1) == V.need[d] - 1) q_push(V, d);
      }
    }
  } else {
    // z = y_s - (first chunk, computed here) - (other chunks, in order)
    const int nch = V.nchunk[s];
    const double* pp = V.part + V.part_off[s] * nrhs;
    if (nrhs == 1) {
      // the other chunks' partials: thread (j, h) sums chunks q = 1 + h, 3 + h, ...
      // with eight loads in flight; fixed order, so still deterministic
      double* psum = zx;  // the chunk rows are consumed: reuse as [2][64]
      if (pre) {  // y_s and the column sums are in registers (c <= blockDim.x)
        if (tid < c) {
          double v = y_pre;
          if (nr > 0) v -= (seg[0][tid] + seg[1][tid]) + (seg[2][tid] + seg[3][tid]);
          if (more) v -= acc_pre;
          zs[tid] = v;
        }
      } else if (nch > 1) {
        const int j = tid & (kSnCols - 1), h = tid / kSnCols;
        double a[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        if (j < c && h < 2) {
          int q = 1 + h;
          for (; q + 14 < nch; q += 16) {
#pragma unroll
            for (int u = 0; u < 8; ++u) a[u] += __ldcg(pp + (int64_t)(q + 2 * u) * c + j);
          }
#pragma unroll
          for (int u = 0; u < 8; ++u)
            if (q + 2 * u < nch) a[u] += __ldcg(pp + (int64_t)(q + 2 * u) * c + j);
        }
        if (h < 2) psum[h * kSnCols + j] = ((a[0] + a[1]) + (a[2] + a[3])) + ((a[4] + a[5]) + (a[6] + a[7]));
        __syncthreads();
      }
      if (!pre) {
        for (int j = tid; j < c; j += blockDim.x) {
          double v = __ldcg(x + f + j);
          if (nr > 0) v -= (seg[0][j] + seg[1][j]) + (seg[2][j] + seg[3][j]);
          if (nch > 1) v -= psum[j] + psum[kSnCols + j];
          zs[j] = v;
        }
      }
    } else {
      for (int idx = tid; idx < c * nrhs; idx += blockDim.x) {
        const int j = idx / nrhs, col = idx % nrhs;
        double v = __ldcg(x + (int64_t)f * nrhs + idx);
        if (nr > 0) {
          double a = 0.0;
          for (int ii = 0; ii < nr; ++ii) a += __ldg(P + (int64_t)j * ld + c + ii) * zx[ii * nrhs + col];
          v -= a;
        }
        for (int q = 1; q < nch; ++q) v -= __ldcg(pp + (int64_t)q * c * nrhs + idx);
        zs[idx] = v;
      }
    }
    load_diag_finish(D, rinv, c, sc);
    diag_solve(D, rinv, zs, c, nrhs, false, sc);
    for (int idx = tid; idx < c * nrhs; idx += blockDim.x) x[(int64_t)f * nrhs + idx] = zs[idx];
    __threadfence();
    __syncthreads();
    if (tid == 0) atomicExch(xdone + s, 1);
    if (V.queue) count_owner_done(V, V.dep_ptr[s], V.dep_ptr[s + 1]);  // x_s is out: every queued task whose rows s owns
  }
}

__global__ void __launch_bounds__(kSolveThreads) k_bwd_persistent(
    int ntask, const SolveTask* __restrict__ tasks, const int* __restrict__ sn_first,
    const int64_t* __restrict__ rows_ptr, const int* __restrict__ sn_rows, const int64_t* __restrict__ Lptr,
    double* const* Lbase, double* x, int nrhs, const int* __restrict__ own_ptr, const int* __restrict__ own,
    const int* __restrict__ nchunk, const int64_t* __restrict__ part_off, double* part, int* sync, int nsn,
    int* err) {
  __shared__ double D[kSnCols][kSnCols + 1];
  __shared__ double rinv[kSnCols];
  __shared__ double seg[4][kSnCols];
  extern __shared__ double zs[];  // max(c, chunk rows) x nrhs
  __shared__ int task_id;
  int* counter = sync + 4 * nsn + 1;
  const SweepView V{tasks, sn_first, rows_ptr, sn_rows, Lptr, Lbase, x, own_ptr, own, nullptr,
                    nchunk, part_off, part, sync, nsn, ntask};
  const double* Lb = *Lbase;
  for (;;) {
    if (threadIdx.x == 0) task_id = atomicAdd(counter, 1);
    __syncthreads();
    const int t = task_id;
    __syncthreads();
    if (t >= ntask) break;
    unsigned long long* rec = g_timeline_b ? g_timeline_b + 4 * (size_t)t : nullptr;
    if (rec && threadIdx.x == 0) rec[0] = gtime();
    bwd_task(V, t, Lb, nrhs, err, D, rinv, seg, zs, rec ? rec + 1 : nullptr);
    if (rec && threadIdx.x == 0) { rec[2] = gtime(); rec[3] = smid(); }
  }
}

// ---------------------------------------------------------------------------
// Runs of column blocks swept by one CTA (single right-hand side).
// A wide supernode is split into blocks of at most 64 columns, one per level,
// each block's rows being the next block's columns followed by the next
// block's rows.  Handed from CTA to CTA, every block costs a publish, a fence
// and a poll on the critical path.  A leader task instead walks the blocks of
// a run itself: the first 128 rows of each block's panel (which, inside the
// run, are the next blocks' columns) are applied locally through a ring of
// run columns in shared memory, and only the other row chunks (ordinary chunk
// tasks of other CTAs) and the rows beyond the run go through global memory
// with atomics and counts, two blocks or more ahead of their use.  The task
// entry of every block (the leader's own, or an absorbed entry past the
// claimable tasks) keeps the owners of its first chunk beyond the run.
//   forward: block q waits for its expected inputs, subtracts the ring, solves,
//            publishes y_q, accumulates its first chunk into the ring or x;
//   backward: block q waits for its other chunks and for the owners beyond
//            the run, takes the run rows' x from the ring, solves, publishes.
// ---------------------------------------------------------------------------
constexpr int kRing = 256;  // run columns held in shared memory (>= 64 + 128 live)
// Most run leaders spanning any one level (a leader holds a CTA while it waits
// for chunk tasks claimed after it; the persistent kernels keep hundreds of
// CTAs resident, so the chunk tasks always find CTAs).
constexpr int kMaxLeaders = 24;

__device__ __forceinline__ int leader_blocks(const SolveTask& T) { return T.kind >> 4; }

__device__ void fwd_leader(const SweepView& V, int t, const double* Lb, int* err, double (*D)[kSnCols + 1],
                           double* rinv, double* ys, double* ring) {
  int* ready = V.sync;
  int* ydone = V.sync + V.nsn;
  double* x = V.x;
  const int tid = threadIdx.x;
  const SolveTask T0 = V.tasks[t];
  const int a = T0.s, e = a + leader_blocks(T0) - 1;
  const int f_run = V.sn_first[a], f_end = V.sn_first[e + 1];
  for (int k = tid; k < kRing; k += blockDim.x) ring[k] = 0.0;
  FwdRegs R;
  {
    const int c = V.sn_first[a + 1] - f_run;
    const int64_t r = V.rows_ptr[a + 1] - V.rows_ptr[a], ld = c + r;
    const double* P = Lb + V.Lptr[a];
    pre_fwd(R, P + c, c, ld, tid, tid < (r < kChunkRows ? r : (int64_t)kChunkRows));
    load_diag_start_1(D, V, Lb, a, P, c, ld);
  }
  const bool sc = V.Dptr != nullptr;
  for (int q = a; q <= e; ++q) {
    const int f = V.sn_first[q], c = V.sn_first[q + 1] - f;
    const int64_t rp = V.rows_ptr[q], r = V.rows_ptr[q + 1] - rp;
    const int r1 = (int)(r < kChunkRows ? r : (int64_t)kChunkRows);
    const int dq = V.diag_task[q];
    if (tid == 0) wait_geq(ready + q, V.expect[q], err, 1, spin_limit(V));
    __syncthreads();
    for (int j = tid; j < c; j += blockDim.x) {
      const int slot = (f + j - f_run) & (kRing - 1);
      ys[j] = __ldcg(x + f + j) + ring[slot];  // the ring holds the negated in-run contributions
      ring[slot] = 0.0;
    }
    load_diag_finish(D, rinv, c, sc);
    diag_solve(D, rinv, ys, c, 1, true, sc);
    for (int j = tid; j < c; j += blockDim.x) x[f + j] = ys[j];
    if (tid < r1) {
      const double v = fin_fwd(R, ys, c);
      const int row = V.sn_rows[rp + tid];
      if (row < f_end) ring[(row - f_run) & (kRing - 1)] -= v;  // inside the run: one writer per row
      else atomicAdd(x + row, -v);
    }
    __threadfence();
    __syncthreads();
    if (tid == 0) atomicExch(ydone + q, 1);
    if (V.queue) {
      count_inputs(V, V.tgt_ptr[dq], V.tgt_ptr[dq + 1]);
    } else if (tid == 0) {
      for (int k = V.tgt_ptr[dq]; k < V.tgt_ptr[dq + 1]; ++k) atomicAdd(ready + V.tgt[k], 1);
    }
    if (q < e) {  // the next block's panel: first chunk into registers, diagonal block into shared memory
      const int fn = V.sn_first[q + 1], cn = V.sn_first[q + 2] - fn;
      const int64_t rn = V.rows_ptr[q + 2] - V.rows_ptr[q + 1], ldn = cn + rn;
      const double* Pn = Lb + V.Lptr[q + 1];
      pre_fwd(R, Pn + cn, cn, ldn, tid, tid < (rn < kChunkRows ? rn : (int64_t)kChunkRows));
      load_diag_start_1(D, V, Lb, q + 1, Pn, cn, ldn);
    }
  }
}

__device__ void bwd_leader(const SweepView& V, int t, const double* Lb, int* err, double (*D)[kSnCols + 1],
                           double* rinv, double (*seg)[kSnCols], double* zs, double* ring) {
  int* cdone = V.sync + 2 * V.nsn;
  int* xdone = V.sync + 3 * V.nsn;
  double* x = V.x;
  const int tid = threadIdx.x;
  const SolveTask T0 = V.tasks[t];
  const int e = T0.s, a = e - leader_blocks(T0) + 1;
  const int f_run = V.sn_first[a], f_end = V.sn_first[e + 1];
  FwdRegs R;
  {
    const int c = V.sn_first[e + 1] - V.sn_first[e];
    const int64_t r = V.rows_ptr[e + 1] - V.rows_ptr[e], ld = c + r;
    const double* P = Lb + V.Lptr[e];
    const int r1 = (int)(r < kChunkRows ? r : (int64_t)kChunkRows);
    if (r1 > 0) pre_fwd(R, P + c, c, ld, tid, tid < r1);
    load_diag_start_1(D, V, Lb, e, P, c, ld);
  }
  const bool sc = V.Dptr != nullptr;
  for (int q = e; q >= a; --q) {
    const int f = V.sn_first[q], c = V.sn_first[q + 1] - f;
    const int64_t rp = V.rows_ptr[q], r = V.rows_ptr[q + 1] - rp;
    const int r1 = (int)(r < kChunkRows ? r : (int64_t)kChunkRows);
    const int dq = V.diag_task[q];
    // the owners of the first chunk's rows beyond the run, and the block's other chunks
    {
      const int q0 = V.tgt_ptr[dq], nq = V.tgt_ptr[dq + 1] - q0;
      for (int k = tid; k < nq; k += blockDim.x) wait_geq(xdone + V.tgt[q0 + k], 1, err, 3, spin_limit(V));
      if (tid == blockDim.x - 1) wait_geq(cdone + q, V.nchunk[q] - (r1 > 0 ? 1 : 0), err, 4, spin_limit(V));
    }
    __syncthreads();
    double* zx = zs + kSnCols;
    if (r1 > 0) {
      double zi = 0.0;
      if (tid < r1) {
        const int row = V.sn_rows[rp + tid];
        zi = row < f_end ? ring[(row - f_run) & (kRing - 1)] : __ldcg(x + row);
      }
      bwd_row_sums(R, zi, seg);
      __syncthreads();
    }
    // z = y_q - (first chunk) - (other chunks, fixed order)
    const int nch = V.nchunk[q];
    const double* pp = V.part + V.part_off[q];
    double* psum = zx;  // the chunk rows are consumed: reuse as [2][64]
    if (nch > 1 && V.bacc) {
      for (int j = tid; j < c; j += blockDim.x) {
        psum[j] = __ldcg(V.bacc + f + j);
        psum[kSnCols + j] = 0.0;
      }
      __syncthreads();
    } else if (nch > 1) {
      const int j = tid & (kSnCols - 1), h = tid / kSnCols;
      double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      if (j < c && h < 2) {
        int k = 1 + h;
        for (; k + 14 < nch; k += 16) {
#pragma unroll
          for (int u = 0; u < 8; ++u) acc[u] += __ldcg(pp + (int64_t)(k + 2 * u) * c + j);
        }
#pragma unroll
        for (int u = 0; u < 8; ++u)
          if (k + 2 * u < nch) acc[u] += __ldcg(pp + (int64_t)(k + 2 * u) * c + j);
      }
      if (h < 2) psum[h * kSnCols + j] = ((acc[0] + acc[1]) + (acc[2] + acc[3])) + ((acc[4] + acc[5]) + (acc[6] + acc[7]));
      __syncthreads();
    }
    for (int j = tid; j < c; j += blockDim.x) {
      double v = __ldcg(x + f + j);
      if (r1 > 0) v -= (seg[0][j] + seg[1][j]) + (seg[2][j] + seg[3][j]);
      if (nch > 1) v -= psum[j] + psum[kSnCols + j];
      zs[j] = v;
    }
    load_diag_finish(D, rinv, c, sc);
    diag_solve(D, rinv, zs, c, 1, false, sc);
    for (int j = tid; j < c; j += blockDim.x) {
      x[f + j] = zs[j];
      ring[(f + j - f_run) & (kRing - 1)] = zs[j];
    }
    __threadfence();
    __syncthreads();
    if (tid == 0) atomicExch(xdone + q, 1);
    if (V.queue) count_owner_done(V, V.dep_ptr[q], V.dep_ptr[q + 1]);  // x_q is out: every queued task whose rows q owns
    if (q > a) {  // the next block (one lower): first chunk into registers, diagonal block into shared memory
      const int fn = V.sn_first[q - 1], cn = f - fn;
      const int64_t rn = V.rows_ptr[q] - V.rows_ptr[q - 1], ldn = cn + rn;
      const double* Pn = Lb + V.Lptr[q - 1];
      const int r1n = (int)(rn < kChunkRows ? rn : (int64_t)kChunkRows);
      if (r1n > 0) pre_fwd(R, Pn + cn, cn, ldn, tid, tid < r1n);
      load_diag_start_1(D, V, Lb, q - 1, Pn, cn, ldn);
    }
  }
}

// The same sweeps scheduled through the ready queue (single right-hand side).
// Instantiated with and without run leaders: the leader code needs many more
// registers, so the plans without leaders get three resident CTAs per SM
// (168 registers) for both sweeps; the backward with leaders two.
template <bool kLeaders>
__global__ void __launch_bounds__(kSolveThreads, 3) k_fwd_queued(const SweepView V, int* err) {
  __shared__ double D[kSnCols][kSnCols + 1];
  __shared__ double rinv[kSnCols];
  __shared__ double ys[kSnCols];
  __shared__ double ring[kRing];
  __shared__ int task_id;
  const double* Lb = *V.Lbase;
  int phase = 0;
  for (;;) {
    const int t = next_task(V, V.sync + 4 * V.nsn, true, err, phase, &task_id);
    if (t < 0) break;
    unsigned long long* rec = g_timeline_f ? g_timeline_f + 4 * (size_t)t : nullptr;
    if (rec && threadIdx.x == 0) rec[0] = gtime();
    if (kLeaders && (V.tasks[t].kind & 15) == 3) {
      if (rec && threadIdx.x == 0) rec[1] = gtime();
      fwd_leader(V, t, Lb, err, D, rinv, ys, ring);
    } else {
      fwd_task(V, t, Lb, 1, err, D, rinv, ys, rec ? rec + 1 : nullptr);
    }
    if (rec && threadIdx.x == 0) { rec[2] = gtime(); rec[3] = smid(); }
  }
}

template <bool kLeaders>
__global__ void __launch_bounds__(kSolveThreads, kLeaders ? 2 : 3) k_bwd_queued(const SweepView V, int* err) {
  __shared__ double D[kSnCols][kSnCols + 1];
  __shared__ double rinv[kSnCols];
  __shared__ double seg[4][kSnCols];
  __shared__ double zs[kSnCols + kChunkRows];
  __shared__ double ring[kRing];
  __shared__ int task_id;
  const double* Lb = *V.Lbase;
  int phase = 0;
  for (;;) {
    const int t = next_task(V, V.sync + 4 * V.nsn + 1, false, err, phase, &task_id);
    if (t < 0) break;
    unsigned long long* rec = g_timeline_b ? g_timeline_b + 4 * (size_t)t : nullptr;
    if (rec && threadIdx.x == 0) rec[0] = gtime();
    if (kLeaders && (V.tasks[t].kind & 15) == 3) {
      if (rec && threadIdx.x == 0) rec[1] = gtime();
      bwd_leader(V, t, Lb, err, D, rinv, seg, zs, ring);
    } else {
      bwd_task(V, t, Lb, 1, err, D, rinv, seg, zs, rec ? rec + 1 : nullptr);
    }
    if (rec && threadIdx.x == 0) { rec[2] = gtime(); rec[3] = smid(); }
  }
}

// ---------------------------------------------------------------------------
// The bottom of the tree, whole subtrees per warp (single right-hand side).
// The supernodes below the tree level form disjoint subtrees, each a
// contiguous range [first, root] of supernode indices (the nested-dissection
// order is a postorder of the tree).  One warp sweeps one subtree at a time,
// supernode by supernode, with no flags and no waits:
//  * forward (before the task kernels): every contribution to a supernode of
//    the subtree comes from its descendants, which the same warp has done;
//  * backward (after them): every row a supernode reads belongs to an
//    ancestor, done earlier by the same warp or, above the root, finished
//    when the task kernels ended.
// Rows inside the subtree (index < first column after the root) have one
// writer, so the forward sweep updates them with plain read-modify-writes;
// rows above it receive FP64 atomics (other subtrees add to them too).  Warps
// order their own accesses with __syncwarp between supernodes.  Panel values
// are read with coalesced 32-row loads: lane i holds row i of the diagonal
// block (forward) or column i (backward), and row i of each 32-row chunk.
// ---------------------------------------------------------------------------
constexpr int kTreeThreads = 128;  // four warps per CTA, one subtree each
constexpr unsigned kFull = 0xffffffffu;

// Optional per-subtree timeline (start, end, SM) of the subtree kernels
// (profiling aid; null unless temf_solve_timeline is running).
__device__ unsigned long long* g_timeline_tf = nullptr;
__device__ unsigned long long* g_timeline_tb = nullptr;

struct TreeView {
  const int2* trees;
  int ntree;
  const int* sn_first;
  const int64_t* rows_ptr;
  const int* sn_rows;
  const int64_t* Lptr;
  double* const* Lbase;
  double* x;
  int* counter;
  const int64_t* Dptr;  // the factor's scaled diagonal copies
};


// Rows below the diagonal block, 32 at a time: push -L21 y (ys: y in shared
// memory), plain writes for rows inside the subtree, atomics above it.
__device__ __forceinline__ void fwd_sn_rows(const TreeView& V, const double* P, int s, int c, int r, int64_t ld,
                                            int inside_end, const double* ys) {
  const int lane = threadIdx.x & 31;
  double* x = V.x;
  const int* rows = V.sn_rows + V.rows_ptr[s];
  for (int q0 = 0; q0 < r; q0 += 32) {
    const int i = q0 + lane;
    if (i < r) {
      const double* col = P + c + i;
      double acc0 = 0.0, acc1 = 0.0;
      for (int h = 0; h < c; h += 32) {  // 32 columns' loads in flight at a time
        double w[32];
#pragma unroll
        for (int k = 0; k < 32; ++k) w[k] = h + k < c ? __ldg(col + (int64_t)(h + k) * ld) : 0.0;
#pragma unroll
        for (int k = 0; k < 32; k += 2) {
          acc0 += w[k] * ys[h + k];
          acc1 += w[k + 1] * ys[h + k + 1];
        }
      }
      const double acc = acc0 + acc1;
      const int row = rows[i];
      if (row < inside_end) x[row] = __ldcg(x + row) - acc;  // one writer: this warp
      else atomicAdd(x + row, -acc);
    }
  }
  __syncwarp();
}

// forward L y = b for supernode s by one warp (ys: this warp's 64 doubles of
// shared memory).  The diagonal block comes from the factor's scaled copy Q
// (c x c column-major: L_ij / L_ii below the diagonal, 1 / L_ii on it), so
// y = D^-1 (b / L_ii) with one FMA per column on the dependent chain; lane i
// holds row i of the block.
__device__ __forceinline__ void fwd_sn_warp(const TreeView& V, const double* Lb, int s, int inside_end, double* ys) {
  const int lane = threadIdx.x & 31;
  const int f = V.sn_first[s];
  const int c = V.sn_first[s + 1] - f;
  const int r = (int)(V.rows_ptr[s + 1] - V.rows_ptr[s]);
  const int64_t ld = c + r;
  const double* P = Lb + V.Lptr[s];
  const double* Q = Lb + V.Dptr[s];
  double* x = V.x;
  const int c0 = min(c, 32);
  double a[32];
#pragma unroll
  for (int j = 0; j < 32; ++j) a[j] = (j < lane && lane < c) ? Q[j * c + lane] : 0.0;
  double v0 = lane < c ? __ldcg(x + f + lane) * Q[lane * c + lane] : 0.0;
#pragma unroll
  for (int j = 0; j < 32; ++j) {
    if (j < c0) {
      const double yj = __shfl_sync(kFull, v0, j);
      if (lane > j) v0 -= a[j] * yj;
    }
  }
  double v1 = 0.0;
  if (c > 32) {  // warp-uniform: rows 32..c-1
    const bool on = 32 + lane < c;
    v1 = on ? __ldcg(x + f + 32 + lane) * Q[(32 + lane) * c + 32 + lane] : 0.0;
#pragma unroll
    for (int j = 0; j < 32; ++j) a[j] = on ? Q[j * c + 32 + lane] : 0.0;
    double acc = 0.0;
#pragma unroll
    for (int j = 0; j < 32; ++j) acc += a[j] * __shfl_sync(kFull, v0, j);
    v1 -= acc;
#pragma unroll
    for (int m = 0; m < 32; ++m) a[m] = (m < lane && on) ? Q[(32 + m) * c + 32 + lane] : 0.0;
#pragma unroll
    for (int m = 0; m < 32; ++m) {
      if (32 + m < c) {
        const double ym = __shfl_sync(kFull, v1, m);
        if (lane > m) v1 -= a[m] * ym;
      }
    }
  }
  if (lane < c) x[f + lane] = v0;
  if (32 + lane < c) x[f + 32 + lane] = v1;
  ys[lane] = lane < c ? v0 : 0.0;
  ys[32 + lane] = 32 + lane < c ? v1 : 0.0;
  __syncwarp();
  fwd_sn_rows(V, P, s, c, r, ld, inside_end, ys);
}

// backward L^T x = y for supernode s by one warp; xs: this warp's kTreeXs
// doubles of shared memory (x at the first rows, kept from the first pass)
constexpr int kTreeXs = 256;
__device__ __forceinline__ void bwd_sn_warp(const TreeView& V, const double* Lb, int s, double* xs) {
  const int lane = threadIdx.x & 31;
  const int f = V.sn_first[s];
  const int c = V.sn_first[s + 1] - f;
  const int64_t rp = V.rows_ptr[s];
  const int r = (int)(V.rows_ptr[s + 1] - rp);
  const int64_t ld = c + r;
  const double* P = Lb + V.Lptr[s];
  double* x = V.x;
  const int* rows = V.sn_rows + rp;
  double v0 = lane < c ? __ldcg(x + f + lane) : 0.0;
  double v1 = 32 + lane < c ? __ldcg(x + f + 32 + lane) : 0.0;
  // z_j = y_j - sum_i L21[i][j] x[rows_i], 32 columns at a time.  The first
  // pass gathers x at the rows one 32-row block ahead (the gather overlaps
  // the block in flight) and keeps the first kTreeXs in shared memory for
  // the second pass.
  double acc[32];
  for (int h = 0; h * 32 < c; ++h) {
#pragma unroll
    for (int k = 0; k < 32; ++k) acc[k] = 0.0;
    double xn = (h == 0 && lane < r) ? __ldcg(x + rows[lane]) : 0.0;
    for (int q0 = 0; q0 < r; q0 += 32) {
      const int i = q0 + lane;
      const bool on = i < r;
      double xi;
      if (h == 0) {
        xi = xn;
        if (on && i < kTreeXs) xs[i] = xi;
        xn = i + 32 < r ? __ldcg(x + rows[i + 32]) : 0.0;
      } else {
        xi = !on ? 0.0 : (i < kTreeXs ? xs[i] : __ldcg(x + rows[i]));
      }
      const double* col = P + c + i;
#pragma unroll
      for (int k = 0; k < 32; ++k) {
        const int j = h * 32 + k;
        acc[k] += (on && j < c) ? __ldg(col + (int64_t)j * ld) * xi : 0.0;
      }
    }
    const double p = lane_transpose_sum(acc);
    if (h == 0) v0 -= p;
    else v1 -= p;
  }
  // diagonal block on the factor's scaled copy Q (c x c column-major,
  // D_ij = L_ij / L_ii below the diagonal, 1 / L_ii on it): D^T w = z with
  // w_i = L_ii x_i, one FMA per column on the dependent chain, then x = w / L_ii
  const double* Q = Lb + V.Dptr[s];
  double b[32];
  if (c > 32) {  // columns c-1 .. 32 (lane m holds column 32 + m)
    const bool on = 32 + lane < c;
#pragma unroll
    for (int m = 0; m < 32; ++m) b[m] = (m > lane && 32 + m < c && on) ? Q[(32 + lane) * c + 32 + m] : 0.0;
#pragma unroll
    for (int m = 31; m >= 0; --m) {
      if (32 + m < c) {
        const double wm = __shfl_sync(kFull, v1, m);
        if (lane < m) v1 -= b[m] * wm;
      }
    }
    // their contribution to columns 0..31 (lane l holds column l)
#pragma unroll
    for (int m = 0; m < 32; ++m) b[m] = (32 + m < c && lane < c) ? Q[lane * c + 32 + m] : 0.0;
    double acc2 = 0.0;
#pragma unroll
    for (int m = 0; m < 32; ++m) acc2 += b[m] * __shfl_sync(kFull, v1, m);
    v0 -= acc2;
    v1 *= on ? Q[(32 + lane) * c + 32 + lane] : 0.0;
  }
  // columns min(c,32)-1 .. 0
  const int c0 = min(c, 32);
#pragma unroll
  for (int m = 0; m < 32; ++m) b[m] = (m > lane && m < c0) ? Q[lane * c + m] : 0.0;
#pragma unroll
  for (int m = 31; m >= 0; --m) {
    if (m < c0) {
      const double wm = __shfl_sync(kFull, v0, m);
      if (lane < m) v0 -= b[m] * wm;
    }
  }
  v0 *= lane < c ? Q[lane * c + lane] : 0.0;
  if (lane < c) x[f + lane] = v0;
  if (32 + lane < c) x[f + 32 + lane] = v1;
  __syncwarp();
}

__global__ void __launch_bounds__(kTreeThreads, 3) k_fwd_subtrees(const TreeView V) {
  __shared__ double ysm[kTreeThreads / 32][kSnCols];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const double* Lb = *V.Lbase;
  for (;;) {
    int t = 0;
    if (lane == 0) t = atomicAdd(V.counter, 1);
    t = __shfl_sync(kFull, t, 0);
    if (t >= V.ntree) break;
    unsigned long long* rec = g_timeline_tf ? g_timeline_tf + 4 * (size_t)t : nullptr;
    if (rec && lane == 0) rec[0] = gtime();
    const int2 tr = V.trees[t];
    const int inside_end = V.sn_first[tr.y + 1];
    for (int s = tr.x; s <= tr.y; ++s) fwd_sn_warp(V, Lb, s, inside_end, ysm[warp]);
    if (rec && lane == 0) { rec[1] = rec[0]; rec[2] = gtime(); rec[3] = smid(); }
  }
}

__global__ void __launch_bounds__(kTreeThreads, 3) k_bwd_subtrees(const TreeView V) {
  __shared__ double xsm[kTreeThreads / 32][kTreeXs];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const double* Lb = *V.Lbase;
  for (;;) {
    int t = 0;
    if (lane == 0) t = atomicAdd(V.counter, 1);
    t = __shfl_sync(kFull, t, 0);
    if (t >= V.ntree) break;
    unsigned long long* rec = g_timeline_tb ? g_timeline_tb + 4 * (size_t)t : nullptr;
    if (rec && lane == 0) rec[0] = gtime();
    const int2 tr = V.trees[t];
    for (int s = tr.y; s >= tr.x; --s) bwd_sn_warp(V, Lb, s, xsm[warp]);
    if (rec && lane == 0) { rec[1] = rec[0]; rec[2] = gtime(); rec[3] = smid(); }
  }
}

// ---------------------------------------------------------------------------
// Many models at once (one right-hand side each): the persistent sweeps over
// the merged task list of all models.  `order` holds (model, task) pairs,
// each model's tasks in its own dependency order, so every wait still targets
// a task claimed earlier; tasks of models whose flag in `active` is 0 are
// skipped.  The dependency chains of the models overlap, which fills the GPU
// where one small model alone leaves most SMs waiting.
// ---------------------------------------------------------------------------
// Next (model, task) of a merged sweep for this CTA; (-1, -1) when done.
// Phase order as next_task: forward queue first, backward queue last.
__device__ __forceinline__ int2 next_model_task(int nstatic, const int2* __restrict__ order,
                                                const int* __restrict__ active, int* counter, int* qhead,
                                                const int* queue, int qlim, bool queue_first, int* err, int& phase,
                                                int2* sh, int spin) {
  for (;;) {
    const bool use_q = (phase == 0) == queue_first;
    if (threadIdx.x == 0) {
      int2 r = make_int2(-1, -1);
      if (use_q) {
        if (queue) {
          const int v = q_pop(qhead, queue, qlim, err, spin);
          if (v >= 0) r = make_int2(v >> 24, v & 0xFFFFFF);
        }
      } else {
        for (;;) {  // skip the tasks of models that are not stepping
          const int i = atomicAdd(counter, 1);
          if (i >= nstatic) break;
          const int2 mt = order[i];
          if (active[mt.x]) {
            r = mt;
            break;
          }
        }
      }
      *sh = r;
    }
    __syncthreads();
    const int2 r = *sh;
    __syncthreads();
    if (r.x >= 0) return r;
    if (phase == 1) return r;
    phase = 1;
  }
}

__global__ void __launch_bounds__(kSolveThreads, 3) k_fwd_models(int nstatic, const int2* __restrict__ order,
                                                                  const SweepView* __restrict__ views,
                                                                  const int* __restrict__ active, int* counter,
                                                                  int* err, int qlim) {
  __shared__ double D[kSnCols][kSnCols + 1];
  __shared__ double rinv[kSnCols];
  __shared__ double ys[kSnCols];
  __shared__ int2 mt_sh;
  const SweepView& V0 = views[0];  // the shared queue lives in every view
  int phase = 0;
  for (;;) {
    const int2 mt = next_model_task(nstatic, order, active, counter, V0.qhead, V0.queue, qlim, true, err, phase,
                                    &mt_sh, spin_limit(V0));
    if (mt.x < 0) break;
    const SweepView V = views[mt.x];
    fwd_task(V, mt.y, *V.Lbase, 1, err, D, rinv, ys);
  }
}

__global__ void __launch_bounds__(kSolveThreads, 3) k_bwd_models(int nstatic, const int2* __restrict__ order,
                                                                  const SweepView* __restrict__ views,
                                                                  const int* __restrict__ active, int* counter,
                                                                  int* err, int qlim) {
  __shared__ double D[kSnCols][kSnCols + 1];
  __shared__ double rinv[kSnCols];
  __shared__ double seg[4][kSnCols];
  __shared__ double zs[kSnCols + kChunkRows];
  __shared__ int2 mt_sh;
  const SweepView& V0 = views[0];
  int phase = 0;
  for (;;) {
    const int2 mt = next_model_task(nstatic, order, active, counter, V0.qhead, V0.queue, qlim, false, err, phase,
                                    &mt_sh, spin_limit(V0));
    if (mt.x < 0) break;
    const SweepView V = views[mt.x];
    bwd_task(V, mt.y, *V.Lbase, 1, err, D, rinv, seg, zs);
  }
}

// ---------------------------------------------------------------------------
// Blocks of up to 64 right-hand sides (many sources on one mesh): the same
// persistent task graph with 64-row chunks.  Per task:
//  * the panel block (64 rows x c columns) and the diagonal block are copied
//    to shared memory with cp.async before any dependency wait, so their
//    latency overlaps the wait;
//  * right-hand-side rows are read with all of a thread's loads in flight at
//    once (register staging; L2-coherent loads, since other CTAs write them);
//  * the 64 x 64 x c chunk products run on the FP64 tensor cores (DMMA);
//  * the c x 64 diagonal solves use two threads per column;
//  * forward chunk updates are pushed into the ancestors' rows with FP64
//    atomics; backward chunk partial sums are accumulated with FP64 atomics
//    into one c x 64 block per supernode (zeroed before each sweep), so the
//    diagonal task reads one block however many chunks the supernode has.
// ---------------------------------------------------------------------------
constexpr int kLdm = 72;  // padded leading dimension of the 64-wide shared tiles

__device__ __forceinline__ void dmma8(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}


struct MultiSmem {
  double D[kSnCols][kSnCols + 1];
  double rinv[kSnCols];
  double A[kSnCols * kLdm];  // panel block, [j][i] (column j of L21, rows of the chunk)
  double Y[kSnCols * kLdm];  // right-hand-side block, [row][col]
};

// C[m][n] += sum_k A(m,k) B(k,n) for a 64 x 64 tile; warps 2x2 of 32x32.
// A(m,k) = Am[m * sam + k * sak], B(k,n) = Bk[k * kLdm + n].
__device__ __forceinline__ void mma_tile64(double acc[4][4][2], const double* Am, int sam, int sak,
                                           const double* Bk, int kdim) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wr = (warp >> 1) * 32, wc = (warp & 1) * 32;
  const int g = lane >> 2, q = lane & 3;
  for (int k0 = 0; k0 < kdim; k0 += 4) {
    double fa[4], fb[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) fa[a] = Am[(wr + a * 8 + g) * sam + (k0 + q) * sak];
#pragma unroll
    for (int b = 0; b < 4; ++b) fb[b] = Bk[(k0 + q) * kLdm + wc + b * 8 + g];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) dmma8(acc[a][b][0], acc[a][b][1], fa[a], fb[b]);
  }
}

// store the accumulators of mma_tile64 to a [m][n] tile with leading dimension kLdm
__device__ __forceinline__ void store_tile64(const double acc[4][4][2], double* C) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wr = (warp >> 1) * 32, wc = (warp & 1) * 32;
  const int g = lane >> 2, q = lane & 3;
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b)
#pragma unroll
      for (int e = 0; e < 2; ++e) C[(wr + a * 8 + g) * kLdm + wc + b * 8 + 2 * q + e] = acc[a][b][e];
}

__device__ __forceinline__ void zero_acc(double acc[4][4][2]) {
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
}

// panel rows [r0, r0+nr) x columns [0, c) of L21 into A[j][i] (zero padded to 64 x 64), asynchronously
__device__ __forceinline__ void load_panel_block_async(double* A, const double* P, int c, int64_t ld, int r0,
                                                       int nr) {
  for (int idx = threadIdx.x; idx < kSnCols * kSnCols; idx += blockDim.x) {
    const int j = idx / kSnCols, i = idx % kSnCols;
    if (j < c && i < nr) cp_async8(A + j * kLdm + i, P + (int64_t)j * ld + c + r0 + i);
    else A[j * kLdm + i] = 0.0;
  }
}
// lower triangle of the diagonal block into D[i][j], asynchronously (rinv after the wait)
__device__ __forceinline__ void load_diag_async(double (*D)[kSnCols + 1], const double* P, int c, int64_t ld) {
  for (int idx = threadIdx.x; idx < c * c; idx += blockDim.x) {
    const int j = idx / c, i = idx % c;
    if (i >= j) cp_async8(&D[i][j], P + (int64_t)j * ld + i);
  }
}
__device__ __forceinline__ void finish_diag(MultiSmem& M, int c) {
  if ((int)threadIdx.x < c) M.rinv[threadIdx.x] = 1.0 / M.D[threadIdx.x][threadIdx.x];
}

// Y[j][col] = x[rows[j]][col] for j < nr, col < k (zero elsewhere); every
// load of a thread is issued before the first store.
template <bool kContiguous>
__device__ __forceinline__ void load_rows(double* Y, const double* x, int64_t ldx, int k, int nr, int f,
                                          const int* __restrict__ rows) {
  constexpr int kPer = kSnCols * kSnCols / kSolveThreads;
  double v[kPer];
#pragma unroll
  for (int u = 0; u < kPer; ++u) {
    const int idx = threadIdx.x + u * kSolveThreads;
    const int j = idx / kSnCols, col = idx % kSnCols;
    const int64_t row = kContiguous ? (int64_t)(f + j) : (j < nr ? (int64_t)rows[j] : 0);
    v[u] = (j < nr && col < k) ? __ldcg(x + row * ldx + col) : 0.0;
  }
#pragma unroll
  for (int u = 0; u < kPer; ++u) {
    const int idx = threadIdx.x + u * kSolveThreads;
    Y[(idx / kSnCols) * kLdm + idx % kSnCols] = v[u];
  }
}

// Y = L11^{-1} Y (forward) or L11^{-T} Y (backward) for 64 columns; two
// threads per column (adjacent lanes) split the rows by parity.
__device__ __forceinline__ void diag_solve_block(MultiSmem& M, int c, bool forward) {
  const int col = threadIdx.x >> 1, h = threadIdx.x & 1;
  double* Y = M.Y;
  if (forward) {
    for (int j = 0; j < c; ++j) {
      if ((j & 1) == h) Y[j * kLdm + col] *= M.rinv[j];
      __syncwarp();
      const double yj = Y[j * kLdm + col];
      int i = j + 1;
      if ((i & 1) != h) ++i;
      for (; i < c; i += 2) Y[i * kLdm + col] -= M.D[i][j] * yj;
    }
  } else {
    for (int j = c - 1; j >= 0; --j) {
      if ((j & 1) == h) Y[j * kLdm + col] *= M.rinv[j];
      __syncwarp();
      const double xj = Y[j * kLdm + col];
      for (int i = h; i < j; i += 2) Y[i * kLdm + col] -= M.D[j][i] * xj;
    }
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kSolveThreads) k_fwd_multi(const SweepView V, int ldx, int k, int* err) {
  extern __shared__ __align__(16) unsigned char smraw[];
  MultiSmem& M = *reinterpret_cast<MultiSmem*>(smraw);
  __shared__ int task_id;
  int* ready = V.sync;
  int* ydone = V.sync + V.nsn;
  double* x = V.x;
  const int tid = threadIdx.x;
  const double* Lb = *V.Lbase;
  int phase = 0;
  for (;;) {
    const int t = next_task(V, V.sync + 4 * V.nsn, true, err, phase, &task_id);
    if (t < 0) break;
    const SolveTask T = V.tasks[t];
    const int s = T.s;
    const int f = V.sn_first[s];
    const int c = V.sn_first[s + 1] - f;
    const int64_t rp = V.rows_ptr[s];
    const int64_t r = V.rows_ptr[s + 1] - rp;
    const int64_t ld = c + r;
    const double* P = Lb + V.Lptr[s];
    const int nr = T.r1 - T.r0;
    // the factor does not depend on the sweep: start its copies before any wait
    if (nr > 0) load_panel_block_async(M.A, P, c, ld, T.r0, nr);
    if (T.kind == 0) load_diag_async(M.D, P, c, ld);
    if (tid == 0 && !in_queue(V, t)) {  // claimed in order: wait for the inputs
      if (T.kind == 0) wait_geq(ready + s, V.expect[s], err, 1, spin_limit(V));
      else wait_geq(ydone + s, 1, err, 2, spin_limit(V));
    }
    __syncthreads();
    load_rows<true>(M.Y, x, ldx, k, c, f, nullptr);
    cp_async_wait_all();
    __syncthreads();
    if (T.kind == 0) {
      finish_diag(M, c);
      __syncthreads();
      diag_solve_block(M, c, true);
      for (int idx = tid; idx < c * k; idx += blockDim.x) {
        const int j = idx / k, col = idx % k;
        x[(int64_t)(f + j) * ldx + col] = M.Y[j * kLdm + col];
      }
      __threadfence();
      __syncthreads();
      if (tid == 0) atomicExch(ydone + s, 1);
      // y_s is out: the other row chunks of s (the tasks right after this one) are ready
      const int nx = max(1, (int)((r + kChunkRowsMulti - 1) / kChunkRowsMulti)) - 1;
      for (int q = tid; q < nx; q += blockDim.x) q_push(V, t + 1 + q);
    }
    if (nr > 0) {
      // U = L21[rows] Y_s (64 x 64 x c), then push -U into the rows' right-hand sides
      double acc[4][4][2];
      zero_acc(acc);
      mma_tile64(acc, M.A, 1, kLdm, M.Y, (c + 3) & ~3);
      __syncthreads();
      store_tile64(acc, M.A);  // reuse A as [row][col]
      __syncthreads();
      const int warp = tid >> 5, lane = tid & 31;
      for (int i = warp; i < nr; i += kSolveThreads / 32) {
        double* dst = x + (int64_t)V.sn_rows[rp + T.r0 + i] * ldx;
        for (int col = lane; col < k; col += 32) atomicAdd(dst + col, -M.A[i * kLdm + col]);
      }
      __threadfence();
      __syncthreads();
      count_inputs(V, V.tgt_ptr[t], V.tgt_ptr[t + 1]);
    }
  }
}

__global__ void __launch_bounds__(kSolveThreads) k_bwd_multi(const SweepView V, int ldx, int k, int* err) {
  extern __shared__ __align__(16) unsigned char smraw[];
  MultiSmem& M = *reinterpret_cast<MultiSmem*>(smraw);
  __shared__ int task_id;
  int* cdone = V.sync + 2 * V.nsn;
  int* xdone = V.sync + 3 * V.nsn;
  double* x = V.x;
  const int tid = threadIdx.x;
  const double* Lb = *V.Lbase;
  int phase = 0;
  for (;;) {
    const int t = next_task(V, V.sync + 4 * V.nsn + 1, false, err, phase, &task_id);
    if (t < 0) break;
    const SolveTask T = V.tasks[t];
    const int s = T.s;
    const int f = V.sn_first[s];
    const int c = V.sn_first[s + 1] - f;
    const int64_t rp = V.rows_ptr[s];
    const int64_t r = V.rows_ptr[s + 1] - rp;
    const int64_t ld = c + r;
    const double* P = Lb + V.Lptr[s];
    const int nr = T.r1 - T.r0;
    if (nr > 0) load_panel_block_async(M.A, P, c, ld, T.r0, nr);
    if (T.kind == 0) load_diag_async(M.D, P, c, ld);
    if (!in_queue(V, t)) {  // claimed in order: wait for the inputs, one polling thread each
      const int q0 = V.tgt_ptr[t], nq = V.tgt_ptr[t + 1] - q0;
      for (int q = tid; q < nq; q += blockDim.x) wait_geq(xdone + V.tgt[q0 + q], 1, err, 3, spin_limit(V));
      if (T.kind == 0 && tid == blockDim.x - 1) wait_geq(cdone + s, max(V.nchunk[s], 1) - 1, err, 4, spin_limit(V));
    }
    __syncthreads();
    // Xr = x[rows] (64 x k); C = L21[rows]^T Xr (c x k)
    if (nr > 0) load_rows<false>(M.Y, x, ldx, k, nr, 0, V.sn_rows + rp + T.r0);
    cp_async_wait_all();
    __syncthreads();
    double acc[4][4][2];
    zero_acc(acc);
    if (nr > 0) {
      mma_tile64(acc, M.A, kLdm, 1, M.Y, 64);
      __syncthreads();
    }
    double* as = V.part + V.part_off[s] * kMultiCols;  // this supernode's c x 64 accumulator
    if (T.kind == 1) {
      store_tile64(acc, M.Y);
      __syncthreads();
      const int warp = tid >> 5, lane = tid & 31;
      for (int j = warp; j < c; j += kSolveThreads / 32)
        for (int col = lane; col < k; col += 32) atomicAdd(as + j * kMultiCols + col, M.Y[j * kLdm + col]);
      __threadfence();
      __syncthreads();
      if (tid == 0) {
        atomicAdd(cdone + s, 1);
        const int d = V.diag_task[s];
        if (in_queue(V, d) && atomicAdd(V.cnt + d, 1) == V.need[d] - 1) q_push(V, d);
      }
    } else {
      // Z = Y_s - (first chunk, here) - (other chunks, accumulated); back-substitute
      finish_diag(M, c);
      store_tile64(acc, M.A);  // first-chunk products as [j][col]
      __syncthreads();
      const bool more = V.nchunk[s] > 1;
      for (int idx = tid; idx < kSnCols * kSnCols; idx += blockDim.x) {
        const int j = idx / kSnCols, col = idx % kSnCols;
        double v = 0.0;
        if (j < c && col < k) {
          v = __ldcg(x + (int64_t)(f + j) * ldx + col);
          if (nr > 0) v -= M.A[j * kLdm + col];
          if (more) v -= __ldcg(as + j * kMultiCols + col);
        }
        M.Y[j * kLdm + col] = v;
      }
      __syncthreads();
      diag_solve_block(M, c, false);
      for (int idx = tid; idx < c * k; idx += blockDim.x) {
        const int j = idx / k, col = idx % k;
        x[(int64_t)(f + j) * ldx + col] = M.Y[j * kLdm + col];
      }
      __threadfence();
      __syncthreads();
      if (tid == 0) atomicExch(xdone + s, 1);
      count_owner_done(V, V.dep_ptr[s], V.dep_ptr[s + 1]);  // x_s is out: every queued task whose rows s owns
    }
  }
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

__global__ void k_add_int(int* p, int d) { *p += d; }

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
namespace {
// Task lists of the persistent sweeps for a given chunk height (see the
// kernels): per task its owner/target supernodes, per supernode the forward
// chunk count it waits for, its row-chunk count and partial-sum offset.
struct Sched {
  std::vector<SolveTask> ft, bt;  // the claimable tasks (nf, nb of them), then the absorbed entries
  std::vector<int> ftp{0}, ftg, btp{0}, btg, expect, nch;
  std::vector<int64_t> poff;
  int nf = 0, nb = 0;
};

// min_level > 0: supernodes below that level (swept by the subtree kernels)
// get no tasks and feed no counts.  lead_level: runs of column blocks (at
// least two, the first at or above that level) are swept by one leader task
// (kind 3 | blocks << 4: forward at the run's first block, backward at its
// last); the diagonal entries of the other blocks become absorbed entries
// (kind 4) after the claimable tasks.  The targets / owners of a run block's
// first chunk exclude the run's own blocks (applied through the leader's
// ring).  Single right-hand side only (128-row first chunks).
// group_from: at levels from this one up, the tasks are ordered for in-order
// claiming.  Forward: a level's diagonal tasks first; each other chunk is held
// back until just before the diagonal tasks of the lowest level it feeds, so
// chunks claimed in order find their own diagonal task long done and the
// next level's diagonal tasks are not queued behind chunks that feed levels
// far above.  Backward: every other chunk of a level, then its diagonal
// tasks.  Only above the queue split: the queued forward tasks rely on a
// supernode's chunks following its diagonal task.
void build_sched(const Symbolic& S, int CH, Sched& o, int min_level = 0, int lead_level = INT_MAX,
                 int group_from = INT_MAX) {
  const int nsn = S.nsn;
  // distinct owner supernodes of rows [r0, r1) of s above `skip_to` (rows ascending -> owners ascending)
  std::vector<int> tmp;
  auto owners = [&](int s, int r0, int r1, int skip_to = -1) {
    tmp.clear();
    const int* rows = S.sn_rows.data() + S.sn_rows_ptr[s];
    for (int i = r0; i < r1; ++i) {
      const int ow = S.col2sn[rows[i]];
      if (ow <= skip_to) continue;
      if (tmp.empty() || tmp.back() != ow) tmp.push_back(ow);
    }
  };
  o.expect.assign(nsn, 0);
  o.nch.assign(nsn, 0);
  o.poff.assign(nsn + 1, 0);
  for (int s = 0; s < nsn; ++s) {
    const int r = (int)(S.sn_rows_ptr[s + 1] - S.sn_rows_ptr[s]);
    o.nch[s] = ceil_div(r, CH);
    o.poff[s + 1] = o.poff[s] + (int64_t)o.nch[s] * (S.sn_first[s + 1] - S.sn_first[s]);
  }
  // runs with a leader: run_a[s] = first block, run_e[s] = last block (-1: none).
  // A leader holds its CTA while it waits for chunk tasks claimed after it, so
  // the leaders that may be active at once must stay well below the resident
  // CTAs of the kernel: runs are taken from the top of the tree down while no
  // level is spanned by more than kMaxLeaders of them.
  std::vector<int> run_a(nsn, -1), run_e(nsn, -1);
  if (lead_level < INT_MAX && CH == kChunkRows) {
    const std::vector<int> rf = block_run_first(S);
    std::vector<std::pair<int, int>> cand;  // (first, last block)
    for (int s0 = 0; s0 < nsn;) {
      int e = s0;
      while (e + 1 < nsn && rf[e + 1] == s0) ++e;
      if (e > s0 && S.sn_level[s0] >= std::max(lead_level, min_level)) cand.push_back({s0, e});
      s0 = e + 1;
    }
    std::stable_sort(cand.begin(), cand.end(), [&](const std::pair<int, int>& x, const std::pair<int, int>& y) {
      return S.sn_level[x.second] > S.sn_level[y.second];
    });
    std::vector<int> span(S.nlevels + 1, 0);  // runs spanning each level
    for (const auto& rn : cand) {
      const int lo = S.sn_level[rn.first], hi = S.sn_level[rn.second];
      bool room = true;
      for (int l = lo; l <= hi && room; ++l) room = span[l] < kMaxLeaders;
      if (!room) continue;
      for (int l = lo; l <= hi; ++l) ++span[l];
      for (int q = rn.first; q <= rn.second; ++q) { run_a[q] = rn.first; run_e[q] = rn.second; }
    }
  }
  std::vector<SolveTask> abs_t;
  std::vector<std::vector<int>> abs_g;
  // forward chunks above group_from, by the lowest level among their targets
  std::vector<std::vector<std::pair<SolveTask, std::vector<int>>>> late(S.nlevels + 1);
  // forward: bottom-up levels; per supernode its diagonal task (with the first
  // row chunk), then the other chunks
  for (int l = std::max(0, min_level); l < S.nlevels; ++l) {
    const bool grouped = l >= group_from;
    for (int q = S.level_ptr[l]; q < S.level_ptr[l + 1]; ++q) {
      const int s = S.level_sn[q];
      const int r = (int)(S.sn_rows_ptr[s + 1] - S.sn_rows_ptr[s]);
      for (int r0 = 0; r0 < std::max(r, 1); r0 += CH) {
        const int r1 = std::min(r, r0 + CH);
        if (grouped && r0 > 0) {  // held back until just before its first consumer's level
          owners(s, r0, r1);
          int mlev = S.nlevels - 1;
          for (int ow : tmp) mlev = std::min(mlev, S.sn_level[ow]);
          late[mlev].push_back({SolveTask{s, 1, r0, r1}, tmp});
          continue;
        }
        if (r0 == 0 && run_a[s] >= 0) {
          owners(s, 0, r1, run_e[s]);
          for (int ow : tmp) o.expect[ow]++;
          if (s == run_a[s]) {
            o.ft.push_back({s, 3 | ((run_e[s] - s + 1) << 4), 0, r1});
            o.ftg.insert(o.ftg.end(), tmp.begin(), tmp.end());
            o.ftp.push_back((int)o.ftg.size());
          } else {
            abs_t.push_back({s, 4, 0, r1});
            abs_g.push_back(tmp);
          }
          continue;
        }
        o.ft.push_back({s, r0 == 0 ? 0 : 1, r0, r1});
        owners(s, r0, r1);
        for (int ow : tmp) { o.ftg.push_back(ow); o.expect[ow]++; }
        o.ftp.push_back((int)o.ftg.size());
      }
    }
    // the chunks whose first consumer is at the next level, before its diagonal tasks
    if (l + 1 < S.nlevels) {
      for (auto& e : late[l + 1]) {
        o.ft.push_back(e.first);
        for (int ow : e.second) { o.ftg.push_back(ow); o.expect[ow]++; }
        o.ftp.push_back((int)o.ftg.size());
      }
      late[l + 1].clear();
    }
  }
  o.nf = (int)o.ft.size();
  for (size_t k = 0; k < abs_t.size(); ++k) {
    o.ft.push_back(abs_t[k]);
    o.ftg.insert(o.ftg.end(), abs_g[k].begin(), abs_g[k].end());
    o.ftp.push_back((int)o.ftg.size());
  }
  abs_t.clear();
  abs_g.clear();
  // backward: top-down levels; per supernode its other chunks, then the
  // diagonal task with the first chunk.  A backward task waits for one owner
  // only: the owner A of its lowest row.  Its rows R' lie in R(s) above A's
  // first column; following the supernodal tree from s up to A, each step
  // keeps R' inside the next supernode's rows (R(child) minus the parent's
  // columns lies in R(parent)), so R' lies in cols(A) and R(A), and A is
  // solved only after every owner of R(A) (check_schedule replays the real
  // row dependencies).  So each task has one dependency, not one per owner.
  auto lowest = [&]() {
    if (tmp.size() > 1) tmp.resize(1);
  };
  for (int l = S.nlevels - 1; l >= std::max(0, min_level); --l)
    for (int pass = 0; pass < (l >= group_from ? 2 : 1); ++pass)
    for (int q = S.level_ptr[l]; q < S.level_ptr[l + 1]; ++q) {
      const int s = S.level_sn[q];
      const int r = (int)(S.sn_rows_ptr[s + 1] - S.sn_rows_ptr[s]);
      if (l < group_from || pass == 0) {
        for (int r0 = CH; r0 < r; r0 += CH) {
          const int r1 = std::min(r, r0 + CH);
          o.bt.push_back({s, 1, r0, r1});
          owners(s, r0, r1);
          lowest();
          o.btg.insert(o.btg.end(), tmp.begin(), tmp.end());
          o.btp.push_back((int)o.btg.size());
        }
      }
      if (l >= group_from && pass == 0) continue;
      const int r1 = std::min(r, CH);
      if (run_a[s] >= 0) {
        owners(s, 0, r1, run_e[s]);
        lowest();
        if (s == run_e[s]) {
          o.bt.push_back({s, 3 | ((run_e[s] - run_a[s] + 1) << 4), 0, r1});
          o.btg.insert(o.btg.end(), tmp.begin(), tmp.end());
          o.btp.push_back((int)o.btg.size());
        } else {
          abs_t.push_back({s, 4, 0, r1});
          abs_g.push_back(tmp);
        }
        continue;
      }
      o.bt.push_back({s, 0, 0, r1});
      owners(s, 0, r1);
      lowest();
      o.btg.insert(o.btg.end(), tmp.begin(), tmp.end());
      o.btp.push_back((int)o.btg.size());
    }
  o.nb = (int)o.bt.size();
  for (size_t k = 0; k < abs_t.size(); ++k) {
    o.bt.push_back(abs_t[k]);
    o.btg.insert(o.btg.end(), abs_g[k].begin(), abs_g[k].end());
    o.btp.push_back((int)o.btg.size());
  }
}
// Ready-queue data of a schedule: diagonal task per supernode (forward,
// backward), backward completion counts and dependants, initially ready
// tasks of both sweeps.
struct QueueData {
  std::vector<int> fdiag, bdiag, bneed, dptr, dep, finit, binit;
};

void build_queue_data(const Sched& a, int nsn, QueueData& q, int f_hi, int b_lo) {
  q.fdiag.assign(nsn, -1);
  q.bdiag.assign(nsn, -1);
  q.bneed.assign(a.bt.size(), 0);
  // diagonal entry per supernode: its diagonal task, its run's leader, or its absorbed entry
  auto diag_kind = [](int k) { k &= 15; return k == 0 || k == 3 || k == 4; };
  for (size_t i = 0; i < a.ft.size(); ++i)
    if (diag_kind(a.ft[i].kind)) q.fdiag[a.ft[i].s] = (int)i;
  for (size_t i = 0; i < a.bt.size(); ++i)
    if (diag_kind(a.bt[i].kind)) q.bdiag[a.bt[i].s] = (int)i;
  q.dptr.assign(nsn + 1, 0);
  for (size_t i = 0; i < a.bt.size(); ++i) {
    const SolveTask& T = a.bt[i];
    // owners of its rows, and for a diagonal task its other row chunks
    q.bneed[i] = (a.btp[i + 1] - a.btp[i]) + (T.kind == 0 ? std::max(a.nch[T.s], 1) - 1 : 0);
    for (int k = a.btp[i]; k < a.btp[i + 1]; ++k) q.dptr[a.btg[k] + 1]++;
  }
  for (int k = 0; k < nsn; ++k) q.dptr[k + 1] += q.dptr[k];
  q.dep.resize(q.dptr[nsn]);
  std::vector<int> fill(q.dptr.begin(), q.dptr.end() - 1);
  for (size_t i = 0; i < a.bt.size(); ++i)
    for (int k = a.btp[i]; k < a.btp[i + 1]; ++k) q.dep[fill[a.btg[k]]++] = (int)i;
  q.finit.clear();
  q.binit.clear();
  for (int i = 0; i < f_hi; ++i)
    if (a.ft[i].kind == 0 && a.expect[a.ft[i].s] == 0) q.finit.push_back(i);
  for (int i = b_lo; i < a.nb; ++i)
    if (q.bneed[i] == 0) q.binit.push_back(i);
}

// queue ranges of a split level: forward tasks below it (a prefix of the
// bottom-up schedule), backward tasks below it (a suffix of the top-down one)
void split_ranges(const Sched& a, const Symbolic& S, int split, int& f_hi, int& b_lo) {
  f_hi = 0;
  while (f_hi < a.nf && S.sn_level[a.ft[f_hi].s] < split) ++f_hi;
  b_lo = a.nb;
  while (b_lo > 0 && S.sn_level[a.bt[b_lo - 1].s] < split) --b_lo;
}

// first level (from the leaves) holding fewer than `width` supernodes
int level_below_width(const Symbolic& S, int width) {
  for (int l = 0; l < S.nlevels; ++l)
    if (S.level_ptr[l + 1] - S.level_ptr[l] < width) return l;
  return S.nlevels;
}
int default_split(const Symbolic& S) { return level_below_width(S, 512); }

void upload_queue_plan(const Sched& a, const Symbolic& S, int split, QueuePlan& Q, cudaStream_t st) {
  const int nsn = S.nsn;
  int f_hi = 0, b_lo = 0;
  split_ranges(a, S, split, f_hi, b_lo);
  QueueData qd;
  build_queue_data(a, nsn, qd, f_hi, b_lo);
  Q.split = split;
  Q.f_hi = f_hi;
  Q.b_lo = b_lo;
  auto up = [&](DBuf<int>& d, const std::vector<int>& v) {
    if (v.empty()) d.alloc(1);
    else d.upload(v.data(), v.size(), st);
  };
  up(Q.fdiag, qd.fdiag);
  up(Q.bdiag, qd.bdiag);
  up(Q.bneed, qd.bneed);
  up(Q.bdep_ptr, qd.dptr);
  up(Q.bdep, qd.dep);
  // queue slots hold task + 1 (0 marks a slot not yet written)
  std::vector<int> fi(qd.finit), bi(qd.binit);
  for (int& v : fi) ++v;
  for (int& v : bi) ++v;
  up(Q.finit, fi);
  up(Q.binit, bi);
  Q.n_finit = (int)qd.finit.size();
  Q.n_binit = (int)qd.binit.size();
  const int tails[2] = {Q.n_finit, Q.n_binit};
  Q.qtails.upload(tails, 2, st);
  Q.qbuf.alloc(a.ft.size() + 2 * a.bt.size() + 4);
  TEMF_CUDA(cudaStreamSynchronize(st));
}

// Host replay of both sweeps' protocols for chunk height CH and queue split
// level `split`: tasks below the split go through the ready queue (handed
// out once, only after their inputs), the others are claimed in schedule
// order and must find their inputs complete when every earlier task is.
// Forward: queue phase, then the ordered phase; backward: the other way
// round, the ordered tasks' completions feeding the queue.  Returns an empty
// string or the first violation.
std::string check_schedule(const Symbolic& S, int CH, int split, int min_level = 0, int lead_level = INT_MAX,
                           bool grouped = false, int group_at = -1) {
  Sched a;
  build_sched(S, CH, a, min_level, lead_level,
              grouped ? (group_at >= 0 ? group_at : std::max(split, min_level)) : INT_MAX);
  int f_hi = 0, b_lo = 0;
  split_ranges(a, S, split, f_hi, b_lo);
  QueueData q;
  build_queue_data(a, S.nsn, q, f_hi, b_lo);
  const int nsn = S.nsn, nf = a.nf, nb = a.nb;
  auto first_rows = [&](int s) { return (int)std::min<int64_t>(S.sn_rows_ptr[s + 1] - S.sn_rows_ptr[s], CH); };
  {
    std::vector<int> ready(nsn, 0), ydone(nsn, 0), seen(nf, 0);
    std::vector<int> queue(q.finit);
    // run leaders in progress: (next block, last block)
    std::vector<std::pair<int, int>> leaders;
    auto feed = [&](int t) {  // the targets of entry t count one input more
      for (int k = a.ftp[t]; k < a.ftp[t + 1]; ++k) {
        const int o = a.ftg[k];
        if (++ready[o] == a.expect[o] && q.fdiag[o] < f_hi) queue.push_back(q.fdiag[o]);
      }
    };
    auto advance = [&]() {  // every leader as far as its inputs allow
      for (bool moved = true; moved;) {
        moved = false;
        for (auto& L : leaders)
          while (L.first <= L.second && ready[L.first] == a.expect[L.first]) {
            ydone[L.first] = 1;
            feed(q.fdiag[L.first]);
            ++L.first;
            moved = true;
          }
      }
    };
    auto run = [&](int t, bool queued) -> std::string {
      if (seen[t]++) return "forward: task handed out twice";
      const SolveTask& T = a.ft[t];
      if ((T.kind & 15) == 3) {
        if (queued) return "forward queue: a run leader in the queue";
        leaders.push_back({T.s, T.s + (T.kind >> 4) - 1});
        advance();
        return std::string();
      }
      advance();
      if (T.kind == 0) {
        if (ready[T.s] != a.expect[T.s]) return queued ? "forward queue: diagonal task before its inputs"
                                                       : "forward: diagonal task claimed before its inputs";
        ydone[T.s] = 1;
        const int r = (int)(S.sn_rows_ptr[T.s + 1] - S.sn_rows_ptr[T.s]);
        const int nx = std::max(1, (r + CH - 1) / CH) - 1;
        for (int k = 0; k < nx; ++k)
          if (t + 1 + k < f_hi) queue.push_back(t + 1 + k);
      } else if (T.kind == 1) {
        if (!ydone[T.s]) return "forward: chunk before its diagonal block is solved";
      } else {
        return "forward: an absorbed entry among the claimable tasks";
      }
      feed(t);
      return std::string();
    };
    for (size_t h = 0; h < queue.size(); ++h) {
      if (queue[h] >= f_hi) return "forward queue: task outside the queue range";
      const std::string w = run(queue[h], true);
      if (!w.empty()) return w;
    }
    if ((int)queue.size() != f_hi) return "forward queue: not every queued task handed out";
    for (int t = f_hi; t < nf; ++t) {
      const std::string w = run(t, false);
      if (!w.empty()) return w;
    }
    advance();
    for (const auto& L : leaders)
      if (L.first <= L.second) return "forward: a run leader cannot finish";
    for (int s = 0; s < nsn; ++s)
      if (S.sn_level[s] >= min_level && !ydone[s]) return "forward: a supernode never solved";
  }
  {
    std::vector<int> xdone(nsn, 0), cdone(nsn, 0), cnt(nb, 0), seen(nb, 0);
    std::vector<int> queue(q.binit);
    std::vector<std::pair<int, int>> leaders;  // (next block, first block), top-down
    // the real inputs: every row [r0, r1) of s owned above `skip_to` is solved
    auto rows_final = [&](int s, int r0, int r1, int skip_to) {
      const int* rows = S.sn_rows.data() + S.sn_rows_ptr[s];
      for (int i = r0; i < r1; ++i) {
        const int ow = S.col2sn[rows[i]];
        if (ow > skip_to && !xdone[ow]) return false;
      }
      return true;
    };
    std::string real_err;
    std::vector<int> run_last(nsn, -1);  // per first block of a leader's run: its last block
    auto count = [&](int d) {
      if (d < nb && ++cnt[d] == q.bneed[d] && d >= b_lo) queue.push_back(d);
    };
    auto solved = [&](int s) {
      xdone[s] = 1;
      for (int k = q.dptr[s]; k < q.dptr[s + 1]; ++k) count(q.dep[k]);
    };
    auto inputs_done = [&](int t, int s) {
      for (int k = a.btp[t]; k < a.btp[t + 1]; ++k)
        if (!xdone[a.btg[k]]) return false;
      return cdone[s] == std::max(a.nch[s], 1) - 1 || (first_rows(s) == 0 && cdone[s] == 0);
    };
    auto advance = [&]() {
      for (bool moved = true; moved;) {
        moved = false;
        for (auto& L : leaders)
          while (L.first >= L.second && inputs_done(q.bdiag[L.first], L.first)) {
            const SolveTask& E = a.bt[q.bdiag[L.first]];
            if (real_err.empty() && !rows_final(E.s, E.r0, E.r1, run_last[L.second]))
              real_err = "backward: a run block solved before an owner of its rows";
            solved(L.first);
            --L.first;
            moved = true;
          }
      }
    };
    auto run = [&](int t, bool queued) -> std::string {
      if (seen[t]++) return "backward: task handed out twice";
      const SolveTask& T = a.bt[t];
      if ((T.kind & 15) == 3) {
        if (queued) return "backward queue: a run leader in the queue";
        leaders.push_back({T.s, T.s - (T.kind >> 4) + 1});
        run_last[T.s - (T.kind >> 4) + 1] = T.s;
        advance();
        return std::string();
      }
      advance();
      if (queued) {
        if (cnt[t] != q.bneed[t]) return "backward queue: task before its inputs";
      } else {
        for (int k = a.btp[t]; k < a.btp[t + 1]; ++k)
          if (!xdone[a.btg[k]]) return "backward: task claimed before an owner of its rows";
        if (T.kind == 0 && cdone[T.s] != std::max(a.nch[T.s], 1) - 1) return "backward: diagonal task before its chunks";
      }
      if (!rows_final(T.s, T.r0, T.r1, -1)) return "backward: task run before an owner of its rows";
      if (T.kind == 1) {
        cdone[T.s]++;
        count(q.bdiag[T.s]);
      } else if (T.kind == 0) {
        solved(T.s);
      } else {
        return "backward: an absorbed entry among the claimable tasks";
      }
      return std::string();
    };
    for (int t = 0; t < b_lo; ++t) {
      const std::string w = run(t, false);
      if (!w.empty()) return w;
    }
    advance();
    for (const auto& L : leaders)
      if (L.first >= L.second) return "backward: a run leader cannot finish";
    for (size_t h = 0; h < queue.size(); ++h) {
      if (queue[h] < b_lo) return "backward queue: task outside the queue range";
      const std::string w = run(queue[h], true);
      if (!w.empty()) return w;
    }
    if ((int)queue.size() != nb - b_lo) return "backward queue: not every queued task handed out";
    if (!real_err.empty()) return real_err;
    for (int s = 0; s < nsn; ++s)
      if (S.sn_level[s] >= min_level && !xdone[s]) return "backward: a supernode never solved";
  }
  return std::string();
}

// Subtrees of the supernodes below `level`: a root is such a supernode whose
// parent is at or above the level (or that has none); its subtree is the
// index range [first descendant, root], which the postorder of the supernodes
// makes contiguous (checked).  Largest stored panels first, so the warps that
// take the last subtrees finish together.
std::vector<int2> build_trees(const Symbolic& S, int level) {
  std::vector<int2> out;
  if (level <= 0) return out;
  const int nsn = S.nsn;
  std::vector<int> first(nsn), cnt(nsn, 1);
  for (int s = 0; s < nsn; ++s) first[s] = s;
  for (int s = 0; s < nsn; ++s) {
    const int p = S.sn_parent[s];
    if (p < 0) continue;
    if (p <= s) throw StateError("supernodes are not in postorder (parent before child)");
    first[p] = std::min(first[p], first[s]);
    cnt[p] += cnt[s];
  }
  std::vector<std::pair<int64_t, int2>> v;
  for (int s = 0; s < nsn; ++s) {
    if (S.sn_level[s] >= level) continue;
    const int p = S.sn_parent[s];
    if (p >= 0 && S.sn_level[p] < level) continue;
    if (cnt[s] != s - first[s] + 1) throw StateError("a subtree is not a contiguous supernode range");
    v.push_back({S.sn_Lptr[s + 1] - S.sn_Lptr[first[s]], make_int2(first[s], s)});
  }
  std::stable_sort(v.begin(), v.end(), [](const std::pair<int64_t, int2>& a, const std::pair<int64_t, int2>& b) {
    return a.first > b.first;
  });
  out.reserve(v.size());
  for (const auto& e : v) out.push_back(e.second);
  return out;
}

// Host check of the subtree protocol at `level`: the subtrees cover every
// supernode below the level exactly once, each supernode's rows are owned by
// later supernodes, rows owned inside its subtree belong to supernodes of
// that subtree, and rows above it to supernodes at or above the level (done
// by the task kernels, never by another subtree).
std::string check_trees(const Symbolic& S, int level) {
  std::vector<int2> trees;
  try {
    trees = build_trees(S, level);
  } catch (const std::exception& e) {
    return e.what();
  }
  std::vector<int> seen(S.nsn, 0);
  for (const int2& t : trees) {
    const int inside_end = S.sn_first[t.y + 1];
    for (int s = t.x; s <= t.y; ++s) {
      if (seen[s]++) return "a supernode in two subtrees";
      if (S.sn_level[s] >= level) return "a subtree holds a supernode at or above the level";
      for (int64_t k = S.sn_rows_ptr[s]; k < S.sn_rows_ptr[s + 1]; ++k) {
        const int row = S.sn_rows[k];
        const int o = S.col2sn[row];
        if (o <= s) return "a row owned by an earlier supernode";
        if (row < inside_end ? (o > t.y) : (S.sn_level[o] < level)) return "a row owned outside the protocol";
      }
    }
  }
  for (int s = 0; s < S.nsn; ++s)
    if (S.sn_level[s] < level && !seen[s]) return "a supernode below the level in no subtree";
  return std::string();
}

// The single-column plan at a subtree level and queue split.
void upload_tree_plan(temf_ctx& c, int level, int split, bool leaders) {
  const Symbolic& S = c.sym;
  TreePlan& T = c.splan.tree;
  cudaStream_t st = c.stream;
  const std::vector<int2> trees = build_trees(S, level);
  Sched a;
  build_sched(S, kChunkRows, a, level, leaders ? std::max(level, split) : INT_MAX, std::max(level, split));
  T.level = level;
  T.leaders = leaders;
  if (T.bacc.n < (size_t)S.n) T.bacc.alloc(S.n);
  T.ntree = (int)trees.size();
  if (trees.empty()) T.trees.alloc(1);
  else T.trees.upload(trees.data(), trees.size(), st);
  T.n_ftask = a.nf;
  T.n_btask = a.nb;
  auto up_tasks = [&](DBuf<SolveTask>& d, const std::vector<SolveTask>& v) {
    if (v.empty()) d.alloc(1);
    else d.upload(v.data(), v.size(), st);
  };
  up_tasks(T.ftask, a.ft);
  up_tasks(T.btask, a.bt);
  T.ftgt_ptr.upload(a.ftp.data(), a.ftp.size(), st);
  T.ftgt.upload(a.ftg.data(), std::max<size_t>(a.ftg.size(), 1), st);
  T.fexpect.upload(a.expect.data(), a.expect.size(), st);
  T.btgt_ptr.upload(a.btp.data(), a.btp.size(), st);
  T.btgt.upload(a.btg.data(), std::max<size_t>(a.btg.size(), 1), st);
  upload_queue_plan(a, S, split, T.q, st);  // synchronises: the host vectors go out of scope
}

// The highest subtree level (up to 11) below which there are still at least
// min_roots subtrees.  The plan built with the analysis uses two subtrees per
// resident warp of the subtree kernels (148 SMs x 12 warps).
int default_tree_level(const Symbolic& S, int min_roots = 2 * 148 * 12) {
  int best = 0;
  for (int l = 1; l < std::min(S.nlevels, 12); ++l) {
    int roots = 0;
    for (int s = 0; s < S.nsn; ++s)
      if (S.sn_level[s] < l && (S.sn_parent[s] < 0 || S.sn_level[S.sn_parent[s]] >= l)) ++roots;
    if (roots < min_roots) break;
    best = l;
  }
  return best;
}
}  // namespace

void upload_multi_plan(temf_ctx& c, int split);

void build_solve_plan(temf_ctx& c) {
  const Symbolic& S = c.sym;
  SolvePlan& P = c.splan;
  const int nsn = S.nsn;
  P.nsn = nsn;
  P.u_len = (int64_t)S.sn_rows.size();
  cudaStream_t st = c.stream;
  Sched a;
  build_sched(S, kChunkRows, a, 0, INT_MAX, default_split(S));  // above the split: ordered for claiming
  P.n_ftask = (int)a.ft.size();
  P.n_btask = (int)a.bt.size();
  P.ftask.upload(a.ft.data(), a.ft.size(), st);
  P.btask.upload(a.bt.data(), a.bt.size(), st);
  P.ftgt_ptr.upload(a.ftp.data(), a.ftp.size(), st);
  P.ftgt.upload(a.ftg.data(), std::max<size_t>(a.ftg.size(), 1), st);
  P.fexpect.upload(a.expect.data(), a.expect.size(), st);
  P.btgt_ptr.upload(a.btp.data(), a.btp.size(), st);
  P.btgt.upload(a.btg.data(), std::max<size_t>(a.btg.size(), 1), st);
  P.nchunk.upload(a.nch.data(), a.nch.size(), st);
  P.part_len = a.poff[nsn];
  P.part_off.upload(a.poff.data(), a.poff.size(), st);
  upload_queue_plan(a, S, default_split(S), P.q1, st);
  TEMF_CUDA(cudaStreamSynchronize(st));  // the host vectors of `a` go out of scope
  upload_multi_plan(c, default_split(S));
  P.sync.alloc(4 * (size_t)nsn + 8);  // + 2 claim counters of the task kernels, 2 of the subtree kernels
  upload_tree_plan(c, default_tree_level(S), default_split(S), true);
  P.tree.tuned = false;
  TEMF_CUDA(cudaStreamSynchronize(st));
}

// The 64-column block sweeps' schedules (64-row chunks) at a queue split:
// the levels above it ordered for in-order claiming (build_sched).
void upload_multi_plan(temf_ctx& c, int split) {
  const Symbolic& S = c.sym;
  SolvePlan& P = c.splan;
  const int nsn = S.nsn;
  cudaStream_t st = c.stream;
  Sched b;
  build_sched(S, kChunkRowsMulti, b, 0, INT_MAX, split);
  P.n_mftask = (int)b.ft.size();
  P.n_mbtask = (int)b.bt.size();
  P.mftask.upload(b.ft.data(), b.ft.size(), st);
  P.mbtask.upload(b.bt.data(), b.bt.size(), st);
  P.mftgt_ptr.upload(b.ftp.data(), b.ftp.size(), st);
  P.mftgt.upload(b.ftg.data(), std::max<size_t>(b.ftg.size(), 1), st);
  P.mfexpect.upload(b.expect.data(), b.expect.size(), st);
  P.mbtgt_ptr.upload(b.btp.data(), b.btp.size(), st);
  P.mbtgt.upload(b.btg.data(), std::max<size_t>(b.btg.size(), 1), st);
  P.mnchunk.upload(b.nch.data(), b.nch.size(), st);
  std::vector<int64_t> aoff(nsn + 1, 0);
  for (int s = 0; s < nsn; ++s) aoff[s + 1] = aoff[s] + (b.nch[s] > 1 ? S.sn_first[s + 1] - S.sn_first[s] : 0);
  P.macc_len = aoff[nsn];
  P.macc_off.upload(aoff.data(), aoff.size(), st);
  upload_queue_plan(b, S, split, P.qm, st);  // synchronises: the host vectors go out of scope
}

void ensure_update_buffer(temf_ctx& c, int nrhs) {
  const SolvePlan& P = c.splan;
  const size_t need = nrhs == 1 ? (size_t)std::max<int64_t>(P.part_len, 1)
                                : (size_t)std::max<int64_t>(P.macc_len, 1) * kMultiCols;
  if (c.d_part.n < need) c.d_part.alloc(need);
}

// CTAs of a persistent kernel: all that fit on the device at once.
template <typename K>
static int persistent_grid(K kernel, size_t smem) {
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, kSolveThreads, smem);
  return std::max(1, sms) * std::max(1, per);
}

static void queued_views(temf_ctx& c, bool block, double* const* Lbase, double* x, SweepView& vf, SweepView& vb);
static void reset_queues(temf_ctx& c, bool block, cudaStream_t st);

static void scale_rows(temf_ctx& c, const double* sgn, double* x, int ld, int ncol, cudaStream_t st);

static void launch_solve_multi(temf_ctx& c, double* const* Lbase, double* x, int nrhs, cudaStream_t st,
                               const double* sgn) {
  SolvePlan& P = c.splan;
  const size_t smem = sizeof(MultiSmem);
  TEMF_CUDA(cudaFuncSetAttribute(k_fwd_multi, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  TEMF_CUDA(cudaFuncSetAttribute(k_bwd_multi, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int gridf = std::min(persistent_grid(k_fwd_multi, smem), std::max(P.n_mftask, 1));
  const int gridb = std::min(persistent_grid(k_bwd_multi, smem), std::max(P.n_mbtask, 1));
  for (int c0 = 0; c0 < nrhs; c0 += kMultiCols) {
    const int k = std::min(kMultiCols, nrhs - c0);
    SweepView vf, vb;
    queued_views(c, true, Lbase, x + c0, vf, vb);
    reset_queues(c, true, st);
    k_fwd_multi<<<gridf, kSolveThreads, smem, st>>>(vf, nrhs, k, c.d_status.p + 1);
    TEMF_CHECK_LAUNCH();
    if (sgn) scale_rows(c, sgn, x + c0, nrhs, k, st);  // indefinite factor: L S L^T
    TEMF_CUDA(cudaMemsetAsync(c.d_part.p, 0, (size_t)std::max<int64_t>(P.macc_len, 1) * kMultiCols * sizeof(double), st));
    k_bwd_multi<<<gridb, kSolveThreads, smem, st>>>(vb, nrhs, k, c.d_status.p + 1);
    TEMF_CHECK_LAUNCH();
  }
}

int solve_launch_count(const temf_ctx& c, int nrhs) {
  if (nrhs > 1) return 2 * ceil_div(nrhs, kMultiCols);
  const TreePlan& T = c.splan.tree;
  return (T.ntree ? 2 : 0) + (T.n_ftask ? 1 : 0) + (T.n_btask ? 1 : 0);
}

// Views of the sweeps through the ready queue: the single-column schedules
// (q1) or the 64-row ones of the block sweeps (qm, backward accumulators in
// place of the partial sums)
static void queued_views(temf_ctx& c, bool block, double* const* Lbase, double* x, SweepView& vf, SweepView& vb) {
  FactorPlan& F = c.fplan;
  SolvePlan& P = c.splan;
  QueuePlan& Q = block ? P.qm : P.q1;
  const int nf = block ? P.n_mftask : P.n_ftask, nb = block ? P.n_mbtask : P.n_btask;
  int* q = Q.qbuf.p;
  int* words = q + (size_t)nf + 2 * (size_t)nb;  // fhead, bhead, ftail, btail
  vf = SweepView{block ? P.mftask.p : P.ftask.p, F.sn_first.p, F.sn_rows_ptr.p, F.sn_rows.p, F.sn_Lptr.p, Lbase, x,
                 block ? P.mftgt_ptr.p : P.ftgt_ptr.p, block ? P.mftgt.p : P.ftgt.p,
                 block ? P.mfexpect.p : P.fexpect.p, nullptr, nullptr, nullptr, P.sync.p, P.nsn, nf,
                 q, words + 0, words + 2, Q.fdiag.p, nullptr, nullptr, nullptr, nullptr, 0, Q.f_hi, 0,
                 c.spin_limit};
  vb = SweepView{block ? P.mbtask.p : P.btask.p, F.sn_first.p, F.sn_rows_ptr.p, F.sn_rows.p, F.sn_Lptr.p, Lbase, x,
                 block ? P.mbtgt_ptr.p : P.btgt_ptr.p, block ? P.mbtgt.p : P.btgt.p, nullptr,
                 block ? P.mnchunk.p : P.nchunk.p, block ? P.macc_off.p : P.part_off.p, c.d_part.p, P.sync.p, P.nsn,
                 nb, q + nf, words + 1, words + 3, Q.bdiag.p, Q.bdep_ptr.p, Q.bdep.p, Q.bneed.p, q + nf + nb,
                 Q.b_lo, nb, 0, c.spin_limit};
}

// clear the sweep words and seed both queues with their initially ready tasks
static void reset_queues(temf_ctx& c, bool block, cudaStream_t st) {
  SolvePlan& P = c.splan;
  QueuePlan& Q = block ? P.qm : P.q1;
  const int nf = block ? P.n_mftask : P.n_ftask, nb = block ? P.n_mbtask : P.n_btask;
  int* q = Q.qbuf.p;
  int* words = q + (size_t)nf + 2 * (size_t)nb;
  TEMF_CUDA(cudaMemsetAsync(P.sync.p, 0, P.sync.bytes(), st));
  TEMF_CUDA(cudaMemsetAsync(q, 0, Q.qbuf.bytes(), st));
  if (Q.n_finit)
    TEMF_CUDA(cudaMemcpyAsync(q, Q.finit.p, Q.n_finit * sizeof(int), cudaMemcpyDeviceToDevice, st));
  if (Q.n_binit)
    TEMF_CUDA(cudaMemcpyAsync(q + nf, Q.binit.p, Q.n_binit * sizeof(int), cudaMemcpyDeviceToDevice, st));
  TEMF_CUDA(cudaMemcpyAsync(words + 2, Q.qtails.p, 2 * sizeof(int), cudaMemcpyDeviceToDevice, st));
}

// Views of the single-column sweeps of the tree plan: its task schedules
// (the supernodes at or above the subtree level) with their ready queue.
static void tree_views(temf_ctx& c, double* const* Lbase, double* x, SweepView& vf, SweepView& vb) {
  FactorPlan& F = c.fplan;
  SolvePlan& P = c.splan;
  TreePlan& T = P.tree;
  QueuePlan& Q = T.q;
  const int nf = T.n_ftask, nb = T.n_btask;
  int* q = Q.qbuf.p;
  int* words = q + (size_t)nf + 2 * (size_t)nb;  // fhead, bhead, ftail, btail
  vf = SweepView{T.ftask.p, F.sn_first.p, F.sn_rows_ptr.p, F.sn_rows.p, F.sn_Lptr.p, Lbase, x, T.ftgt_ptr.p,
                 T.ftgt.p, T.fexpect.p, nullptr, nullptr, nullptr, P.sync.p, P.nsn, nf,
                 q, words + 0, words + 2, Q.fdiag.p, nullptr, nullptr, nullptr, nullptr, 0, Q.f_hi, 0,
                 c.spin_limit};
  vb = SweepView{T.btask.p, F.sn_first.p, F.sn_rows_ptr.p, F.sn_rows.p, F.sn_Lptr.p, Lbase, x, T.btgt_ptr.p,
                 T.btgt.p, nullptr, P.nchunk.p, P.part_off.p, c.d_part.p, P.sync.p, P.nsn, nb,
                 q + nf, words + 1, words + 3, Q.bdiag.p, Q.bdep_ptr.p, Q.bdep.p, Q.bneed.p, q + nf + nb,
                 Q.b_lo, nb, 0, c.spin_limit};
  vb.bacc = T.bacc.p;  // allocated with the plan
  vf.Dptr = vb.Dptr = F.sn_Dptr.p;
}

static void reset_tree_queues(temf_ctx& c, cudaStream_t st) {
  SolvePlan& P = c.splan;
  TreePlan& T = P.tree;
  QueuePlan& Q = T.q;
  const int nf = T.n_ftask, nb = T.n_btask;
  int* q = Q.qbuf.p;
  int* words = q + (size_t)nf + 2 * (size_t)nb;
  TEMF_CUDA(cudaMemsetAsync(P.sync.p, 0, P.sync.bytes(), st));
  TEMF_CUDA(cudaMemsetAsync(q, 0, Q.qbuf.bytes(), st));
  if (Q.n_finit)
    TEMF_CUDA(cudaMemcpyAsync(q, Q.finit.p, Q.n_finit * sizeof(int), cudaMemcpyDeviceToDevice, st));
  if (Q.n_binit)
    TEMF_CUDA(cudaMemcpyAsync(q + nf, Q.binit.p, Q.n_binit * sizeof(int), cudaMemcpyDeviceToDevice, st));
  TEMF_CUDA(cudaMemcpyAsync(words + 2, Q.qtails.p, 2 * sizeof(int), cudaMemcpyDeviceToDevice, st));
}

static int tree_grid() {
  static int g = 0;
  if (!g) {
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_fwd_subtrees, kTreeThreads, 0);
    int perb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perb, k_bwd_subtrees, kTreeThreads, 0);
    g = std::max(1, sms) * std::max(1, std::min(per, perb));
  }
  return g;
}

// x[i * ld + k] *= sgn[i] for the k < ncol columns of a row-major block
__global__ void k_scale_rows(int64_t n, int ld, int ncol, const double* __restrict__ sgn, double* __restrict__ x) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n * ncol) x[(q / ncol) * ld + q % ncol] *= sgn[q / ncol];
}

static void scale_rows(temf_ctx& c, const double* sgn, double* x, int ld, int ncol, cudaStream_t st) {
  const int64_t n = c.pat.n;
  k_scale_rows<<<ceil_div(n * ncol, 256), 256, 0, st>>>(n, ld, ncol, sgn, x);
  TEMF_CHECK_LAUNCH();
}

// r = b - (a X + b2 Y) x on the permuted full pattern, nrhs columns (row-major)
__global__ void k_residual(int n, int nrhs, const int* __restrict__ rowptr, const int* __restrict__ col,
                           const double* __restrict__ X, double a, const double* __restrict__ Y, double b2,
                           const double* __restrict__ x, const double* __restrict__ b, double* __restrict__ r) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (int64_t)n * nrhs) return;
  const int i = (int)(q / nrhs), k = (int)(q % nrhs);
  double acc = 0.0;
  for (int p = rowptr[i]; p < rowptr[i + 1]; ++p) {
    const double v = a * X[p] + (Y ? b2 * Y[p] : 0.0);
    acc += v * x[(int64_t)col[p] * nrhs + k];
  }
  r[q] = b[q] - acc;
}

void launch_residual(temf_ctx& c, const FactorSlot& fs, const double* x, const double* b, double* r, int nrhs,
                     cudaStream_t st) {
  const int n = c.pat.n;
  k_residual<<<ceil_div((int64_t)n * nrhs, 256), 256, 0, st>>>(n, nrhs, c.d_rowptr.p, c.d_col.p, fs.X, fs.a,
                                                               fs.Y, fs.b, x, b, r);
  TEMF_CHECK_LAUNCH();
}

void launch_solve(temf_ctx& c, double* const* Lbase, double* x, int nrhs, cudaStream_t st, const double* sgn) {
  SolvePlan& P = c.splan;
  ensure_update_buffer(c, nrhs);
  if (nrhs > 1) {
    launch_solve_multi(c, Lbase, x, nrhs, st, sgn);
    return;
  }
  // single column: subtrees (forward), task kernels above the subtree level
  // (forward, backward), subtrees (backward)
  TreePlan& T = P.tree;
  SweepView vf, vb;
  tree_views(c, Lbase, x, vf, vb);
  reset_tree_queues(c, st);
  // failure-detection test: one more input expected for the last supernode
  // than any task provides, so its wait (or its queue slot) runs out
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  TEMF_CUDA(cudaStreamIsCapturing(st, &cap));
  const bool inject = c.inject_wait && T.n_ftask > 0 && cap == cudaStreamCaptureStatusNone;
  int* inject_word = inject ? T.fexpect.p + (P.nsn - 1) : nullptr;
  if (inject) {
    c.inject_wait = 0;
    k_add_int<<<1, 1, 0, st>>>(inject_word, 1);
    TEMF_CHECK_LAUNCH();
  }
  int* tcount = P.sync.p + 4 * (size_t)P.nsn + 4;
  const int tgrid = std::min(tree_grid(), std::max(1, ceil_div(T.ntree, kTreeThreads / 32)));
  if (T.ntree) {
    k_fwd_subtrees<<<tgrid, kTreeThreads, 0, st>>>(TreeView{T.trees.p, T.ntree, c.fplan.sn_first.p,
                                                            c.fplan.sn_rows_ptr.p, c.fplan.sn_rows.p,
                                                            c.fplan.sn_Lptr.p, Lbase, x, tcount,
                                                            c.fplan.sn_Dptr.p});
    TEMF_CHECK_LAUNCH();
  }
  if (T.n_ftask) {
    if (T.leaders) {
      const int grid = std::min(persistent_grid(k_fwd_queued<true>, 0), T.n_ftask);
      k_fwd_queued<true><<<grid, kSolveThreads, 0, st>>>(vf, c.d_status.p + 1);
    } else {
      const int grid = std::min(persistent_grid(k_fwd_queued<false>, 0), T.n_ftask);
      k_fwd_queued<false><<<grid, kSolveThreads, 0, st>>>(vf, c.d_status.p + 1);
    }
    TEMF_CHECK_LAUNCH();
  }
  if (inject) {
    k_add_int<<<1, 1, 0, st>>>(inject_word, -1);
    TEMF_CHECK_LAUNCH();
  }
  if (sgn) scale_rows(c, sgn, x, 1, 1, st);  // indefinite factor: L S L^T
  TEMF_CUDA(cudaMemsetAsync(T.bacc.p, 0, (size_t)c.n_edges * sizeof(double), st));
  if (T.n_btask) {
    if (T.leaders) {
      const int gridb = std::min(persistent_grid(k_bwd_queued<true>, 0), T.n_btask);
      k_bwd_queued<true><<<gridb, kSolveThreads, 0, st>>>(vb, c.d_status.p + 1);
    } else {
      const int gridb = std::min(persistent_grid(k_bwd_queued<false>, 0), T.n_btask);
      k_bwd_queued<false><<<gridb, kSolveThreads, 0, st>>>(vb, c.d_status.p + 1);
    }
    TEMF_CHECK_LAUNCH();
  }
  if (T.ntree) {
    k_bwd_subtrees<<<tgrid, kTreeThreads, 0, st>>>(TreeView{T.trees.p, T.ntree, c.fplan.sn_first.p,
                                                            c.fplan.sn_rows_ptr.p, c.fplan.sn_rows.p,
                                                            c.fplan.sn_Lptr.p, Lbase, x, tcount + 1,
                                                            c.fplan.sn_Dptr.p});
    TEMF_CHECK_LAUNCH();
  }
}

void launch_solve_scratch(temf_ctx& c, double* const* Lbase, double* x, int* sync, double* part, int* err,
                          cudaStream_t st) {
  FactorPlan& F = c.fplan;
  SolvePlan& P = c.splan;
  const size_t smem = (size_t)(kSnCols + kChunkRows) * sizeof(double);
  TEMF_CUDA(cudaMemsetAsync(sync, 0, (4 * (size_t)P.nsn + 4) * sizeof(int), st));
  const int grid = std::min(persistent_grid(k_fwd_persistent, smem), std::max(P.n_ftask, 1));
  k_fwd_persistent<<<grid, kSolveThreads, smem, st>>>(P.n_ftask, P.ftask.p, F.sn_first.p, F.sn_rows_ptr.p,
                                                      F.sn_rows.p, F.sn_Lptr.p, Lbase, x, 1, P.ftgt_ptr.p, P.ftgt.p,
                                                      P.fexpect.p, sync, P.nsn, err);
  TEMF_CHECK_LAUNCH();
  const int gridb = std::min(persistent_grid(k_bwd_persistent, smem), std::max(P.n_btask, 1));
  k_bwd_persistent<<<gridb, kSolveThreads, smem, st>>>(P.n_btask, P.btask.p, F.sn_first.p, F.sn_rows_ptr.p,
                                                       F.sn_rows.p, F.sn_Lptr.p, Lbase, x, 1, P.btgt_ptr.p, P.btgt.p,
                                                       P.nchunk.p, P.part_off.p, part, sync, P.nsn, err);
  TEMF_CHECK_LAUNCH();
}

int solve_error_flag(temf_ctx& c) {
  int v = 0;
  TEMF_CUDA(cudaMemcpyAsync(&v, c.d_status.p + 1, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  TEMF_CUDA(cudaStreamSynchronize(c.stream));
  return v;
}

void clear_solve_error_flag(temf_ctx& c) {
  TEMF_CUDA(cudaMemsetAsync(c.d_status.p + 1, 0, sizeof(int), c.stream));
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

// --- many models at once -----------------------------------------------------
SweepView fwd_view(temf_ctx& c, double* const* Lbase, double* x, int* sync) {
  FactorPlan& F = c.fplan;
  SolvePlan& P = c.splan;
  SweepView v{P.ftask.p, F.sn_first.p, F.sn_rows_ptr.p, F.sn_rows.p, F.sn_Lptr.p, Lbase, x, P.ftgt_ptr.p,
              P.ftgt.p, P.fexpect.p, nullptr, nullptr, nullptr, sync, P.nsn, P.n_ftask};
  v.spin = c.spin_limit;
  return v;
}

SweepView bwd_view(temf_ctx& c, double* const* Lbase, double* x, int* sync) {
  FactorPlan& F = c.fplan;
  SolvePlan& P = c.splan;
  ensure_update_buffer(c, 1);
  SweepView v{P.btask.p, F.sn_first.p, F.sn_rows_ptr.p, F.sn_rows.p, F.sn_Lptr.p, Lbase, x, P.btgt_ptr.p,
              P.btgt.p, nullptr, P.nchunk.p, P.part_off.p, c.d_part.p, sync, P.nsn, P.n_btask};
  v.spin = c.spin_limit;
  return v;
}

int models_grid(bool forward) {
  return forward ? persistent_grid(k_fwd_models, 0) : persistent_grid(k_bwd_models, 0);
}

void launch_solve_models(int nf, const int2* order_f, const SweepView* vf, int nb, const int2* order_b,
                         const SweepView* vb, const int* active, int* counters, int* err, int grid_f, int grid_b,
                         int qlim_f, int qlim_b, cudaStream_t st) {
  k_fwd_models<<<std::max(1, std::min(grid_f, nf + qlim_f)), kSolveThreads, 0, st>>>(nf, order_f, vf, active,
                                                                                      counters, err, qlim_f);
  TEMF_CHECK_LAUNCH();
  k_bwd_models<<<std::max(1, std::min(grid_b, nb + qlim_b)), kSolveThreads, 0, st>>>(nb, order_b, vb, active,
                                                                                      counters + 1, err, qlim_b);
  TEMF_CHECK_LAUNCH();
}

void queue_ranges(const temf_ctx& c, int& f_hi, int& b_lo) {
  f_hi = c.splan.q1.f_hi;
  b_lo = c.splan.q1.b_lo;
}

void queue_init_lists(const temf_ctx& c, std::vector<int>& finit, std::vector<int>& binit) {
  const QueuePlan& Q = c.splan.q1;
  finit.resize(Q.n_finit);
  binit.resize(Q.n_binit);
  // stored as task + 1
  if (Q.n_finit) TEMF_CUDA(cudaMemcpy(finit.data(), Q.finit.p, Q.n_finit * sizeof(int), cudaMemcpyDeviceToHost));
  if (Q.n_binit) TEMF_CUDA(cudaMemcpy(binit.data(), Q.binit.p, Q.n_binit * sizeof(int), cudaMemcpyDeviceToHost));
  for (int& v : finit) --v;
  for (int& v : binit) --v;
}

// One single-column solve of b with the per-task timeline recorded.
// out: 8 words per task, forward tasks then backward tasks: start, dependency
// satisfied, end (ns), SM, supernode, kind, first row, supernode level.
void solve_timeline(temf_ctx& c, int slot, const double* b_perm, int64_t cap, unsigned long long* out,
                    int* n_fwd, int* n_bwd) {
  SolvePlan& P = c.splan;
  TreePlan& T = P.tree;
  const int nf = T.ntree + T.n_ftask, nb = T.n_btask + T.ntree;
  const int64_t nt = (int64_t)nf + nb;
  *n_fwd = nf;
  *n_bwd = nb;
  if (!out) return;
  if (cap < 8 * nt) throw ArgError("timeline buffer too small: need 8 words per task");
  cudaStream_t st = c.stream;
  // stamps: forward subtrees, forward tasks, backward tasks, backward subtrees
  DBuf<unsigned long long> rec;
  rec.alloc(4 * (size_t)std::max<int64_t>(nt, 1));
  TEMF_CUDA(cudaMemsetAsync(rec.p, 0, rec.bytes(), st));
  DBuf<double> x;
  x.upload(b_perm, c.n_edges, st);
  DBuf<double*> lb;
  lb.alloc(1);
  double* Lp = c.slots[slot].L.p;
  TEMF_CUDA(cudaMemcpyAsync(lb.p, &Lp, sizeof(double*), cudaMemcpyHostToDevice, st));
  unsigned long long* ptf = rec.p;
  unsigned long long* pf = rec.p + 4 * (size_t)T.ntree;
  unsigned long long* pb = rec.p + 4 * (size_t)nf;
  unsigned long long* ptb = rec.p + 4 * ((size_t)nf + T.n_btask);
  unsigned long long* none = nullptr;
  TEMF_CUDA(cudaMemcpyToSymbolAsync(g_timeline_f, &pf, sizeof(pf), 0, cudaMemcpyHostToDevice, st));
  TEMF_CUDA(cudaMemcpyToSymbolAsync(g_timeline_b, &pb, sizeof(pb), 0, cudaMemcpyHostToDevice, st));
  TEMF_CUDA(cudaMemcpyToSymbolAsync(g_timeline_tf, &ptf, sizeof(ptf), 0, cudaMemcpyHostToDevice, st));
  TEMF_CUDA(cudaMemcpyToSymbolAsync(g_timeline_tb, &ptb, sizeof(ptb), 0, cudaMemcpyHostToDevice, st));
  launch_solve(c, lb.p, x.p, 1, st);
  TEMF_CUDA(cudaMemcpyToSymbolAsync(g_timeline_f, &none, sizeof(none), 0, cudaMemcpyHostToDevice, st));
  TEMF_CUDA(cudaMemcpyToSymbolAsync(g_timeline_b, &none, sizeof(none), 0, cudaMemcpyHostToDevice, st));
  TEMF_CUDA(cudaMemcpyToSymbolAsync(g_timeline_tf, &none, sizeof(none), 0, cudaMemcpyHostToDevice, st));
  TEMF_CUDA(cudaMemcpyToSymbolAsync(g_timeline_tb, &none, sizeof(none), 0, cudaMemcpyHostToDevice, st));
  std::vector<unsigned long long> h(4 * (size_t)std::max<int64_t>(nt, 1));
  std::vector<SolveTask> tf(T.n_ftask), tb(T.n_btask);
  std::vector<int2> tr(T.ntree);
  TEMF_CUDA(cudaMemcpyAsync(h.data(), rec.p, rec.bytes(), cudaMemcpyDeviceToHost, st));
  if (T.n_ftask)
    TEMF_CUDA(cudaMemcpyAsync(tf.data(), T.ftask.p, tf.size() * sizeof(SolveTask), cudaMemcpyDeviceToHost, st));
  if (T.n_btask)
    TEMF_CUDA(cudaMemcpyAsync(tb.data(), T.btask.p, tb.size() * sizeof(SolveTask), cudaMemcpyDeviceToHost, st));
  if (T.ntree) TEMF_CUDA(cudaMemcpyAsync(tr.data(), T.trees.p, tr.size() * sizeof(int2), cudaMemcpyDeviceToHost, st));
  TEMF_CUDA(cudaStreamSynchronize(st));
  for (int64_t i = 0; i < nt; ++i) {
    // which list row i is in, and its task / subtree
    SolveTask t{0, 0, 0, 0};
    if (i < T.ntree) {
      const int2 q = tr[i];
      t = SolveTask{q.y, 2, q.x, 0};
    } else if (i < nf) {
      t = tf[i - T.ntree];
    } else if (i < nf + T.n_btask) {
      t = tb[i - nf];
    } else {
      const int2 q = tr[i - nf - T.n_btask];
      t = SolveTask{q.y, 2, q.x, 0};
    }
    unsigned long long* o = out + 8 * i;
    for (int q = 0; q < 4; ++q) o[q] = h[4 * i + q];
    o[4] = (unsigned long long)t.s;
    o[5] = (unsigned long long)(t.kind & 15);
    o[6] = (unsigned long long)t.r0;
    o[7] = (unsigned long long)c.sym.sn_level[t.s];
  }
}

// Structure of the supernodal partition (the analogue of pardiso_checker,
// src/FETD_UTILITY.f90:993-1027, for the factor): row lists ascending and
// below the diagonal block, the parent owning the first row, and every row
// of a child either a column or a row of its parent (the Schur update of
// the child lands inside the parent's panel).
static std::string check_structure(const Symbolic& S) {
  for (int s = 0; s < S.nsn; ++s) {
    const int f = S.sn_first[s], l = S.sn_first[s + 1];
    if (l <= f) return "empty supernode";
    const int* b = S.sn_rows.data() + S.sn_rows_ptr[s];
    const int* e = S.sn_rows.data() + S.sn_rows_ptr[s + 1];
    for (const int* q = b; q < e; ++q) {
      if (*q < l || *q >= S.n) return "row list outside the lower triangle";
      if (q > b && q[-1] >= *q) return "row list not ascending";
    }
    const int p = S.sn_parent[s];
    if (b == e) {
      if (p >= 0) return "supernode without rows has a parent";
      continue;
    }
    if (p != S.col2sn[*b]) return "parent does not own the first row";
    const int fp = S.sn_first[p], lp = S.sn_first[p + 1];
    const int* pb = S.sn_rows.data() + S.sn_rows_ptr[p];
    const int* pe = S.sn_rows.data() + S.sn_rows_ptr[p + 1];
    for (const int* q = b; q < e; ++q) {
      if (*q >= fp && *q < lp) continue;
      if (!std::binary_search(pb, pe, *q)) return "child row missing from its parent";
    }
    if (S.sn_level[p] <= S.sn_level[s]) return "parent not on a higher level";
  }
  return std::string();
}

static std::vector<int> split_candidates(const Symbolic& S, int level);

std::string check_schedules(const Symbolic& S) {
  {
    const std::string w = check_structure(S);
    if (!w.empty()) return "supernode structure: " + w;
  }
  {
    const std::string w = check_update_groups(S);
    if (!w.empty()) return "factor update groups: " + w;
  }
  const int splits[5] = {0, level_below_width(S, 2048), default_split(S), level_below_width(S, 64), S.nlevels};
  for (int sp : splits) {
    std::string w = check_schedule(S, kChunkRows, sp);
    if (!w.empty()) return "128-row chunks, split " + std::to_string(sp) + ": " + w;
    w = check_schedule(S, kChunkRows, sp, 0, INT_MAX, true);
    if (!w.empty()) return "128-row chunks, split " + std::to_string(sp) + ", grouped levels: " + w;
    // the allocation-free path (everything claimed in order) and the model batches (queue split
    // at the default): their schedule is grouped at the default split
    if (sp <= default_split(S)) {
      w = check_schedule(S, kChunkRows, sp, 0, INT_MAX, true, default_split(S));
      if (!w.empty()) return "128-row chunks, split " + std::to_string(sp) + ", grouped at the default: " + w;
    }
    w = check_schedule(S, kChunkRows, sp, 0, sp, true);
    if (!w.empty()) return "128-row chunks, split " + std::to_string(sp) + ", run leaders: " + w;
    w = check_schedule(S, kChunkRowsMulti, sp, 0, INT_MAX, true);
    if (!w.empty()) return "64-row chunks, split " + std::to_string(sp) + ": " + w;
  }
  // the single-column plans with subtrees: every level the tuner may pick,
  // the subtree protocol and the task schedules above it at each queue split
  for (int l = 1; l <= std::max(default_tree_level(S, 148), std::min(S.nlevels, 3)); ++l) {
    std::string w = check_trees(S, l);
    if (!w.empty()) return "subtrees below level " + std::to_string(l) + ": " + w;
    for (int sp : split_candidates(S, l)) {
      w = check_schedule(S, kChunkRows, sp, l, INT_MAX, true);
      if (!w.empty()) return "subtree level " + std::to_string(l) + ", split " + std::to_string(sp) + ": " + w;
      w = check_schedule(S, kChunkRows, sp, l, std::max(l, sp), true);
      if (!w.empty())
        return "subtree level " + std::to_string(l) + ", split " + std::to_string(sp) + ", run leaders: " + w;
    }
  }
  return std::string();
}

// Autotuner of the queue split: times one solve (right-hand side all ones,
// nrhs columns) for each candidate split level and keeps the fastest.
static int tune_tree(temf_ctx& c, int slot);

int tune_solve(temf_ctx& c, int slot, int nrhs) {
  if (nrhs == 1) return tune_tree(c, slot);
  const Symbolic& S = c.sym;
  SolvePlan& P = c.splan;
  const bool block = nrhs > 1;
  QueuePlan& Q = block ? P.qm : P.q1;
  cudaStream_t st = c.stream;
  Sched a;
  if (!block) build_sched(S, kChunkRows, a);
  std::vector<int> cand = {0, level_below_width(S, 4096), level_below_width(S, 1024), level_below_width(S, 512),
                           level_below_width(S, 148), level_below_width(S, 32), S.nlevels};
  std::sort(cand.begin(), cand.end());
  cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
  const size_t vec = (size_t)c.n_edges * nrhs;
  DBuf<double> ones, x;
  std::vector<double> h(vec, 1.0);
  ones.upload(h.data(), vec, st);
  x.alloc(vec);
  DBuf<double*> lb;
  lb.alloc(1);
  double* Lp = c.slots[slot].L.p;
  TEMF_CUDA(cudaMemcpyAsync(lb.p, &Lp, sizeof(double*), cudaMemcpyHostToDevice, st));
  cudaEvent_t e0, e1;
  TEMF_CUDA(cudaEventCreate(&e0));
  TEMF_CUDA(cudaEventCreate(&e1));
  Q.tune_ms.clear();
  Q.tune_split.clear();
  int best = Q.split;
  double best_ms = 1e30;
  for (int sp : cand) {
    if (block) upload_multi_plan(c, sp);
    else upload_queue_plan(a, S, sp, Q, st);
    double tot = 0.0;
    for (int rep = 0; rep < 4; ++rep) {
      TEMF_CUDA(cudaMemcpyAsync(x.p, ones.p, vec * sizeof(double), cudaMemcpyDeviceToDevice, st));
      TEMF_CUDA(cudaEventRecord(e0, st));
      launch_solve(c, lb.p, x.p, nrhs, st);
      TEMF_CUDA(cudaEventRecord(e1, st));
      TEMF_CUDA(cudaEventSynchronize(e1));
      float ms = 0;
      TEMF_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      if (rep > 0) tot += ms;  // the first solve warms up
    }
    tot /= 3.0;
    Q.tune_ms.push_back(tot);
    Q.tune_split.push_back(sp);
    if (tot < best_ms) {
      best_ms = tot;
      best = sp;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (block) upload_multi_plan(c, best);
  else upload_queue_plan(a, S, best, Q, st);
  Q.tuned = true;
  return best;
}

// Candidate queue splits above a subtree level (the level itself: no queue).
static std::vector<int> split_candidates(const Symbolic& S, int level) {
  std::vector<int> cand = {level};
  for (int w : {4096, 1024, 512, 148, 32}) {
    const int l = level_below_width(S, w);
    if (l > level) cand.push_back(l);
  }
  std::sort(cand.begin(), cand.end());
  cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
  return cand;
}

// Autotuner of the single-column plan: first the subtree level (0 = none, and
// the levels below which there are enough subtrees to fill the GPU twice),
// each with the default queue split, then the queue split at the best level,
// both without run leaders, then the best plan with them.
// Times one solve (right-hand side all ones) per candidate, keeps the fastest.
static int tune_tree(temf_ctx& c, int slot) {
  const Symbolic& S = c.sym;
  TreePlan& T = c.splan.tree;
  cudaStream_t st = c.stream;
  const size_t vec = (size_t)c.n_edges;
  DBuf<double> ones, x;
  std::vector<double> h(vec, 1.0);
  ones.upload(h.data(), vec, st);
  x.alloc(vec);
  DBuf<double*> lb;
  lb.alloc(1);
  double* Lp = c.slots[slot].L.p;
  TEMF_CUDA(cudaMemcpyAsync(lb.p, &Lp, sizeof(double*), cudaMemcpyHostToDevice, st));
  cudaEvent_t e0, e1;
  TEMF_CUDA(cudaEventCreate(&e0));
  TEMF_CUDA(cudaEventCreate(&e1));
  std::vector<int> lv_c, sp_c;
  std::vector<double> ms_c;
  auto time_plan = [&](int level, int split, bool leaders = false) {
    upload_tree_plan(c, level, split, leaders);
    double tot = 0.0;
    for (int rep = 0; rep < 4; ++rep) {
      TEMF_CUDA(cudaMemcpyAsync(x.p, ones.p, vec * sizeof(double), cudaMemcpyDeviceToDevice, st));
      TEMF_CUDA(cudaEventRecord(e0, st));
      launch_solve(c, lb.p, x.p, 1, st);
      TEMF_CUDA(cudaEventRecord(e1, st));
      TEMF_CUDA(cudaEventSynchronize(e1));
      float ms = 0;
      TEMF_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      if (rep > 0) tot += ms;  // the first solve warms up
    }
    lv_c.push_back(level);
    sp_c.push_back(split);
    ms_c.push_back(tot / 3.0);
    return tot / 3.0;
  };
  // levels with at least one subtree per SM (resident warps: about 12 per SM)
  std::vector<int> levels = {0};
  const int top = default_tree_level(S, 148);
  for (int l = 2; l <= top; ++l) levels.push_back(l);
  int best_level = 0, best_split = default_split(S);
  double best = 1e30;
  for (int l : levels) {
    const int sp = std::max(l, default_split(S));
    const double ms = time_plan(l, sp);
    if (ms < best) { best = ms; best_level = l; best_split = sp; }
  }
  // the split candidates at the chosen level (at most 6, with the one timed above)
  std::vector<int> sps = {best_split};
  std::vector<double> sms = {best};
  for (int sp : split_candidates(S, best_level)) {
    if (sp == sps[0]) continue;
    const double ms = time_plan(best_level, sp);
    sps.push_back(sp);
    sms.push_back(ms);
    if (ms < best) { best = ms; best_split = sp; }
  }
  // and the chosen plan with run leaders (the level and split candidates are
  // timed without: the leader instances carry more registers)
  bool best_leaders = false;
  {
    const double ms = time_plan(best_level, best_split, true);
    if (ms < best) { best = ms; best_leaders = true; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  upload_tree_plan(c, best_level, best_split, best_leaders);
  T.q.tune_ms = sms;
  T.q.tune_split = sps;
  T.tune_level = lv_c;
  T.q.tuned = true;
  T.tuned = true;
  return best_split;
}

void set_tree_plan(temf_ctx& c, int level, int split, bool leaders) {
  const Symbolic& S = c.sym;
  if (level < 0 || level > S.nlevels) throw ArgError("subtree level out of range");
  if (split < 0 || split > S.nlevels) throw ArgError("queue split level out of range");
  if (level > 0) {
    const std::string w = check_trees(S, level);
    if (!w.empty()) throw StateError("subtrees below level " + std::to_string(level) + ": " + w);
  }
  upload_tree_plan(c, level, split, leaders);
  c.splan.tree.q.tuned = true;
  c.splan.tree.tuned = true;
}

}  // namespace temf
